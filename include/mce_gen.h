/*
 * mce_gen.h - seeded synthetic graph generators of libmce.so.
 *
 * The reference benchmarks on public SNAP / Network Repository graphs that
 * are downloaded at run time (download.py:21-96).  These generators stand in
 * for them with seeded, deterministic graphs of the shapes the benchmark
 * configurations name.  Every generator returns a normalised CSR (symmetric,
 * sorted rows, no self-loops, no duplicates) in an mce_hgraph_t that the
 * caller releases with mce_hgraph_free().  The output depends only on the
 * arguments, not on the number of host threads.
 */
#ifndef MCE_GEN_H
#define MCE_GEN_H

#include "mce.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Erdos-Renyi G(n, p) plus `planted` cliques whose sizes are uniform in
 * [clique_min, clique_max], each on a uniformly random vertex set.         */
int mce_gen_er(int64_t n, double p, uint64_t seed, int32_t planted, int32_t clique_min,
               int32_t clique_max, mce_hgraph_t *out);

/* R-MAT: 2^scale vertices, edge_factor * 2^scale edge samples, quadrant
 * probabilities (a, b, c, 1-a-b-c); symmetrised, deduplicated, no loops.   */
int mce_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                 uint64_t seed, mce_hgraph_t *out);

/* Barabasi-Albert preferential attachment (n vertices, m edges per new
 * vertex, starting from a clique on m+1 vertices) plus `planted` cliques of
 * size uniform in [clique_min, clique_max] drawn from a shared pool of
 * planted * (clique_min + clique_max) / 4 vertices, so that they overlap.  */
int mce_gen_ba(int64_t n, int32_t m, uint64_t seed, int32_t planted, int32_t clique_min,
               int32_t clique_max, mce_hgraph_t *out);

/* A batch of independent Chung-Lu graphs (one mce_hgraph_t with
 * num_graphs > 1).  Graph i has n_i log-uniform in [n_min, n_max], weights
 * w_j ~ (j+1)^(-1/(gamma-1)) scaled to a mean degree uniform in
 * [deg_min, deg_max] (the edge sampler's target before deduplication), and
 * a uniform number in [0, max_planted] of planted cliques of size uniform in
 * [clique_min, clique_max] (capped at n_i).                                */
int mce_gen_chung_lu_batch(int32_t num_graphs, int64_t n_min, int64_t n_max, double gamma,
                           double deg_min, double deg_max, int32_t max_planted,
                           int32_t clique_min, int32_t clique_max, uint64_t seed,
                           mce_hgraph_t *out);

/* Relabel a graph by a seeded random permutation (for invariance tests). */
int mce_gen_permute(const mce_hgraph_t *in, uint64_t seed, mce_hgraph_t *out);

/* Disjoint union of a batch's graphs as one CSR (for running a batch
 * through the single-graph path).                                          */
int mce_hgraph_union(const mce_hgraph_t *batch, mce_hgraph_t *out);

/* The 2-hop ego subgraph of `seed_vertex`: the seed, its neighbours in row
 * order, then 2-hop vertices in discovery order (the rows of the
 * neighbours, in turn) until `cap` vertices are taken; relabelled 0..k-1 in
 * ascending original id.  If vertex_map_out is not NULL it receives the
 * original ids (cap entries).  The serving kernel extracts the same graph. */
int mce_ego_subgraph(const int32_t *row_ptr, const int32_t *col, int64_t n,
                     int64_t seed_vertex, int64_t cap, mce_hgraph_t *out,
                     int32_t *vertex_map_out);

#ifdef __cplusplus
}
#endif
#endif /* MCE_GEN_H */
