// Workload generation for the checker side (test infrastructure only).
//
// bench.py's reference arm times the reference binary on the benchmark's
// seeded 4,096-graph Chung-Lu batch.  That process must not map libmce.so,
// the library under test, so the same seeded generators are compiled a
// second time into liboracle.so (sources: mce-gpu_b200/host/gen.cpp,
// hgraph.cpp and bel.cpp, with hidden visibility) and reached through the
// oracle_* entry points below.  The graphs are byte-identical to the ones
// libmce.so's generators return (tests/test_oracle.py checks it).
#include <cstdint>
#include <cstdlib>

#include "../include/mce.h"
#include "../include/mce_gen.h"

#define ORACLE_API extern "C" __attribute__((visibility("default")))

// The disjoint union of a seeded Chung-Lu batch (mce_gen_chung_lu_batch's
// arguments), as one CSR, plus each graph's first vertex in the union
// (graph_start, num_graphs + 1 entries, malloc'd).  Release with
// oracle_hgraph_free / free.
ORACLE_API int oracle_gen_batch_union(int32_t num_graphs, int64_t n_min, int64_t n_max,
                                      double gamma, double deg_min, double deg_max,
                                      int32_t max_planted, int32_t clique_min,
                                      int32_t clique_max, uint64_t seed, mce_hgraph_t *out,
                                      int64_t **graph_start) {
  mce_hgraph_t b{};
  int rc = mce_gen_chung_lu_batch(num_graphs, n_min, n_max, gamma, deg_min, deg_max, max_planted,
                                  clique_min, clique_max, seed, &b);
  if (rc) return rc;
  int64_t *gs = (int64_t *)malloc(sizeof(int64_t) * (size_t)(num_graphs + 1));
  if (!gs) {
    mce_hgraph_free(&b);
    return MCE_ENOMEM;
  }
  // graph g's local rows occupy vtx_offsets[g] .. vtx_offsets[g+1] (n_g + 1
  // entries), so its first union vertex is vtx_offsets[g] - g
  for (int32_t g = 0; g <= num_graphs; ++g) gs[g] = b.vtx_offsets[g] - g;
  rc = mce_hgraph_union(&b, out);
  mce_hgraph_free(&b);
  if (rc) {
    free(gs);
    return rc;
  }
  *graph_start = gs;
  return 0;
}

// A single graph from the Barabasi-Albert / R-MAT / Erdos-Renyi generators
// (mce_gen_ba / mce_gen_rmat / mce_gen_er arguments).
ORACLE_API int oracle_gen_ba(int64_t n, int32_t m, uint64_t seed, int32_t planted, int32_t cmin,
                             int32_t cmax, mce_hgraph_t *out) {
  return mce_gen_ba(n, m, seed, planted, cmin, cmax, out);
}

ORACLE_API int oracle_gen_rmat(int32_t scale, int32_t ef, double a, double b, double c,
                               uint64_t seed, mce_hgraph_t *out) {
  return mce_gen_rmat(scale, ef, a, b, c, seed, out);
}

ORACLE_API int oracle_gen_er(int64_t n, double p, uint64_t seed, int32_t planted, int32_t cmin,
                             int32_t cmax, mce_hgraph_t *out) {
  return mce_gen_er(n, p, seed, planted, cmin, cmax, out);
}

// The .bel writer (the record layout of graph::convert_to_bel,
// include/fileop.h:62-71).
ORACLE_API int oracle_bel_write(const char *path, const mce_hgraph_t *g) {
  return mce_bel_write(path, g);
}

// The 2-hop ego subgraph of a seed vertex (mce_ego_subgraph's arguments).
ORACLE_API int oracle_ego_subgraph(const int32_t *row_ptr, const int32_t *col, int64_t n,
                                   int64_t seed_vertex, int64_t cap, mce_hgraph_t *out) {
  return mce_ego_subgraph(row_ptr, col, n, seed_vertex, cap, out, nullptr);
}

ORACLE_API void oracle_hgraph_free(mce_hgraph_t *g) { mce_hgraph_free(g); }
