/*
 * mce.h - C ABI of the B200 maximal-clique enumerator (libmce.so).
 *
 * The library counts the maximal cliques (size >= 2) of an undirected simple
 * graph with the method of yen-hsiang-chang/mce-gpu: a degeneracy order from
 * k-core peeling, then one Bron-Kerbosch search per root vertex with Tomita
 * pivoting over the bitmap-encoded subgraph induced by the root's
 * later-ordered neighbours.  Isolated vertices (maximal cliques of size 1)
 * are never counted, exactly as in the reference (mce/mce_kernel_wl.cuh:70-79:
 * a root with no later neighbour yields nothing).
 *
 * Conventions (all entry points):
 *   - return MCE_OK (0) or a negative MCE_E* code; nothing calls exit();
 *   - the caller owns every host buffer it passes in; buffers the library
 *     returns (mce_hgraph_t arrays) are released with mce_hgraph_free();
 *   - device memory is owned by the handle that allocated it;
 *   - a handle is used by one host thread at a time; its work is queued on
 *     the stream given in mce_opts_t.stream (or the handle's own stream).
 *
 * Vertex ids and CSR offsets are int32 (the reference's DataType is uint32,
 * include/defs.h:10); graphs with 2^31 or more arcs are rejected.
 */
#ifndef MCE_H
#define MCE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MCE_OK 0
#define MCE_EINVAL (-1)   /* bad argument                                   */
#define MCE_ENOMEM (-2)   /* host or device allocation failed               */
#define MCE_ECUDA (-3)    /* CUDA runtime error                             */
#define MCE_EIO (-4)      /* file could not be opened / read / written      */
#define MCE_EFORMAT (-5)  /* malformed input (.bel or CSR)                  */
#define MCE_ELIMIT (-6)   /* a size cap was exceeded (degree, depth, queue) */
#define MCE_ETIMEOUT (-7) /* a bounded device wait ran out                  */
#define MCE_ENODEV (-8)   /* no usable CUDA device                          */
#define MCE_ESTATE (-9)   /* call out of order (e.g. serve handle closed)   */
#define MCE_EAGAIN (-10) /* not finished yet (mce_serve_poll)              */

/* Clique-size histogram length: hist[s] counts maximal cliques of size s.  */
#define MCE_HIST_MAX 4096

/* Largest later-neighbour count (bitmap width) a root may have.  The
 * reference caps this at MAX_DEGEN = 2048 (mce/parameter.cuh:3); so do we.  */
#define MCE_MAX_LATER_DEGREE 2048

/* ---- options ------------------------------------------------------------ */
/* -p (include/config.h:52-61): level of the subtrees that are parallelised.
 * L1: a root's subtrees go to idle warps once its walk is under way
 * (donate_after nodes).  L2: the reference's edge-rooted scheme
 * (mce/mce_kernel_wl.cuh:307-485): every oriented edge (r, v) is a unit
 * whose candidates are the triangle list N+(r) & N+(v), whose pivot comes
 * from them alone, and whose outside set is the neighbours of r before v in
 * the degeneracy order adjacent to v; units are offered to idle warps at
 * once.  Same counts; the trees are the reference's L2 trees.              */
#define MCE_LEVEL_L1 1
#define MCE_LEVEL_L2 2
/* -i (include/config.h:72-81): which sets the induced subgraph is built on */
#define MCE_INDUCED_P 1
#define MCE_INDUCED_PX 2
/* -w (include/config.h:92-101): worker list (donation) off / on           */
#define MCE_WL_OFF 1
#define MCE_WL_ON 2
/* root scheduling */
#define MCE_SCHED_PLAIN 0   /* roots in vertex-id order (the reference's order) */
#define MCE_SCHED_DEGREE 1  /* roots sorted by a degree-based cost estimate     */
#define MCE_SCHED_LEARNED 2 /* roots sorted by the cost MLP's prediction        */

typedef struct mce_opts {
  int32_t level;            /* MCE_LEVEL_*                                    */
  int32_t induced;          /* MCE_INDUCED_*                                  */
  int32_t worker_list;      /* MCE_WL_*                                       */
  int32_t sched;            /* MCE_SCHED_*                                    */
  int32_t bitmap_width;     /* 0 = auto; 32 or 64: word width of the rows of
                               roots with at most 32 later neighbours          */
  int32_t warps_per_root;   /* 0 = auto (1); k = 1..32: each root is searched
                               by k warps, warp j taking the root's
                               first-level branches j, j+k, j+2k, ... (the
                               same tree, split by its first level; the
                               counterpart of the reference's PSIZE lanes per
                               candidate, src/main.cu:158-165).  Buckets
                               without their own value use this one; runs
                               with warp_log and mce_list use one warp       */
  int32_t donate_threshold; /* 0 = default (10, the reference's SZTH,
                               mce/parameter.cuh:5): smallest candidate set a
                               subtree must have to be donated                 */
  int32_t log_roots;        /* 1 = record per-root search-tree node counts    */
  int32_t x_pivot;          /* 1 = also take pivots from the root's earlier
                               neighbours adjacent to the chosen set, and prune
                               a subtree when one of them covers P (the -i px
                               rule; also set by induced = MCE_INDUCED_PX).
                               All engines; the count is unchanged, the
                               search trees are not                          */
  int32_t peel_solo_max;    /* 0 = default (off); < 0 = off; > 0: frontiers of at most
                               this many vertices are peeled by one block           */
  int32_t donate_after;     /* 0 = default (256): a warp shares subtrees of a
                               root only after walking this many of its nodes */
  int32_t cuda_graph;       /* 1 = capture the search launches in a CUDA graph
                               once and replay it (default for batches)      */
  int32_t heavy_log2;       /* 0 = default (12): with a cost schedule, roots
                               whose predicted tree has at least 2^heavy_log2
                               nodes run first, largest first                */
  int32_t share_log2;       /* 0 = default (16): with MCE_SCHED_LEARNED, roots
                               predicted at least 2^share_log2 nodes share
                               subtrees from their first node on             */
  int32_t warp_log;         /* 1 = record per search warp its SM, tree nodes
                               and donations; 2 = also its clock cycles per
                               phase (read both with mce_warp_log)           */
  int32_t wide_blocks;      /* 0 = default (4): blocks per SM of the wide
                               engine (d+ > 64); 8 = its 64-register variant */
  int32_t wait_limit_ms;    /* 0 = default (30 s): a search warp waiting for
                               subtrees gives up after this long without
                               progress anywhere and the call returns
                               MCE_ETIMEOUT (the device stays usable)       */
  int32_t count_ops;        /* 1 = run the counting variants of the engines:
                               mce_stats_t.word_ops gets the algorithmic
                               32-bit word operations of the IP walk (per
                               root too with log_roots, mce_root_ops); not
                               with x_pivot, warp_log or mce_list (MCE_EINVAL).
                               Same counts and trees; slower (a measurement
                               run, not a timed one)                        */
  /* Per bucket of roots - the engine classes, by bitmap width: [0] roots
   * with d+ <= 32 (one 32- or 64-bit row per lane), [1] 33..64 (two 64-bit
   * rows per lane), [2] wider (rows in a slab) - the settings above for that
   * bucket alone; 0 = the value above.  The autotuner fills them.         */
  int32_t bucket_warps_per_root[3];
  int32_t bucket_donate_threshold[3];
  int32_t bucket_donate_after[3];
  int32_t stage_lists;      /* 1 = the 32-bit engine (d+ <= 32, one warp per
                               root, IP) copies each group of later lists it
                               encodes into shared memory with 1-D bulk
                               copies (16-byte windows, one mbarrier per
                               warp) and reads them there; groups that do not
                               fit 2 KB are read from global memory         */
  void *stream;             /* cudaStream_t to queue work on; NULL = own      */
  void *model;              /* mce_model_t for MCE_SCHED_LEARNED (NULL: the
                               degree heuristic is used instead)              */
} mce_opts_t;

/* Fill *o with the defaults: L1, P, worker list on, plain schedule, auto.   */
void mce_opts_default(mce_opts_t *o);

/* Per-call statistics; device times are CUDA-event times on the call's stream. */
typedef struct mce_stats {
  double peel_ms;           /* k-core peeling (degeneracy order)              */
  double orient_ms;         /* orientation / split CSR + root classification  */
  double count_ms;          /* Bron-Kerbosch search                           */
  double total_ms;          /* first kernel to last copy back                 */
  int32_t degeneracy;       /* max core number                                */
  int32_t max_later_degree; /* largest later-neighbour count of any root      */
  int64_t max_degree;
  int64_t roots;            /* vertices with at least one later neighbour     */
  uint64_t tree_nodes;      /* search-tree nodes visited (branches taken)     */
  uint64_t donations;       /* subtrees handed to another warp                */
  int32_t kernel_launches;  /* this library's kernels launched by the call    */
  uint32_t error_flags;     /* device-side status bits (0 = clean)            */
  int64_t class_roots[8];   /* roots per engine class                         */
  int64_t peel_rounds;      /* synchronous peel rounds                        */
  int64_t peel_solo_sections; /* runs of rounds peeled by a single block      */
  double peel_scan_ms;      /* peel time split as seen by one block: level    */
  double peel_round_ms;     /* scans, round work, and waits at grid barriers  */
  double peel_wait_ms;
  uint64_t word_ops;        /* opts.count_ops: algorithmic 32-bit word ops of
                               the search, W = ceil(d+/32) words per row:
                               2W per candidate of every pivot selection
                               (AND + POPC, mce/mce_utils.cuh:338-402) + 4W per
                               tree node for the child sets (:321-336)       */
  double class_ms[4];       /* search launch time per engine class: 32-bit
                               rows (d+ <= 32), 64-bit rows (33..64), wide   */
} mce_stats_t;

/* ---- host graphs -------------------------------------------------------- */
/* A CSR graph in host memory whose arrays belong to the library.  For a
 * batch of graphs, the arrays hold every graph's CSR back to back:
 *   graph g's rows are row_ptr[vtx_offsets[g] .. vtx_offsets[g+1]) (n_g + 1
 *   entries, local offsets starting at 0) and its arcs are
 *   col[arc_offsets[g] .. arc_offsets[g+1]) (local vertex ids).
 * For a single graph num_graphs = 1, vtx_offsets = {0, n+1},
 * arc_offsets = {0, m}.                                                      */
typedef struct mce_hgraph {
  int64_t n;             /* total vertices (sum over graphs)                */
  int64_t m;             /* total directed arcs (2 x undirected edges)      */
  int32_t *row_ptr;      /* n + num_graphs entries                          */
  int32_t *col;          /* m entries                                       */
  int32_t num_graphs;
  int64_t *vtx_offsets;  /* num_graphs + 1 entries, into row_ptr            */
  int64_t *arc_offsets;  /* num_graphs + 1 entries, into col                */
} mce_hgraph_t;

/* Release the arrays of *g and zero it. */
void mce_hgraph_free(mce_hgraph_t *g);

/* Build a normalised CSR from an undirected edge list: both directions are
 * added, self-loops dropped, duplicates removed, rows sorted - the same
 * normalisation as graph::convert_to_bel (include/fileop.h:28-41).
 * n = max(n_hint, max id + 1).                                               */
int mce_hgraph_from_edges(const int64_t *src, const int64_t *dst, int64_t count,
                          int64_t n_hint, mce_hgraph_t *out);

/* Check that a CSR is a valid simple undirected graph: offsets monotone,
 * ids in range, rows strictly increasing, no self-loops, symmetric.         */
int mce_csr_validate(const int32_t *row_ptr, const int32_t *col, int64_t n, int64_t m);

/* ---- .bel files ---------------------------------------------------------- */
/* Read a .bel file (24-byte records: u64 dst, u64 src, u64 0; sorted by
 * (src, dst)).  Replaces graph::read_bel (include/fileop.h:81-129) followed by
 * CSRCOO::from_edgelist (include/csrcoo.cuh:41-81): n = max src + 1, empty
 * rows are filled, ids are narrowed to 32 bits.  Returns MCE_EFORMAT if the
 * records are not sorted by source (the reference asserts this,
 * include/csrcoo.cuh:57-61) or the file size is not a multiple of 24.       */
int mce_bel_read(const char *path, mce_hgraph_t *out);

/* Write a host CSR as a .bel file (the record layout written by
 * graph::convert_to_bel, include/fileop.h:62-71).                          */
int mce_bel_write(const char *path, const mce_hgraph_t *g);

/* Text edge list -> .bel.  Replaces graph::convert_to_bel
 * (include/fileop.h:13-79): lines not starting with a digit are skipped,
 * "u v" lines with u != v add both directions, then sort + unique.  On
 * success *n_out = max id + 1 and *undirected_edges_out = m / 2 (the two
 * numbers the reference prints).                                           */
int mce_convert_to_bel(const char *txt_path, const char *bel_path, int64_t *n_out,
                       int64_t *undirected_edges_out);

/* The same conversion on device `device`: the text is parsed, and the arcs
 * sorted and deduplicated, on the GPU; the output file and the two numbers
 * are those of mce_convert_to_bel, byte for byte (lines are read up to
 * 65,535 bytes by both).  Replaces graph::convert_to_bel
 * (include/fileop.h:13-79).  `stream` may be NULL (a stream of the call's
 * own).                                                                    */
int mce_convert_to_bel_device(const char *txt_path, const char *bel_path, int32_t device,
                              void *stream, int64_t *n_out, int64_t *undirected_edges_out);

/* ---- device graphs -------------------------------------------------------- */
typedef struct mce_graph *mce_graph_t;

/* Copy a CSR (host pointers, pageable or pinned) to device `device` and
 * create a handle.  Replaces the managed-memory upload in main
 * (src/main.cu:53-93).  `stream` may be NULL (the handle's own stream).     */
int mce_graph_upload(const int32_t *row_ptr, const int32_t *col, int64_t n, int64_t m,
                     int32_t device, void *stream, mce_graph_t *out);

/* Replace the CSR of an existing handle with a new one of the same or
 * smaller size, reusing its device buffers (no allocation when it fits).    */
int mce_graph_reload(mce_graph_t g, const int32_t *row_ptr, const int32_t *col, int64_t n,
                     int64_t m, void *stream);

/* Vertex and arc count of a handle. */
int mce_graph_size(mce_graph_t g, int64_t *n, int64_t *m);

/* Free a handle and every device buffer it owns. */
int mce_graph_free(mce_graph_t g);

/* Read a .bel file straight into a device handle: the records stream
 * through pinned staging buffers to the device, where they are decoded and
 * checked and the row offsets are built (the host reader's checks, same
 * MCE_EFORMAT cases).  Replaces read_bel + from_edgelist + the upload
 * (include/fileop.h:81-129, include/csrcoo.cuh:41-81, src/main.cu:53-93)
 * for callers that do not need the graph on the host.                      */
int mce_bel_load(const char *path, int32_t device, void *stream, mce_graph_t *out);

/* Read a text edge list straight into a device handle, without a .bel file:
 * the graph mce_bel_load builds from mce_convert_to_bel's output
 * (include/fileop.h:13-79 followed by :81-129 and include/csrcoo.cuh:41-81).
 * MCE_ELIMIT when a narrowed id is above the int32 CSR's range, MCE_EFORMAT
 * when two ids narrow to the same vertex (a self-loop the .bel reader
 * rejects).                                                                */
int mce_text_load(const char *txt_path, int32_t device, void *stream, mce_graph_t *out);

/* Degeneracy order of the uploaded graph.  Replaces
 * graph::SingleGPU_Kcore::findKcoreIncremental_async (include/kcore.cuh:233-316).
 * priority_out[v] (nullable, n entries) is the synchronous peel round in
 * which v was removed, with the reference's numbering: rounds are numbered
 * from 0 over all levels, and the vertices of the final round keep the value
 * m (include/kcore.cuh:258,276).  core_out[v] (nullable) is v's core number;
 * *degeneracy (nullable) the max core number (include/kcore.cuh:313-315).   */
int mce_degeneracy(mce_graph_t g, uint32_t *priority_out, int32_t *core_out,
                   int32_t *degeneracy);

/* Oriented ("split") CSR after mce_degeneracy/mce_count: split_out[v]
 * (n entries) is where v's later neighbours begin, col_out (m entries) holds
 * each row as [earlier neighbours | later neighbours], both parts sorted by
 * id.  Replaces set_priority/split_pointer/split_data
 * (include/main_support.cuh:6-84, driven from src/main.cu:102-146).        */
int mce_split_csr(mce_graph_t g, int32_t *split_out, int32_t *col_out);

/* Count the maximal cliques (size >= 2).  Runs peeling, orientation and the
 * search on the device; replaces MultiGPU_MCE::mce_count + show
 * (mce/mce.cuh:107-422).  hist (nullable, MCE_HIST_MAX entries) receives the
 * clique-size histogram; stats (nullable) the timings and counters.         */
int mce_count(mce_graph_t g, const mce_opts_t *opts, uint64_t *total, uint64_t *hist,
              mce_stats_t *stats);

/* List the maximal cliques (size >= 2): clique k is
 * ids_out[offsets_out[k] .. offsets_out[k+1]), the root first, k <
 * *count_out, in no particular order (the search's leaves are reached in
 * parallel).  offsets_out holds cliques_cap + 1 entries.  If the listing
 * does not fit (more than ids_cap ids or cliques_cap cliques), nothing is
 * written, *count_out and *ids_needed (nullable) get the sizes it needs and
 * MCE_ELIMIT is returned.  No counterpart in the reference, which only
 * counts (mce/mce_utils.cuh:522-523).                                      */
int mce_list(mce_graph_t g, const mce_opts_t *opts, int32_t *ids_out, int64_t ids_cap,
             int64_t *offsets_out, int64_t cliques_cap, uint64_t *count_out, int64_t *ids_needed);

/* Per-root search-tree node counts of the last mce_count that ran with
 * opts.log_roots = 1 (n entries, 0 for non-roots).                          */
int mce_root_log(mce_graph_t g, uint64_t *nodes_out);

/* Per-root maximal-clique counts of the last mce_count that ran with
 * opts.log_roots = 1 (n entries, 0 for non-roots).                          */
int mce_root_counts(mce_graph_t g, uint64_t *count_out);

/* Per-root algorithmic word operations (mce_stats_t.word_ops, split by
 * root) of the last mce_count that ran with opts.log_roots = 1 and
 * opts.count_ops = 1 (n entries); MCE_ESTATE otherwise.  No counterpart in
 * the reference; it measures the work of the reference's walk
 * (mce/mce_utils.cuh:321-402) root by root.                                */
int mce_root_ops(mce_graph_t g, uint64_t *ops_out);

/* Per-warp load of the last mce_count that ran with opts.warp_log >= 1: for
 * every search warp (all engine classes, widest class first) the SM it ran
 * on, the search-tree nodes it walked (its roots and the subtrees it took)
 * and the subtrees it handed to other warps; with warp_log = 2 also its
 * clock cycles in the seven phases of the reference's breakdown, in its
 * order (other, building induced subgraphs, worker list, selecting pivots,
 * set operations, testing maximality, branching and backtracking; 7 per
 * warp in cycles_out).  The counterpart of the reference's -m mce-lb-eval /
 * mce-donor-eval / mce-bd-eval per-block lines (mce/mce_kernel_wl_lb.cuh:157,
 * mce/mce_kernel_wl_donor.cuh:157, mce/mce_kernel_wl_bd.cuh:270), with a
 * warp as the unit of work.  Arrays (nullable) take up to `cap` warps;
 * *count_out gets the number of warps.                                      */
int mce_warp_log(mce_graph_t g, uint32_t *sm_out, uint64_t *nodes_out, uint64_t *donations_out,
                 uint64_t *cycles_out, int64_t cap, int64_t *count_out);

/* ---- batches of graphs ------------------------------------------------------ */
typedef struct mce_batch *mce_batch_t;

/* Upload many graphs at once (host pointers).  Graph g's CSR is
 * row_ptr[vtx_offsets[g] .. vtx_offsets[g+1]) (n_g + 1 local offsets) and
 * col[arc_offsets[g] .. arc_offsets[g+1]) (local ids) - the layout of a
 * batch mce_hgraph_t.  On the device the graphs become one disjoint union
 * with a vertex -> graph map, so one peel, one orientation and one search
 * launch per engine class serve the whole batch.  No counterpart in the
 * reference, which counts one graph per run (src/main.cu:18-187).          */
int mce_batch_upload(const int32_t *row_ptr, const int32_t *col, const int64_t *vtx_offsets,
                     const int64_t *arc_offsets, int32_t num_graphs, int32_t device,
                     void *stream, mce_batch_t *out);

/* Replace the graphs of a batch handle, reusing its device memory when the
 * new batch fits.                                                           */
int mce_batch_reload(mce_batch_t b, const int32_t *row_ptr, const int32_t *col,
                     const int64_t *vtx_offsets, const int64_t *arc_offsets, int32_t num_graphs,
                     void *stream);

/* Count every graph of the batch: per_graph_total (num_graphs entries) gets
 * each graph's maximal cliques, *total their sum, hist (nullable) the size
 * histogram over the batch.  opts NULL = defaults with cuda_graph = 1: the
 * search launches are captured once and replayed on later calls.           */
int mce_batch_count(mce_batch_t b, const mce_opts_t *opts, uint64_t *per_graph_total,
                    uint64_t *total, uint64_t *hist, mce_stats_t *stats);

/* mce_batch_reload followed by mce_batch_count in one call, for a batch in
 * host memory: batches of 2^20 arcs or more are copied in up to six parts
 * of whole graphs on a stream of the handle's own, and each part is rebased,
 * peeled, oriented and - for counts in plain or degree order without
 * per-root or per-warp logs - its roots with at most 32 later and 256
 * earlier neighbours are searched while the next parts are still being
 * copied (parts of 2, 4, 7, 11, 16 and 24 64ths of the arcs): the host
 * enqueues a part's rebase and peel once its copy has landed, its
 * orientation once the search of the part before it has ended, and its
 * search once it is oriented; the other roots of every part (hub roots,
 * wider bitmaps) follow in one search.  In the other modes one search over
 * the whole batch follows.
 * Same results as the two calls.  Pinned host memory lets the copies
 * overlap.  In the part-by-part mode stats->peel_ms is the time until the
 * first part is ready, orient_ms 0 and count_ms the rest.  With the
 * environment variable MCE_TRACE_PARTS=1 the part-by-part mode prints the
 * call's timeline (copies, peels, orientations, searches; ms from the
 * call's start) to stderr, for diagnostics.                               */
int mce_batch_count_host(mce_batch_t b, const int32_t *row_ptr, const int32_t *col,
                         const int64_t *vtx_offsets, const int64_t *arc_offsets,
                         int32_t num_graphs, const mce_opts_t *opts, uint64_t *per_graph_total,
                         uint64_t *total, uint64_t *hist, mce_stats_t *stats);

int mce_batch_free(mce_batch_t b);


/* ---- learned scheduling ------------------------------------------------------ */
/* A cost model predicts each root's search-tree size (log2(1 + nodes)) from
 * eight features (later / earlier / total degree, core number, density and
 * largest degree of the subgraph induced by the later neighbours, first-level
 * branches left by that degree, later-list mass).  Network 8 -> 64 -> 64 -> 1
 * with ReLU, FP16 weights and FP32 accumulation; trained on the device by
 * this library's own forward/backward/Adam kernels on the tree sizes that
 * mce_count logs (opts.log_roots = 1).  With opts.sched = MCE_SCHED_LEARNED
 * and opts.model set, roots run longest-predicted first and only roots
 * predicted large share subtrees.  The count never depends on the model.
 * No counterpart in the reference, whose only static choice is per graph
 * (table.py:127).                                                           */
#define MCE_MLP_INPUTS 8
#define MCE_MLP_HIDDEN 64
#define MCE_MLP_PARAMS 4801  /* W1 64x8, b1 64, W2 64x64, b2 64, W3 64, b3 1 */
typedef struct mce_model *mce_model_t;

/* A model with seeded He-uniform weights and zero biases. */
int mce_model_create(int32_t device, uint64_t seed, mce_model_t *out);
int mce_model_free(mce_model_t m);
/* Set the FP32 master weights (MCE_MLP_PARAMS, layout above); the FP16
 * copy used by the kernels is their round-to-nearest.                      */
int mce_model_set(mce_model_t m, const float *params);
/* Read the FP32 master weights and/or the FP16 copy (either nullable).     */
int mce_model_get(mce_model_t m, float *params_out, uint16_t *fp16_out);
/* Features of every vertex (n x MCE_MLP_INPUTS, zeros for non-roots). */
int mce_root_features(mce_graph_t g, float *features_out);
/* Train on the roots of g with at least 16 later neighbours (the roots the
 * model ranks; smaller trees are not worth scheduling) against the tree
 * sizes of the last mce_count that ran with log_roots = 1 (MCE_ESTATE
 * otherwise): `epochs` passes of Adam
 * over seeded shuffles in minibatches of `batch`; loss_out (nullable,
 * `epochs` entries) gets each epoch's mean squared error.                  */
int mce_model_train(mce_model_t m, mce_graph_t g, int32_t epochs, int32_t batch, float lr,
                    uint64_t seed, float *loss_out);
/* Predicted log2(1 + tree nodes) of every vertex of g (n entries). */
int mce_model_predict(mce_model_t m, mce_graph_t g, float *pred_out);
/* Forward pass on host features (count x MCE_MLP_INPUTS). */
int mce_model_eval(mce_model_t m, const float *X, int64_t count, float *out);
/* Gradient of the mean squared error over (X, Y) (host arrays) with respect
 * to the parameters, as the training kernel computes it (FP16 weights, FP32
 * accumulation); the model is not updated.                                  */
int mce_model_grad(mce_model_t m, const float *X, const float *Y, int64_t count,
                   float *grad_out, float *loss_out);

/* ---- allocation-free search ------------------------------------------------ */
/* Bytes of the file-scope device array that mce_count_oriented_noalloc uses
 * as scratch.  Every GPU that loads libmce.so holds this array until the
 * process exits.                                                             */
#define MCE_NOALLOC_SCRATCH_BYTES (32u << 20)

/* Search an oriented graph that is already in device memory without
 * allocating anything.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc - a process whose device memory is
 * owned by another allocator (for example a framework's caching allocator
 * that reserved the GPU), or a latency-critical loop where cudaMalloc's
 * implicit device synchronisation is not acceptable.
 *
 * Inputs (device pointers, caller-owned): d_row_ptr (n+1), d_split (n) and
 * d_col_split (m) - the oriented CSR that mce_split_csr returns - with its
 * vertex count n, and d_roots (num_roots vertex ids).  Output: d_hist
 * (MCE_HIST_MAX uint64, device) receives the number of maximal cliques of
 * each size found from those roots (zeroed by the call once the roots have
 * passed its checks; left untouched when it returns an error).  A root id
 * outside [0, n) is caught before anything is read at it: nothing is
 * searched and MCE_EINVAL is returned.  Every root must have 1 to 32 later
 * and at most 1024 earlier neighbours; otherwise nothing is searched and
 * MCE_ELIMIT is returned.  Work is queued on `stream` (NULL = legacy default
 * stream) and the call synchronises that stream twice before it returns.
 * The call uses the
 * MCE_NOALLOC_SCRATCH_BYTES array (its address on the current device is
 * looked up on every call); calls that overlap on the GPU race on the
 * array, so serialise them.                                                  */
int mce_count_oriented_noalloc(const int32_t *d_row_ptr, const int32_t *d_split,
                               const int32_t *d_col_split, int64_t n, const int32_t *d_roots,
                               int64_t num_roots, uint64_t *d_hist, void *stream);

/* ---- autotuner ------------------------------------------------------------ */
/* Per graph-shape class, the search settings (donation gate and threshold,
 * bitmap word width of narrow roots, single-block peeling of small
 * frontiers, blocks per SM of the wide engine, X-in-subgraph pivots) that
 * ran fastest in timed trials, kept in a text table with one
 * line per class.  A class is floor(log2) of the vertex count, mean degree
 * and degeneracy (and of the graph count for a batch), e.g. "n23-a4-k5" or
 * "b12-n23-a4-k7".  No counterpart in the reference (its per-graph variant
 * choice is a rule of thumb in table.py:127).                               */
typedef struct mce_tune_result {
  char key[48];       /* shape class                                        */
  mce_opts_t best;    /* the base options with the tuned fields set         */
  double best_ms;     /* device time of one count with `best`               */
  double default_ms;  /* ... with the base options                          */
  int32_t trials_run; /* counts timed by this call (0 when from the table)  */
  int32_t from_table; /* 1: the class was in the table, nothing was timed   */
} mce_tune_result_t;

/* Shape class of a graph / a batch (runs the peel for the degeneracy).     */
int mce_shape_key(mce_graph_t g, char *key_out, size_t len);
int mce_batch_shape_key(mce_batch_t b, char *key_out, size_t len);
/* Set the tuned fields of *inout from the table's line for `key`;
 * MCE_EIO: no table, MCE_ESTATE: no line for the class.                    */
int mce_tune_lookup(const char *table_path, const char *key, mce_opts_t *inout);
/* Tune the graph's class unless the table (nullable) has it already (force
 * = 1: tune anyway); each setting is timed `reps` times (best kept) and
 * must return the same count (else MCE_ESTATE).  The table is rewritten
 * with the class's new line.                                               */
int mce_autotune(mce_graph_t g, const mce_opts_t *base, const char *table_path, int32_t reps,
                 int32_t force, mce_tune_result_t *out);
int mce_batch_autotune(mce_batch_t b, const mce_opts_t *base, const char *table_path,
                       int32_t reps, int32_t force, mce_tune_result_t *out);

/* ---- serving ------------------------------------------------------------ */
/* A serving session answers requests against a resident graph from one
 * persistent kernel (no counterpart in the reference, which runs one graph
 * per process).  A request is a seed vertex; its answer is the number of
 * maximal cliques of the seed's 2-hop ego subgraph, the graph that
 * mce_ego_subgraph (mce_gen.h) builds with the same cap.  Each resident
 * block (a slot) takes one request at a time; requests are admitted as
 * slots free up, so a request never waits for a batch to fill.  The graph
 * handle must outlive the session and must not be reloaded meanwhile.
 * A request whose ego graph has at least 1,024 vertices opens its root
 * search to slots that have nothing to do, so a large request does not
 * run on one block alone while the GPU idles.
 * Admission by footprint: with small_cap > 0 the slots come in two
 * classes.  The first big_slots blocks are whole-block slots (1,024
 * threads) for any request; every other block holds four 256-thread slots
 * for requests whose bound deg(seed) + sum of its neighbours' degrees + 1
 * is at most small_cap (computed for every vertex at open), so many small
 * requests run side by side instead of one per block.  Such a request goes
 * to the small slots only while every whole-block slot holds a request
 * (submitted and not yet polled): below that load a whole block answers it
 * sooner.  Request ids carry the class in bit 0.
 * While requests keep coming the kernel stays resident on every SM; a
 * cudaDeviceSynchronize by the caller returns only after the slots have
 * been idle for idle_ms (or after mce_serve_close).                       */
typedef struct mce_serve *mce_serve_t;

typedef struct mce_serve_opts {
  int32_t ego_cap;  /* ego-graph vertex cap, 2..16384 (default 1024)         */
  int32_t slots;    /* resident blocks; <= 0: as many as fit                 */
  uint32_t ring;    /* requests submitted and not yet polled (default 4096)  */
  int32_t idle_ms;  /* a slot idle this long leaves; the next submit or poll
                       relaunches the kernel (default 1000)                  */
  int64_t max_arcs; /* arcs per ego graph; 0: 128 * ego_cap (capped at
                       ego_cap * (ego_cap - 1)).  More: status MCE_ELIMIT    */
  int64_t max_nodes; /* search-tree nodes per request; 0: no limit.  More:
                        status MCE_ELIMIT (the request's search stops)       */
  int32_t small_cap; /* footprint bound of the 256-thread slots' requests:
                        0 one class only; < 0 automatic (1,024 when ego_cap
                        is above 2,048, else 0); else 2..ego_cap            */
  int32_t big_slots; /* whole-block slots when small_cap is on; <= 0: half
                        the blocks (at least one block stays split)         */
  int64_t reserved[2];
} mce_serve_opts_t;

typedef struct mce_serve_result {
  uint64_t count;     /* maximal cliques of the ego graph                   */
  int64_t seed;
  int32_t status;     /* MCE_OK, MCE_EINVAL (seed out of range) or
                         MCE_ELIMIT (see `limits`)                          */
  int32_t ego_n;      /* ego-graph vertices                                 */
  int32_t ego_arcs;   /* ego-graph arcs (2 x edges)                         */
  uint32_t limits;    /* MCE_SERVE_* bits of the limits a request hit       */
  uint64_t device_ns; /* time the slot spent on the request                 */
  uint32_t extract_ns; /* ... building the ego graph                        */
  uint32_t order_ns;   /* ... peeling and orienting it                      */
  uint32_t search_ns;  /* ... searching its roots                           */
  uint32_t pad2;
} mce_serve_result_t;

#define MCE_SERVE_OVER_BUDGET 0x20u /* search passed max_nodes             */
#define MCE_SERVE_OVER_ARCS 0x40u   /* ego graph above max_arcs             */
#define MCE_SERVE_TOO_WIDE 0x0Cu    /* a root with more than 256 later (0x8)
                                       or a slab's earlier rows (0x4)       */

typedef struct mce_serve_stats {
  int32_t slots, running;   /* slots of both classes                          */
  uint32_t ring, pad;
  uint64_t submitted, served, tree_nodes;
  int64_t kernel_launches;
  uint64_t arena_bytes, slab_bytes;
  uint64_t helps;     /* times an idle slot joined another slot's search    */
  int32_t small_slots; /* of `slots`: the 256-thread ones                   */
  int32_t small_cap;   /* their footprint bound (0: one class)              */
  uint64_t peak_in_flight; /* most requests held by slots at once           */
} mce_serve_stats_t;

void mce_serve_opts_default(mce_serve_opts_t *o);
/* Start a session on graph g (uploaded with mce_graph_upload). */
int mce_serve_open(mce_graph_t g, const mce_serve_opts_t *opts, mce_serve_t *out);
/* Publish one request; *id_out names it.  MCE_ELIMIT: `ring` requests are
 * outstanding - poll some first.                                          */
int mce_serve_submit(mce_serve_t s, int64_t seed, uint64_t *id_out);
/* MCE_OK and *res filled once the answer is there (each id is taken once),
 * MCE_EAGAIN while it is not.                                             */
int mce_serve_poll(mce_serve_t s, uint64_t id, mce_serve_result_t *res);
/* Poll until done or timeout_ms (< 0: no limit) -> MCE_ETIMEOUT.          */
int mce_serve_wait(mce_serve_t s, uint64_t id, int64_t timeout_ms, mce_serve_result_t *res);
/* Open-loop trace: request i (seeds[i]) is submitted arrival_us[i]
 * microseconds after the call (NULL: all at once, as the ring admits);
 * results[i] and latency_us[i] (completion seen minus arrival; may be NULL)
 * are filled.                                                             */
int mce_serve_run(mce_serve_t s, const int64_t *seeds, const double *arrival_us, int64_t count,
                  int64_t timeout_ms, mce_serve_result_t *results, double *latency_us);
int mce_serve_stats(mce_serve_t s, mce_serve_stats_t *st);
/* Finish the published requests, stop the kernel and free the session.    */
int mce_serve_close(mce_serve_t s);

/* Text for a status code. */
const char *mce_strerror(int code);

/* Library version string. */
const char *mce_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MCE_H */
