// Launch wrappers shared by the .cu files of libmce.so (internal).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "queue.cuh"

namespace mce {

// ---- peeling ---------------------------------------------------------------
struct PeelArgs {
  int64_t n, m;
  const int32_t *rp, *col;
  int32_t *deg, *core;
  uint32_t *prio;
  int32_t *alistA, *alistB, *front0, *front1, *front2;
  int32_t *hb0, *hb1, *hb2;  // heavy chunk bases per frontier slot (n + 1 each)
  void *ctl;  // peel_ctl_bytes() of device memory
  uint64_t wait_limit_ns;
  uint32_t solo_max;  // frontiers up to this size are peeled by block 0 alone (0: never)
};
size_t peel_ctl_bytes();
int peel_launch(const PeelArgs &a, cudaStream_t s, int *launches);
// Batches: each graph of the disjoint union peeled by one block (order:
// graph ids, largest first).
// part >= 0 (0..3): one part of a batch still arriving, peeled concurrently
// with the others; the control block was zeroed before the first part and
// each part takes graphs from its own counter.  part < 0: the whole batch.
// max_n: the most vertices of a graph of the launch (0: unknown); graphs up
// to 16,384 vertices are peeled with their state in shared memory.
// `order` holds the large graphs (more than PEEL_MID_N vertices) first, g_big
// of them, peeled by 512-thread blocks; then g_mid middle ones (at most
// PEEL_MID_N) by 256-thread blocks and the small rest (at most PEEL_SMALL_N)
// by 128-thread blocks, those two launches on the side streams (forked from
// s by `fork`, joined back by `join`; all null: on s after the others), so
// that the smaller graphs' blocks, which need less shared memory, run many
// at a time beside the large ones.
constexpr int64_t PEEL_SMALL_N = 2048;
constexpr int64_t PEEL_MID_N = 8192;
// A host batch is copied, prepared and searched in at most this many parts.
constexpr int MAX_BATCH_PARTS = 6;
struct PeelSide {
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
};
int peel_segments_launch(const PeelArgs &a, const int64_t *vtx_off, const int64_t *arc_off,
                         const int32_t *order, int32_t G, int32_t g_big, int32_t g_mid,
                         cudaStream_t s, const PeelSide &ps, int *launches, int part = -1,
                         int64_t max_n = 0);
int peel_read(const void *ctl_dev, int32_t *degeneracy, uint32_t *err, uint32_t *rounds,
              uint32_t *solo_sections, cudaStream_t s, double *phase_ms = nullptr);

// ---- orientation + root classes ------------------------------------------------
// Engine classes of a root (by later degree d+ and earlier degree d-).
enum RootClass : uint32_t {
  CLS_R32 = 0,   // 1 <= d+ <= 32, d- <= REG_XCAP_MAX: warp engine, rows in registers
  CLS_R64 = 1,   // 33 <= d+ <= 64, d- <= REG_XCAP_MAX: warp engine, two rows per lane
  CLS_MEM = 2,   // any other root with d+ <= 2048: warp engine, rows in a slab
  CLS_NONE = 3,  // d+ == 0: not a root
  CLS_BIG = 4,   // d+ > 2048: rejected (the reference's MAX_DEGEN)
  NCLS = 5
};
// Earlier-neighbour rows a register-engine warp keeps: REG_XCAP in the
// serving slots and the allocation-free entry point; in mce_count and
// mce_batch_count the slab is sized per graph (BKArgs::rxcap, a power of two
// from REG_XCAP up to REG_XCAP_MAX covering the largest d- of those roots),
// so hubs with few later neighbours stay in the register engines.
constexpr int REG_XCAP = 1024;
constexpr int REG_XCAP_MAX = 16384;
// Register-class roots with more earlier neighbours than this ("hubs") get
// their earlier-neighbour rows from a parallel pass before the search, one
// warp per 32 of them, instead of walking them serially in the root's warp.
constexpr int HUB_XMIN = 256;

// Per-call summary the device writes and the host reads once.
struct ShapeInfo {
  uint32_t cls_cnt[8];
  uint32_t cls_off[9];
  uint32_t max_dplus;      // over all roots
  uint32_t max_dminus_mem; // over roots of CLS_MEM
  uint32_t max_deg;
  uint32_t max_dminus_reg; // over roots of CLS_R32 and CLS_R64
  uint32_t hub_cnt;        // register-class roots with d- > HUB_XMIN
  uint32_t hub_r32;        // ... of them in CLS_R32
  unsigned long long hub_rows;  // their earlier degrees, each rounded up to 32
};

struct OrientArgs {
  int64_t n;
  const int32_t *rp, *col;
  const uint32_t *prio;
  int32_t *split, *cs;
  uint32_t *keys_in;    // sort keys (class / cost), n
  int32_t *vals_in;     // vertex ids, n
  ShapeInfo *shape;     // zeroed by the launcher
  const float *cost;    // nullable: per-vertex cost estimate (larger first)
  int sched;
  int32_t *hub_of;      // nullable, n: index of the vertex in hub_list, or -1
  int32_t *hub_list;    // n: the hub roots, in no particular order
  int64_t v0 = 0;       // vertices [v0, n) are oriented (a batch part: its range)
  bool keep_shape = false;  // add to the summary of earlier parts instead of zeroing it
  uint32_t *next = nullptr; // two counters (zeroed by the launcher): the launch's row groups
                            // and its long rows; launches that run at the same time need
                            // their own
  int32_t *long_list = nullptr;  // room for the vertices of [v0, n) whose rows are long
                                 // (any scratch of n - v0 ints, free until the roots' sort)
};
int orient_launch(const OrientArgs &a, cudaStream_t s, int *launches);

// Earlier-neighbour rows of the hub roots (orient's hub_list, cnt of them):
// off[j] = first row of hub j (rows padded to 32 per hub), rows[k] = the
// bitmap over the hub's later list of one earlier neighbour's later list.
// nx[j] = -1: hub j's distinct rows are not known yet (the search sets it).
// hub_of[list[i]] = i for the cnt hubs of `list` (one hub numbering for
// hub lists gathered from several parts of a batch).
int hub_index_launch(const int32_t *list, uint32_t cnt, int32_t *hub_of, cudaStream_t s,
                     int *launches);
int hub_rows_launch(const int32_t *rp, const int32_t *split, const int32_t *cs,
                    const int32_t *hub_list, uint32_t cnt, int64_t total_rows, int64_t *off,
                    int32_t *nx, unsigned long long *rows, int sms, cudaStream_t s,
                    int *launches);

// Sort roots by key (stable) and compute class offsets.  temp grows on demand.
int roots_sort(int64_t n, const uint32_t *keys_in, uint32_t *keys_out, const int32_t *vals_in,
               int32_t *vals_out, int end_bit, void **temp, size_t *temp_bytes,
               ShapeInfo *shape, cudaStream_t s, int *launches);

// ---- search ------------------------------------------------------------------
struct BKArgs {
  const int32_t *rp, *split, *cs;
  const int32_t *roots;          // class-sorted roots
  const ShapeInfo *shape;        // cls_off on the device
  uint32_t *fetch;               // [NCLS] root fetch counters, zeroed per call
  unsigned long long *hist;      // [MCE_HIST_MAX]
  unsigned long long *nodes;     // total tree nodes
  unsigned long long *root_nodes;  // nullable [n]: search-tree nodes per root
  unsigned long long *root_count;  // nullable [n]: maximal cliques per root
  const int32_t *graph_of;       // nullable [n]: graph of each vertex (batch)
  unsigned long long *graph_count; // nullable [num_graphs]
  uint32_t *err;
  unsigned long long *slab;      // per-warp scratch
  size_t slab_words;             // u64 words per warp
  int32_t dcap, xcap;            // slab capacities (later degree, x rows)
  int32_t rxcap;                 // register engines' x rows (0: REG_XCAP)
  const int32_t *hub_of;         // nullable, n: hub index of a root (-1: none) ...
  const int64_t *hub_off;        // ... its first precomputed earlier-neighbour row ...
  unsigned long long *hub_rows;  // ... in these rows (hub_rows_launch) ...
  int32_t *hub_nx;               // ... of which the first hub_nx are distinct once >= 0
  QueueView q;                   // task queue (q.hdr == nullptr: no sharing)
  int32_t donate_min;            // hand off children with at least this many candidates
  uint32_t donate_after;         // ... once this many nodes of the root/task were walked
  uint64_t wait_limit_ns;        // an idle warp gives up after this long without progress
  const uint8_t *policy;         // nullable [n]: 1 = root may share subtrees at once
  unsigned long long node_budget;  // 0: none; else a tree stops past this many nodes
  unsigned long long *warp_log;  // nullable: per warp of the launch {SM id, tree nodes, donations,
                                 // cycles per phase[7]}
  int32_t warp_cycles;           // 1: also the per-phase cycle breakdown
  int32_t wide8;                 // 1: the wide engine's 8-blocks-per-SM variant
  int32_t level2;                // 1 (-p l2): edge-rooted units, offered to idle warps at once
  const uint32_t *prio;          // peel priorities (the degeneracy order of the L2 units)
  int32_t x_pivot;               // 1 (-i px): register engines also pivot on earlier neighbours
  int32_t *list_buf;             // nullable: clique records {size, root, members...}
  unsigned long long *list_words;  // words taken in list_buf (also past list_cap)
  unsigned long long list_cap;   // words list_buf holds
  int32_t parts;                 // warps per root of the launched class (<= 1: one); each
                                 // takes every parts-th first-level branch of the root
  int32_t stage;                 // 1: the 32-bit engine stages its lists by bulk copies
                                 // (cs must have 16 readable bytes past its end)
  int32_t count_ops;             // 1: the counting variants sum the algorithmic word ops ...
  unsigned long long *ops;       // ... into *ops ...
  unsigned long long *root_ops;  // ... and per root (nullable [n])
};

// Launch the engine of one class.  warps_out: number of warps launched (slab sizing).
int bk_warps_for_class(int cls, int sms, int wide_blocks, int *warps, int *block, int *smem);
size_t bk_slab_words(int cls, int dcap, int xcap, int rxcap = REG_XCAP);
uint32_t bk_task_words(int cls, int dcap);
int queue_launch_init(const QueueView &q, cudaStream_t s, int *launches);

// ---- cost model -----------------------------------------------------------------
constexpr int MLP_IN = 8, MLP_HIDDEN = 64;
constexpr int MLP_MIN_LATER = 16;  // roots the model sees: at least this many later neighbours
// The learned schedule runs the model only on the roots whose trees decide
// the tails of the search (the 64-bit-row and wide roots); the others keep
// the degree heuristic.  With every root from MLP_MIN_LATER on, the feature
// pass cost 5.3 ms per call on the 4,096-graph batch.
constexpr int SCHED_MIN_LATER = 33;
constexpr int MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN +
                           MLP_HIDDEN + 1;
// Features of the roots with at least min_later later neighbours (0:
// MLP_MIN_LATER), listed in cand / *cand_count.
int features_launch(int64_t n, const int32_t *rp, const int32_t *split, const int32_t *cs,
                    const int32_t *core, float *out, int32_t *cand, uint32_t *cand_count, int sms,
                    cudaStream_t s, int *launches, int min_later = 0);
int mlp_forward_launch(const void *wh, const float *X, const int32_t *idx, const uint32_t *idx_count,
                       int64_t count, float *out, int sms, cudaStream_t s, int *launches);
int mlp_grad_launch(const void *wh, const float *X, const float *Y, const int32_t *idx,
                    int64_t begin, int64_t end, float *grad, float *loss, cudaStream_t s);
int mlp_adam_launch(float *master, void *wh, float *grad, float *m1, float *m2, float lr,
                    int step, cudaStream_t s);
// Sort keys by cost: with `cost`, roots with at least cost_min later
// neighbours take it and the others the degree heuristic.
// hub_of (nullable, the same n vertices): hub roots sort before the other
// roots of their class (key bit 27; the cost keeps 27 bits).
int rekey_launch(int64_t n, uint32_t *keys, const float *cost, const int32_t *rp,
                 const int32_t *split, uint8_t *policy, float heavy_cost, float share_cost,
                 int sms, cudaStream_t s, int *launches, int cost_min = 0,
                 const int32_t *hub_of = nullptr);

// ---- batches ------------------------------------------------------------------
int batch_rebase_launch(const int32_t *rp_local, const int32_t *col_local,
                        const int64_t *vtx_off, const int64_t *arc_off, int32_t G, int64_t n,
                        int64_t m, int32_t *rp, int32_t *col, int32_t *graph_of, int sms,
                        cudaStream_t s, int *launches);
// The same for the graphs [g0, g1) of the batch only (uploaded rows
// [row0, row1) and arcs [arc0, arc1)); also writes rp[vend] = rp_end, the
// offset the part's last row ends at (the next part's first row).
int batch_rebase_part_launch(const int32_t *rp_local, const int32_t *col_local,
                             const int64_t *vtx_off, const int64_t *arc_off, int32_t G,
                             int64_t row0, int64_t row1, int64_t arc0, int64_t arc1, int64_t vend,
                             int32_t rp_end, int32_t *rp, int32_t *col, int32_t *graph_of, int sms,
                             cudaStream_t s, int *launches);
int bk_launch(int cls, int word_bits, const BKArgs &a, int grid, int block, int smem,
              cudaStream_t s, int *launches);

}  // namespace mce
