// C ABI of libmce.so: device graph handles and the counting pipeline.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

#include "../host/host.h"
#include "common.cuh"
#include "kernels.h"

namespace mce {

static thread_local char g_last_detail[512];

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  std::snprintf(g_last_detail, sizeof(g_last_detail), "%s: %s (%s:%d)", cudaGetErrorString(e),
                what, file, line);
}

template <typename T>
static int dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  MCE_CUDA(cudaMalloc((void **)p, sizeof(T) * count));
  return MCE_OK;
}

template <typename T>
static void dfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

}  // namespace mce

using namespace mce;

struct mce_graph {
  int device = 0;
  int sms = 0;
  cudaStream_t own = nullptr;
  int64_t n = 0, m = 0, cap_n = -1, cap_m = -1;
  // graph
  int32_t *rp = nullptr, *col = nullptr, *cs = nullptr, *split = nullptr;
  // peeling
  uint32_t *prio = nullptr;
  int32_t *core = nullptr, *deg = nullptr, *alA = nullptr, *alB = nullptr;
  int32_t *f0 = nullptr, *f1 = nullptr, *f2 = nullptr;
  int32_t *hb0 = nullptr, *hb1 = nullptr, *hb2 = nullptr;
  void *peel_ctl = nullptr;
  // roots
  uint32_t *keys_in = nullptr, *keys_out = nullptr;
  int32_t *vals_in = nullptr, *roots = nullptr;
  int32_t *hub_of = nullptr, *hub_list = nullptr;  // roots with many earlier neighbours
  int64_t *hub_off = nullptr;                      // ... their first precomputed row
  int32_t *hub_nx = nullptr;                       // ... and their number of distinct rows
  unsigned long long *hub_rows = nullptr;          // ... and the rows
  int64_t hub_off_cap = 0, hub_rows_cap = 0;
  ShapeInfo *shape = nullptr;
  void *sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  // search
  uint32_t *fetch = nullptr, *err = nullptr;
  uint32_t *orient_next = nullptr;  // orientation counters, two per launch: [0] whole graph,
                                    // [2 + 2p] part p
  unsigned long long *hist = nullptr, *nodes = nullptr;
  unsigned long long *root_nodes = nullptr, *root_count = nullptr;
  unsigned long long *root_ops = nullptr;  // per-root word operations (opts.count_ops)
  unsigned long long *wlog = nullptr;     // per-warp {SM, nodes, donations} (opts.warp_log)
  int64_t wlog_cap = 0, wlog_count = 0;
  float *feat = nullptr, *pred = nullptr;  // per-vertex features (n x 8) and predicted cost
  int32_t *cand = nullptr;                // the roots the model scores ...
  uint32_t *cand_n = nullptr;             // ... and their number (device)
  uint8_t *policy = nullptr;              // per-root sharing policy from the model
  unsigned long long *slab = nullptr;
  size_t slab_bytes = 0;
  void *qbuf[NCLS] = {nullptr};   // task queue per engine class
  size_t qbytes[NCLS] = {0};
  bool logged = false;
  bool logged_ops = false;
  // host copies of the last call
  ShapeInfo shape_h{};
  int32_t degeneracy = 0;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t cls_ev[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  // a batch arriving in parts: one stream per part, forked from and joined
  // to the caller's stream
  cudaStream_t part_s[MAX_BATCH_PARTS] = {nullptr};
  cudaEvent_t part_fork = nullptr, part_done[MAX_BATCH_PARTS] = {nullptr};
  cudaEvent_t part_sdone = nullptr;  // the latest part search of a call has ended
  // opt-in timeline of a part-by-part batch call (environment MCE_TRACE_PARTS=1):
  // events on the streams it uses, printed to stderr in ms from the call's start
  static constexpr int TRACE_MAX = 64;
  cudaEvent_t trace_ev[TRACE_MAX] = {nullptr};
  char trace_name[TRACE_MAX][12];
  int trace_n = -1;  // < 0: off for this call
  // a batch's per-graph peel: the middle and small graphs' launches run on
  // side streams ([k][0] whole batch, [k][1 + p] part p)
  cudaStream_t seg_side[2][1 + MAX_BATCH_PARTS] = {{nullptr}};
  cudaEvent_t seg_fork[1 + MAX_BATCH_PARTS] = {nullptr};
  cudaEvent_t seg_join[2][1 + MAX_BATCH_PARTS] = {{nullptr}};
  // a batch searched part by part as it arrives (mce_batch_count_host):
  // per part its roots' summary and its search's (device and pinned host),
  // root fetch counters and sort scratch; the same for the deferred search
  ShapeInfo *part_shape = nullptr, *part_shape_h = nullptr;
  uint32_t *part_fetch = nullptr;
  void *part_tmp[MAX_BATCH_PARTS] = {nullptr};
  size_t part_tmp_bytes[MAX_BATCH_PARTS] = {0};
  // search launches captured as a CUDA graph, replayed while the key matches
  cudaGraphExec_t search_exec = nullptr;
  unsigned char search_key[320] = {0};
};

namespace {

constexpr uint64_t WAIT_LIMIT_NS = 20ull * 1000 * 1000 * 1000;  // 20 s per barrier wait
constexpr uint64_t IDLE_LIMIT_NS = 30ull * 1000 * 1000 * 1000;  // 30 s without any progress
constexpr uint32_t QUEUE_CAP = 1u << 14;                        // tasks per class queue
constexpr int DEFAULT_DONATE_MIN = 10;
constexpr int64_t BATCH_PART_MIN_ARCS = 1 << 20;  // mce_batch_count_host: smaller batches in one part
constexpr uint32_t DEFAULT_SOLO_MAX = 0;     // measured slower than grid-wide rounds
constexpr uint32_t DEFAULT_DONATE_AFTER = 256;  // the reference's SZTH (mce/parameter.cuh:5)

constexpr int MAX_PARTS = MAX_BATCH_PARTS;

void free_graph_bufs(mce_graph *g) {
  dfree(g->rp); dfree(g->col); dfree(g->cs); dfree(g->split);
  dfree(g->prio); dfree(g->core); dfree(g->deg); dfree(g->alA); dfree(g->alB);
  dfree(g->f0); dfree(g->f1); dfree(g->f2);
  dfree(g->hb0); dfree(g->hb1); dfree(g->hb2);
  dfree(g->keys_in); dfree(g->keys_out); dfree(g->vals_in); dfree(g->roots);
  dfree(g->hub_of); dfree(g->hub_list); dfree(g->hub_off); dfree(g->hub_rows); dfree(g->hub_nx);
  g->hub_off_cap = g->hub_rows_cap = 0;
  dfree(g->root_nodes); dfree(g->root_count); dfree(g->root_ops);
  dfree(g->feat); dfree(g->pred); dfree(g->policy); dfree(g->wlog); dfree(g->cand);
  dfree(g->cand_n);
  g->cap_n = g->cap_m = -1;
}

int alloc_graph_bufs(mce_graph *g, int64_t n, int64_t m) {
  free_graph_bufs(g);
  const size_t N = (size_t)n + 1, M = (size_t)m;
  int rc;
  // cs: 4 spare entries, so that a list's 16-byte window never ends past
  // the allocation (the bulk-copy staging of the search rounds it up)
  if ((rc = dalloc(&g->rp, N)) || (rc = dalloc(&g->col, M)) || (rc = dalloc(&g->cs, M + 4)) ||
      (rc = dalloc(&g->split, N)) || (rc = dalloc(&g->prio, N)) || (rc = dalloc(&g->core, N)) ||
      (rc = dalloc(&g->deg, N)) || (rc = dalloc(&g->alA, N)) || (rc = dalloc(&g->alB, N)) ||
      (rc = dalloc(&g->f0, N)) || (rc = dalloc(&g->f1, N)) || (rc = dalloc(&g->f2, N)) ||
      (rc = dalloc(&g->hb0, N)) || (rc = dalloc(&g->hb1, N)) || (rc = dalloc(&g->hb2, N)) ||
      (rc = dalloc(&g->keys_in, N)) || (rc = dalloc(&g->keys_out, N)) ||
      (rc = dalloc(&g->vals_in, N)) || (rc = dalloc(&g->roots, N)) ||
      (rc = dalloc(&g->hub_of, N)) || (rc = dalloc(&g->hub_list, N))) {
    free_graph_bufs(g);
    return rc;
  }
  g->cap_n = n;
  g->cap_m = m;
  return MCE_OK;
}

int alloc_fixed_bufs(mce_graph *g) {
  int rc;
  if ((rc = dalloc((char **)&g->peel_ctl, peel_ctl_bytes())) || (rc = dalloc(&g->shape, 1)) ||
      (rc = dalloc(&g->orient_next, 2 * (1 + MAX_PARTS))) ||
      (rc = dalloc(&g->fetch, 8)) || (rc = dalloc(&g->err, 4)) ||
      (rc = dalloc(&g->hist, MCE_HIST_MAX)) || (rc = dalloc(&g->nodes, 4)))
    return rc;
  for (auto &e : g->ev) MCE_CUDA(cudaEventCreate(&e));
  for (auto &pr : g->cls_ev)
    for (auto &e : pr) MCE_CUDA(cudaEventCreate(&e));
  return MCE_OK;
}

cudaStream_t pick_stream(mce_graph *g, void *s) { return s ? (cudaStream_t)s : g->own; }

// Per-graph counting of a batch handle.
// A batch still arriving from the host in parts (mce_batch_count_host):
// graphs [g[p], g[p+1]) are on the device once ready[p] has fired.
struct BatchParts {
  int k;
  int64_t g[MAX_PARTS + 1];
  cudaEvent_t ready[MAX_PARTS];
  const int32_t *rp_local, *col_local;  // device: the uploaded concatenations
  const int64_t *vo_h, *ao_h;           // host: the layout
};

// the most vertices of a graph of part p
// The per-graph peel's size class of a graph of n vertices: 0 more than
// PEEL_MID_N, 1 more than PEEL_SMALL_N, 2 the rest.
inline int peel_class(int64_t n) { return n > PEEL_MID_N ? 0 : n > PEEL_SMALL_N ? 1 : 2; }

// Graphs [g0, g1) of the large and middle peel classes.
inline void count_classes(const int64_t *vo, int64_t g0, int64_t g1, int32_t *big, int32_t *mid) {
  *big = *mid = 0;
  for (int64_t g = g0; g < g1; ++g) {
    const int c = peel_class(vo[g + 1] - vo[g] - 1);
    *big += c == 0;
    *mid += c == 1;
  }
}

// The per-graph peel's order of graphs [g0, g1): by size class (each class
// its own launch), each class largest first.
void order_graphs(int32_t *order, int64_t g0, int64_t g1, const int64_t *vo, const int64_t *ao) {
  std::stable_sort(order + g0, order + g1, [&](int32_t x, int32_t y) {
    const int cx = peel_class(vo[x + 1] - vo[x] - 1), cy = peel_class(vo[y + 1] - vo[y] - 1);
    if (cx != cy) return cx < cy;
    return ao[x + 1] - ao[x] > ao[y + 1] - ao[y];
  });
}

// One search's root summary, written on the device.
__global__ void shape_set_kernel(ShapeInfo *dst, ShapeInfo v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = v;
}

// The opt-in timeline (diagnostics only): trace_mark records an event on a
// stream under a short name, trace_dump prints the call's events once the
// last has completed.
void trace_mark(mce_graph *g, cudaStream_t st, const char *what, int i = -1) {
  if (g->trace_n < 0 || g->trace_n >= mce_graph::TRACE_MAX) return;
  const int k = g->trace_n++;
  if (!g->trace_ev[k] && cudaEventCreate(&g->trace_ev[k]) != cudaSuccess) {
    g->trace_ev[k] = nullptr;
    g->trace_n = -1;
    return;
  }
  if (i >= 0)
    snprintf(g->trace_name[k], sizeof(g->trace_name[k]), "%s%d", what, i);
  else
    snprintf(g->trace_name[k], sizeof(g->trace_name[k]), "%s", what);
  cudaEventRecord(g->trace_ev[k], st);
}

void trace_dump(mce_graph *g) {
  if (g->trace_n <= 0) return;
  const int n = g->trace_n;
  g->trace_n = -1;
  for (int k = 0; k < n; ++k) cudaEventSynchronize(g->trace_ev[k]);
  fprintf(stderr, "mce parts timeline (ms):");
  for (int k = 0; k < n; ++k) {
    float ms = 0;
    cudaEventElapsedTime(&ms, g->trace_ev[0], g->trace_ev[k]);
    fprintf(stderr, " %s=%.2f", g->trace_name[k], ms);
  }
  fprintf(stderr, "\n");
}

// The side streams and events of a per-graph peel launch (i: 0 whole batch,
// 1 + p part p), made on first use.
int seg_side(mce_graph *g, int i, PeelSide *ps) {
  for (int k = 0; k < 2; ++k) {
    if (!g->seg_side[k][i])
      MCE_CUDA(cudaStreamCreateWithFlags(&g->seg_side[k][i], cudaStreamNonBlocking));
    if (!g->seg_join[k][i])
      MCE_CUDA(cudaEventCreateWithFlags(&g->seg_join[k][i], cudaEventDisableTiming));
    ps->side[k] = g->seg_side[k][i];
    ps->join[k] = g->seg_join[k][i];
  }
  if (!g->seg_fork[i]) MCE_CUDA(cudaEventCreateWithFlags(&g->seg_fork[i], cudaEventDisableTiming));
  ps->fork = g->seg_fork[i];
  return MCE_OK;
}

inline int64_t part_max_n(const BatchParts &P, int p) {
  int64_t mx = 0;
  for (int64_t g = P.g[p]; g < P.g[p + 1]; ++g) {
    const int64_t n = P.vo_h[g + 1] - P.vo_h[g] - 1;
    if (n > mx) mx = n;
  }
  return mx;
}

struct BatchCtx {
  const int32_t *graph_of;             // device, n
  unsigned long long *graph_count;     // device, G
  uint64_t *per_graph_out;             // host, G
  int64_t G;
  const int64_t *vtx_off, *arc_off;    // device, G + 1: the uploaded layout
  const int32_t *order;                // device, G: graphs largest first (within each part)
  const BatchParts *parts = nullptr;   // nullable: rebase, peel and orient part by part
  int64_t max_n = 0;                   // the most vertices of a graph (0: unknown)
  int32_t g_big = 0, g_mid = 0;        // graphs of `order` in the large and middle peel classes
};

int check_args(const int32_t *row_ptr, const int32_t *col, int64_t n, int64_t m) {
  if (n < 0 || m < 0 || (n > 0 && !row_ptr) || (m > 0 && !col)) return MCE_EINVAL;
  if (n >= ((int64_t)1 << 31) - 1 || m >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  return MCE_OK;
}

int upload_csr(mce_graph *g, const int32_t *row_ptr, const int32_t *col, int64_t n, int64_t m,
               cudaStream_t s) {
  if (n > g->cap_n || m > g->cap_m) {
    int rc = alloc_graph_bufs(g, n, m);
    if (rc) return rc;
  }
  g->n = n;
  g->m = m;
  if (n > 0)
    MCE_CUDA(cudaMemcpyAsync(g->rp, row_ptr, sizeof(int32_t) * (size_t)(n + 1),
                             cudaMemcpyHostToDevice, s));
  if (m > 0)
    MCE_CUDA(cudaMemcpyAsync(g->col, col, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
  g->logged = false;
  return MCE_OK;
}

// Stage 1: peel -> prio, core.
PeelArgs peel_args(mce_graph *g, int solo_opt);

int run_peel(mce_graph *g, cudaStream_t s, int *launches, int solo_opt = 0,
             const BatchCtx *bc = nullptr) {
  if (g->n == 0) return MCE_OK;
  const PeelArgs pa = peel_args(g, solo_opt);
  if (bc) {  // a batch: every graph peeled by one block, no grid-wide rounds
    PeelSide ps;
    int rc = seg_side(g, 0, &ps);
    if (rc) return rc;
    return peel_segments_launch(pa, bc->vtx_off, bc->arc_off, bc->order, (int32_t)bc->G,
                                bc->g_big, bc->g_mid, s, ps, launches, -1, bc->max_n);
  }
  return peel_launch(pa, s, launches);
}

PeelArgs peel_args(mce_graph *g, int solo_opt) {
  PeelArgs pa;
  pa.n = g->n;
  pa.m = g->m;
  pa.rp = g->rp;
  pa.col = g->col;
  pa.deg = g->deg;
  pa.core = g->core;
  pa.prio = g->prio;
  pa.alistA = g->alA;
  pa.alistB = g->alB;
  pa.front0 = g->f0;
  pa.front1 = g->f1;
  pa.front2 = g->f2;
  pa.hb0 = g->hb0;
  pa.hb1 = g->hb1;
  pa.hb2 = g->hb2;
  pa.ctl = g->peel_ctl;
  pa.wait_limit_ns = WAIT_LIMIT_NS;
  pa.solo_max = solo_opt < 0 ? 0u : solo_opt == 0 ? DEFAULT_SOLO_MAX : (uint32_t)solo_opt;
  return pa;
}

// Stage 2: orient + classify + sort roots (keys plain: class only).
int run_sort(mce_graph *g, int end_bit, cudaStream_t s, int *launches) {
  return roots_sort(g->n, g->keys_in, g->keys_out, g->vals_in, g->roots, end_bit, &g->sort_tmp,
                    &g->sort_tmp_bytes, g->shape, s, launches);
}

OrientArgs orient_args(mce_graph *g) {
  OrientArgs oa;
  oa.n = g->n;
  oa.rp = g->rp;
  oa.col = g->col;
  oa.prio = g->prio;
  oa.split = g->split;
  oa.cs = g->cs;
  oa.keys_in = g->keys_in;
  oa.vals_in = g->vals_in;
  oa.shape = g->shape;
  oa.cost = nullptr;
  oa.sched = MCE_SCHED_PLAIN;
  oa.hub_of = g->hub_of;
  oa.hub_list = g->hub_list;
  oa.next = g->orient_next;
  oa.long_list = reinterpret_cast<int32_t *>(g->keys_out);  // free until the roots' sort
  return oa;
}

int run_orient(mce_graph *g, cudaStream_t s, int *launches, bool skip_sort = false) {
  int rc = orient_launch(orient_args(g), s, launches);
  if (rc) return rc;
  return skip_sort ? MCE_OK : run_sort(g, 3, s, launches);  // keys: class only
}

// A batch arriving in parts: as each part's copy lands, its graphs are
// rebased, peeled (one block per graph) and their vertices oriented, on a
// stream per part so that the parts' peels (each bound by its largest
// graphs' round chains) overlap; the roots' summary accumulates over them.
int run_parts(mce_graph *g, cudaStream_t s, int *launches, const BatchCtx *bc, int solo_opt) {
  const BatchParts &P = *bc->parts;
  const PeelArgs pa = peel_args(g, solo_opt);
  for (int p = 0; p < P.k; ++p) {
    if (!g->part_s[p]) MCE_CUDA(cudaStreamCreateWithFlags(&g->part_s[p], cudaStreamNonBlocking));
    if (!g->part_done[p])
      MCE_CUDA(cudaEventCreateWithFlags(&g->part_done[p], cudaEventDisableTiming));
  }
  if (!g->part_fork) MCE_CUDA(cudaEventCreateWithFlags(&g->part_fork, cudaEventDisableTiming));
  // zeroed once for all parts: the peel's control block and the roots' summary
  MCE_CUDA(cudaMemsetAsync(g->peel_ctl, 0, peel_ctl_bytes(), s));
  MCE_CUDA(cudaMemsetAsync(g->shape, 0, sizeof(ShapeInfo), s));
  MCE_CUDA(cudaEventRecord(g->part_fork, s));
  for (int p = 0; p < P.k; ++p) {
    cudaStream_t sp = g->part_s[p];
    const int64_t g0 = P.g[p], g1 = P.g[p + 1];
    const int64_t vbeg = P.vo_h[g0] - g0, vend = P.vo_h[g1] - g1;
    MCE_CUDA(cudaStreamWaitEvent(sp, g->part_fork, 0));
    MCE_CUDA(cudaStreamWaitEvent(sp, P.ready[p], 0));
    int rc = batch_rebase_part_launch(P.rp_local, P.col_local, bc->vtx_off, bc->arc_off,
                                      (int32_t)bc->G, P.vo_h[g0], P.vo_h[g1], P.ao_h[g0],
                                      P.ao_h[g1], vend, (int32_t)P.ao_h[g1], g->rp, g->col,
                                      const_cast<int32_t *>(bc->graph_of), g->sms, sp, launches);
    if (rc) return rc;
    // a part's peel in two launches, its large and middle graphs together:
    // a third launch per part measured slower end to end (53.1 against 51.3 ms)
    PeelSide ps;
    int32_t nbig = 0, nmid = 0;
    if ((rc = seg_side(g, 1 + p, &ps))) return rc;
    if (vend > vbeg &&
        (count_classes(P.vo_h, g0, g1, &nbig, &nmid),
         rc = peel_segments_launch(pa, bc->vtx_off, bc->arc_off, bc->order + g0,
                                   (int32_t)(g1 - g0), nbig + nmid, 0, sp, ps, launches, p,
                                   part_max_n(P, p))))
      return rc;
    OrientArgs oa = orient_args(g);
    oa.v0 = vbeg;
    oa.n = vend;
    oa.keep_shape = true;
    oa.next = g->orient_next + 2 + 2 * p;  // the parts' orientations run at the same time
    oa.long_list = reinterpret_cast<int32_t *>(g->keys_out) + vbeg;
    if ((rc = orient_launch(oa, sp, launches))) return rc;
    MCE_CUDA(cudaEventRecord(g->part_done[p], sp));
  }
  for (int p = 0; p < P.k; ++p) MCE_CUDA(cudaStreamWaitEvent(s, g->part_done[p], 0));
  return MCE_OK;
}

int read_shape(mce_graph *g, cudaStream_t s) {
  MCE_CUDA(cudaMemcpyAsync(&g->shape_h, g->shape, sizeof(ShapeInfo), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  return MCE_OK;
}

// Queue of class c laid out in one buffer: header | seq[cap] | payload.
int ensure_queue(mce_graph *g, int c, uint32_t words, QueueView *out) {
  const size_t hdr = 256, seq = (size_t)QUEUE_CAP * 4;
  const size_t need = hdr + seq + (size_t)QUEUE_CAP * words * 8;
  if (need > g->qbytes[c]) {
    dfree(g->qbuf[c]);
    g->qbytes[c] = 0;
    MCE_CUDA(cudaMalloc(&g->qbuf[c], need));
    g->qbytes[c] = need;
  }
  char *b = (char *)g->qbuf[c];
  out->hdr = (QueueHdr *)b;
  out->seq = (uint32_t *)(b + hdr);
  out->pay = (unsigned long long *)(b + hdr + seq);
  out->cap = QUEUE_CAP;
  out->words = words;
  return MCE_OK;
}

int graph_create(int32_t device, mce_graph **out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MCE_ENODEV;
  if (device < 0 || device >= ndev) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(device));
  mce_graph *g = new (std::nothrow) mce_graph();
  if (!g) return MCE_ENOMEM;
  g->device = device;
  if (cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&g->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete g;
    return MCE_ECUDA;
  }
  int rc = alloc_fixed_bufs(g);
  if (rc) {
    mce_graph_free(g);
    return rc;
  }
  *out = g;
  return MCE_OK;
}

int ensure_slab(mce_graph *g, size_t bytes) {
  if (bytes <= g->slab_bytes) return MCE_OK;
  dfree(g->slab);
  g->slab_bytes = 0;
  MCE_CUDA(cudaMalloc((void **)&g->slab, bytes));
  g->slab_bytes = bytes;
  return MCE_OK;
}

}  // namespace

namespace mce {
// A new handle sized for n vertices and m arcs whose CSR the caller writes
// on the device (the .bel loader): row_ptr, col, and the m-entry split-CSR
// array as scratch (orientation rewrites it).
int graph_adopt(int32_t device, int64_t n, int64_t m, struct ::mce_graph **out, int32_t **rp,
                int32_t **col, int32_t **scratch, cudaStream_t *own) {
  int rc;
  if (n < 0 || m < 0 || n >= ((int64_t)1 << 31) - 1 || m >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  mce_graph *g = nullptr;
  if ((rc = graph_create(device, &g))) return rc;
  if ((rc = alloc_graph_bufs(g, n, m))) {
    mce_graph_free(g);
    return rc;
  }
  g->n = n;
  g->m = m;
  *out = g;
  *rp = g->rp;
  *col = g->col;
  *scratch = g->cs;
  *own = g->own;
  return MCE_OK;
}

// sizes of a graph handle and the union graph of a batch (autotuner)
int graph_shape(const struct ::mce_graph *g, int64_t *n, int64_t *m) {
  if (!g) return MCE_EINVAL;
  *n = g->n;
  *m = g->m;
  return MCE_OK;
}
struct ::mce_graph *batch_union(struct ::mce_batch *b, int32_t *num_graphs);

// device CSR of a graph handle, for the serving sessions (serve.cu)
int graph_device_view(const struct ::mce_graph *g, const int32_t **rp, const int32_t **col,
                      int64_t *n, int *device) {
  if (!g || !g->rp) return MCE_ESTATE;
  *rp = g->rp;
  *col = g->col;
  *n = g->n;
  *device = g->device;
  return MCE_OK;
}
}  // namespace mce

extern "C" {

void mce_opts_default(mce_opts_t *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->level = MCE_LEVEL_L1;
  o->induced = MCE_INDUCED_P;
  o->worker_list = MCE_WL_ON;
  o->sched = MCE_SCHED_PLAIN;
  o->bitmap_width = 0;
  o->warps_per_root = 0;
  o->donate_threshold = 0;
  o->log_roots = 0;
  o->x_pivot = 0;
  o->stream = nullptr;
}

const char *mce_strerror(int code) {
  switch (code) {
    case MCE_OK: return "ok";
    case MCE_EINVAL: return "invalid argument";
    case MCE_ENOMEM: return "out of memory";
    case MCE_ECUDA: return g_last_detail[0] ? g_last_detail : "CUDA error";
    case MCE_EIO: return "I/O error";
    case MCE_EFORMAT: return "malformed input";
    case MCE_ELIMIT: return "size limit exceeded";
    case MCE_ETIMEOUT: return "device wait limit reached";
    case MCE_ENODEV: return "no usable CUDA device";
    case MCE_ESTATE: return "call out of order";
    case MCE_EAGAIN: return "not finished yet";
    default: return "unknown error";
  }
}

const char *mce_version(void) { return "mce-b200 0.1 (sm_100a)"; }

int mce_graph_upload(const int32_t *row_ptr, const int32_t *col, int64_t n, int64_t m,
                     int32_t device, void *stream, mce_graph_t *out) {
  if (!out) return MCE_EINVAL;
  *out = nullptr;
  int rc = check_args(row_ptr, col, n, m);
  if (rc) return rc;
  mce_graph *g = nullptr;
  if ((rc = graph_create(device, &g))) return rc;
  rc = upload_csr(g, row_ptr, col, n, m, pick_stream(g, stream));
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(pick_stream(g, stream));
    if (e != cudaSuccess) rc = MCE_ECUDA;
  }
  if (rc) {
    mce_graph_free(g);
    return rc;
  }
  *out = g;
  return MCE_OK;
}

int mce_graph_reload(mce_graph_t g, const int32_t *row_ptr, const int32_t *col, int64_t n,
                     int64_t m, void *stream) {
  if (!g) return MCE_EINVAL;
  int rc = check_args(row_ptr, col, n, m);
  if (rc) return rc;
  MCE_CUDA(cudaSetDevice(g->device));
  return upload_csr(g, row_ptr, col, n, m, pick_stream(g, stream));
}

int mce_graph_size(mce_graph_t g, int64_t *n, int64_t *m) {
  if (!g || !n || !m) return MCE_EINVAL;
  *n = g->n;
  *m = g->m;
  return MCE_OK;
}

int mce_graph_free(mce_graph_t g) {
  if (!g) return MCE_OK;
  cudaSetDevice(g->device);
  if (g->own) cudaStreamSynchronize(g->own);
  free_graph_bufs(g);
  dfree(g->peel_ctl);
  dfree(g->shape);
  dfree(g->orient_next);
  dfree(g->fetch);
  dfree(g->err);
  dfree(g->hist);
  dfree(g->nodes);
  dfree(g->slab);
  dfree(g->sort_tmp);
  for (auto &q : g->qbuf) dfree(q);
  if (g->search_exec) cudaGraphExecDestroy(g->search_exec);
  for (auto &e : g->ev)
    if (e) cudaEventDestroy(e);
  for (auto &pr : g->cls_ev)
    for (auto &e : pr)
      if (e) cudaEventDestroy(e);
  dfree(g->part_shape);
  dfree(g->part_fetch);
  if (g->part_shape_h) cudaFreeHost(g->part_shape_h);
  for (int p = 0; p < MAX_PARTS; ++p) {
    dfree(g->part_tmp[p]);
  }
  for (int p = 0; p < MAX_PARTS; ++p) {
    if (g->part_s[p]) cudaStreamDestroy(g->part_s[p]);
    if (g->part_done[p]) cudaEventDestroy(g->part_done[p]);
  }
  if (g->part_fork) cudaEventDestroy(g->part_fork);
  if (g->part_sdone) cudaEventDestroy(g->part_sdone);
  for (cudaEvent_t e : g->trace_ev)
    if (e) cudaEventDestroy(e);
  for (int i = 0; i < 1 + MAX_PARTS; ++i) {
    for (int k = 0; k < 2; ++k) {
      if (g->seg_side[k][i]) cudaStreamDestroy(g->seg_side[k][i]);
      if (g->seg_join[k][i]) cudaEventDestroy(g->seg_join[k][i]);
    }
    if (g->seg_fork[i]) cudaEventDestroy(g->seg_fork[i]);
  }
  if (g->own) cudaStreamDestroy(g->own);
  delete g;
  return MCE_OK;
}

int mce_degeneracy(mce_graph_t g, uint32_t *priority_out, int32_t *core_out,
                   int32_t *degeneracy) {
  if (!g) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = g->own;
  int launches = 0, rc = run_peel(g, s, &launches);
  if (rc) return rc;
  int32_t dg = 0;
  uint32_t err = 0, rounds = 0;
  if (g->n > 0) {
    rc = peel_read(g->peel_ctl, &dg, &err, &rounds, nullptr, s);
    if (rc) return rc;
    if (err) return MCE_ETIMEOUT;
    if (priority_out)
      MCE_CUDA(cudaMemcpyAsync(priority_out, g->prio, sizeof(uint32_t) * (size_t)g->n,
                               cudaMemcpyDeviceToHost, s));
    if (core_out)
      MCE_CUDA(cudaMemcpyAsync(core_out, g->core, sizeof(int32_t) * (size_t)g->n,
                               cudaMemcpyDeviceToHost, s));
    MCE_CUDA(cudaStreamSynchronize(s));
  }
  g->degeneracy = dg;
  if (degeneracy) *degeneracy = dg;
  return MCE_OK;
}

int mce_split_csr(mce_graph_t g, int32_t *split_out, int32_t *col_out) {
  if (!g) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = g->own;
  int launches = 0, rc = run_peel(g, s, &launches);
  if (!rc) rc = run_orient(g, s, &launches);
  if (rc) return rc;
  if (split_out && g->n)
    MCE_CUDA(cudaMemcpyAsync(split_out, g->split, sizeof(int32_t) * (size_t)g->n,
                             cudaMemcpyDeviceToHost, s));
  if (col_out && g->m)
    MCE_CUDA(cudaMemcpyAsync(col_out, g->cs, sizeof(int32_t) * (size_t)g->m,
                             cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  return MCE_OK;
}

}  // extern "C"

namespace {

}  // namespace

struct mce_model {
  int device = 0;
  int sms = 0;
  cudaStream_t own = nullptr;
  float *master = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr, *loss = nullptr;
  __half *wh = nullptr;
  int step = 0;
};

namespace {

constexpr int WLOG_WORDS = 10;  // per-warp log record: SM, nodes, donations, 7 phase cycles
constexpr int DEFAULT_HEAVY_LOG2 = 12;  // predicted log2(tree nodes) from which a root runs first
constexpr int DEFAULT_SHARE_LOG2 = 16;  // ... and (learned schedule) shares from its first node

int ensure_feat(mce_graph *g) {
  int rc;
  if (!g->feat && (rc = dalloc(&g->feat, (size_t)(g->cap_n + 1) * MLP_IN))) return rc;
  if (!g->pred && (rc = dalloc(&g->pred, (size_t)g->cap_n + 1))) return rc;
  if (!g->policy && (rc = dalloc(&g->policy, (size_t)g->cap_n + 1))) return rc;
  if (!g->cand && (rc = dalloc(&g->cand, (size_t)g->cap_n + 1))) return rc;
  if (!g->cand_n && (rc = dalloc(&g->cand_n, 1))) return rc;
  return MCE_OK;
}

// Features of the candidate roots (at least MLP_MIN_LATER later neighbours)
// of the peeled, oriented graph into g->feat, their list into g->cand; with
// zero_rest the other rows are zeroed too (mce_root_features returns them).
int compute_features(mce_graph *g, cudaStream_t s, int *launches, bool zero_rest,
                     int min_later = MLP_MIN_LATER) {
  int rc = ensure_feat(g);
  if (rc) return rc;
  if (zero_rest && g->n)
    MCE_CUDA(cudaMemsetAsync(g->feat, 0, sizeof(float) * MLP_IN * (size_t)g->n, s));
  return features_launch(g->n, g->rp, g->split, g->cs, g->core, g->feat, g->cand, g->cand_n,
                         g->sms, s, launches, min_later);
}

// Predicted cost of every vertex into g->pred: the model on the candidate
// roots, 0 (light) elsewhere.
int predict_candidates(mce_graph *g, const void *wh, cudaStream_t s, int *launches) {
  if (g->n == 0) return MCE_OK;
  MCE_CUDA(cudaMemsetAsync(g->pred, 0, sizeof(float) * (size_t)g->n, s));
  return mlp_forward_launch(wh, g->feat, g->cand, g->cand_n, g->n, g->pred, g->sms, s, launches);
}

// The counting pipeline shared by mce_count and mce_batch_count.  With a
// batch context, each root's count also goes to its graph's counter.
// Clique listing: device buffer for the {size, root, members...} records.
struct ListCtx {
  int32_t *buf;
  unsigned long long *words;
  unsigned long long cap;
};

int count_impl(mce_graph *g, const mce_opts_t &o, uint64_t *total, uint64_t *hist,
               mce_stats_t *stats, const BatchCtx *bc, const ListCtx *lc = nullptr) {
  if (o.bitmap_width != 0 && o.bitmap_width != 32 && o.bitmap_width != 64) return MCE_EINVAL;
  if (o.wide_blocks != 0 && o.wide_blocks != 4 && o.wide_blocks != 8) return MCE_EINVAL;
  // the word-op count follows the IP walk; it is not an evaluation or listing run
  if (o.count_ops &&
      (o.x_pivot || o.induced == MCE_INDUCED_PX || o.warp_log || lc || o.level == MCE_LEVEL_L2))
    return MCE_EINVAL;
  if (o.warps_per_root < 0 || o.warps_per_root > 32) return MCE_EINVAL;
  for (int c = 0; c < 3; ++c)
    if (o.bucket_warps_per_root[c] < 0 || o.bucket_warps_per_root[c] > 32 ||
        o.bucket_donate_threshold[c] < 0 || o.bucket_donate_after[c] < 0)
      return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = pick_stream(g, o.stream);
  int launches = 0, rc;
  mce_stats_t st;
  std::memset(&st, 0, sizeof(st));
  MCE_CUDA(cudaEventRecord(g->ev[0], s));
  const bool parted = bc && bc->parts;
  if ((rc = parted ? run_parts(g, s, &launches, bc, o.peel_solo_max)
                   : run_peel(g, s, &launches, o.peel_solo_max, bc)))
    return rc;
  MCE_CUDA(cudaEventRecord(g->ev[1], s));
  // Root order: plain = vertex id within each engine class; degree = a
  // degree-based cost; learned = the model's predicted tree size.  Larger
  // costs first; the learned order also sets which roots share subtrees.
  const mce_model *model = (const mce_model *)o.model;
  const int sched = o.sched == MCE_SCHED_LEARNED && !model ? MCE_SCHED_DEGREE : o.sched;
  if (parted) {  // oriented part by part already; plain order sorts by class only
    if (sched == MCE_SCHED_PLAIN && (rc = run_sort(g, 3, s, &launches))) return rc;
  } else if ((rc = run_orient(g, s, &launches, sched != MCE_SCHED_PLAIN))) {
    return rc;
  }
  const uint8_t *policy = nullptr;
  const float heavy = (float)(o.heavy_log2 > 0 ? o.heavy_log2 : DEFAULT_HEAVY_LOG2);
  const float share_cost = (float)(o.share_log2 > 0 ? o.share_log2 : DEFAULT_SHARE_LOG2);
  if (sched == MCE_SCHED_DEGREE && g->n > 0) {
    if ((rc = rekey_launch(g->n, g->keys_in, nullptr, g->rp, g->split, nullptr, heavy, heavy,
                           g->sms, s, &launches)) ||
        (rc = run_sort(g, 32, s, &launches)))
      return rc;
  } else if (sched == MCE_SCHED_LEARNED && g->n > 0) {
    if (model->device != g->device) return MCE_EINVAL;
    if ((rc = compute_features(g, s, &launches, false, SCHED_MIN_LATER)) ||
        (rc = predict_candidates(g, model->wh, s, &launches)) ||
        (rc = rekey_launch(g->n, g->keys_in, g->pred, g->rp, g->split, g->policy, heavy, share_cost,
                           g->sms, s, &launches, SCHED_MIN_LATER)) ||
        (rc = run_sort(g, 32, s, &launches)))
      return rc;
    policy = g->policy;
  }
  MCE_CUDA(cudaEventRecord(g->ev[2], s));
  if ((rc = read_shape(g, s))) return rc;
  const ShapeInfo &sh = g->shape_h;
  if (sh.cls_cnt[CLS_BIG]) return MCE_ELIMIT;
  // earlier-neighbour rows of the hub roots, built by many warps at once
  if (sh.hub_cnt > 0) {
    const int64_t need_off = (int64_t)sh.hub_cnt + 2, need_rows = (int64_t)sh.hub_rows;
    if (need_off > g->hub_off_cap) {
      dfree(g->hub_off);
      dfree(g->hub_nx);
      g->hub_off_cap = 0;
      if ((rc = dalloc(&g->hub_off, (size_t)need_off)) || (rc = dalloc(&g->hub_nx, (size_t)need_off)))
        return rc;
      g->hub_off_cap = need_off;
    }
    if (need_rows > g->hub_rows_cap) {
      dfree(g->hub_rows);
      g->hub_rows_cap = 0;
      if ((rc = dalloc(&g->hub_rows, (size_t)need_rows))) return rc;
      g->hub_rows_cap = need_rows;
    }
    if ((rc = hub_rows_launch(g->rp, g->split, g->cs, g->hub_list, sh.hub_cnt, need_rows,
                              g->hub_off, g->hub_nx, g->hub_rows, g->sms, s, &launches)))
      return rc;
  }
  // search scratch
  const bool share = o.worker_list != MCE_WL_OFF;
  int grid[NCLS] = {0}, block[NCLS] = {0}, smem[NCLS] = {0};
  const int dcap = (int)(sh.max_dplus > 0 ? sh.max_dplus : 1);
  const int xcap = (int)(sh.max_dminus_mem > 0 ? sh.max_dminus_mem : 1);
  int rxcap = REG_XCAP;  // a power of two covering the register classes' earlier degrees
  while (rxcap < (int)sh.max_dminus_reg && rxcap < REG_XCAP_MAX) rxcap <<= 1;
  size_t slab_need = 0;
  // per bucket (engine class): warps per root, donation threshold and gate
  int parts[NCLS] = {1, 1, 1, 1, 1}, dmin[NCLS] = {0}, dafter[NCLS] = {0};
  for (int c = CLS_R32; c <= CLS_MEM; ++c) {
    const int w = o.bucket_warps_per_root[c] ? o.bucket_warps_per_root[c] : o.warps_per_root;
    // evaluation, listing and L2 (whose units split a root already): one warp
    parts[c] = w > 1 && !o.warp_log && !lc && o.level != MCE_LEVEL_L2 ? w : 1;
    const int t = o.bucket_donate_threshold[c] ? o.bucket_donate_threshold[c] : o.donate_threshold;
    dmin[c] = t > 0 ? t : DEFAULT_DONATE_MIN;
    const int af = o.bucket_donate_after[c] ? o.bucket_donate_after[c] : o.donate_after;
    dafter[c] = af > 0 ? af : (int)DEFAULT_DONATE_AFTER;
  }
  for (int c = CLS_R32; c <= CLS_MEM; ++c) {
    if (!sh.cls_cnt[c]) continue;
    int warps = 0;
    if ((rc = bk_warps_for_class(c, g->sms, o.wide_blocks, &warps, &block[c], &smem[c]))) return rc;
    // never more warps than units of work (a root's parts; rounded up to
    // whole blocks); with task sharing keep at least a full wave so idle
    // warps can take subtrees
    const int wpb = block[c] / 32;
    int64_t want = (int64_t)sh.cls_cnt[c] * parts[c];
    if (share) want = want > warps ? want : warps;
    if (want < warps) warps = (int)((want + wpb - 1) / wpb) * wpb;
    grid[c] = warps / wpb;
    const size_t need = (size_t)warps * bk_slab_words(c, dcap, xcap, rxcap) * 8;
    if (need > slab_need) slab_need = need;
  }
  if ((rc = ensure_slab(g, slab_need))) return rc;
  if (o.log_roots && !g->root_nodes) {
    if ((rc = dalloc(&g->root_nodes, (size_t)g->cap_n + 1))) return rc;
    if ((rc = dalloc(&g->root_count, (size_t)g->cap_n + 1))) return rc;
  }
  const bool log_ops = o.log_roots && o.count_ops;
  if (log_ops && !g->root_ops && (rc = dalloc(&g->root_ops, (size_t)g->cap_n + 1))) return rc;
  int64_t wlog_base[NCLS] = {0}, wlog_total = 0;
  for (int c : {CLS_MEM, CLS_R64, CLS_R32}) {  // the launch order below
    wlog_base[c] = wlog_total;
    if (grid[c]) wlog_total += (int64_t)grid[c] * (block[c] / 32);
  }
  if (o.warp_log && wlog_total > g->wlog_cap) {
    dfree(g->wlog);
    if ((rc = dalloc(&g->wlog, WLOG_WORDS * (size_t)wlog_total))) return rc;
    g->wlog_cap = wlog_total;
  }
  g->wlog_count = o.warp_log ? wlog_total : 0;
  BKArgs a;
  std::memset(&a, 0, sizeof(a));
  a.rp = g->rp;
  a.split = g->split;
  a.cs = g->cs;
  a.roots = g->roots;
  a.shape = g->shape;
  a.fetch = g->fetch;
  a.hist = g->hist;
  a.nodes = g->nodes;
  a.root_nodes = o.log_roots ? g->root_nodes : nullptr;
  a.root_count = o.log_roots ? g->root_count : nullptr;
  a.graph_of = bc ? bc->graph_of : nullptr;
  a.graph_count = bc ? bc->graph_count : nullptr;
  a.err = g->err;
  a.slab = g->slab;
  a.dcap = dcap;
  a.xcap = xcap;
  a.rxcap = rxcap;
  a.hub_of = sh.hub_cnt > 0 ? g->hub_of : nullptr;
  a.hub_off = g->hub_off;
  a.hub_rows = g->hub_rows;
  a.hub_nx = g->hub_nx;
  a.donate_min = dmin[CLS_R32];  // set per class at each launch below
  a.donate_after = (uint32_t)dafter[CLS_R32];
  a.wait_limit_ns = o.wait_limit_ms > 0 ? (uint64_t)o.wait_limit_ms * 1000000ull : IDLE_LIMIT_NS;
  a.policy = policy;
  a.wide8 = o.wide_blocks == 8 ? 1 : 0;
  a.level2 = o.level == MCE_LEVEL_L2 ? 1 : 0;
  a.prio = g->prio;
  a.x_pivot = (o.x_pivot || o.induced == MCE_INDUCED_PX) ? 1 : 0;
  a.count_ops = o.count_ops ? 1 : 0;
  a.stage = o.stage_lists ? 1 : 0;
  a.ops = g->nodes + 1;
  a.root_ops = log_ops ? g->root_ops : nullptr;
  if (lc) {
    a.list_buf = lc->buf;
    a.list_words = lc->words;
    a.list_cap = lc->cap;
  }
  const int wbits = o.bitmap_width == 64 ? 64 : 32;
  QueueView qv[NCLS];
  for (int c = CLS_R32; c <= CLS_MEM; ++c)
    if (share && grid[c] && (rc = ensure_queue(g, c, bk_task_words(c, dcap), &qv[c]))) return rc;
  // Everything from here to the end of the search is a fixed sequence of
  // memsets and launches whose arguments depend only on `key`: with
  // opts.cuda_graph it is captured once and replayed.
  struct SearchKey {
    int grid[NCLS], block[NCLS];
    int dcap, xcap, rxcap, wbits, share, log, wide8, level2, xpiv, ops, stage;
    int parts[NCLS], dmin[NCLS], dafter[NCLS];
    uint64_t wlimit;
    const void *slab, *graph_count, *graph_of, *root_nodes, *policy, *q[NCLS], *bufs[4], *wlog;
    const void *hub[4];
    int64_t n, G;
  } key;
  std::memset(&key, 0, sizeof(key));
  for (int c = 0; c < NCLS; ++c) {
    key.grid[c] = grid[c];
    key.block[c] = block[c];
    key.q[c] = qv[c].hdr;
  }
  key.dcap = dcap;
  key.xcap = xcap;
  key.rxcap = rxcap;
  key.wbits = wbits;
  key.share = share;
  for (int c = 0; c < NCLS; ++c) {
    key.parts[c] = parts[c];
    key.dmin[c] = dmin[c];
    key.dafter[c] = dafter[c];
  }
  key.wlimit = a.wait_limit_ns;
  key.log = o.log_roots != 0;
  key.wide8 = a.wide8;
  key.level2 = a.level2;
  key.xpiv = a.x_pivot;
  key.ops = a.count_ops + (log_ops ? 2 : 0);
  key.stage = a.stage;
  key.slab = g->slab;
  key.graph_count = a.graph_count;
  key.root_nodes = a.root_nodes;
  key.graph_of = a.graph_of;
  key.policy = a.policy;
  key.wlog = o.warp_log ? g->wlog : nullptr;
  key.bufs[0] = g->rp;
  key.bufs[1] = g->split;
  key.bufs[2] = g->cs;
  key.bufs[3] = g->roots;
  key.hub[0] = a.hub_of;
  key.hub[1] = a.hub_off;
  key.hub[2] = a.hub_rows;
  key.hub[3] = a.hub_nx;
  key.n = g->n;
  key.G = bc ? bc->G : 0;
  static_assert(sizeof(SearchKey) <= sizeof(g->search_key), "search key");
  // per-class launch times: plain event records, or external event nodes
  // while the launches are being captured
  bool capturing = false;
  auto mark = [&](cudaEvent_t e) {
    return capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal)
                     : cudaEventRecord(e, s);
  };
  auto record = [&]() -> int {
    int r2;
    if (o.log_roots) {
      MCE_CUDA(cudaMemsetAsync(g->root_nodes, 0, sizeof(unsigned long long) * (size_t)(g->n + 1), s));
      MCE_CUDA(cudaMemsetAsync(g->root_count, 0, sizeof(unsigned long long) * (size_t)(g->n + 1), s));
    }
    if (log_ops)
      MCE_CUDA(cudaMemsetAsync(g->root_ops, 0, sizeof(unsigned long long) * (size_t)(g->n + 1), s));
    if (bc) MCE_CUDA(cudaMemsetAsync(bc->graph_count, 0, sizeof(unsigned long long) * bc->G, s));
    MCE_CUDA(cudaMemsetAsync(g->fetch, 0, sizeof(uint32_t) * 8, s));
    MCE_CUDA(cudaMemsetAsync(g->err, 0, sizeof(uint32_t) * 4, s));
    MCE_CUDA(cudaMemsetAsync(g->hist, 0, sizeof(unsigned long long) * MCE_HIST_MAX, s));
    MCE_CUDA(cudaMemsetAsync(g->nodes, 0, sizeof(unsigned long long) * 4, s));
    if (o.warp_log)
      MCE_CUDA(cudaMemsetAsync(g->wlog, 0, sizeof(unsigned long long) * WLOG_WORDS * (size_t)wlog_total,
                               s));
    if (lc) MCE_CUDA(cudaMemsetAsync(lc->words, 0, sizeof(unsigned long long), s));
    // widest roots first so the long trees start early
    const int order[3] = {CLS_MEM, CLS_R64, CLS_R32};
    for (int c : order) {
      if (!grid[c]) continue;
      a.slab_words = bk_slab_words(c, dcap, xcap, rxcap);
      a.parts = parts[c];
      a.donate_min = dmin[c];
      a.donate_after = (uint32_t)dafter[c];
      a.q = share ? qv[c] : QueueView();
      a.warp_log = o.warp_log ? g->wlog + WLOG_WORDS * wlog_base[c] : nullptr;
      a.warp_cycles = o.warp_log == 2 ? 1 : 0;
      if (share && (r2 = queue_launch_init(a.q, s, &launches))) return r2;
      MCE_CUDA(mark(g->cls_ev[c][0]));
      if ((r2 = bk_launch(c, wbits, a, grid[c], block[c], smem[c], s, &launches))) return r2;
      MCE_CUDA(mark(g->cls_ev[c][1]));
    }
    return MCE_OK;
  };
  if (o.cuda_graph && !lc) {
    if (!g->search_exec || std::memcmp(g->search_key, &key, sizeof(key)) != 0) {
      if (g->search_exec) {
        cudaGraphExecDestroy(g->search_exec);
        g->search_exec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      MCE_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int lc = launches;
      capturing = true;
      rc = record();
      capturing = false;
      cudaError_t e = cudaStreamEndCapture(s, &graph);
      launches = lc;
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (e != cudaSuccess) return MCE_ECUDA;
      e = cudaGraphInstantiate(&g->search_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        g->search_exec = nullptr;
        return MCE_ECUDA;
      }
      std::memcpy(g->search_key, &key, sizeof(key));
    }
    MCE_CUDA(cudaGraphLaunch(g->search_exec, s));
    for (int c = CLS_R32; c <= CLS_MEM; ++c) launches += grid[c] ? (share ? 2 : 1) : 0;
  } else {
    if ((rc = record())) return rc;
  }
  MCE_CUDA(cudaEventRecord(g->ev[3], s));
  unsigned long long h_hist[MCE_HIST_MAX];
  unsigned long long h_nodes[2] = {0, 0};
  uint32_t h_err = 0;
  MCE_CUDA(cudaMemcpyAsync(h_hist, g->hist, sizeof(h_hist), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaMemcpyAsync(h_nodes, g->nodes, sizeof(h_nodes), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaMemcpyAsync(&h_err, g->err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
  QueueHdr qh[NCLS];
  bool qused[NCLS] = {false};
  for (int c = 0; c < NCLS; ++c)
    if (share && grid[c] && g->qbuf[c]) {
      MCE_CUDA(cudaMemcpyAsync(&qh[c], g->qbuf[c], sizeof(QueueHdr), cudaMemcpyDeviceToHost, s));
      qused[c] = true;
    }
  MCE_CUDA(cudaEventRecord(g->ev[4], s));
  if (bc) MCE_CUDA(cudaMemcpyAsync(bc->per_graph_out, bc->graph_count,
                                   sizeof(unsigned long long) * bc->G, cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  int32_t dg = 0;
  uint32_t perr = 0, rounds = 0, solo = 0;
  double pms[3] = {0, 0, 0};
  if (g->n > 0 && (rc = peel_read(g->peel_ctl, &dg, &perr, &rounds, &solo, s, pms))) return rc;
  g->degeneracy = dg;
  g->logged = o.log_roots != 0;
  g->logged_ops = log_ops;
  uint64_t pushed = 0;
  for (int c = 0; c < NCLS; ++c)
    if (qused[c]) pushed += qh[c].pushed;
  uint64_t tot = 0;
  for (int i = 0; i < MCE_HIST_MAX; ++i) tot += h_hist[i];
  *total = tot;
  if (hist)
    for (int i = 0; i < MCE_HIST_MAX; ++i) hist[i] = h_hist[i];
  float ms = 0;
  cudaEventElapsedTime(&ms, g->ev[0], g->ev[1]);
  st.peel_ms = ms;
  cudaEventElapsedTime(&ms, g->ev[1], g->ev[2]);
  st.orient_ms = ms;
  cudaEventElapsedTime(&ms, g->ev[2], g->ev[3]);
  st.count_ms = ms;
  cudaEventElapsedTime(&ms, g->ev[0], g->ev[4]);
  st.total_ms = ms;
  for (int c = CLS_R32; c <= CLS_MEM; ++c)
    if (grid[c] && cudaEventElapsedTime(&ms, g->cls_ev[c][0], g->cls_ev[c][1]) == cudaSuccess)
      st.class_ms[c] = ms;
  st.degeneracy = dg;
  st.max_later_degree = (int32_t)sh.max_dplus;
  st.max_degree = sh.max_deg;
  st.roots = (int64_t)sh.cls_cnt[CLS_R32] + sh.cls_cnt[CLS_R64] + sh.cls_cnt[CLS_MEM];
  st.tree_nodes = h_nodes[0];
  st.word_ops = o.count_ops ? h_nodes[1] : 0;
  st.kernel_launches = launches;
  st.error_flags = h_err | (perr ? MCE_ERR_WAIT_TIMEOUT : 0);
  for (int c = 0; c < NCLS && c < 8; ++c) st.class_roots[c] = sh.cls_cnt[c];
  st.peel_rounds = rounds;
  st.peel_solo_sections = solo;
  st.peel_scan_ms = pms[0];
  st.peel_round_ms = pms[1];
  st.peel_wait_ms = pms[2];
  st.donations = pushed;
  if (stats) *stats = st;
  if (perr) return MCE_ETIMEOUT;
  if (h_err & MCE_ERR_WAIT_TIMEOUT) return MCE_ETIMEOUT;
  if (h_err) return MCE_ELIMIT;
  return MCE_OK;
}

}  // namespace

namespace {

// mce_batch_count_host, pipelined: each part of a batch arriving from the
// host is rebased, peeled, oriented and its roots sorted on a stream of its
// own as soon as its copy lands; the host reads the part's summary and
// queues its search (hub rows, then the engine classes) on the call's stream,
// so part p is searched while parts p+1.. are still being copied and peeled.
// A part's graphs share no vertex with other parts, so its search reads only
// its own rows.  Buffers that a later part outgrows are replaced and the old
// ones freed after the call (earlier parts' searches may still use them).
// Counting only: plain or degree order; the other modes take count_impl.
int count_pipelined(mce_graph *g, const mce_opts_t &o, uint64_t *total, uint64_t *hist,
                    mce_stats_t *stats, const BatchCtx *bc) {
  const BatchParts &P = *bc->parts;
  MCE_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = pick_stream(g, o.stream);
  int launches = 0, rc = MCE_OK;
  mce_stats_t st;
  std::memset(&st, 0, sizeof(st));
  // part shapes: [0, MAX_PARTS) the parts', [MAX_PARTS, 2 MAX_PARTS) their searches',
  // [2 MAX_PARTS] the deferred roots'
  if (!g->part_shape && (rc = dalloc(&g->part_shape, 2 * MAX_PARTS + 1))) return rc;
  if (!g->part_fetch && (rc = dalloc(&g->part_fetch, 8 * (MAX_PARTS + 1)))) return rc;
  if (!g->part_shape_h &&
      cudaHostAlloc((void **)&g->part_shape_h, sizeof(ShapeInfo) * (2 * MAX_PARTS + 1),
                    cudaHostAllocDefault) != cudaSuccess)
    return MCE_ENOMEM;
  for (int p = 0; p < P.k; ++p) {
    if (!g->part_s[p]) MCE_CUDA(cudaStreamCreateWithFlags(&g->part_s[p], cudaStreamNonBlocking));
    if (!g->part_done[p])
      MCE_CUDA(cudaEventCreateWithFlags(&g->part_done[p], cudaEventDisableTiming));
  }
  if (!g->part_fork) MCE_CUDA(cudaEventCreateWithFlags(&g->part_fork, cudaEventDisableTiming));
  std::vector<void *> retired;  // freed after the call's last search
  auto finish = [&](int code) {
    for (int p = 0; p < P.k; ++p) cudaStreamSynchronize(g->part_s[p]);
    cudaStreamSynchronize(s);
    for (void *q : retired) cudaFree(q);
    return code;
  };
  const bool share = o.worker_list != MCE_WL_OFF;
  const bool degree = o.sched == MCE_SCHED_DEGREE;
  const float heavy = (float)(o.heavy_log2 > 0 ? o.heavy_log2 : DEFAULT_HEAVY_LOG2);
  MCE_CUDA(cudaEventRecord(g->ev[0], s));
  MCE_CUDA(cudaMemsetAsync(g->peel_ctl, 0, peel_ctl_bytes(), s));
  MCE_CUDA(cudaMemsetAsync(g->part_fetch, 0, sizeof(uint32_t) * 8 * (MAX_PARTS + 1), s));
  MCE_CUDA(cudaMemsetAsync(bc->graph_count, 0, sizeof(unsigned long long) * bc->G, s));
  MCE_CUDA(cudaMemsetAsync(g->err, 0, sizeof(uint32_t) * 4, s));
  MCE_CUDA(cudaMemsetAsync(g->hist, 0, sizeof(unsigned long long) * MCE_HIST_MAX, s));
  MCE_CUDA(cudaMemsetAsync(g->nodes, 0, sizeof(unsigned long long) * 4, s));
  MCE_CUDA(cudaEventRecord(g->part_fork, s));
  const PeelArgs pa = peel_args(g, o.peel_solo_max);
  int64_t vb[MAX_PARTS + 1];
  for (int p = 0; p <= P.k; ++p) vb[p] = P.vo_h[P.g[p]] - P.g[p];
  // a part's preparation, on its own stream
  auto prep = [&](int p) -> int {
    cudaStream_t sp = g->part_s[p];
    const int64_t g0 = P.g[p], g1 = P.g[p + 1], vbeg = vb[p], vend = vb[p + 1];
    MCE_CUDA(cudaStreamWaitEvent(sp, g->part_fork, 0));
    MCE_CUDA(cudaStreamWaitEvent(sp, P.ready[p], 0));
    if ((rc = batch_rebase_part_launch(P.rp_local, P.col_local, bc->vtx_off, bc->arc_off,
                                       (int32_t)bc->G, P.vo_h[g0], P.vo_h[g1], P.ao_h[g0],
                                       P.ao_h[g1], vend, (int32_t)P.ao_h[g1], g->rp, g->col,
                                       const_cast<int32_t *>(bc->graph_of), g->sms, sp,
                                       &launches)))
      return rc;
    // a part's peel in two launches, its large and middle graphs together:
    // a third launch per part measured slower end to end (53.1 against 51.3 ms)
    PeelSide ps;
    int32_t nbig = 0, nmid = 0;
    if ((rc = seg_side(g, 1 + p, &ps))) return rc;
    if (vend > vbeg &&
        (count_classes(P.vo_h, g0, g1, &nbig, &nmid),
         rc = peel_segments_launch(pa, bc->vtx_off, bc->arc_off, bc->order + g0,
                                   (int32_t)(g1 - g0), nbig + nmid, 0, sp, ps, &launches, p,
                                   part_max_n(P, p))))
      return rc;
    trace_mark(g, sp, "peel", p);
    return MCE_OK;
  };
  // ... then its orientation and root sort
  auto prep_b = [&](int p) -> int {
    cudaStream_t sp = g->part_s[p];
    const int64_t vbeg = vb[p], vend = vb[p + 1];
    OrientArgs oa = orient_args(g);
    oa.v0 = vbeg;
    oa.n = vend;
    oa.shape = g->part_shape + p;
    oa.hub_list = g->hub_list + vbeg;  // hub indices are the part's own
    oa.next = g->orient_next + 2 + 2 * p;
    oa.long_list = reinterpret_cast<int32_t *>(g->keys_out) + vbeg;
    if ((rc = orient_launch(oa, sp, &launches))) return rc;
    const int64_t np = vend - vbeg;
    // keys: class, hubs first, then (degree order) the cost; vertex order
    // within a key (plain order: no cost)
    if (np > 0 && (rc = rekey_launch(np, g->keys_in + vbeg, nullptr, g->rp + vbeg,
                                     g->split + vbeg, nullptr, degree ? heavy : 1e30f,
                                     degree ? heavy : 1e30f, g->sms, sp, &launches, 0,
                                     g->hub_of + vbeg)))
      return rc;
    if ((rc = roots_sort(np, g->keys_in + vbeg, g->keys_out + vbeg, g->vals_in + vbeg,
                         g->roots + vbeg, 32, &g->part_tmp[p], &g->part_tmp_bytes[p],
                         g->part_shape + p, sp, &launches)))
      return rc;
    MCE_CUDA(cudaMemcpyAsync(g->part_shape_h + p, g->part_shape + p, sizeof(ShapeInfo),
                             cudaMemcpyDeviceToHost, sp));
    MCE_CUDA(cudaEventRecord(g->part_done[p], sp));
    trace_mark(g, sp, "prep", p);
    return MCE_OK;
  };
  // The searches, in order on the call's stream.  As each part lands, its
  // 32-bit roots without hub rows are searched (most of the work).  Every
  // other root - the hubs of all classes, the 64-bit and wide classes, whose
  // largest trees set a launch's tail - waits for one search at the end,
  // with one hub table built over all parts: one tail instead of one per part.
  uint32_t err_limit = 0;
  const bool share_q = share;
  const int wbits = o.bitmap_width == 64 ? 64 : 32;
  ShapeInfo *sh_search = g->part_shape + MAX_PARTS;   // [MAX_PARTS]: per-part searches
  ShapeInfo *sh_final = g->part_shape + 2 * MAX_PARTS;
  ShapeInfo *hs_final = g->part_shape_h + 2 * MAX_PARTS;
  struct Seg {
    int64_t at, cnt;
  };
  std::vector<Seg> defer[3];  // by class: R32 hubs, R64, MEM (offsets into g->roots)
  std::vector<Seg> hubsegs;   // the parts' hub lists (offsets into g->hub_list)
  uint64_t hub_rows_total = 0;
  uint32_t mx_dplus = 0, mx_dm_mem = 0, mx_dm_reg = 0, mx_deg = 0;
  // grid, slab and queue of one class launch; returns MCE_OK or an error
  auto plan = [&](int c, int64_t roots, int dcap, int xcap, int rxcap, int *grid, int *block,
                  int *smem, int *parts_c, int *dmin_c, int *dafter_c, QueueView *qv) -> int {
    int r;
    const int w = o.bucket_warps_per_root[c] ? o.bucket_warps_per_root[c] : o.warps_per_root;
    *parts_c = w > 1 && o.level != MCE_LEVEL_L2 ? w : 1;
    const int t = o.bucket_donate_threshold[c] ? o.bucket_donate_threshold[c] : o.donate_threshold;
    *dmin_c = t > 0 ? t : DEFAULT_DONATE_MIN;
    const int af = o.bucket_donate_after[c] ? o.bucket_donate_after[c] : o.donate_after;
    *dafter_c = af > 0 ? af : (int)DEFAULT_DONATE_AFTER;
    int warps = 0;
    if ((r = bk_warps_for_class(c, g->sms, o.wide_blocks, &warps, block, smem))) return r;
    const int wpb = *block / 32;
    int64_t want = roots * *parts_c;
    if (share_q) want = want > warps ? want : warps;
    if (want < warps) warps = (int)((want + wpb - 1) / wpb) * wpb;
    *grid = warps / wpb;
    const size_t need = (size_t)warps * bk_slab_words(c, dcap, xcap, rxcap) * 8;
    if (need > g->slab_bytes) {  // earlier searches of the call keep the old slab
      if (g->slab) retired.push_back(g->slab);
      g->slab = nullptr;
      g->slab_bytes = 0;
      MCE_CUDA(cudaMalloc((void **)&g->slab, need));
      g->slab_bytes = need;
    }
    if (share_q) {
      const uint32_t words = bk_task_words(c, dcap);
      const size_t qneed = 256 + (size_t)QUEUE_CAP * 4 + (size_t)QUEUE_CAP * words * 8;
      if (qneed > g->qbytes[c] && g->qbuf[c]) {  // ensure_queue would free it in use
        retired.push_back(g->qbuf[c]);
        g->qbuf[c] = nullptr;
        g->qbytes[c] = 0;
      }
      if ((r = ensure_queue(g, c, words, qv))) return r;
    }
    return MCE_OK;
  };
  auto base_args = [&](BKArgs &a, int dcap, int xcap, int rxcap) {
    std::memset(&a, 0, sizeof(a));
    a.rp = g->rp;
    a.split = g->split;
    a.cs = g->cs;
    a.hist = g->hist;
    a.nodes = g->nodes;
    a.graph_of = bc->graph_of;
    a.graph_count = bc->graph_count;
    a.err = g->err;
    a.dcap = dcap;
    a.xcap = xcap;
    a.rxcap = rxcap;
    a.wait_limit_ns = o.wait_limit_ms > 0 ? (uint64_t)o.wait_limit_ms * 1000000ull : IDLE_LIMIT_NS;
    a.wide8 = o.wide_blocks == 8 ? 1 : 0;
    a.level2 = o.level == MCE_LEVEL_L2 ? 1 : 0;
    a.prio = g->prio;
    a.x_pivot = (o.x_pivot || o.induced == MCE_INDUCED_PX) ? 1 : 0;
    a.stage = o.stage_lists ? 1 : 0;
  };
  auto run_class = [&](int c, BKArgs &a, int grid, int block, int smem, int parts_c, int dmin_c,
                       int dafter_c, const QueueView &qv, int dcap, int xcap, int rxcap) -> int {
    int r;
    a.slab = g->slab;  // after plan(): the slab may have grown
    a.slab_words = bk_slab_words(c, dcap, xcap, rxcap);
    a.parts = parts_c;
    a.donate_min = dmin_c;
    a.donate_after = (uint32_t)dafter_c;
    a.q = share_q ? qv : QueueView();
    if (share_q && (r = queue_launch_init(a.q, s, &launches))) return r;
    return bk_launch(c, wbits, a, grid, block, smem, s, &launches);
  };
  // a part's search, once its preparation is done
  auto search = [&](int p) -> int {
    MCE_CUDA(cudaEventSynchronize(g->part_done[p]));
    const ShapeInfo sh = g->part_shape_h[p];
    MCE_CUDA(cudaStreamWaitEvent(s, g->part_done[p], 0));
    if (p == 0) MCE_CUDA(cudaEventRecord(g->ev[1], s));
    if (sh.cls_cnt[CLS_BIG]) {
      err_limit = 1;
      return MCE_OK;
    }
    const int64_t vbeg = vb[p];
    // roots of the part, class-sorted, hubs first within a class
    const int64_t n32 = (int64_t)sh.cls_cnt[CLS_R32] - sh.hub_r32;
    defer[0].push_back({vbeg + sh.cls_off[CLS_R32], (int64_t)sh.hub_r32});
    defer[1].push_back({vbeg + sh.cls_off[CLS_R64], (int64_t)sh.cls_cnt[CLS_R64]});
    defer[2].push_back({vbeg + sh.cls_off[CLS_MEM], (int64_t)sh.cls_cnt[CLS_MEM]});
    hubsegs.push_back({vbeg, (int64_t)sh.hub_cnt});
    hub_rows_total += sh.hub_rows;
    mx_dplus = std::max(mx_dplus, sh.max_dplus);
    mx_dm_mem = std::max(mx_dm_mem, sh.max_dminus_mem);
    mx_dm_reg = std::max(mx_dm_reg, sh.max_dminus_reg);
    mx_deg = std::max(mx_deg, sh.max_deg);
    st.roots += (int64_t)sh.cls_cnt[CLS_R32] + sh.cls_cnt[CLS_R64] + sh.cls_cnt[CLS_MEM];
    for (int c = 0; c < NCLS && c < 8; ++c) st.class_roots[c] += sh.cls_cnt[c];
    if ((int32_t)sh.max_dplus > st.max_later_degree) st.max_later_degree = (int32_t)sh.max_dplus;
    if ((int64_t)sh.max_deg > st.max_degree) st.max_degree = sh.max_deg;
    if (n32 <= 0) return MCE_OK;
    // the part's 32-bit roots after its hubs: earlier degree <= HUB_XMIN, no hub rows
    ShapeInfo ss{};
    for (int c = 1; c < 9; ++c) ss.cls_off[c] = (uint32_t)n32;
    ss.cls_cnt[CLS_R32] = (uint32_t)n32;
    // written by a kernel rather than copied from the host on the call's
    // stream, whose copy would share the copy engine with the part copies
    // still in flight (0.3 ms end to end)
    shape_set_kernel<<<1, 32, 0, s>>>(sh_search + p, ss);
    MCE_CUDA(cudaGetLastError());
    launches += 1;
    const int dcap = 32, xcap = 1, rxcap = REG_XCAP;
    int grid = 0, block = 0, smem = 0, pc = 1, dm = 0, da = 0;
    QueueView qv;
    if ((rc = plan(CLS_R32, n32, dcap, xcap, rxcap, &grid, &block, &smem, &pc, &dm, &da, &qv)))
      return rc;
    BKArgs a;
    base_args(a, dcap, xcap, rxcap);
    a.roots = g->roots + vbeg + sh.cls_off[CLS_R32] + sh.hub_r32;
    a.shape = sh_search + p;
    a.fetch = g->part_fetch + 8 * p;
    trace_mark(g, s, "sb", p);
    if ((rc = run_class(CLS_R32, a, grid, block, smem, pc, dm, da, qv, dcap, xcap, rxcap)))
      return rc;
    trace_mark(g, s, "se", p);
    return MCE_OK;
  };
  // Each part's rebase and peel are enqueued once its copy has landed, its
  // orientation and sort once the search before it has ended, and its
  // search once those are done: no stream then waits on an event at the
  // head of a hardware queue that other streams share.
  if (!g->part_sdone) MCE_CUDA(cudaEventCreateWithFlags(&g->part_sdone, cudaEventDisableTiming));
  int na = 0, nb = 0, ns = 0;
  auto ready = [&](cudaEvent_t e, int *bad) {
    const cudaError_t q = cudaEventQuery(e);
    if (q != cudaSuccess && q != cudaErrorNotReady) *bad = 1;
    return q == cudaSuccess;
  };
  int bad = 0;
  while (ns < P.k && !err_limit && !bad) {
    if (na < P.k && ready(P.ready[na], &bad)) {
      if ((rc = prep(na++))) return finish(rc);
      continue;
    }
    if (nb < na && (nb == 0 || (ns == nb && ready(g->part_sdone, &bad)))) {
      if ((rc = prep_b(nb++))) return finish(rc);
      continue;
    }
    if (ns < nb && ready(g->part_done[ns], &bad)) {
      if ((rc = search(ns++))) return finish(rc);
      MCE_CUDA(cudaEventRecord(g->part_sdone, s));
      continue;
    }
    std::this_thread::yield();
  }
  if (bad) return finish(MCE_ECUDA);
  // the deferred roots of every part: one list (R32 hubs, R64, MEM) in the
  // sort's key buffer and one hub list in its value buffer, both free now
  int64_t ncls[3] = {0, 0, 0};
  int32_t *dlist = reinterpret_cast<int32_t *>(g->keys_out);
  int32_t *hlist = g->vals_in;
  if (!err_limit) {
    int64_t at = 0;
    for (int c = 0; c < 3; ++c)
      for (const Seg &sg : defer[c]) {
        if (sg.cnt > 0)
          MCE_CUDA(cudaMemcpyAsync(dlist + at, g->roots + sg.at, sizeof(int32_t) * (size_t)sg.cnt,
                                   cudaMemcpyDeviceToDevice, s));
        at += sg.cnt;
        ncls[c] += sg.cnt;
      }
    trace_mark(g, s, "defer");
    int64_t nh = 0;
    for (const Seg &sg : hubsegs) {
      if (sg.cnt > 0)
        MCE_CUDA(cudaMemcpyAsync(hlist + nh, g->hub_list + sg.at, sizeof(int32_t) * (size_t)sg.cnt,
                                 cudaMemcpyDeviceToDevice, s));
      nh += sg.cnt;
    }
    if (nh > 0) {
      if ((rc = hub_index_launch(hlist, (uint32_t)nh, g->hub_of, s, &launches))) return finish(rc);
      const int64_t need_off = nh + 2, need_rows = (int64_t)hub_rows_total;
      if (need_off > g->hub_off_cap) {
        if (g->hub_off) retired.push_back(g->hub_off);
        if (g->hub_nx) retired.push_back(g->hub_nx);
        g->hub_off = nullptr;
        g->hub_nx = nullptr;
        g->hub_off_cap = 0;
        if ((rc = dalloc(&g->hub_off, (size_t)need_off)) ||
            (rc = dalloc(&g->hub_nx, (size_t)need_off)))
          return finish(rc);
        g->hub_off_cap = need_off;
      }
      if (need_rows > g->hub_rows_cap) {
        if (g->hub_rows) retired.push_back(g->hub_rows);
        g->hub_rows = nullptr;
        g->hub_rows_cap = 0;
        if ((rc = dalloc(&g->hub_rows, (size_t)need_rows))) return finish(rc);
        g->hub_rows_cap = need_rows;
      }
      if ((rc = hub_rows_launch(g->rp, g->split, g->cs, hlist, (uint32_t)nh, need_rows,
                                g->hub_off, g->hub_nx, g->hub_rows, g->sms, s, &launches)))
        return finish(rc);
    }
    trace_mark(g, s, "hubrows");
    const int64_t nd = ncls[0] + ncls[1] + ncls[2];
    if (nd > 0) {
      // the 32-bit hubs run in the 64-bit launch, ahead of its roots: one
      // launch and one tail less (48.1 against 49.3 ms end to end on the
      // 4,096-graph batch; the 64-bit engine takes any root of d+ <= 64)
      const bool fold = ncls[0] > 0 && ncls[1] > 0;
      int64_t nrun[3] = {ncls[0], ncls[1], ncls[2]};
      if (fold) {
        nrun[1] += nrun[0];
        nrun[0] = 0;
      }
      ShapeInfo fs{};
      fs.cls_cnt[CLS_R32] = (uint32_t)nrun[0];
      fs.cls_cnt[CLS_R64] = (uint32_t)nrun[1];
      fs.cls_cnt[CLS_MEM] = (uint32_t)nrun[2];
      fs.cls_off[CLS_R32] = 0;
      fs.cls_off[CLS_R64] = (uint32_t)nrun[0];
      fs.cls_off[CLS_MEM] = (uint32_t)(ncls[0] + ncls[1]);
      for (int c = CLS_MEM + 1; c < 9; ++c) fs.cls_off[c] = (uint32_t)nd;
      hs_final[0] = fs;
      MCE_CUDA(cudaMemcpyAsync(sh_final, hs_final, sizeof(ShapeInfo), cudaMemcpyHostToDevice, s));
      const int dcap = (int)(mx_dplus > 0 ? mx_dplus : 1);
      const int xcap = (int)(mx_dm_mem > 0 ? mx_dm_mem : 1);
      int rxcap = REG_XCAP;
      while (rxcap < (int)mx_dm_reg && rxcap < REG_XCAP_MAX) rxcap <<= 1;
      const int cls_of[3] = {CLS_R32, CLS_R64, CLS_MEM};
      int grid[3] = {0}, block[3] = {0}, smem[3] = {0}, pc[3] = {1, 1, 1}, dm[3] = {0},
          da[3] = {0};
      QueueView qv[3];
      for (int i = 0; i < 3; ++i)
        if (nrun[i] > 0 && (rc = plan(cls_of[i], nrun[i], dcap, xcap, rxcap, &grid[i], &block[i],
                                      &smem[i], &pc[i], &dm[i], &da[i], &qv[i])))
          return finish(rc);
      BKArgs a;
      base_args(a, dcap, xcap, rxcap);
      a.roots = dlist;
      a.shape = sh_final;
      a.fetch = g->part_fetch + 8 * MAX_PARTS;
      a.hub_of = nh > 0 ? g->hub_of : nullptr;
      a.hub_off = g->hub_off;
      a.hub_rows = g->hub_rows;
      a.hub_nx = g->hub_nx;
      for (int i : {2, 1, 0})  // wide, 64-bit, then the 32-bit hubs
        if (nrun[i] > 0 && (rc = run_class(cls_of[i], a, grid[i], block[i], smem[i], pc[i], dm[i],
                                           da[i], qv[i], dcap, xcap, rxcap)))
          return finish(rc);
    }
  }
  trace_mark(g, s, "final");
  MCE_CUDA(cudaEventRecord(g->ev[3], s));
  unsigned long long h_hist[MCE_HIST_MAX];
  unsigned long long h_nodes[2] = {0, 0};
  uint32_t h_err = 0;
  MCE_CUDA(cudaMemcpyAsync(h_hist, g->hist, sizeof(h_hist), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaMemcpyAsync(h_nodes, g->nodes, sizeof(h_nodes), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaMemcpyAsync(&h_err, g->err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaMemcpyAsync(bc->per_graph_out, bc->graph_count,
                           sizeof(unsigned long long) * bc->G, cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaEventRecord(g->ev[4], s));
  finish(MCE_OK);
  int32_t dg = 0;
  uint32_t perr = 0, rounds = 0, solo = 0;
  if (g->n > 0 && (rc = peel_read(g->peel_ctl, &dg, &perr, &rounds, &solo, s, nullptr))) return rc;
  g->degeneracy = dg;
  g->logged = false;
  g->search_key[0] ^= 0xFF;  // buffers may have moved: mce_batch_count captures anew
  if (err_limit) return MCE_ELIMIT;
  uint64_t tot = 0;
  for (int i = 0; i < MCE_HIST_MAX; ++i) tot += h_hist[i];
  *total = tot;
  if (hist)
    for (int i = 0; i < MCE_HIST_MAX; ++i) hist[i] = h_hist[i];
  float ms = 0;
  // overlapped phases: until the first part is oriented, then every search
  cudaEventElapsedTime(&ms, g->ev[0], g->ev[1]);
  st.peel_ms = ms;
  st.orient_ms = 0;
  cudaEventElapsedTime(&ms, g->ev[1], g->ev[3]);
  st.count_ms = ms;
  cudaEventElapsedTime(&ms, g->ev[0], g->ev[4]);
  st.total_ms = ms;
  st.degeneracy = dg;
  st.tree_nodes = h_nodes[0];
  st.kernel_launches = launches;
  st.error_flags = h_err | (perr ? MCE_ERR_WAIT_TIMEOUT : 0);
  st.peel_rounds = rounds;
  st.peel_solo_sections = solo;
  if (stats) *stats = st;
  if (perr) return MCE_ETIMEOUT;
  if (h_err & MCE_ERR_WAIT_TIMEOUT) return MCE_ETIMEOUT;
  if (h_err) return MCE_ELIMIT;
  return MCE_OK;
}

}  // namespace

extern "C" {

int mce_count(mce_graph_t g, const mce_opts_t *opts, uint64_t *total, uint64_t *hist,
              mce_stats_t *stats) {
  if (!g || !total) return MCE_EINVAL;
  mce_opts_t o;
  if (opts)
    o = *opts;
  else
    mce_opts_default(&o);
  return count_impl(g, o, total, hist, stats, nullptr);
}

int mce_list(mce_graph_t g, const mce_opts_t *opts, int32_t *ids_out, int64_t ids_cap,
             int64_t *offsets_out, int64_t cliques_cap, uint64_t *count_out, int64_t *ids_needed) {
  if (!g || !count_out || ids_cap < 0 || cliques_cap < 0 || (ids_cap > 0 && !ids_out) ||
      !offsets_out)
    return MCE_EINVAL;
  mce_opts_t o;
  if (opts)
    o = *opts;
  else
    mce_opts_default(&o);
  MCE_CUDA(cudaSetDevice(g->device));
  // the records hold a size word per clique beside the ids
  const unsigned long long cap = (unsigned long long)ids_cap + (unsigned long long)cliques_cap;
  ListCtx lc{nullptr, nullptr, cap};
  int rc = dalloc(&lc.buf, (size_t)(cap > 0 ? cap : 1));
  if (!rc) rc = dalloc(&lc.words, 1);
  uint64_t total = 0;
  if (!rc) rc = count_impl(g, o, &total, nullptr, nullptr, nullptr, &lc);
  unsigned long long words = 0;
  if (!rc && cudaMemcpy(&words, lc.words, sizeof(words), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = MCE_ECUDA;
  *count_out = total;
  if (ids_needed) *ids_needed = (int64_t)(words - total);
  if (!rc && (words > cap || total > (uint64_t)cliques_cap)) rc = MCE_ELIMIT;
  if (!rc) {
    std::vector<int32_t> h((size_t)words);
    if (words && cudaMemcpy(h.data(), lc.buf, sizeof(int32_t) * (size_t)words,
                            cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = MCE_ECUDA;
    int64_t pos = 0, k = 0;
    for (size_t w = 0; !rc && w < (size_t)words; ++k) {
      const int32_t sz = h[w];
      offsets_out[k] = pos;
      std::memcpy(ids_out + pos, &h[w + 1], sizeof(int32_t) * (size_t)sz);
      pos += sz;
      w += (size_t)sz + 1;
    }
    if (!rc) offsets_out[k] = pos;
  }
  dfree(lc.buf);
  dfree(lc.words);
  return rc;
}

int mce_root_log(mce_graph_t g, uint64_t *nodes_out) {
  if (!g || !nodes_out) return MCE_EINVAL;
  if (!g->logged || !g->root_nodes) return MCE_ESTATE;
  MCE_CUDA(cudaSetDevice(g->device));
  MCE_CUDA(cudaMemcpy(nodes_out, g->root_nodes, sizeof(uint64_t) * (size_t)g->n,
                      cudaMemcpyDeviceToHost));
  return MCE_OK;
}

int mce_warp_log(mce_graph_t g, uint32_t *sm_out, uint64_t *nodes_out, uint64_t *donations_out,
                 uint64_t *cycles_out, int64_t cap, int64_t *count_out) {
  if (!g || cap < 0) return MCE_EINVAL;
  if (count_out) *count_out = g->wlog_count;
  const int64_t k = cap < g->wlog_count ? cap : g->wlog_count;
  if (k == 0) return MCE_OK;
  MCE_CUDA(cudaSetDevice(g->device));
  std::vector<unsigned long long> h(WLOG_WORDS * (size_t)k);
  MCE_CUDA(cudaMemcpy(h.data(), g->wlog, sizeof(unsigned long long) * WLOG_WORDS * (size_t)k,
                      cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < k; ++i) {
    const unsigned long long *r = &h[WLOG_WORDS * (size_t)i];
    if (sm_out) sm_out[i] = (uint32_t)r[0];
    if (nodes_out) nodes_out[i] = r[1];
    if (donations_out) donations_out[i] = r[2];
    if (cycles_out)
      for (int p = 0; p < 7; ++p) cycles_out[7 * i + p] = r[3 + p];
  }
  return MCE_OK;
}

int mce_root_ops(mce_graph_t g, uint64_t *ops_out) {
  if (!g || !ops_out) return MCE_EINVAL;
  if (!g->logged_ops || !g->root_ops) return MCE_ESTATE;
  MCE_CUDA(cudaSetDevice(g->device));
  MCE_CUDA(cudaMemcpy(ops_out, g->root_ops, sizeof(uint64_t) * (size_t)g->n,
                      cudaMemcpyDeviceToHost));
  return MCE_OK;
}

int mce_root_counts(mce_graph_t g, uint64_t *count_out) {
  if (!g || !count_out) return MCE_EINVAL;
  if (!g->logged || !g->root_count) return MCE_ESTATE;
  MCE_CUDA(cudaSetDevice(g->device));
  MCE_CUDA(cudaMemcpy(count_out, g->root_count, sizeof(uint64_t) * (size_t)g->n,
                      cudaMemcpyDeviceToHost));
  return MCE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches of graphs
// ---------------------------------------------------------------------------
struct mce_batch {
  mce_graph *g = nullptr;  // the disjoint union, resident
  int32_t G = 0;
  int32_t *graph_of = nullptr;
  unsigned long long *graph_count = nullptr;
  int32_t *rp_local = nullptr, *col_local = nullptr;  // uploaded concatenations
  int64_t *vtx_off = nullptr, *arc_off = nullptr;
  int32_t *order = nullptr;    // graph ids by arc count, largest first (per-graph peel)
  int32_t *order_h = nullptr;  // its pinned host staging copy
  int64_t cap_rows = -1, cap_m = -1, cap_g = -1;
  int64_t max_n = 0;           // the most vertices of a graph of the batch
  int32_t g_big = 0, g_mid = 0;  // its graphs in the large and middle peel classes
  // mce_batch_count_host: copies on their own stream, one event per part
  cudaStream_t copy = nullptr;
  cudaEvent_t start = nullptr, ready[MAX_PARTS] = {nullptr};
};

namespace {

int batch_check(const int32_t *row_ptr, const int32_t *col, const int64_t *vo, const int64_t *ao,
                int32_t G, int64_t *n, int64_t *m) {
  if (G < 1 || !row_ptr || !vo || !ao) return MCE_EINVAL;
  if (vo[0] != 0 || ao[0] != 0) return MCE_EINVAL;
  for (int32_t g = 0; g < G; ++g)
    if (vo[g + 1] < vo[g] + 1 || ao[g + 1] < ao[g]) return MCE_EINVAL;
  *n = vo[G] - G;
  *m = ao[G];
  if (*m > 0 && !col) return MCE_EINVAL;
  if (*n >= ((int64_t)1 << 31) - 1 || *m >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  return MCE_OK;
}

void batch_free_bufs(mce_batch *b) {
  dfree(b->graph_of);
  dfree(b->graph_count);
  dfree(b->rp_local);
  dfree(b->col_local);
  dfree(b->vtx_off);
  dfree(b->arc_off);
  dfree(b->order);
  if (b->order_h) cudaFreeHost(b->order_h);
  b->order_h = nullptr;
  b->cap_rows = b->cap_m = b->cap_g = -1;
}

// Device buffers for a batch of G graphs, n vertices and m arcs.
int batch_alloc(mce_batch *b, int32_t G, int64_t n, int64_t m) {
  mce_graph *g = b->g;
  int rc;
  if (n > g->cap_n || m > g->cap_m) {
    if ((rc = alloc_graph_bufs(g, n, m))) return rc;
  }
  const int64_t rows = n + G;
  if (rows > b->cap_rows || m > b->cap_m || G > b->cap_g) {
    batch_free_bufs(b);
    if ((rc = dalloc(&b->graph_of, (size_t)n + 1)) || (rc = dalloc(&b->graph_count, (size_t)G)) ||
        (rc = dalloc(&b->rp_local, (size_t)rows)) || (rc = dalloc(&b->col_local, (size_t)m)) ||
        (rc = dalloc(&b->vtx_off, (size_t)G + 1)) || (rc = dalloc(&b->arc_off, (size_t)G + 1)) ||
        (rc = dalloc(&b->order, (size_t)G)))
      return rc;
    if (cudaHostAlloc((void **)&b->order_h, sizeof(int32_t) * (size_t)G, cudaHostAllocDefault) !=
        cudaSuccess)
      return MCE_ENOMEM;
    b->cap_rows = rows;
    b->cap_m = m;
    b->cap_g = G;
  }
  b->G = G;
  g->n = n;
  g->m = m;
  g->logged = false;
  return MCE_OK;
}

int batch_load(mce_batch *b, const int32_t *row_ptr, const int32_t *col, const int64_t *vo,
               const int64_t *ao, int32_t G, int64_t n, int64_t m, cudaStream_t s) {
  mce_graph *g = b->g;
  int rc = batch_alloc(b, G, n, m);
  if (rc) return rc;
  const int64_t rows = n + G;
  MCE_CUDA(cudaMemcpyAsync(b->rp_local, row_ptr, sizeof(int32_t) * (size_t)rows,
                           cudaMemcpyHostToDevice, s));
  if (m > 0)
    MCE_CUDA(cudaMemcpyAsync(b->col_local, col, sizeof(int32_t) * (size_t)m,
                             cudaMemcpyHostToDevice, s));
  MCE_CUDA(cudaMemcpyAsync(b->vtx_off, vo, sizeof(int64_t) * (size_t)(G + 1),
                           cudaMemcpyHostToDevice, s));
  MCE_CUDA(cudaMemcpyAsync(b->arc_off, ao, sizeof(int64_t) * (size_t)(G + 1),
                           cudaMemcpyHostToDevice, s));
  // the previous call's copy out of order_h finished before that call returned
  int32_t *order = b->order_h;
  for (int32_t i = 0; i < G; ++i) order[i] = i;
  b->max_n = 0;
  for (int32_t i = 0; i < G; ++i) b->max_n = std::max<int64_t>(b->max_n, vo[i + 1] - vo[i] - 1);
  order_graphs(order, 0, G, vo, ao);
  count_classes(vo, 0, G, &b->g_big, &b->g_mid);
  MCE_CUDA(cudaMemcpyAsync(b->order, order, sizeof(int32_t) * (size_t)G, cudaMemcpyHostToDevice,
                           s));
  return batch_rebase_launch(b->rp_local, b->col_local, b->vtx_off, b->arc_off, G, n, m, g->rp,
                             g->col, b->graph_of, g->sms, s, nullptr);
}

}  // namespace

extern "C" {

int mce_batch_upload(const int32_t *row_ptr, const int32_t *col, const int64_t *vtx_offsets,
                     const int64_t *arc_offsets, int32_t num_graphs, int32_t device,
                     void *stream, mce_batch_t *out) {
  if (!out) return MCE_EINVAL;
  *out = nullptr;
  int64_t n = 0, m = 0;
  int rc = batch_check(row_ptr, col, vtx_offsets, arc_offsets, num_graphs, &n, &m);
  if (rc) return rc;
  mce_batch *b = new (std::nothrow) mce_batch();
  if (!b) return MCE_ENOMEM;
  if ((rc = graph_create(device, &b->g))) {
    delete b;
    return rc;
  }
  cudaStream_t s = pick_stream(b->g, stream);
  rc = batch_load(b, row_ptr, col, vtx_offsets, arc_offsets, num_graphs, n, m, s);
  if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = MCE_ECUDA;
  if (rc) {
    mce_batch_free(b);
    return rc;
  }
  *out = b;
  return MCE_OK;
}

int mce_batch_reload(mce_batch_t b, const int32_t *row_ptr, const int32_t *col,
                     const int64_t *vtx_offsets, const int64_t *arc_offsets, int32_t num_graphs,
                     void *stream) {
  if (!b) return MCE_EINVAL;
  int64_t n = 0, m = 0;
  int rc = batch_check(row_ptr, col, vtx_offsets, arc_offsets, num_graphs, &n, &m);
  if (rc) return rc;
  MCE_CUDA(cudaSetDevice(b->g->device));
  return batch_load(b, row_ptr, col, vtx_offsets, arc_offsets, num_graphs, n, m,
                    pick_stream(b->g, stream));
}

}  // extern "C"

namespace mce {
struct ::mce_graph *batch_union(struct ::mce_batch *b, int32_t *num_graphs) {
  if (!b) return nullptr;
  if (num_graphs) *num_graphs = b->G;
  return b->g;
}
}  // namespace mce

extern "C" {

int mce_batch_count(mce_batch_t b, const mce_opts_t *opts, uint64_t *per_graph_total,
                    uint64_t *total, uint64_t *hist, mce_stats_t *stats) {
  if (!b || !total || !per_graph_total) return MCE_EINVAL;
  mce_opts_t o;
  if (opts)
    o = *opts;
  else {
    mce_opts_default(&o);
    o.cuda_graph = 1;
  }
  BatchCtx bc{b->graph_of, b->graph_count, per_graph_total, b->G, b->vtx_off, b->arc_off, b->order};
  bc.max_n = b->max_n;
  bc.g_big = b->g_big;
  bc.g_mid = b->g_mid;
  return count_impl(b->g, o, total, hist, stats, &bc);
}

int mce_batch_count_host(mce_batch_t b, const int32_t *row_ptr, const int32_t *col,
                         const int64_t *vtx_offsets, const int64_t *arc_offsets,
                         int32_t num_graphs, const mce_opts_t *opts, uint64_t *per_graph_total,
                         uint64_t *total, uint64_t *hist, mce_stats_t *stats) {
  if (!b || !total || !per_graph_total) return MCE_EINVAL;
  int64_t n = 0, m = 0;
  int rc = batch_check(row_ptr, col, vtx_offsets, arc_offsets, num_graphs, &n, &m);
  if (rc) return rc;
  mce_opts_t o;
  if (opts) {
    o = *opts;
  } else {
    mce_opts_default(&o);
    o.cuda_graph = 1;
  }
  const int32_t G = num_graphs;
  const int64_t *vo = vtx_offsets, *ao = arc_offsets;
  // Parts of whole graphs; small batches in one.  When the parts are
  // searched as they arrive, they grow (2, 4, 7, 11, 16 and 24 64ths of the
  // arcs): the first search starts after a short copy, and since the copy
  // moves arcs faster than the narrow roots are searched, each part lands
  // before the search stream reaches it; parts growing 2x per step left the
  // stream waiting for the last ones, and 3, 5, 8, 12, 16, 20 measured
  // 0.3 ms slower end to end.  Otherwise they are equal.
  const bool pipelined = !o.log_roots && !o.warp_log && !o.count_ops &&
                         (o.sched == MCE_SCHED_PLAIN || o.sched == MCE_SCHED_DEGREE);
  static const int64_t kGeo[MAX_PARTS] = {2, 6, 13, 24, 40, 64};  // cumulative 64ths
  int k = m >= BATCH_PART_MIN_ARCS ? MAX_PARTS : 1;
  if (k > G) k = G;
  BatchParts P;
  P.k = 0;
  P.g[0] = 0;
  for (int p = 1; p < k; ++p) {
    int64_t gp = P.g[P.k];
    const int64_t want = pipelined && k == MAX_PARTS ? m * kGeo[p - 1] / 64 : m * p / k;
    while (gp < G && ao[gp] < want) ++gp;
    if (gp > P.g[P.k] && gp < G) P.g[++P.k] = gp;
  }
  P.g[++P.k] = G;
  if (P.k == 1)
    return (rc = mce_batch_reload(b, row_ptr, col, vo, ao, G, o.stream)) ? rc
           : mce_batch_count(b, &o, per_graph_total, total, hist, stats);
  MCE_CUDA(cudaSetDevice(b->g->device));
  cudaStream_t s = pick_stream(b->g, o.stream);
  if ((rc = batch_alloc(b, G, n, m))) return rc;
  if (!b->copy) MCE_CUDA(cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking));
  if (!b->start) MCE_CUDA(cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming));
  for (int p = 0; p < MAX_PARTS; ++p)
    if (!b->ready[p]) MCE_CUDA(cudaEventCreateWithFlags(&b->ready[p], cudaEventDisableTiming));
  // graphs largest first within each part (the per-graph peel's order)
  int32_t *order = b->order_h;
  for (int32_t i = 0; i < G; ++i) order[i] = i;
  b->max_n = 0;
  for (int32_t i = 0; i < G; ++i) b->max_n = std::max<int64_t>(b->max_n, vo[i + 1] - vo[i] - 1);
  for (int p = 0; p < P.k; ++p) order_graphs(order, P.g[p], P.g[p + 1], vo, ao);
  b->g_big = G;  // the order is per part now: a later resident count peels all in one launch
  b->g_mid = 0;
  // the copies wait for earlier work on the caller's stream, then run on
  // their own stream while the caller's stream processes the parts already
  // on the device
  {
    const char *tr = getenv("MCE_TRACE_PARTS");
    b->g->trace_n = tr && *tr && *tr != '0' ? 0 : -1;
  }
  trace_mark(b->g, s, "start");
  MCE_CUDA(cudaEventRecord(b->start, s));
  MCE_CUDA(cudaStreamWaitEvent(b->copy, b->start, 0));
  MCE_CUDA(cudaMemcpyAsync(b->vtx_off, vo, sizeof(int64_t) * (size_t)(G + 1),
                           cudaMemcpyHostToDevice, b->copy));
  MCE_CUDA(cudaMemcpyAsync(b->arc_off, ao, sizeof(int64_t) * (size_t)(G + 1),
                           cudaMemcpyHostToDevice, b->copy));
  MCE_CUDA(cudaMemcpyAsync(b->order, order, sizeof(int32_t) * (size_t)G, cudaMemcpyHostToDevice,
                           b->copy));
  for (int p = 0; p < P.k; ++p) {
    const int64_t r0 = vo[P.g[p]], r1 = vo[P.g[p + 1]], a0 = ao[P.g[p]], a1 = ao[P.g[p + 1]];
    MCE_CUDA(cudaMemcpyAsync(b->rp_local + r0, row_ptr + r0, sizeof(int32_t) * (size_t)(r1 - r0),
                             cudaMemcpyHostToDevice, b->copy));
    if (a1 > a0)
      MCE_CUDA(cudaMemcpyAsync(b->col_local + a0, col + a0, sizeof(int32_t) * (size_t)(a1 - a0),
                               cudaMemcpyHostToDevice, b->copy));
    MCE_CUDA(cudaEventRecord(b->ready[p], b->copy));
    trace_mark(b->g, b->copy, "copy", p);
    P.ready[p] = b->ready[p];
  }
  P.rp_local = b->rp_local;
  P.col_local = b->col_local;
  P.vo_h = vo;
  P.ao_h = ao;
  BatchCtx bc{b->graph_of, b->graph_count, per_graph_total, b->G, b->vtx_off, b->arc_off, b->order};
  bc.parts = &P;
  bc.max_n = b->max_n;
  bc.g_big = b->g_big;
  bc.g_mid = b->g_mid;
  rc = pipelined ? count_pipelined(b->g, o, total, hist, stats, &bc)
                 : count_impl(b->g, o, total, hist, stats, &bc);
  trace_dump(b->g);
  if (rc) cudaStreamSynchronize(b->copy);  // no copy outlives a failed call
  return rc;
}

int mce_batch_free(mce_batch_t b) {
  if (!b) return MCE_OK;
  if (b->g) {
    cudaSetDevice(b->g->device);
    cudaStreamSynchronize(b->g->own);
    if (b->copy) {
      cudaStreamSynchronize(b->copy);
      cudaStreamDestroy(b->copy);
    }
    if (b->start) cudaEventDestroy(b->start);
    for (cudaEvent_t e : b->ready)
      if (e) cudaEventDestroy(e);
  }
  batch_free_bufs(b);
  if (b->g) mce_graph_free(b->g);
  delete b;
  return MCE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Cost model
// ---------------------------------------------------------------------------
namespace {

int model_upload(mce_model *m, const float *params) {
  std::vector<__half> h(MLP_PARAMS);
  for (int i = 0; i < MLP_PARAMS; ++i) h[i] = __float2half_rn(params[i]);
  MCE_CUDA(cudaMemcpyAsync(m->master, params, sizeof(float) * MLP_PARAMS, cudaMemcpyHostToDevice,
                           m->own));
  MCE_CUDA(cudaMemcpyAsync(m->wh, h.data(), sizeof(__half) * MLP_PARAMS, cudaMemcpyHostToDevice,
                           m->own));
  MCE_CUDA(cudaMemsetAsync(m->m1, 0, sizeof(float) * MLP_PARAMS, m->own));
  MCE_CUDA(cudaMemsetAsync(m->m2, 0, sizeof(float) * MLP_PARAMS, m->own));
  MCE_CUDA(cudaMemsetAsync(m->grad, 0, sizeof(float) * MLP_PARAMS, m->own));
  MCE_CUDA(cudaStreamSynchronize(m->own));
  m->step = 0;
  return MCE_OK;
}

}  // namespace

extern "C" {

int mce_model_create(int32_t device, uint64_t seed, mce_model_t *out) {
  if (!out) return MCE_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MCE_ENODEV;
  if (device < 0 || device >= ndev) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(device));
  mce_model *m = new (std::nothrow) mce_model();
  if (!m) return MCE_ENOMEM;
  m->device = device;
  int rc;
  if (cudaStreamCreateWithFlags(&m->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    delete m;
    return MCE_ECUDA;
  }
  if ((rc = dalloc(&m->master, MLP_PARAMS)) || (rc = dalloc(&m->grad, MLP_PARAMS)) ||
      (rc = dalloc(&m->m1, MLP_PARAMS)) || (rc = dalloc(&m->m2, MLP_PARAMS)) ||
      (rc = dalloc(&m->loss, 4)) || (rc = dalloc(&m->wh, MLP_PARAMS))) {
    mce_model_free(m);
    return rc;
  }
  // He-uniform weights, zero biases (seeded)
  std::vector<float> p(MLP_PARAMS, 0.f);
  mce::Rng rng(seed, 0x4d4c50ull);
  const int F = MLP_IN, H = MLP_HIDDEN;
  auto fill = [&](int off, int count, float fan_in) {
    const float lim = std::sqrt(6.0f / fan_in);
    for (int i = 0; i < count; ++i) p[off + i] = (float)((rng.uniform() * 2.0 - 1.0) * lim);
  };
  fill(0, H * F, (float)F);
  fill(H * F + H, H * H, (float)H);
  fill(H * F + H + H * H + H, H, (float)H);
  if ((rc = model_upload(m, p.data()))) {
    mce_model_free(m);
    return rc;
  }
  *out = m;
  return MCE_OK;
}

int mce_model_free(mce_model_t m) {
  if (!m) return MCE_OK;
  cudaSetDevice(m->device);
  if (m->own) cudaStreamSynchronize(m->own);
  dfree(m->master);
  dfree(m->grad);
  dfree(m->m1);
  dfree(m->m2);
  dfree(m->loss);
  dfree(m->wh);
  if (m->own) cudaStreamDestroy(m->own);
  delete m;
  return MCE_OK;
}

int mce_model_set(mce_model_t m, const float *params) {
  if (!m || !params) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(m->device));
  return model_upload(m, params);
}

int mce_model_get(mce_model_t m, float *params_out, uint16_t *fp16_out) {
  if (!m || (!params_out && !fp16_out)) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(m->device));
  if (params_out)
    MCE_CUDA(cudaMemcpyAsync(params_out, m->master, sizeof(float) * MLP_PARAMS,
                             cudaMemcpyDeviceToHost, m->own));
  if (fp16_out)
    MCE_CUDA(cudaMemcpyAsync(fp16_out, m->wh, sizeof(uint16_t) * MLP_PARAMS,
                             cudaMemcpyDeviceToHost, m->own));
  MCE_CUDA(cudaStreamSynchronize(m->own));
  return MCE_OK;
}

int mce_root_features(mce_graph_t g, float *features_out) {
  if (!g) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = g->own;
  int launches = 0, rc;
  if ((rc = run_peel(g, s, &launches)) || (rc = run_orient(g, s, &launches)) ||
      (rc = compute_features(g, s, &launches, true)))
    return rc;
  if (features_out && g->n)
    MCE_CUDA(cudaMemcpyAsync(features_out, g->feat, sizeof(float) * MLP_IN * (size_t)g->n,
                             cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  return MCE_OK;
}

int mce_model_train(mce_model_t m, mce_graph_t g, int32_t epochs, int32_t batch, float lr,
                    uint64_t seed, float *loss_out) {
  if (!m || !g || epochs < 1 || batch < 1 || !(lr > 0.f)) return MCE_EINVAL;
  if (m->device != g->device) return MCE_EINVAL;
  if (!g->logged || !g->root_nodes) return MCE_ESTATE;  // needs a count with log_roots = 1
  MCE_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = m->own;
  // the logged tree sizes belong to the current orientation; recompute features for it
  std::vector<unsigned long long> nodes((size_t)g->n);
  MCE_CUDA(cudaMemcpy(nodes.data(), g->root_nodes, sizeof(unsigned long long) * (size_t)g->n,
                      cudaMemcpyDeviceToHost));
  int rc = mce_root_features(g, nullptr);
  if (rc) return rc;
  std::vector<int32_t> split((size_t)g->n), rp((size_t)g->n + 1);
  MCE_CUDA(cudaMemcpy(split.data(), g->split, sizeof(int32_t) * (size_t)g->n,
                      cudaMemcpyDeviceToHost));
  MCE_CUDA(cudaMemcpy(rp.data(), g->rp, sizeof(int32_t) * (size_t)(g->n + 1),
                      cudaMemcpyDeviceToHost));
  std::vector<int32_t> idx;
  std::vector<float> y((size_t)g->n, 0.f);
  for (int64_t v = 0; v < g->n; ++v)
    if (nodes[v] && rp[v + 1] - split[v] >= MLP_MIN_LATER) {  // the roots the model ranks
      idx.push_back((int32_t)v);
      y[v] = std::log2(1.0f + (float)nodes[v]);
    }
  const int64_t N = (int64_t)idx.size();
  if (N == 0) return MCE_EINVAL;
  float *dy = nullptr;
  int32_t *didx = nullptr;
  if ((rc = dalloc(&dy, (size_t)g->n)) || (rc = dalloc(&didx, (size_t)N))) {
    dfree(dy);
    return rc;
  }
  MCE_CUDA(cudaMemcpyAsync(dy, y.data(), sizeof(float) * (size_t)g->n, cudaMemcpyHostToDevice, s));
  mce::Rng rng(seed, 0x5452ull);
  for (int e = 0; e < epochs && !rc; ++e) {
    for (int64_t i = N - 1; i > 0; --i) std::swap(idx[i], idx[(int64_t)rng.below(i + 1)]);
    if (cudaMemcpyAsync(didx, idx.data(), sizeof(int32_t) * (size_t)N, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(m->loss, 0, sizeof(float), s) != cudaSuccess) {
      rc = MCE_ECUDA;
      break;
    }
    for (int64_t b = 0; b < N && !rc; b += batch) {
      const int64_t end = std::min<int64_t>(N, b + batch);
      rc = mlp_grad_launch(m->wh, g->feat, dy, didx, b, end, m->grad, m->loss, s);
      if (!rc) rc = mlp_adam_launch(m->master, m->wh, m->grad, m->m1, m->m2, lr, ++m->step, s);
    }
    float l = 0.f;
    if (!rc && cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess) {
      if (loss_out) loss_out[e] = l / (float)N;
    } else if (!rc) {
      rc = MCE_ECUDA;
    }
  }
  cudaStreamSynchronize(s);
  dfree(dy);
  dfree(didx);
  return rc;
}

int mce_model_predict(mce_model_t m, mce_graph_t g, float *pred_out) {
  if (!m || !g) return MCE_EINVAL;
  if (m->device != g->device) return MCE_EINVAL;
  int rc = mce_root_features(g, nullptr);
  if (rc) return rc;
  cudaStream_t s = g->own;
  if ((rc = predict_candidates(g, m->wh, s, nullptr))) return rc;
  if (pred_out && g->n)
    MCE_CUDA(cudaMemcpyAsync(pred_out, g->pred, sizeof(float) * (size_t)g->n,
                             cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  return MCE_OK;
}

int mce_model_eval(mce_model_t m, const float *X, int64_t count, float *out) {
  if (!m || count < 0 || (count > 0 && (!X || !out))) return MCE_EINVAL;
  if (count == 0) return MCE_OK;
  MCE_CUDA(cudaSetDevice(m->device));
  float *dx = nullptr, *dout = nullptr;
  int rc;
  if ((rc = dalloc(&dx, (size_t)count * MLP_IN)) || (rc = dalloc(&dout, (size_t)count))) {
    dfree(dx);
    return rc;
  }
  cudaStream_t s = m->own;
  if (cudaMemcpyAsync(dx, X, sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    rc = MCE_ECUDA;
  if (!rc) rc = mlp_forward_launch(m->wh, dx, nullptr, nullptr, count, dout, m->sms, s, nullptr);
  if (!rc && (cudaMemcpyAsync(out, dout, sizeof(float) * (size_t)count, cudaMemcpyDeviceToHost,
                              s) != cudaSuccess ||
              cudaStreamSynchronize(s) != cudaSuccess))
    rc = MCE_ECUDA;
  dfree(dx);
  dfree(dout);
  return rc;
}

int mce_model_grad(mce_model_t m, const float *X, const float *Y, int64_t count, float *grad_out,
                   float *loss_out) {
  if (!m || count < 1 || !X || !Y || !grad_out) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(m->device));
  float *dx = nullptr, *dy = nullptr;
  int rc;
  if ((rc = dalloc(&dx, (size_t)count * MLP_IN)) || (rc = dalloc(&dy, (size_t)count))) {
    dfree(dx);
    return rc;
  }
  cudaStream_t s = m->own;
  float l = 0.f;
  if (cudaMemcpyAsync(dx, X, sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(dy, Y, sizeof(float) * (size_t)count, cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemsetAsync(m->grad, 0, sizeof(float) * MLP_PARAMS, s) != cudaSuccess ||
      cudaMemsetAsync(m->loss, 0, sizeof(float), s) != cudaSuccess)
    rc = MCE_ECUDA;
  if (!rc) rc = mlp_grad_launch(m->wh, dx, dy, nullptr, 0, count, m->grad, m->loss, s);
  if (!rc && (cudaMemcpyAsync(grad_out, m->grad, sizeof(float) * MLP_PARAMS,
                              cudaMemcpyDeviceToHost, s) != cudaSuccess ||
              cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s) !=
                  cudaSuccess ||
              cudaMemsetAsync(m->grad, 0, sizeof(float) * MLP_PARAMS, s) != cudaSuccess ||
              cudaStreamSynchronize(s) != cudaSuccess))
    rc = MCE_ECUDA;
  if (loss_out) *loss_out = l / (float)count;
  dfree(dx);
  dfree(dy);
  return rc;
}

}  // extern "C"
