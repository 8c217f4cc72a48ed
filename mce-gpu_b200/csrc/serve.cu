// Serving: a device-resident request loop over a resident graph.
//
// No counterpart in the reference, which runs one graph per process
// (src/main.cu).  A request is a seed vertex; its answer is the number of
// maximal cliques (size >= 2) of the seed's 2-hop ego subgraph: the seed,
// its neighbours in row order, then 2-hop vertices in discovery order, at
// most `ego_cap` vertices, relabelled in ascending id order
// (mce_ego_subgraph builds the same graph on the host).
//
// Persistent kernels serve a session.  Each block is a slot: it claims the
// next published request, extracts the ego subgraph into its own arena,
// peels and orients it with block barriers (the same synchronous rounds and
// orientation rule as peel.cu / orient.cu), searches its roots with its
// warps (the engines of engine.cuh) and writes the count back to mapped
// host memory.  Requests that arrive while others run are taken by
// whichever slot frees first, so unrelated requests overlap on the device:
// continuous batching at request granularity with no launch per request.
// Two slot classes, one kernel each: class 0, 1,024-thread blocks, takes
// any request; class 1, 256-thread blocks (four in the room of one class-0
// block), takes the requests whose footprint bound (deg(seed) + the sum of
// its neighbours' degrees + 1) fits its smaller cap, which the host routes
// there while every class-0 slot holds a request.  Each class has its own
// ring; class-0 slots also take class-1 requests when their ring is empty.
//
// Ring protocol (mapped pinned host memory): the host writes entry
// id % ring, then releases `tail` = id + 1.  On the device one waiting
// thread at a time (the poller duty, at most every SV_POLL_NS) reads the
// host tail and stop flag over the bus and mirrors them into device memory;
// waiting slots watch the mirror and claim with a CAS on `next` only when a
// request is published, so a slot that leaves never holds an unserved
// request.  A slot with nothing to do for `idle_ms` leaves; the host
// relaunches the kernel when requests are pending and no slot is left.
// Every device wait is bounded.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "kernels.h"

namespace mce {

namespace {

// 32 warps per slot: a large request's block-wide phases (extraction, peel)
// take half the windows of 512 threads.  Measured on the 4e6-vertex BA trace
// at 2,000 req/s: p99 4.27 ms (512 threads: 4.80 ms), burst capacity 130 k
// req/s (143 k; the search inside a slot spills at 64 registers).
constexpr int SV_BLOCK = 1024;
constexpr int SV_WARPS = SV_BLOCK / 32;
// Small requests (their footprint bound fits the class-1 cap) run in
// 256-thread blocks: four at once in the room of one whole-block slot.
constexpr int SV_SMALL = 256;
constexpr int SV_DCAP = 256;            // widest root (later neighbours) a slot searches
// The host tail of ring 0 is read at most every SV_POLL_NS, ring 1's every
// 4 x SV_POLL_NS (at 500 ns both, the bus reads of the second ring cost
// 0.04 ms of median latency at 2,000 requests/s; ring 1 fills under load,
// when 2 us is small beside a request's service time).
constexpr uint64_t SV_POLL_NS = 500;
constexpr int SV_MAX_EGO = 16384;
constexpr int SV_RUN = 4;  // consecutive positions a thread takes per window of the extraction passes

struct SvEntry {             // one request, in mapped host memory
  int64_t seed;              // host -> device
  unsigned long long count;  // device -> host
  unsigned long long device_ns;
  int32_t status, ego_n, ego_arcs;
  uint32_t limits;           // MCE_ERR_* bits of the limits the request hit
  uint32_t done;             // id + 1 once the answer is written
  uint32_t extract_ns, order_ns, search_ns;  // the request's phases on the slot
};

struct SvHostHdr {           // mapped host memory, host-written
  uint32_t tail;
  uint32_t pad0[15];
  uint32_t stop;
  uint32_t pad1[15];
};

struct SvCtl {               // device memory
  uint32_t next, dtail, dstop;
  uint32_t board_n;          // entries on the help board (class 0's counts them)
  unsigned long long poll_ns, served, nodes, helped;
  unsigned long long inflight, peak;  // requests on the device (class 0's counts both classes)
};

// The root work of a slot's current request, shared with helping slots.
struct SvHelp {
  uint32_t state;            // SV_OPEN | number of helping slots inside
  uint32_t rootnext;         // next root (ego vertex) to search
  int32_t n;                 // roots
  uint32_t pad;
  unsigned long long total, nodes;
};
constexpr uint32_t SV_OPEN = 0x80000000u;
constexpr int SV_BOARD = 64;                  // requests open for help at a time
constexpr int SV_HELP_MIN = 1024;             // roots from which a request takes helpers
constexpr uint32_t SV_HELP = 0x40000000u;     // claim(): help slot (value & 0xFFFFFF)
constexpr uint64_t SV_HELP_WAIT_NS = 60ull * 1000 * 1000 * 1000;

// A class of slots with its own request ring and arenas: class 0, whole
// blocks, takes requests of any footprint up to ego_cap vertices; class 1,
// 256-thread quarters of blocks, the requests whose footprint bound fits its
// smaller cap (the host routes each request by it).
struct SvClass {
  const SvHostHdr *hdr;       // device views of the class's mapped ring
  SvEntry *ent;
  uint32_t ring;
  SvCtl *ctl;
  char *arena;                // per-slot ego-graph arenas
  size_t arena_bytes;
  int32_t ego_cap, arc_cap, hcap;
  int32_t slots;
  unsigned long long *slab;   // per-warp engine scratch of the class's kernel, by block and warp
};

struct ServeArgs {
  const int32_t *grp, *gcol;  // resident graph
  int64_t gn;
  SvClass cls[2];
  size_t slab_words, reg_words;  // per warp: register engines' part, then the wide engine's
  uint64_t idle_ns;
  unsigned long long node_budget;  // per request; 0: none
  SvHelp *help;                    // per class-0 slot
  uint32_t *board;                 // slot + 1 of requests open for help (0: empty)
};

struct Arena {
  int32_t *hkey, *hval, *hfirst, *V, *rp, *col, *split, *cs, *deg, *core, *fa, *fb, *off;
  int32_t *rs;  // resident-row start of each row being walked (row_offsets)
  uint32_t *prio, *err;
  unsigned long long *hist;  // clique sizes above the engines' register bins
};

__host__ __device__ inline size_t arena_layout(int ego_cap, int arc_cap, int hcap, char *base,
                                               Arena *a) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *p = base ? base + off : nullptr;
    off += (bytes + 255) & ~(size_t)255;
    return p;
  };
  Arena x;
  x.hkey = (int32_t *)take(4 * (size_t)hcap);
  x.hval = (int32_t *)take(4 * (size_t)hcap);
  x.hfirst = (int32_t *)take(4 * (size_t)hcap);
  x.V = (int32_t *)take(4 * (size_t)ego_cap);
  x.rp = (int32_t *)take(4 * ((size_t)ego_cap + 1));
  x.col = (int32_t *)take(4 * (size_t)arc_cap);
  x.split = (int32_t *)take(4 * (size_t)ego_cap);
  x.cs = (int32_t *)take(4 * (size_t)arc_cap);
  x.deg = (int32_t *)take(4 * (size_t)ego_cap);
  x.core = (int32_t *)take(4 * (size_t)ego_cap);
  x.fa = (int32_t *)take(4 * (size_t)ego_cap);
  x.fb = (int32_t *)take(4 * (size_t)ego_cap);
  x.off = (int32_t *)take(4 * ((size_t)ego_cap + 1));
  x.rs = (int32_t *)take(4 * ((size_t)ego_cap + 1));
  x.prio = (uint32_t *)take(4 * (size_t)ego_cap);
  x.err = (uint32_t *)take(4);
  x.hist = (unsigned long long *)take(8 * (size_t)MCE_HIST_MAX);
  if (a) *a = x;
  return off;
}

__device__ __forceinline__ uint32_t ld_acquire_sys(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.sys.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t hslot(int32_t key, int hcap) {
  return (uint32_t)(((uint64_t)(uint32_t)key * 0x9E3779B97F4A7C15ull) >> 32) & (uint32_t)(hcap - 1);
}

// local id of a vertex, or -1 (not in the ego graph, or cut by the cap)
__device__ __forceinline__ int32_t hget(const Arena &A, int hcap, int32_t key) {
  uint32_t h = hslot(key, hcap);
  for (int p = 0; p < hcap; ++p) {
    const int32_t k = A.hkey[h];
    if (k == key) return A.hval[h];
    if (k == -1) return -1;
    h = (h + 1) & (uint32_t)(hcap - 1);
  }
  return -1;
}

// insert key if absent; *slot receives its entry; true if this call inserted it
__device__ __forceinline__ bool hput(const Arena &A, int hcap, int32_t key, uint32_t *slot) {
  uint32_t h = hslot(key, hcap);
  for (int p = 0; p < hcap; ++p) {
    const int32_t old = atomicCAS(&A.hkey[h], -1, key);
    if (old == -1 || old == key) {
      *slot = h;
      return old == -1;
    }
    h = (h + 1) & (uint32_t)(hcap - 1);
  }
  return false;  // cannot happen: the table has twice the keys it can receive
}

// A slot's threads: one block of G threads (SV_BLOCK for class 0, SV_SMALL
// for class 1), so a slot's barriers are the block's.
template <int G>
struct Grp {
  __device__ static int tid() { return (int)threadIdx.x; }
  __device__ static void sync() { __syncthreads(); }
  // the number of the slot's threads with p set (and a barrier)
  __device__ static int count(bool p) { return __syncthreads_count(p); }
};

// exclusive scan of one value per thread over the slot; returns the total
template <int G>
__device__ __forceinline__ int block_scan(int x, int *excl, int *ws) {
  using Gp = Grp<G>;
  const int lane = (int)lane_id(), w = Gp::tid() >> 5;
  const int incl = warp_incl_scan(x);
  if (lane == 31) ws[w] = incl;
  Gp::sync();
  int base = 0, total = 0;
#pragma unroll
  for (int i = 0; i < (G / 32); ++i) {
    base += i < w ? ws[i] : 0;
    total += ws[i];
  }
  *excl = base + incl - x;
  Gp::sync();
  return total;
}

// bitonic sort of buf[0 .. n_pow2) in shared memory
template <int G>
__device__ void block_sort(int32_t *buf, int n_pow2) {
  using Gp = Grp<G>;
  for (int k = 2; k <= n_pow2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = Gp::tid(); i < n_pow2; i += G) {
        const int p = i ^ j;
        if (p > i) {
          const bool up = (i & k) == 0;
          const int32_t a = buf[i], b = buf[p];
          if ((a > b) == up) {
            buf[i] = b;
            buf[p] = a;
          }
        }
      }
      Gp::sync();
    }
}

struct SvShared {  // one per slot
  uint32_t req;
  int32_t rcls;  // the ring of the claimed request
  int32_t posted, broken;
  int32_t k, fcnt, ncnt, todo, level, minv, acnt, carry;
  unsigned long long total, nodes;
  int ws[SV_WARPS];
};

constexpr int32_t SV_PENDING = -3;  // hval of a vertex first seen in the current window

// inclusive max over the block (one value per thread)
template <int G>
__device__ __forceinline__ int block_max_scan(int x, int *ws) {
  using Gp = Grp<G>;
  const int lane = (int)lane_id(), w = Gp::tid() >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(MCE_FULL, x, o);
    if (lane >= o) x = max(x, y);
  }
  if (lane == 31) ws[w] = x;
  Gp::sync();
  int before = -1;
  for (int i = 0; i < w; ++i) before = max(before, ws[i]);
  Gp::sync();
  return max(x, before);
}

// off[0 .. nrows] = exclusive prefix of the resident-row lengths of the
// vertices list[0 .. nrows), rs[i] = where row i starts in the resident
// graph (a window's elements then need one load less); returns the total.
template <int G>
__device__ int row_offsets(const ServeArgs &S, const int32_t *list, int nrows, int32_t *off,
                           int32_t *rs, SvShared &sh) {
  using Gp = Grp<G>;
  int base = 0;
  for (int i0 = 0; i0 < nrows; i0 += G) {
    const int i = i0 + Gp::tid();
    int len = 0;
    if (i < nrows) {
      const int32_t g = list[i];
      const int32_t r0 = S.grp[g];
      len = S.grp[g + 1] - r0;
      rs[i] = r0;
    }
    int ex;
    const int tot = block_scan<G>(len, &ex, sh.ws);
    if (i < nrows) off[i] = base + ex;
    base += tot;
  }
  if (Gp::tid() == 0) off[nrows] = base;
  Gp::sync();
  return base;
}

// The rows list[0 .. nrows) of the resident graph are walked as one
// flattened sequence, G elements per window.  This returns the row
// that owns position e0 + (the thread's index in its slot): the last row starting at or before
// it (`carry`, the owner of the previous window's last position, covers a
// window in which no row starts before a thread's position).  [ia, ib) are
// the rows starting in the window; ia comes in as the previous window's ib
// (0 at the start): starts are ascending, so they are found by one pass of
// coalesced loads, not a search.
template <int G>
__device__ int window_owner(const int32_t *off, int nrows, int e0, int carry, int &ia, int &ib,
                            int32_t *own_sm, SvShared &sh) {
  using Gp = Grp<G>;
  own_sm[Gp::tid()] = -1;
  Gp::sync();
  const int B = G;
  int count = 0;
  for (;;) {
    const int i = ia + count + Gp::tid();
    const bool in = i < nrows && off[i] < e0 + B;
    // rows of length 0 start where the next row starts: the larger index wins
    if (in) atomicMax(&own_sm[off[i] - e0], i);
    const int c = Gp::count(in);
    count += c;
    if (c < B) break;
  }
  ib = ia + count;
  return max(block_max_scan<G>(own_sm[Gp::tid()], sh.ws), carry);
}

// Append the vertices first met in the rows of list[0 .. nrows) (row order,
// then position: discovery order) to the ego list, up to the cap.  A vertex
// seen at several positions of one window is appended at the first.  As in
// the induced-row pass, a window holds SV_RUN consecutive positions per
// thread, each thread finding the row of its first one by a binary search.
template <int G>
__device__ void ego_discover(const ServeArgs &S, const SvClass &C, const Arena &A, const int32_t *list, int nrows,
                             int32_t *own_sm, SvShared &sh) {
  using Gp = Grp<G>;
  constexpr int K = SV_RUN;
  const int cap = C.ego_cap, hc = C.hcap;
  const int T = row_offsets<G>(S, list, nrows, A.off, A.rs, sh);
  for (int w0 = 0; w0 < T; w0 += G * K) {
    const int k0 = sh.k;  // read by all before thread 0 updates it below
    if (k0 >= cap) break;
    const int p0 = w0 + Gp::tid() * K;
    int32_t wv[K];
    uint32_t slot[K];
    bool cand[K];
    if (p0 < T) {
      int lo = 0, hi = nrows + 1;  // the first row starting after p0
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (A.off[mid] <= p0)
          lo = mid + 1;
        else
          hi = mid;
      }
      int r = lo - 1;  // the last row starting at or before p0
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int e = p0 + k;
        wv[k] = -1;
        slot[k] = 0;
        cand[k] = false;
        if (e < T) {
          while (A.off[r + 1] <= e) ++r;  // stops at nrows at the latest: off[nrows] = T > e
          wv[k] = S.gcol[A.rs[r] + (e - A.off[r])];
          hput(A, hc, wv[k], &slot[k]);  // inserts or finds the vertex
          cand[k] = A.hval[slot[k]] == SV_PENDING;
          if (cand[k]) atomicMin(&A.hfirst[slot[k]], e);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        wv[k] = -1;
        slot[k] = 0;
        cand[k] = false;
      }
    }
    Gp::sync();
    bool fresh[K];
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      fresh[k] = cand[k] && A.hfirst[slot[k]] == p0 + k;
      cnt += fresh[k];
    }
    int pos;
    const int tot = block_scan<G>(cnt, &pos, sh.ws);
    int at = k0 + pos;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (fresh[k]) {
        if (at < cap) {
          A.hval[slot[k]] = at;
          A.V[at] = wv[k];
        } else {
          A.hval[slot[k]] = -1;  // beyond the cap: not in the ego graph
        }
        ++at;
      }
    }
    if (Gp::tid() == 0) sh.k = min(cap, k0 + tot);
    Gp::sync();
  }
}

// Build the ego graph of `seed` in the arena: sorted local CSR in rp/col.
// Returns its vertex count, or -1 if it has more arcs than the arena holds.
template <int G>
__device__ int ego_extract(const ServeArgs &S, const SvClass &C, const Arena &A, int64_t seed,
                           int32_t *sortbuf,
                           int32_t *own_sm, SvShared &sh) {
  using Gp = Grp<G>;
  const int hc = C.hcap;
  for (int i = Gp::tid(); i < hc; i += G) {
    A.hkey[i] = -1;
    A.hval[i] = SV_PENDING;
    A.hfirst[i] = INT_MAX;
  }
  Gp::sync();
  if (Gp::tid() == 0) {
    uint32_t slot = 0;
    hput(A, hc, (int32_t)seed, &slot);
    A.hval[slot] = 0;
    A.V[0] = (int32_t)seed;
    sh.k = 1;
  }
  Gp::sync();
  ego_discover<G>(S, C, A, A.V, 1, own_sm, sh);  // 1-hop: the seed's row
  const int k1 = sh.k;
  if (k1 < C.ego_cap && k1 > 1) ego_discover<G>(S, C, A, A.V + 1, k1 - 1, own_sm, sh);  // 2-hop
  const int n = sh.k;
  // local ids in ascending resident-graph id
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  for (int i = Gp::tid(); i < np2; i += G) sortbuf[i] = i < n ? A.V[i] : INT_MAX;
  Gp::sync();
  block_sort<G>(sortbuf, np2);
  for (int i = Gp::tid(); i < n; i += G) {
    const int32_t w = sortbuf[i];
    A.V[i] = w;
    uint32_t h = hslot(w, hc);
    for (int p = 0; p < hc && A.hkey[h] != w; ++p) h = (h + 1) & (uint32_t)(hc - 1);
    A.hval[h] = i;
  }
  Gp::sync();
  // induced rows in one flattened pass: the i-th kept element overall is
  // col[i] (rows in order, each filtered row stays sorted), and a row starts
  // at the count of kept elements before its first one.  A window holds
  // SV_RUN * G positions, SV_RUN consecutive ones per thread: a thread finds
  // the row of its first position by a binary search over the row offsets,
  // looks its elements up with their loads in flight together, and after one
  // scan of the threads' kept counts writes them and the starts of the rows
  // that begin in its positions (four times fewer windows and barriers than
  // one position per thread).
  const int T = row_offsets<G>(S, A.V, n, A.off, A.rs, sh);
  int kept = 0;
  constexpr int K = SV_RUN;
  for (int w0 = 0; w0 < T; w0 += G * K) {
    const int p0 = w0 + Gp::tid() * K;
    int r0 = -1;  // the last row starting at or before p0 - 1 (off[0] = 0, off[n] = T)
    int32_t loc[K];
    int cnt = 0;
    if (p0 < T) {
      int lo = 0, hi = n + 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (A.off[mid] <= p0 - 1)
          lo = mid + 1;
        else
          hi = mid;
      }
      r0 = lo - 1;
    }
    int r = r0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int e = p0 + k;
      loc[k] = -1;
      if (e < T) {
        while (A.off[r + 1] <= e) ++r;  // stops at n at the latest: off[n] = T > e
        loc[k] = hget(A, hc, S.gcol[A.rs[r] + (e - A.off[r])]);
        cnt += loc[k] >= 0;
      }
    }
    int pos;
    const int tot = block_scan<G>(cnt, &pos, sh.ws);
    if (p0 < T) {
      int q = kept + pos;
      r = r0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int e = p0 + k;
        if (e < T) {
          while (A.off[r + 1] <= e) A.rp[++r] = q;  // rows (empty ones too) starting at e
          if (loc[k] >= 0) {
            if (q < C.arc_cap) A.col[q] = loc[k];
            ++q;
          }
        }
      }
    }
    kept += tot;
    Gp::sync();  // the scan's shared words are reused by the next window
  }
  for (int i = Gp::tid(); i <= n; i += G)  // rows starting at the end (empty)
    if (A.off[i] == T) A.rp[i] = kept;
  Gp::sync();
  return kept > C.arc_cap ? -1 : n;
}

// Degeneracy priorities of the ego graph: synchronous peeling rounds over
// all levels, the final round keeping priority m (peel.cu's order).
template <int G>
__device__ void ego_peel(const Arena &A, int n, SvShared &sh) {
  using Gp = Grp<G>;
  const int m = A.rp[n];
  for (int i = Gp::tid(); i < n; i += G) {
    A.deg[i] = A.rp[i + 1] - A.rp[i];
    A.core[i] = -1;
    A.prio[i] = (uint32_t)m;
  }
  if (Gp::tid() == 0) {
    sh.todo = n;
    sh.level = 0;
  }
  Gp::sync();
  uint32_t priority = 0;
  const int lane = (int)lane_id(), w = Gp::tid() >> 5;
  while (sh.todo > 0) {
    const int level = sh.level;
    Gp::sync();
    if (Gp::tid() == 0) {
      sh.fcnt = 0;
      sh.minv = INT_MAX;
    }
    Gp::sync();
    for (int i = Gp::tid(); i < n; i += G)
      if (A.core[i] == -1) {
        if (A.deg[i] <= level) {  // == level: a remaining vertex never has less
          A.core[i] = level;
          A.fa[atomicAdd(&sh.fcnt, 1)] = i;
        } else {
          atomicMin(&sh.minv, A.deg[i]);
        }
      }
    Gp::sync();
    if (sh.fcnt == 0) {  // no vertex at this level: go to the lowest remaining degree
      Gp::sync();
      if (Gp::tid() == 0) sh.level = sh.minv;
      Gp::sync();
      continue;
    }
    int32_t *F = A.fa, *Nx = A.fb;
    for (;;) {
      const int cnt = sh.fcnt;
      Gp::sync();
      if (cnt == 0) break;
      if (Gp::tid() == 0) {
        sh.todo -= cnt;
        sh.ncnt = 0;
      }
      Gp::sync();
      if (sh.todo == 0) break;  // the final round keeps priority m
      for (int i = Gp::tid(); i < cnt; i += G) A.prio[F[i]] = priority;
      for (int i = w; i < cnt; i += (G / 32)) {
        const int v = F[i];
        for (int j = A.rp[v] + lane; j < A.rp[v + 1]; j += 32) {
          const int u = A.col[j];
          if (*(volatile int32_t *)&A.core[u] == -1) {
            const int old = atomicSub(&A.deg[u], 1);
            if (old == level + 1) {
              A.core[u] = level;
              Nx[atomicAdd(&sh.ncnt, 1)] = u;
            }
          }
        }
      }
      Gp::sync();
      if (Gp::tid() == 0) sh.fcnt = sh.ncnt;
      int32_t *t = F;
      F = Nx;
      Nx = t;
      ++priority;
      Gp::sync();
    }
    if (Gp::tid() == 0) sh.level = level + 1;
    Gp::sync();
  }
}

// Rows become [earlier | later]; u is later than v iff
// prio[v] == prio[u] ? v < u : prio[v] < prio[u] (include/main_support.cuh:14).
template <int G>
__device__ void ego_orient(const Arena &A, int n) {
  using Gp = Grp<G>;
  const int lane = (int)lane_id(), w = Gp::tid() >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (int v = w; v < n; v += (G / 32)) {
    const int b = A.rp[v], e = A.rp[v + 1];
    const uint32_t pv = A.prio[v];
    int ne = 0;
    for (int j0 = b; j0 < e; j0 += 32) {
      const int j = j0 + lane;
      bool earlier = false;
      if (j < e) {
        const int u = A.col[j];
        const uint32_t pu = A.prio[u];
        earlier = !(pv == pu ? v < u : pv < pu);
      }
      ne += __popc(__ballot_sync(MCE_FULL, earlier));
    }
    int eo = b, lo = b + ne;
    for (int j0 = b; j0 < e; j0 += 32) {
      const int j = j0 + lane;
      const bool valid = j < e;
      bool later = false;
      int u = 0;
      if (valid) {
        u = A.col[j];
        const uint32_t pu = A.prio[u];
        later = pv == pu ? v < u : pv < pu;
      }
      const uint32_t mL = __ballot_sync(MCE_FULL, valid && later);
      const uint32_t mE = __ballot_sync(MCE_FULL, valid && !later);
      if (valid) A.cs[later ? lo + __popc(mL & lt) : eo + __popc(mE & lt)] = u;
      eo += __popc(mE);
      lo += __popc(mL);
    }
    if (lane == 0) A.split[v] = b + ne;
  }
  Gp::sync();
}

union WarpSmem {
  RegSmem<uint32_t, 1> r32;
  RegSmem<u64, 2> r64;
  MemSmem mem;
};

constexpr uint32_t SV_EXIT = 0xFFFFFFFFu;

// Mirror the class's host tail and stop flag into device memory (one
// thread at a time, at most every SV_POLL_NS); stop first: the host
// publishes its last request before stopping, so a tail read after a stop
// read sees that request.
__device__ __forceinline__ void poll_ring(const SvClass &C, uint64_t now, uint64_t every) {
  SvCtl *c = C.ctl;
  const unsigned long long last = ld_volatile(&c->poll_ns);
  if (now - last >= every && atomicCAS(&c->poll_ns, last, now) == last) {
    const uint32_t st = ld_acquire_sys(&C.hdr->stop);
    const uint32_t t = ld_acquire_sys(&C.hdr->tail);
    atomicMax(&c->dtail, t);
    __threadfence();
    if (st) atomicExch(&c->dstop, 1u);
  }
}

// Claim the next published request of class C: its id, or SV_EXIT if none
// is waiting (*stop: the class is stopping).
__device__ __forceinline__ uint32_t try_claim(const SvClass &C, bool *stop) {
  SvCtl *c = C.ctl;
  *stop = ld_volatile(&c->dstop) != 0;  // before dtail, as poll_ring writes them
  __threadfence();
  for (;;) {
    const uint32_t k = ld_volatile(&c->next);
    if (k >= ld_volatile(&c->dtail)) return SV_EXIT;
    if (atomicCAS(&c->next, k, k + 1) == k) {
      __threadfence_system();  // the entry's seed is read after this
      return k;
    }
  }
}

// Thread 0 of a slot of class `mine`: wait for a published request and
// claim it (*cls: the ring it came from); SV_HELP | j to help class-0 slot
// j's search; SV_EXIT when the session stops or the slot has been idle for
// idle_ns.  A class-0 slot also takes class-1 requests (its arena holds
// them) when its own ring is empty.
__device__ uint32_t claim(const ServeArgs &S, int mine, int *cls) {
  const uint64_t t_idle = globaltimer_ns();
  uint32_t ns = 64;
  for (;;) {
    const uint64_t now = globaltimer_ns();
    bool stop0 = true, stop1 = true;
    for (int c = mine; c < 2; ++c) {
      if (S.cls[c].slots == 0 && c != mine) continue;
      poll_ring(S.cls[c], now, c == 0 ? SV_POLL_NS : 4 * SV_POLL_NS);
      bool st = false;
      const uint32_t k = try_claim(S.cls[c], &st);
      if (k != SV_EXIT) {
        *cls = c;
        return k;
      }
      (c == 0 ? stop0 : stop1) = st;
    }
    if (mine == 0 ? (stop0 && (stop1 || S.cls[1].slots == 0)) : stop1) return SV_EXIT;
    if (now - t_idle > S.idle_ns) return SV_EXIT;
    // no new request: join the search of a large one a class-0 slot runs
    // (the board is scanned only when something is posted: hundreds of idle
    // slots reading its 64 words saturated the L2 slices that hold them)
    const int posted = ld_volatile(&S.cls[0].ctl->board_n) != 0 ? SV_BOARD : 0;
    for (int e = 0; e < posted; ++e) {
      const uint32_t j1 = ld_volatile(&S.board[e]);
      if (j1 == 0) continue;
      SvHelp *h = &S.help[j1 - 1];
      uint32_t st = ld_volatile(&h->state);
      while ((st & SV_OPEN) && ld_volatile(&h->rootnext) < (uint32_t)ld_volatile((uint32_t *)&h->n)) {
        const uint32_t prev = atomicCAS(&h->state, st, st + 1);
        if (prev == st) {
          __threadfence();  // the owner's arena was written before it opened
          return SV_HELP | (j1 - 1);
        }
        st = prev;
      }
    }
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
}

// The warps of a block search roots of the request whose shared state is h
// (the block's own or, when helping, another slot's): a holds the request's
// arena for the wide engine, ar for the register engines; slabs and shared
// memory are the block's own.
__device__ void search_roots(const ServeArgs &S, const BKArgs &a, const BKArgs &ar,
                             const Slab &msl, const RegSlab<uint32_t> &rs32,
                             const RegSlab<u64> &rs64, WarpSmem &sm, SvHelp *h) {
  const int lane = (int)lane_id();
  const int n = (int)ld_volatile((const uint32_t *)&h->n);
  unsigned long long mine = 0, h0 = 0, h1 = 0;
  RegRoot<uint32_t> rt32;
  RegRoot<u64> rt64;
  MemRoot rtm;
  for (;;) {  // warps take roots in id order until done or over a limit
    uint32_t r = 0;
    if (lane == 0) {
      const bool over = S.node_budget && ld_volatile(&h->nodes) > S.node_budget;
      if (over) atomicOr(a.err, MCE_ERR_BUDGET);
      r = (over || ld_volatile(a.err)) ? 0xFFFFFFFFu : atomicAdd(&h->rootnext, 1u);
    }
    r = __shfl_sync(MCE_FULL, r, 0);
    if (r >= (uint32_t)n) break;
    const int dp = a.rp[r + 1] - a.split[r], dm = a.split[r] - a.rp[r];
    if (dp == 0) continue;
    unsigned long long nd = 0, cnt = 0;
    if (dp <= 32 && dm <= REG_XCAP) {
      reg_encode<uint32_t, 1>(ar, sm.r32, rs32, (int32_t)r, rt32);
      reg_tree<uint32_t, 1, true>(ar, sm.r32, rs32, rt32, WOps<uint32_t>::low(dp), 0u, 0u, h0, h1,
                                  nd, cnt);
    } else if (dp <= 64 && dm <= REG_XCAP) {
      reg_encode<u64, 2>(ar, sm.r64, rs64, (int32_t)r, rt64);
      reg_tree<u64, 2, true>(ar, sm.r64, rs64, rt64, WOps<u64>::low(dp), 0ull, 0ull, h0, h1, nd,
                             cnt);
    } else {  // mem_encode flags roots wider than SV_DCAP
      mem_encode(a, sm.mem, msl, (int32_t)r, rtm);
      if (rtm.d > 0) {
        const int Wr = rtm.Wr;
        if (lane < Wr) {  // root frame: P = all of N+(r), X = 0, S = 0
          msl.stk[lane] = (lane == Wr - 1 && (dp & 63)) ? ((1ull << (dp & 63)) - 1ull) : ~0ull;
          msl.stk[Wr + lane] = 0;
          msl.stk[3 * Wr + lane] = 0;
        }
        __syncwarp();
        mem_tree<true>(a, msl, rtm, h0, h1, nd, cnt);
      }
    }
    mine += cnt;
    if (lane == 0 && nd) atomicAdd(&h->nodes, nd);
  }
  if (lane == 0 && mine) atomicAdd(&h->total, mine);
}

// One slot: one block, of SV_BLOCK threads (class 0) or SV_SMALL (class 1),
// with its own shared state sh and windows own_sm (one int per thread), its
// sort buffer (the next power of two >= its class's cap, ints), its arena,
// and its warps' engine state and slabs.
template <bool BIG>
__device__ __forceinline__ void serve_slot(const ServeArgs &S, int slot, SvShared &sh,
                                           int32_t *own_sm, int32_t *sortbuf, WarpSmem *wsm) {
  constexpr bool big = BIG;
  constexpr int G = BIG ? SV_BLOCK : SV_SMALL;
  const int mine = big ? 0 : 1;
  const int tid = (int)threadIdx.x;
  const int w = (int)(threadIdx.x >> 5);
  const SvClass &M = S.cls[mine];
  Arena A;
  arena_layout(M.ego_cap, M.arc_cap, M.hcap, M.arena + (size_t)slot * M.arena_bytes, &A);
  unsigned long long *wslab =
      M.slab + ((size_t)blockIdx.x * (G / 32) + (size_t)w) * S.slab_words;
  // engine arguments (no task sharing, no per-root logs); the slabs are laid
  // out for class 0's cap; the arena fields are set per search
  BKArgs a;
  memset(&a, 0, sizeof(a));
  a.dcap = SV_DCAP;
  a.xcap = S.cls[0].ego_cap;
  a.node_budget = S.node_budget;
  a.slab = wslab + S.reg_words;
  a.slab_words = 0;
  const Slab msl = slab_of(a, 0);
  BKArgs ar = a;
  ar.slab = wslab;
  const RegSlab<uint32_t> rs32 = reg_slab<uint32_t>(ar, 0);
  const RegSlab<u64> rs64 = reg_slab<u64>(ar, 0);
  SvHelp *own = &S.help[mine == 0 ? slot : S.cls[0].slots + slot];
  SvCtl *inflight = S.cls[0].ctl;  // requests on the device, over both classes
  for (;;) {
    if (tid == 0) {
      int c = mine;
      sh.req = claim(S, mine, &c);
      sh.rcls = c;
    }
    __syncthreads();
    const uint32_t req = sh.req;
    const int rc_cls = sh.rcls;
    if (req == SV_EXIT) break;
    const bool helping = (req & SV_HELP) != 0;
    // the request whose roots this slot searches: a class-0 slot's (helping)
    // or its own
    Arena X = A;
    SvHelp *h = own;
    const SvClass &R = S.cls[rc_cls];
    SvEntry *E = nullptr;
    int32_t status = MCE_OK;
    uint32_t limits = 0;
    int n = 0;
    uint64_t t0 = 0, t1 = 0, t2 = 0;
    if (helping) {
      const uint32_t j = req & 0xFFFFFFu;
      const SvClass &B0 = S.cls[0];
      arena_layout(B0.ego_cap, B0.arc_cap, B0.hcap, B0.arena + (size_t)j * B0.arena_bytes, &X);
      h = &S.help[j];
    } else {
      if (tid == 0) {
        *A.err = 0;
        sh.posted = -1;
        sh.broken = 0;
        sh.total = 0;
        sh.nodes = 0;
        const unsigned long long on = atomicAdd(&inflight->inflight, 1ull) + 1;
        atomicMax(&inflight->peak, on);
      }
      __syncthreads();
      t0 = t1 = t2 = globaltimer_ns();
      E = R.ent + (req % R.ring);
      const int64_t seed = *(volatile int64_t *)&E->seed;
      if (seed < 0 || seed >= S.gn) {
        status = MCE_EINVAL;
      } else {
        n = ego_extract<G>(S, M, A, seed, sortbuf, own_sm, sh);
        t1 = t2 = globaltimer_ns();
        if (n < 0) {
          status = MCE_ELIMIT;
          limits = MCE_ERR_ARCS;
          n = 0;
        }
      }
      if (status == MCE_OK) {
        ego_peel<G>(A, n, sh);
        ego_orient<G>(A, n);
        t2 = globaltimer_ns();
        if (tid == 0) {  // open the roots; large requests also to helping slots
          own->rootnext = 0;
          own->n = n;
          own->total = 0;
          own->nodes = 0;
          __threadfence();  // the arena and the fields above before the opening
          if (mine == 0 && n >= SV_HELP_MIN) {
            atomicExch(&own->state, SV_OPEN);
            for (int e = 0; e < SV_BOARD; ++e)
              if (atomicCAS(&S.board[e], 0u, (uint32_t)slot + 1) == 0u) {
                atomicAdd(&S.cls[0].ctl->board_n, 1u);
                sh.posted = e;
                break;
              }
          }
        }
        __syncthreads();
      }
    }
    if (status == MCE_OK) {
      a.rp = ar.rp = X.rp;
      a.split = ar.split = X.split;
      a.cs = ar.cs = X.cs;
      a.hist = ar.hist = X.hist;
      a.err = ar.err = X.err;
      search_roots(S, a, ar, msl, rs32, rs64, wsm[w], h);
    }
    __syncthreads();
    if (helping) {
      if (tid == 0) {
        __threadfence();  // this slot's counts land before it leaves
        atomicSub(&h->state, 1u);
        atomicAdd(&M.ctl->helped, 1ull);
      }
      continue;
    }
    if (status == MCE_OK) {
      if (tid == 0) {  // close, then wait (bounded) for the helpers to leave
        if (sh.posted >= 0) {
          atomicExch(&S.board[sh.posted], 0u);
          atomicSub(&S.cls[0].ctl->board_n, 1u);
        }
        atomicAnd(&own->state, ~SV_OPEN);
        const uint64_t tw = globaltimer_ns();
        while ((ld_volatile(&own->state) & 0xFFFFFFu) != 0) {
          if (globaltimer_ns() - tw > SV_HELP_WAIT_NS) {
            sh.broken = 1;
            break;
          }
          __nanosleep(256);
        }
        __threadfence();
        sh.total = ld_volatile(&own->total);
        sh.nodes = ld_volatile(&own->nodes);
      }
      __syncthreads();
      limits = ld_volatile(A.err);
      if (limits) status = MCE_ELIMIT;
      if (sh.broken) status = MCE_ETIMEOUT;
    }
    __syncthreads();
    if (tid == 0) {
      E->count = status == MCE_OK ? sh.total : 0ull;
      const uint64_t t3 = globaltimer_ns();
      E->device_ns = t3 - t0;
      auto clamp32 = [](uint64_t x) { return (uint32_t)(x > 0xFFFFFFFFull ? 0xFFFFFFFFull : x); };
      E->extract_ns = clamp32(t1 - t0);
      E->order_ns = clamp32(t2 - t1);
      E->search_ns = clamp32(t2 > t0 ? t3 - t2 : 0ull);
      E->status = status;
      E->limits = limits;
      E->ego_n = n;
      E->ego_arcs = n > 0 ? A.rp[n] : 0;
      __threadfence_system();
      *(volatile uint32_t *)&E->done = req + 1;
      atomicAdd(&R.ctl->served, 1ull);
      atomicAdd(&R.ctl->nodes, sh.nodes);
      atomicAdd(&inflight->inflight, ~0ull);  // minus one
    }
    __syncthreads();
    // a helper that never left may still read the arena: the slot retires
    if (sh.broken) break;
  }
}

// One kernel per slot class, launched side by side on two streams: a block
// of serve_kernel<true> (SV_BLOCK threads) is one class-0 slot, a block of
// serve_kernel<false> (SV_SMALL threads, four to an SM's room of one
// class-0 block) one class-1 slot.  Dynamic shared memory: the warps'
// engine state, then the sort buffer.
template <bool BIG>
__global__ void __launch_bounds__(BIG ? SV_BLOCK : SV_SMALL, BIG ? 1 : SV_BLOCK / SV_SMALL)
    serve_kernel(ServeArgs S) {
  constexpr int G = BIG ? SV_BLOCK : SV_SMALL;
  extern __shared__ __align__(16) unsigned char sv_dyn[];
  WarpSmem *wsm = (WarpSmem *)sv_dyn;
  int32_t *sortbuf = (int32_t *)(sv_dyn + sizeof(WarpSmem) * (G / 32));
  __shared__ SvShared sh;
  __shared__ int32_t own[G];
  serve_slot<BIG>(S, (int)blockIdx.x, sh, own, sortbuf, wsm);
}

// Per vertex: deg(v) + the sum of its neighbours' degrees, capped at
// INT32_MAX - a bound on the 2-hop ego graph's size minus one (one warp per
// vertex).
__global__ void footprint_kernel(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                 int64_t n, int32_t *__restrict__ bound) {
  const int lane = (int)lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = gw; v < n; v += nw) {
    const int32_t b = rp[v], e = rp[v + 1];
    long long acc = 0;
    for (int32_t j = b + lane; j < e; j += 32) {
      const int32_t u = col[j];
      acc += rp[u + 1] - rp[u];
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(MCE_FULL, acc, o);
    if (lane == 0) {
      acc += e - b;
      bound[v] = (int32_t)(acc > 0x7FFFFFFFll ? 0x7FFFFFFFll : acc);
    }
  }
}

}  // namespace

int graph_device_view(const struct ::mce_graph *g, const int32_t **rp, const int32_t **col,
                      int64_t *n, int *device);

}  // namespace mce

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace mce;

// One class's request ring in mapped pinned memory, its arenas and control.
struct SvRing {
  char *host = nullptr;        // mapped: SvHostHdr then the ring entries
  SvHostHdr *hdr = nullptr;    // host views
  SvEntry *ent = nullptr;
  uint32_t tail = 0;           // requests published
  uint32_t low = 0;            // lowest id whose entry is not yet free
  uint32_t open = 0;           // submitted, answer not yet taken
  std::vector<uint8_t> taken;  // per entry: answer handed to the caller
  char *arena = nullptr;
  SvCtl *ctl = nullptr;
};

struct mce_serve {
  int device = 0;
  cudaStream_t stream[2] = {nullptr, nullptr};  // one kernel per class
  ServeArgs args{};
  size_t smem[2] = {0, 0};
  uint32_t grid[2] = {0, 0};    // blocks of each class's kernel
  uint32_t blocks = 0, ring = 0;
  SvRing cls[2];                // 0: whole-block slots, 1: quarter-block slots
  std::vector<int32_t> bound;   // per vertex: its footprint bound (2-hop degree sum)
  int32_t small_cap = 0;        // class-1 cap (0: one class)
  unsigned long long *slab = nullptr;
  SvHelp *help = nullptr;
  uint32_t *board = nullptr;
  int64_t launches = 0;
  bool closed = false;
  std::chrono::steady_clock::time_point checked[2];  // last look at each kernel's stream
};

namespace {

// a request id names its ring in bit 0 and its place in the ring above it
inline int id_cls(uint64_t id) { return (int)(id & 1u); }
inline uint32_t id_local(uint64_t id) { return (uint32_t)(id >> 1); }

int sv_launch(mce_serve *s, int c) {
  if (c == 0)
    serve_kernel<true><<<s->grid[0], SV_BLOCK, s->smem[0], s->stream[0]>>>(s->args);
  else
    serve_kernel<false><<<s->grid[1], SV_SMALL, s->smem[1], s->stream[1]>>>(s->args);
  MCE_CUDA(cudaGetLastError());
  ++s->launches;
  return MCE_OK;
}

// relaunch a class's kernel when requests of its ring wait and every slot
// of that kernel has left.  Each stream is looked at most every 100 us (a
// kernel leaves only after idle_ms): with a driver call per poll of every
// open request, the median host-observed latency at 2,000 requests/s was
// 0.06 ms higher with two slot classes.
int sv_ensure_running(mce_serve *s) {
  const auto now = std::chrono::steady_clock::now();
  for (int c = 0; c < 2; ++c) {
    if (!s->cls[c].ctl || now - s->checked[c] < std::chrono::microseconds(100)) continue;
    s->checked[c] = now;
    const cudaError_t q = cudaStreamQuery(s->stream[c]);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return MCE_ECUDA;
    SvCtl ct;
    MCE_CUDA(cudaMemcpy(&ct, s->cls[c].ctl, sizeof(ct), cudaMemcpyDeviceToHost));
    if (ct.next < s->cls[c].tail) {  // something unclaimed
      const int rc = sv_launch(s, c);
      if (rc != MCE_OK) return rc;
    }
  }
  return MCE_OK;
}

bool sv_done(const mce_serve *s, int c, uint32_t id) {
  const SvEntry &e = s->cls[c].ent[id % s->ring];
  return __atomic_load_n(&e.done, __ATOMIC_ACQUIRE) == id + 1;
}

void sv_retire(mce_serve *s, int c) {
  SvRing &R = s->cls[c];
  while (R.low < R.tail && R.taken[R.low % s->ring]) {
    R.taken[R.low % s->ring] = 0;
    ++R.low;
  }
}

void sv_free(mce_serve *s) {
  for (cudaStream_t st : s->stream)
    if (st) cudaStreamDestroy(st);
  for (SvRing &R : s->cls) {
    if (R.host) cudaFreeHost(R.host);
    if (R.arena) cudaFree(R.arena);
    if (R.ctl) cudaFree(R.ctl);
  }
  if (s->slab) cudaFree(s->slab);
  if (s->help) cudaFree(s->help);
  if (s->board) cudaFree(s->board);
  delete s;
}

// The table also takes the vertices of the discovery window that crosses
// the cap: up to threads * SV_RUN of them (a window's positions).
int hash_cap_for(int ego_cap, int threads) {
  int hcap = 32;
  while (hcap < 2 * (ego_cap + threads * SV_RUN)) hcap <<= 1;
  return hcap;
}

}  // namespace

extern "C" void mce_serve_opts_default(mce_serve_opts_t *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->ego_cap = 1024;
  o->max_arcs = 0;
  o->slots = 0;
  o->ring = 4096;
  o->idle_ms = 1000;
  o->small_cap = -1;  // automatic
  o->big_slots = 0;
}

extern "C" int mce_serve_open(mce_graph_t g, const mce_serve_opts_t *opts, mce_serve_t *out) {
  if (!g || !out) return MCE_EINVAL;
  mce_serve_opts_t o;
  mce_serve_opts_default(&o);
  if (opts) o = *opts;
  if (o.ego_cap < 2 || o.ego_cap > SV_MAX_EGO || o.ring < 1 || o.ring > (1u << 24) ||
      o.idle_ms < 1 || o.max_arcs < 0 || o.max_nodes < 0 || o.small_cap > o.ego_cap ||
      o.big_slots < 0)
    return MCE_EINVAL;
  // class 1 (quarter-block slots) for requests whose footprint bound fits
  // small_cap vertices; automatic: 1,024 when the cap is above 2,048
  const int32_t small_cap = o.small_cap < 0 ? (o.ego_cap > 2048 ? 1024 : 0)
                                            : (o.small_cap >= 2 ? o.small_cap : 0);
  const int32_t *rp = nullptr, *col = nullptr;
  int64_t n = 0;
  int device = 0;
  const int rc = graph_device_view(g, &rp, &col, &n, &device);
  if (rc != MCE_OK) return rc;
  MCE_CUDA(cudaSetDevice(device));
  int sms = 0;
  MCE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  mce_serve *s = new mce_serve();
  s->device = device;
  s->ring = o.ring;
  s->small_cap = small_cap;
  int np2 = 1, np2s = 1;
  while (np2 < o.ego_cap) np2 <<= 1;
  while (np2s < small_cap) np2s <<= 1;
  s->smem[0] = sizeof(WarpSmem) * SV_WARPS + sizeof(int32_t) * (size_t)np2;
  s->smem[1] = sizeof(WarpSmem) * (SV_SMALL / 32) + sizeof(int32_t) * (size_t)np2s;
  auto fail = [&](int code) {
    sv_free(s);
    return code;
  };
  // blocks resident at once on the device: class 0 takes `big` SMs' room,
  // class 1 the rest, per_small blocks in the room of one class-0 block
  int per_sm = 0, per_small = 0;
  if (cudaFuncSetAttribute(serve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)s->smem[0]) != cudaSuccess ||
      cudaFuncSetAttribute(serve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)s->smem[1]) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel<true>, SV_BLOCK,
                                                    s->smem[0]) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_small, serve_kernel<false>, SV_SMALL,
                                                    s->smem[1]) != cudaSuccess ||
      per_sm < 1 || per_small < 1)
    return fail(MCE_ECUDA);
  const uint32_t fit = (uint32_t)(sms * per_sm);
  s->blocks = o.slots > 0 ? std::min((uint32_t)o.slots, fit) : fit;
  uint32_t big = s->blocks;
  if (small_cap && s->blocks >= 2)
    big = o.big_slots > 0 ? std::min<uint32_t>((uint32_t)o.big_slots, s->blocks - 1)
                          : (s->blocks + 1) / 2;
  const uint32_t small_slots =
      (s->blocks - big) * (uint32_t)std::min(per_small / per_sm, SV_BLOCK / SV_SMALL);
  if (!small_slots) s->small_cap = 0;  // one class: every request to class 0
  s->grid[0] = big;
  s->grid[1] = small_slots;
  for (int c = 0; c < 2; ++c)
    if (cudaStreamCreateWithFlags(&s->stream[c], cudaStreamNonBlocking) != cudaSuccess)
      return fail(MCE_ECUDA);
  ServeArgs &A = s->args;
  A.grp = rp;
  A.gcol = col;
  A.gn = n;
  const int64_t full = (int64_t)o.ego_cap * (o.ego_cap - 1);
  const int64_t want = o.max_arcs > 0 ? o.max_arcs : (int64_t)o.ego_cap * 128;
  const int32_t arc0 =
      (int32_t)std::max<int64_t>(1, std::min<int64_t>(std::min(full, want), INT32_MAX / 2));
  for (int c = 0; c < 2; ++c) {
    SvRing &R = s->cls[c];
    SvClass &C = A.cls[c];
    std::memset(&C, 0, sizeof(C));
    if (c == 1 && small_slots == 0) continue;
    const size_t host_bytes = sizeof(SvHostHdr) + sizeof(SvEntry) * (size_t)o.ring;
    if (cudaHostAlloc((void **)&R.host, host_bytes, cudaHostAllocMapped) != cudaSuccess)
      return fail(MCE_ENOMEM);
    std::memset(R.host, 0, host_bytes);
    R.hdr = (SvHostHdr *)R.host;
    R.ent = (SvEntry *)(R.host + sizeof(SvHostHdr));
    R.taken.assign(o.ring, 0);
    char *dh = nullptr;
    if (cudaHostGetDevicePointer((void **)&dh, R.host, 0) != cudaSuccess) return fail(MCE_ECUDA);
    C.hdr = (const SvHostHdr *)dh;
    C.ent = (SvEntry *)(dh + sizeof(SvHostHdr));
    C.ring = o.ring;
    C.slots = (int32_t)(c == 0 ? big : small_slots);
    C.ego_cap = c == 0 ? o.ego_cap : small_cap;
    C.hcap = hash_cap_for(C.ego_cap, c == 0 ? SV_BLOCK : SV_SMALL);
    // class 1 holds every arc its vertices can have (up to class 0's limit)
    C.arc_cap = c == 0 ? arc0
                       : (int32_t)std::max<int64_t>(
                             1, std::min<int64_t>((int64_t)small_cap * (small_cap - 1), arc0));
    C.arena_bytes = arena_layout(C.ego_cap, C.arc_cap, C.hcap, nullptr, nullptr);
    if (cudaMalloc((void **)&R.arena, C.arena_bytes * (size_t)C.slots) != cudaSuccess ||
        cudaMalloc((void **)&R.ctl, sizeof(SvCtl)) != cudaSuccess ||
        cudaMemset(R.ctl, 0, sizeof(SvCtl)) != cudaSuccess)
      return fail(MCE_ENOMEM);
    C.arena = R.arena;
    C.ctl = R.ctl;
  }
  A.reg_words = bk_slab_words(CLS_R64, 0, 0);
  A.slab_words = A.reg_words + bk_slab_words(CLS_MEM, SV_DCAP, o.ego_cap);
  A.idle_ns = (uint64_t)o.idle_ms * 1000000ull;
  A.node_budget = (unsigned long long)o.max_nodes;
  const size_t helps = (size_t)big + small_slots;
  const size_t warps = (size_t)big * SV_WARPS + (size_t)small_slots * (SV_SMALL / 32);
  if (cudaMalloc((void **)&s->slab, A.slab_words * 8 * warps) != cudaSuccess ||
      cudaMalloc((void **)&s->help, sizeof(SvHelp) * helps) != cudaSuccess ||
      cudaMalloc((void **)&s->board, sizeof(uint32_t) * SV_BOARD) != cudaSuccess)
    return fail(MCE_ENOMEM);
  if (cudaMemset(s->help, 0, sizeof(SvHelp) * helps) != cudaSuccess ||
      cudaMemset(s->board, 0, sizeof(uint32_t) * SV_BOARD) != cudaSuccess)
    return fail(MCE_ECUDA);
  A.help = s->help;
  A.board = s->board;
  A.cls[0].slab = s->slab;
  A.cls[1].slab = s->slab + A.slab_words * SV_WARPS * (size_t)big;
  if (small_slots) {  // the footprint bound of every seed, for routing on the host
    int32_t *db = nullptr;
    if (cudaMalloc((void **)&db, sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)) !=
        cudaSuccess)
      return fail(MCE_ENOMEM);
    s->bound.assign((size_t)n, 0);
    footprint_kernel<<<sms * 8, 256, 0, s->stream[0]>>>(rp, col, n, db);
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpyAsync(s->bound.data(), db, sizeof(int32_t) * (size_t)n,
                                    cudaMemcpyDeviceToHost, s->stream[0]) == cudaSuccess &&
                    cudaStreamSynchronize(s->stream[0]) == cudaSuccess;
    cudaFree(db);
    if (!ok) return fail(MCE_ECUDA);
  }
  // the graph's upload (queued on its own stream) completes first
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(MCE_ECUDA);
  for (int c = 0; c < 2; ++c)
    if (s->grid[c] && sv_launch(s, c) != MCE_OK) return fail(MCE_ECUDA);
  *out = s;
  return MCE_OK;
}

extern "C" int mce_serve_submit(mce_serve_t s, int64_t seed, uint64_t *id_out) {
  if (!s || !id_out) return MCE_EINVAL;
  if (s->closed) return MCE_ESTATE;
  // admission by footprint: a seed whose 2-hop bound fits the class-1 cap
  // goes to the 256-thread slots once every whole-block slot has a request
  // (below that load a whole block answers it sooner); any other seed to the
  // whole-block slots
  const bool fits = s->small_cap && seed >= 0 && seed < (int64_t)s->bound.size() &&
                    (int64_t)s->bound[(size_t)seed] + 1 <= s->small_cap;
  const int c = fits && s->cls[0].open >= s->grid[0] ? 1 : 0;
  SvRing &R = s->cls[c];
  sv_retire(s, c);
  if (R.tail - R.low >= s->ring) return MCE_ELIMIT;  // ring full: take answers first
  if (R.tail >= 0x3FFFFFF0u) return MCE_ELIMIT;      // ids exhausted (below SV_HELP)
  const uint32_t id = R.tail;
  SvEntry &e = R.ent[id % s->ring];
  e.seed = seed;
  __atomic_store_n(&e.done, 0u, __ATOMIC_RELAXED);
  R.tail = id + 1;
  ++R.open;
  __atomic_store_n(&R.hdr->tail, R.tail, __ATOMIC_RELEASE);
  *id_out = ((uint64_t)id << 1) | (uint64_t)c;
  return sv_ensure_running(s);
}

extern "C" int mce_serve_poll(mce_serve_t s, uint64_t id, mce_serve_result_t *res) {
  if (!s || !res) return MCE_EINVAL;
  const int c = id_cls(id);
  const uint32_t i = id_local(id);
  SvRing &R = s->cls[c];
  if (!R.host || i >= R.tail || i < R.low || R.taken[i % s->ring]) return MCE_EINVAL;
  if (!sv_done(s, c, i)) {
    const int rc = s->closed ? MCE_OK : sv_ensure_running(s);
    return rc != MCE_OK ? rc : MCE_EAGAIN;
  }
  const SvEntry &e = R.ent[i % s->ring];
  res->count = e.count;
  res->seed = e.seed;
  res->status = e.status;
  res->ego_n = e.ego_n;
  res->ego_arcs = e.ego_arcs;
  res->limits = e.limits;
  res->device_ns = e.device_ns;
  res->extract_ns = e.extract_ns;
  res->order_ns = e.order_ns;
  res->search_ns = e.search_ns;
  R.taken[i % s->ring] = 1;
  --R.open;
  sv_retire(s, c);
  return MCE_OK;
}

extern "C" int mce_serve_wait(mce_serve_t s, uint64_t id, int64_t timeout_ms,
                              mce_serve_result_t *res) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const int rc = mce_serve_poll(s, id, res);
    if (rc != MCE_EAGAIN) return rc;
    const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                        std::chrono::steady_clock::now() - t0)
                        .count();
    if (timeout_ms >= 0 && ms > timeout_ms) return MCE_ETIMEOUT;
    std::this_thread::yield();
  }
}

extern "C" int mce_serve_run(mce_serve_t s, const int64_t *seeds, const double *arrival_us,
                             int64_t count, int64_t timeout_ms, mce_serve_result_t *results,
                             double *latency_us) {
  if (!s || count < 0 || (count > 0 && (!seeds || !results))) return MCE_EINVAL;
  if (s->closed) return MCE_ESTATE;
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  auto now_us = [&]() { return std::chrono::duration<double, std::micro>(clk::now() - t0).count(); };
  std::vector<uint64_t> ids((size_t)count);
  std::vector<int64_t> open;  // submitted, answer not yet taken
  open.reserve(2 * s->ring);
  int64_t next = 0, finished = 0;
  while (finished < count) {
    const double t = now_us();
    while (next < count && (!arrival_us || arrival_us[next] <= t)) {
      uint64_t id = 0;
      const int rc = mce_serve_submit(s, seeds[next], &id);
      if (rc == MCE_ELIMIT) break;  // ring full: admit once answers are taken
      if (rc != MCE_OK) return rc;
      ids[(size_t)next] = id;
      open.push_back(next++);
    }
    size_t keep = 0;
    for (size_t q = 0; q < open.size(); ++q) {
      const int64_t r = open[q];
      const int rc = mce_serve_poll(s, ids[(size_t)r], &results[r]);
      if (rc == MCE_OK) {
        if (latency_us) latency_us[r] = now_us() - (arrival_us ? arrival_us[r] : 0.0);
        ++finished;
      } else if (rc == MCE_EAGAIN) {
        open[keep++] = r;
      } else {
        return rc;
      }
    }
    open.resize(keep);
    if (timeout_ms >= 0 && now_us() > 1000.0 * (double)timeout_ms) return MCE_ETIMEOUT;
  }
  return MCE_OK;
}

extern "C" int mce_serve_stats(mce_serve_t s, mce_serve_stats_t *st) {
  if (!s || !st) return MCE_EINVAL;
  std::memset(st, 0, sizeof(*st));
  for (int c = 0; c < 2; ++c) {
    const SvRing &R = s->cls[c];
    if (!R.ctl) continue;
    SvCtl ct;
    MCE_CUDA(cudaMemcpy(&ct, R.ctl, sizeof(ct), cudaMemcpyDeviceToHost));
    st->submitted += R.tail;
    st->served += ct.served;
    st->tree_nodes += ct.nodes;
    st->helps += ct.helped;
    st->arena_bytes += (uint64_t)s->args.cls[c].arena_bytes * (uint64_t)s->args.cls[c].slots;
    if (c == 0) st->peak_in_flight = ct.peak;
  }
  st->slots = s->args.cls[0].slots + s->args.cls[1].slots;
  st->small_slots = s->args.cls[1].slots;
  st->small_cap = s->small_cap;
  st->ring = s->ring;
  st->kernel_launches = s->launches;
  st->slab_bytes = (uint64_t)s->args.slab_words * 8 *
                   ((uint64_t)s->grid[0] * SV_WARPS + (uint64_t)s->grid[1] * (SV_SMALL / 32));
  for (cudaStream_t q : s->stream)
    if (q && cudaStreamQuery(q) == cudaErrorNotReady) st->running = 1;
  return MCE_OK;
}

extern "C" int mce_serve_close(mce_serve_t s) {
  if (!s) return MCE_EINVAL;
  if (!s->closed) {
    s->closed = true;
    for (SvRing &R : s->cls)
      if (R.hdr) __atomic_store_n(&R.hdr->stop, 1u, __ATOMIC_RELEASE);
  }
  // Every slot finishes its request and leaves once nothing is published.
  // A request published just as the last slot left idle is served by one
  // more launch (which sees the stop flags and leaves when done).
  int rc = MCE_OK;
  for (int pass = 0; pass < 3 && rc == MCE_OK; ++pass) {
    for (cudaStream_t q : s->stream)
      if (q && cudaStreamSynchronize(q) != cudaSuccess) rc = MCE_ECUDA;
    if (rc != MCE_OK) break;
    bool pending = false;
    for (int c = 0; c < 2 && rc == MCE_OK; ++c) {
      const SvRing &R = s->cls[c];
      if (!R.ctl) continue;
      SvCtl ct;
      if (cudaMemcpy(&ct, R.ctl, sizeof(ct), cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = MCE_ECUDA;
      } else if (ct.next < R.tail) {
        pending = true;
        rc = sv_launch(s, c);
      }
    }
    if (!pending) break;
  }
  sv_free(s);
  return rc;
}
