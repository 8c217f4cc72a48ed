// Search-engine device code shared by the counting kernels (bk.cu) and
// the serving kernel (serve.cu): the register engine (reg_encode /
// reg_tree) and the wide engine (mem_encode / mem_tree) walk the search
// tree of one root - or one shared subtree - per warp.
#pragma once

#include <climits>

#include "common.cuh"
#include "kernels.h"
#include "queue.cuh"

namespace mce {
namespace {


using u64 = unsigned long long;

template <typename W>
struct WOps;
template <>
struct WOps<uint32_t> {
  static __device__ __forceinline__ int popc(uint32_t x) { return __popc(x); }
  static __device__ __forceinline__ int ctz(uint32_t x) { return __ffs(x) - 1; }
  static __device__ __forceinline__ uint32_t bit(int i) { return 1u << i; }
  static __device__ __forceinline__ uint32_t low(int d) { return d >= 32 ? ~0u : ((1u << d) - 1u); }
};
template <>
struct WOps<u64> {
  static __device__ __forceinline__ int popc(u64 x) { return __popcll(x); }
  static __device__ __forceinline__ int ctz(u64 x) { return __ffsll((long long)x) - 1; }
  static __device__ __forceinline__ u64 bit(int i) { return 1ull << i; }
  static __device__ __forceinline__ u64 low(int d) { return d >= 64 ? ~0ull : ((1ull << d) - 1ull); }
};

constexpr int REG_BLOCK = 256;  // 8 warps
constexpr int MEM_BLOCK = 128;  // 4 warps
constexpr int REG_CHUNK = 1;    // roots fetched per atomic by the register engine

__device__ __forceinline__ int warp_incl_scan(int x) {
  const int lane = (int)lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(MCE_FULL, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ uint32_t hash_word(u64 x) {
  return (uint32_t)((x * 0x9E3779B97F4A7C15ull) >> 32);
}

// warp-uniform answer to "should this warp hand a child to the queue?"
__device__ __forceinline__ bool wants_task(const QueueView &q) {
  int w = 0;
  if (lane_id() == 0) w = q_wants(q) ? 1 : 0;
  return __shfl_sync(MCE_FULL, w, 0) != 0;
}

// Per-warp evaluation log (opts.warp_log): this warp's record in the launch:
// {SM, tree nodes, donations, cycles per phase[7]}.
constexpr int WLOG_WORDS = 10;
__device__ __forceinline__ u64 *warp_record(const BKArgs &a) {
  return a.warp_log + WLOG_WORDS * (((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
}

// Cycle breakdown of a warp (opts.warp_log = 2) in the categories of the
// reference's -m mce-bd-eval (mce/mce.cuh:385-390): time is charged to the
// current phase whenever the warp switches to another one.
enum BdPhase { BD_OTHER, BD_ENCODE, BD_QUEUE, BD_PIVOT, BD_SETS, BD_MAXIMAL, BD_BRANCH };
struct Bd {
  u64 acc[7];
  u64 last;
  int cur;
  __device__ void start() {
    for (int i = 0; i < 7; ++i) acc[i] = 0;
    last = clock64();
    cur = BD_OTHER;
  }
  __device__ void to(int k) {
    const u64 t = clock64();
    acc[cur] += t - last;
    last = t;
    cur = k;
  }
};
#define MCE_BD(k)                    \
  do {                               \
    if constexpr (EV == 2) bd->to(k); \
  } while (0)

__device__ __forceinline__ uint32_t sm_id() {
  uint32_t id;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
  return id;
}

// Per-root outputs shared by donor and takers: accumulate.
__device__ __forceinline__ void root_done(const BKArgs &a, int32_t r, u64 nodes, u64 cnt) {
  if (lane_id() != 0) return;
  if (a.root_nodes && nodes) atomicAdd(&a.root_nodes[r], nodes);
  if (a.root_count && cnt) atomicAdd(&a.root_count[r], cnt);
  if (a.graph_count && cnt) atomicAdd(&a.graph_count[a.graph_of[r]], cnt);
}

// opts.count_ops: the algorithmic 32-bit word operations of a root's (or a
// task's) walk, per root when roots are logged.
__device__ __forceinline__ void root_ops_done(const BKArgs &a, int32_t r, u64 ops) {
  if (lane_id() == 0 && a.root_ops && ops) atomicAdd(&a.root_ops[r], ops);
}

// Idle phase shared by the engines: take tasks until no work is left.
// `run(words)` processes one task whose words were stored by `put`.
template <typename Put, typename Run>
__device__ void idle_phase(const BKArgs &a, Put put, Run run) {
  const QueueView &q = a.q;
  const uint32_t lane = lane_id();
  if (lane == 0) atomicAdd(&q.hdr->idle, 1u);
  uint32_t last_epoch = 0;
  uint64_t t_last = 0;
  if (lane == 0) {
    last_epoch = ld_volatile(&q.hdr->epoch);
    t_last = globaltimer_ns();
  }
  uint32_t ns = 64;
  for (;;) {
    if (q_pop(q, put)) {
      if (lane == 0) atomicSub(&q.hdr->idle, 1u);
      run();
      if (lane == 0) {
        atomicSub(&q.hdr->work, 1u);
        atomicAdd(&q.hdr->epoch, 1u);
        atomicAdd(&q.hdr->idle, 1u);
        t_last = globaltimer_ns();
      }
      ns = 64;
      continue;
    }
    int stop = 0;
    if (lane == 0) {
      if (ld_volatile(&q.hdr->work) == 0) {
        stop = 1;
      } else {
        const uint32_t e = ld_volatile(&q.hdr->epoch);
        const uint64_t now = globaltimer_ns();
        if (e != last_epoch) {
          last_epoch = e;
          t_last = now;
        } else if (now - t_last > a.wait_limit_ns) {
          atomicOr(a.err, MCE_ERR_WAIT_TIMEOUT);  // no progress anywhere: give up
          stop = 1;
        }
      }
    }
    if (__shfl_sync(MCE_FULL, stop, 0)) break;
    __nanosleep(ns);
    if (ns < 8192) ns <<= 1;
  }
  if (lane == 0) atomicSub(&q.hdr->idle, 1u);
}

// ---------------------------------------------------------------------------
// Register engine: d+ <= 32 * NR; lane i holds rows i (and i + 32).
// ---------------------------------------------------------------------------
template <typename Word, int NR>
struct RegSmem {
  Word rows[32 * NR];       // induced-subgraph rows while they are built
  Word xs[32];              // earlier-neighbour rows while they are built
  Word stk[32 * NR + 1][NR == 1 ? 5 : 4]; // DFS frames: P, X, branch set, chosen set
                                          // (+ pending leaves, 32-bit rows)
  int32_t pl[32 * NR];      // the root's later neighbours (sorted ids), padded
  int32_t off[32];          // flattened-walk prefix offsets of the items' lists
  int32_t beg[32];          // ... and the lists' starts
  int32_t own[32];          // ... and the item whose list starts at a window position
  int32_t hkey[128];        // hash of P (128 slots for up to 32 * NR ids): vertex id (-1: empty) ...
  uint8_t hidx[128];        // ... and its index in P
  Word xl0[32];             // the first 32 leaf-filter rows (the rest: slab xl)
  // Long leaf-filter lists (hub roots) are compacted on the way down: lb is
  // where the current list starts in the slab (-1: xl0 + xl), and each DFS
  // frame keeps its list's start and length to return to.
  int32_t lb;
  int32_t flb[32 * NR + 1], fln[32 * NR + 1];
};

// Flattened walk over the concatenated lists of up to 32 items (lane t
// holds item t's list start b and length len; the lists live in cs): calls
// f(t, element) for every element, 32 at a time.  The owner of a position
// is the last item whose list starts at or before it, read from a bitmask
// of the list starts inside the current window.
template <typename F>
__device__ __forceinline__ void flat_walk(const int32_t *__restrict__ cs, int32_t b, int len,
                                          int32_t *off_sm, int32_t *beg_sm, int32_t *own_sm,
                                          F f) {
  const int lane = (int)lane_id();
  const int incl = warp_incl_scan(len);
  const int T = __shfl_sync(MCE_FULL, incl, 31);
  const int off = incl - len;
  off_sm[lane] = off;
  beg_sm[lane] = b;
  int carry = 0;
  for (int e0 = 0; e0 < T; e0 += 32) {
    const bool st = len > 0 && off >= e0 && off < e0 + 32;
    if (st) own_sm[off - e0] = lane;
    const uint32_t mask = __reduce_or_sync(MCE_FULL, st ? 1u << (off - e0) : 0u);
    __syncwarp();
    const uint32_t below = mask & (0xFFFFFFFFu >> (31 - lane));
    const int t = below ? own_sm[31 - __clz(below)] : carry;
    carry = __shfl_sync(MCE_FULL, t, 31);
    const int e = e0 + lane;
    if (e < T) f(t, cs[beg_sm[t] + (e - off_sm[t])]);
    __syncwarp();
  }
}

// Staging of the lists a flattened walk reads (opts.stage_lists, the 32-bit
// engine): each lane copies its list's 16-byte window - start rounded down,
// end rounded up - from global to shared memory with one 1-D bulk copy, the
// warp waits on its mbarrier, and the walk reads shared memory.  Per warp
// of the block: STAGE_WORDS ints of buffer, the mbarrier, and a state word
// (bit 0: parity of the barrier's next phase; bit 1: staging off after a
// wait ran out - the warp then loads from global memory).  Only the kernels
// that stage reference these arrays, so only they allocate them.  Lists
// whose windows do not fit together take flat_walk.
constexpr int STAGE_WORDS = 512;
constexpr uint64_t STAGE_WAIT_NS = 2000000000ull;  // a copy of a few KB takes microseconds
__shared__ __align__(16) int32_t stage_buf[REG_BLOCK / 32][STAGE_WORDS];
__shared__ unsigned long long stage_bar[REG_BLOCK / 32];
__shared__ uint32_t stage_state[REG_BLOCK / 32];

__device__ __forceinline__ void stage_init() {
  const int w = (int)(threadIdx.x >> 5);
  if (lane_id() == 0) {
    mbar_init(&stage_bar[w], 1);
    stage_state[w] = 0;
  }
  __syncwarp();
}

template <typename F>
__device__ __forceinline__ bool flat_walk_staged(const int32_t *__restrict__ cs, int32_t b, int len,
                                                 int32_t *off_sm, int32_t *beg_sm, int32_t *own_sm,
                                                 uint32_t *err, F f) {
  const int lane = (int)lane_id(), w = (int)(threadIdx.x >> 5);
  const uint32_t st0 = stage_state[w];
  if (st0 & 2u) return false;
  const int32_t *src = cs + b;
  const int pad = (int)(((uintptr_t)src >> 2) & 3u);  // ints before the list in its window
  const int words = len > 0 ? ((pad + len + 3) & ~3) : 0;
  const int wincl = warp_incl_scan(words);
  const int total = __shfl_sync(MCE_FULL, wincl, 31);
  if (total == 0 || total > STAGE_WORDS) return false;
  const int wbeg = wincl - words;
  __syncwarp();  // the buffer's last contents are read
  fence_proxy_async_smem();
  if (lane == 0) mbar_arrive_expect_tx(&stage_bar[w], (uint32_t)total * 4u);
  __syncwarp();
  if (words > 0) bulk_copy_g2s(&stage_buf[w][wbeg], src - pad, (uint32_t)words * 4u, &stage_bar[w]);
  const uint32_t ph = st0 & 1u;
  const bool ok = __all_sync(MCE_FULL, mbar_wait(&stage_bar[w], ph, err, STAGE_WAIT_NS));
  __syncwarp();
  if (lane == 0) stage_state[w] = (st0 ^ 1u) | (ok ? 0u : 2u);
  if (!ok) {  // let the copies in flight land before the buffer is given up
    mbar_wait(&stage_bar[w], ph, err, STAGE_WAIT_NS);
    __syncwarp();
    return false;
  }
  const int32_t *buf = stage_buf[w];
  const int incl = warp_incl_scan(len);
  const int T = __shfl_sync(MCE_FULL, incl, 31);
  const int off = incl - len;
  off_sm[lane] = off;
  beg_sm[lane] = wbeg + pad;  // the list's first element in the buffer
  int carry = 0;
  for (int e0 = 0; e0 < T; e0 += 32) {
    const bool st = len > 0 && off >= e0 && off < e0 + 32;
    if (st) own_sm[off - e0] = lane;
    const uint32_t mask = __reduce_or_sync(MCE_FULL, st ? 1u << (off - e0) : 0u);
    __syncwarp();
    const uint32_t below = mask & (0xFFFFFFFFu >> (31 - lane));
    const int t = below ? own_sm[31 - __clz(below)] : carry;
    carry = __shfl_sync(MCE_FULL, t, 31);
    const int e = e0 + lane;
    if (e < T) f(t, buf[beg_sm[t] + (e - off_sm[t])]);
    __syncwarp();
  }
  return true;
}

// Hash of the root's later neighbours (ids are distinct): 128 slots, so that
// the probes of the many later-list elements outside P end within ~1.4 slots
// for the 32-bit engine (4 slots per id) and ~2.5 for the 64-bit one (2).
template <typename Word, int NR>
__device__ __forceinline__ uint32_t p_slot(int32_t w) {
  return ((uint32_t)w * 0x9E3779B1u) >> 25;
}

template <typename Word, int NR>
__device__ __forceinline__ void p_hash_build(RegSmem<Word, NR> &sm, int d) {
  const int lane = (int)lane_id();
  for (int i = lane; i < 128; i += 32) sm.hkey[i] = -1;
  __syncwarp();
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int i = lane + 32 * k;
    if (i < d) {
      const int32_t w = sm.pl[i];
      uint32_t h = p_slot<Word, NR>(w);
      while (atomicCAS(&sm.hkey[h], -1, w) != -1) h = (h + 1) & 127u;
      sm.hidx[h] = (uint8_t)i;
    }
  }
  __syncwarp();
}

// index of w in P, or -1
template <typename Word, int NR>
__device__ __forceinline__ int p_find(const RegSmem<Word, NR> &sm, int32_t w) {
  uint32_t h = p_slot<Word, NR>(w);
  for (;;) {
    const int32_t k = sm.hkey[h];
    if (k == w) return sm.hidx[h];
    if (k == -1) return -1;
    h = (h + 1) & 127u;
  }
}

// Per-warp slab of the register engine, in Words, for xc = the x-row
// capacity (a power of two): a hash set used while the earlier-neighbour
// rows are built (2 xc), the distinct rows (xc) and the rows adjacent to the
// current branch (xc).
template <typename Word>
struct RegSlab {
  Word *hash, *xr, *xl;
  int xc;
};

__device__ __forceinline__ int reg_xcap(const BKArgs &a) { return a.rxcap ? a.rxcap : REG_XCAP; }

template <typename Word>
__device__ __forceinline__ RegSlab<Word> reg_slab(const BKArgs &a, int64_t gw) {
  Word *base = (Word *)(a.slab + (size_t)gw * a.slab_words);
  RegSlab<Word> s;
  s.xc = reg_xcap(a);
  s.hash = base;
  s.xr = base + 2 * s.xc;
  s.xl = s.xr + s.xc;
  return s;
}

template <typename Word, int NR>
__device__ __forceinline__ Word row_of(Word r0, Word r1, int j) {
  if constexpr (NR == 2) return __shfl_sync(MCE_FULL, j >= 32 ? r1 : r0, j & 31);
  return __shfl_sync(MCE_FULL, r0, j & 31);
}

// Encoded state of the root a warp currently works on.
template <typename Word>
struct RegRoot {
  int32_t r = -1;
  int d = 0, nX = 0;
  Word r0 = 0, r1 = 0;
};

// STAGE: the lists are staged in shared memory by bulk copies (*stg).
template <typename Word, int NR, bool STAGE = false>
__device__ void reg_encode(const BKArgs &a, RegSmem<Word, NR> &sm, const RegSlab<Word> &sl,
                           int32_t r, RegRoot<Word> &rt) {
  using O = WOps<Word>;
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  auto walk = [&](int32_t b, int len, auto f) {
    if constexpr (STAGE)
      if (flat_walk_staged(a.cs, b, len, sm.off, sm.beg, sm.own, a.err, f)) return;
    flat_walk(a.cs, b, len, sm.off, sm.beg, sm.own, f);
  };
  const int32_t sb = a.split[r], d = a.rp[r + 1] - sb, ub = a.rp[r], u = sb - ub;
  if (u > sl.xc) {  // more earlier neighbours than the slab's rows (classification bounds it)
    if (lane == 0) atomicOr(a.err, MCE_ERR_XROWS);
    rt.r = r;
    rt.d = 0;
    rt.nX = 0;
    return;
  }

  // setup_stack_original_L1_IP (mce/mce_utils.cuh:565-611): P = N+(r)
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int i = lane + 32 * k;
    sm.pl[i] = i < d ? a.cs[sb + i] : INT_MAX;
    sm.rows[i] = 0;
  }
  __syncwarp();

  p_hash_build(sm, d);

  if (d + u <= 32) {
    // Small root: one flattened walk over the later lists of the P vertices
    // (lanes [0, d)) and of the earlier neighbours (lanes [d, d + u)).
    int b = 0, len = 0;
    if (lane < d + u) {
      const int32_t item = lane < d ? sm.pl[lane] : a.cs[ub + lane - d];
      b = a.split[item];
      len = a.rp[item + 1] - b;
    }
    sm.xs[lane] = 0;
    __syncwarp();
    walk(b, len, [&](int t, int32_t w) {
      const int i = p_find(sm, w);
      if (i >= 0) {
        if (t < d) {
          atomicOr(&sm.rows[t], O::bit(i));
          atomicOr(&sm.rows[i], O::bit(t));
        } else {
          atomicOr(&sm.xs[t - d], O::bit(i));
        }
      }
    });
    __syncwarp();
    rt.r0 = sm.rows[lane];
    rt.r1 = 0;
    if constexpr (NR == 2) rt.r1 = sm.rows[lane + 32];
    // the distinct non-empty earlier-neighbour rows, in lane order
    const Word row = lane < u ? sm.xs[lane] : (Word)0;
    const uint32_t same = __match_any_sync(MCE_FULL, row);
    const bool fresh = lane < u && row != 0 && (same & lt) == 0;
    const uint32_t mk = __ballot_sync(MCE_FULL, fresh);
    if (fresh) sl.xr[__popc(mk & lt)] = row;
    __syncwarp();
    rt.r = r;
    rt.d = d;
    rt.nX = __popc(mk);
    return;
  }

  // warp_sorted_count_and_encode_full (mce/mce_utils.cuh:90-117): bit (j, i)
  // and (i, j) for every later neighbour w = P[i] of v = P[j].  The later
  // lists of 32 P vertices are flattened over the lanes.
  for (int c = 0; c * 32 < d; ++c) {
    const int items = min(32, d - c * 32);
    int vb = 0, vlen = 0;
    if (lane < items) {
      const int32_t v = sm.pl[c * 32 + lane];
      vb = a.split[v];
      vlen = a.rp[v + 1] - vb;
    }
    walk(vb, vlen, [&](int t, int32_t w) {
      const int i = p_find(sm, w);
      if (i >= 0) {
        const int j = c * 32 + t;
        atomicOr(&sm.rows[j], O::bit(i));
        atomicOr(&sm.rows[i], O::bit(j));
      }
    });
    __syncwarp();
  }
  rt.r0 = sm.rows[lane];
  rt.r1 = 0;
  if constexpr (NR == 2) rt.r1 = sm.rows[lane + 32];

  // Earlier neighbours x of r: row(x) = N(x) & P, kept once per distinct
  // non-empty value; x is earlier than every vertex of P, so N(x) & P lies
  // in N+(x).  Up to 32 of them are deduplicated with one match over the
  // warp; more go through a hash set in the slab.
  int nX = 0;
  // A hub's rows were built before the search (hub_rows_launch); its first
  // encode writes the distinct ones back there and publishes their number
  // (hub_nx), so the warps that take its subtrees later only copy them.
  const int32_t hub = (u > 0 && a.hub_of) ? a.hub_of[r] : -1;
  unsigned long long *hrows = hub >= 0 ? a.hub_rows + a.hub_off[hub] : nullptr;
  int kept = -1;
  if (hrows) {
    if (lane == 0) kept = (int)ld_acquire(reinterpret_cast<const uint32_t *>(a.hub_nx + hub));
    kept = __shfl_sync(MCE_FULL, kept, 0);
    __syncwarp();  // the other lanes read after lane 0's acquire
  }
  if (kept >= 0) {
    for (int i = lane; i < kept; i += 32) sl.xr[i] = (Word)__ldcg(hrows + i);  // from L2
    __syncwarp();
    nX = kept;
  } else if (u > 0) {
    const bool hashed = u > 32;
    int hc = 32;
    if (hashed) {
      while (hc < 2 * u && hc < 2 * sl.xc) hc <<= 1;
      for (int i = lane; i < hc; i += 32) sl.hash[i] = 0;
    }
    for (int c = 0; c * 32 < u; ++c) {
      const int items = min(32, u - c * 32);
      Word row;
      if (hrows) {
        row = (Word)hrows[c * 32 + lane];  // zero past the list (padding)
      } else {
        int xb = 0, xlen = 0;
        if (lane < items) {
          const int32_t x = a.cs[ub + c * 32 + lane];
          xb = a.split[x];
          xlen = a.rp[x + 1] - xb;
        }
        sm.xs[lane] = 0;
        __syncwarp();
        walk(xb, xlen, [&](int t, int32_t w) {
          const int i = p_find(sm, w);
          if (i >= 0) atomicOr(&sm.xs[t], O::bit(i));
        });
        __syncwarp();
        row = sm.xs[lane];
      }
      bool fresh = false;
      if (!hashed) {
        const uint32_t same = __match_any_sync(MCE_FULL, row);
        fresh = lane < items && row != 0 && (same & lt) == 0;  // first lane of its value
      } else if (lane < items && row != 0) {
        uint32_t h = hash_word((u64)row) & (uint32_t)(hc - 1);
        for (int probe = 0; probe < hc; ++probe) {
          const Word old = atomicCAS(&sl.hash[h], (Word)0, row);
          if (old == 0) {
            fresh = true;
            break;
          }
          if (old == row) break;
          h = (h + 1) & (uint32_t)(hc - 1);
        }
      }
      const uint32_t mk = __ballot_sync(MCE_FULL, fresh);
      if (fresh) sl.xr[nX + __popc(mk & lt)] = row;
      nX += __popc(mk);
      __syncwarp();
    }
    // rows [0, nX) of the hub's region are no longer read as built; with
    // several warps per root two of them may encode the hub at once, so
    // then the rows stay as built and every warp deduplicates them itself
    if (hrows && a.parts <= 1) {
      for (int i = lane; i < nX; i += 32) hrows[i] = (u64)sl.xr[i];
      __threadfence();
      __syncwarp();
      if (lane == 0) st_release(reinterpret_cast<uint32_t *>(a.hub_nx + hub), (uint32_t)nX);
    }
  }
  rt.r = r;
  rt.d = d;
  rt.nX = nX;
}

// Rows [32, nL) of the leaf filter (in the slab): does one contain S?  Four
// windows of loads are in flight per step; hub roots keep thousands.
template <typename Word>
__device__ __forceinline__ bool xl_covers(const Word *xl, int nL, Word S) {
  const int lane = (int)lane_id();
  for (int i0 = 32; i0 < nL; i0 += 128) {
    bool hit = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + 32 * q + lane;
      if (i < nL) hit |= (xl[i] & S) == S;
    }
    if (__any_sync(MCE_FULL, hit)) return true;
  }
  return false;
}

// The leaf filter of a depth-0 branch: the rows of xr[0, nX) adjacent to
// branch vertex vb, the first 32 into xl0 (shared memory), the rest into xl.
template <typename Word>
__device__ __forceinline__ int xl_filter(const Word *xr, int nX, Word vb, Word *xl0, Word *xl) {
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  int nL = 0;
  for (int i0 = 0; i0 < nX; i0 += 128) {
    Word rw[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + 32 * q + lane;
      rw[q] = i < nX ? xr[i] : (Word)0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool has = (rw[q] & vb) != 0;
      const uint32_t mk = __ballot_sync(MCE_FULL, has);
      if (has) {
        const int at = nL + __popc(mk & lt);
        (at < 32 ? xl0 : xl)[at] = rw[q];
      }
      nL += __popc(mk);
    }
  }
  return nL;
}

// The rows of a leaf-filter list (i < 32 at l0[i], the rest at l1[i]) that
// contain every vertex of S, appended to dst; returns their number.  Not
// inlined: only hub roots' long lists take this path, and the search loop
// keeps its registers.
template <typename Word>
__device__ __noinline__ int xl_compact(const Word *l0, const Word *l1, int nL, Word S, Word *dst) {
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  int k = 0;
  for (int i0 = 0; i0 < nL; i0 += 32) {
    const int i = i0 + lane;
    const Word row = i < nL ? (i < 32 ? l0[i] : l1[i]) : (Word)0;
    const bool keep = i < nL && (row & S) == S;
    const uint32_t mk = __ballot_sync(MCE_FULL, keep);
    if (keep) dst[k + __popc(mk & lt)] = row;
    k += __popc(mk);
  }
  __syncwarp();
  return k;
}

// Leaf-filter row i: the first 32 in shared memory, the rest in the slab.
template <typename Word>
__device__ __forceinline__ Word xrow(const Word *first32, const Word *rest, int i) {
  return i < 32 ? first32[i] : rest[i];
}

// X-in-subgraph pivoting (-i px, opts.x_pivot): among the root's earlier
// neighbours adjacent to the whole chosen set (rows[0 .. cnt) containing
// `chosen`), the one with the most neighbours in Pn - the reference's
// select_pivot_from_Xx (mce/mce_utils.cuh:404-472).  Returns the key
// ((score + 1) << 11 | (2047 - row)) or 0; *elim: one of them is adjacent to
// all of Pn, so no clique below is maximal.
template <typename Word>
__device__ __forceinline__ int outside_pivot(const Word *first32, const Word *rest, int cnt,
                                             Word chosen, Word Pn, int pcn, bool *elim) {
  const int lane = (int)lane_id();
  int k = 0;
  bool el = false;
  for (int i0 = 0; i0 < cnt; i0 += 32) {
    const int i = i0 + lane;
    if (i < cnt) {
      const Word row = xrow(first32, rest, i);
      if ((row & chosen) == chosen) {
        const int sc = WOps<Word>::popc(Pn & row);
        el |= sc == pcn;
        // the key holds 11 bits of index: rows past 2,047 prune but are not pivots
        if (i < 2048) k = max(k, ((sc + 1) << 11) | (2047 - i));
      }
    }
  }
  *elim = __any_sync(MCE_FULL, el);
  return (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
}

// Clique listing (mce_list): each maximal clique becomes the record
// {size, root, members...} at a position of a.list_buf taken with one
// atomicAdd; a record past a.list_cap is counted but not written.
template <typename Word, int NR>
__device__ __forceinline__ void reg_emit(const BKArgs &a, const RegSmem<Word, NR> &sm, int32_t r,
                                         Word Sc) {
  const int lane = (int)lane_id();
  const int sz = WOps<Word>::popc(Sc) + 1;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(a.list_words, (unsigned long long)(sz + 1));
  base = __shfl_sync(MCE_FULL, base, 0);
  if (base + (unsigned long long)sz + 1 > a.list_cap) return;
  if (lane == 0) {
    a.list_buf[base] = sz;
    a.list_buf[base + 1] = r;
  }
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int i = lane + 32 * k;
    if ((Sc >> i) & 1)
      a.list_buf[base + 2 + WOps<Word>::popc(Sc & WOps<Word>::low(i))] = sm.pl[i];
  }
}

// Walk the subtree under node (P, X, S) of root rt.r.  For the root itself
// S = 0; for a task S holds the vertices chosen above the node.  With
// Budget, the walk stops once it has visited a.node_budget nodes; with EV
// (opts.warp_log) >= 1 the warp's donations are counted in its a.warp_log
// record, with EV == 2 its cycles are charged to *bd by phase.
//
// OPS (opts.count_ops) counts the algorithmic work of the reference's walk
// in 32-bit word operations into *ops, with W = ceil(d+ / 32) words per row
// whatever the engine's word width: 2W per candidate of a pivot selection
// (AND + POPC over P' | X', select_pivot_from_P_and_Xp,
// mce/mce_utils.cuh:366-402) plus 4W per node for the child sets
// (populate_xl_and_cl, :321-336); a root's first pivot costs 2W per later
// neighbour (select_pivot_from_P, :338-364).  A donated node is counted by
// the warp that created it.  The clique shortcuts are off, so every node of
// the tree is walked (same nodes, counts and histogram).
// SPLIT: the variant for several warps per root (part / parts below).
// L2: the variant that carries an L2 unit's outside rows (XO); the others
// ignore XO.
template <typename Word, int NR, bool Budget = false, int EV = 0, bool LIST = false,
          bool XP = false, bool OPS = false, bool SPLIT = false, bool L2 = false>
__device__ void reg_tree(const BKArgs &a, RegSmem<Word, NR> &sm, const RegSlab<Word> &sl,
                         const RegRoot<Word> &rt, Word P, Word X, Word S, u64 &h0, u64 &h1,
                         u64 &nodes, u64 &cnt, Bd *bd = nullptr, u64 *ops = nullptr,
                         int part = 0, int parts = 1, Word XO = 0) {
  using O = WOps<Word>;
  const u64 w32 = (u64)((rt.d + 31) >> 5);
  MCE_BD(BD_PIVOT);
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const Word r0 = rt.r0, r1 = rt.r1;
  const int nX = rt.nX;
  const bool share = a.q.hdr != nullptr;
  // A root whose later neighbours are pairwise adjacent: Tomita's walk is one
  // path of d nodes (every pivot leaves exactly itself to branch on) ending
  // in the clique P, which is maximal unless an earlier neighbour of the
  // root is adjacent to all of it.  Same nodes and count, no walk.
  if constexpr (!XP && !OPS) {
    const int d = rt.d;
    if (S == 0 && X == 0 && P == O::low(d) && d > 0) {
      bool full = lane >= d || ((r0 | O::bit(lane)) & P) == P;
      if constexpr (NR == 2) full = full && (lane + 32 >= d || ((r1 | O::bit(lane + 32)) & P) == P);
      if (__all_sync(MCE_FULL, full)) {
        if (part != 0) {  // one path: part 0 walks it
          MCE_BD(BD_OTHER);
          return;
        }
        bool covered = false;
        for (int i0 = 0; !covered && i0 < nX; i0 += 32) {
          const int i = i0 + lane;
          covered = __any_sync(MCE_FULL, i < nX && (sl.xr[i] & P) == P);
        }
        nodes += (u64)d;
        if (!covered) {
          ++cnt;
          if constexpr (LIST) reg_emit<Word, NR>(a, sm, rt.r, P);
          const int bin = d - 1;  // clique size - 2
          if (lane == (bin & 31)) {
            if (bin < 32)
              ++h0;
            else
              ++h1;
          }
        }
        MCE_BD(BD_OTHER);
        return;
      }
    }
  }
  // Leaf filter: for the root it is rebuilt at every depth-0 branch (rows
  // adjacent to that branch vertex); for a task it is built once (rows
  // containing the whole chosen set).
  // List compaction runs in the 64-bit engine, where hub roots' long lists
  // set the class's length; the 32-bit engine keeps its registers.
  constexpr bool kCompact = NR == 2;
  const bool per_branch = (S == 0);
  int nL = 0;
  if (!per_branch && nX > 0) {
    for (int i0 = 0; i0 < nX; i0 += 32) {
      const int i = i0 + lane;
      const Word row = i < nX ? sl.xr[i] : (Word)0;
      const bool has = i < nX && (row & S) == S;
      const uint32_t mk = __ballot_sync(MCE_FULL, has);
      if (has) {
        const int at = nL + __popc(mk & lt);
        (at < 32 ? sm.xl0 : sl.xl)[at] = row;
      }
      nL += __popc(mk);
    }
  }
  if (L2 && XO) {  // an L2 unit's outside rows: the root's later neighbours earlier than its edge
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const Word row = k == 0 ? r0 : r1;
      const bool has = ((XO >> (lane + 32 * k)) & 1) && (row & S) == S;
      const uint32_t mk = __ballot_sync(MCE_FULL, has);
      if (nL + __popc(mk) > 32 + sl.xc) {  // the list's capacity (never reached: nL <= d-)
        if (lane == 0) atomicOr(a.err, MCE_ERR_XROWS);
        return;
      }
      if (has) {
        const int at = nL + __popc(mk & lt);
        (at < 32 ? sm.xl0 : sl.xl)[at] = row;
      }
      nL += __popc(mk);
    }
  }
  if (kCompact && lane == 0) sm.lb = -1;
  __syncwarp();
  // pivot of the start node (select_pivot_from_P / _and_Xp, mce/mce_utils.cuh:338-402)
  int start_k = 0;
  Word start_row = 0;
  bool start_out = false;
  bool iso0 = false, iso1 = false;  // this lane's candidate has no neighbour in P
  {
    const Word cand = P | X;
    const int pc = O::popc(P);
    if constexpr (OPS)
      if (S == 0 && part == 0) *ops += 2 * w32 * (u64)O::popc(cand);  // the root's first pivot
    int k = 0;
    bool el = false;
    if ((cand >> lane) & 1) {
      const int s = O::popc(P & r0);
      k = ((s + 1) << 7) | (127 - lane);
      el = ((X >> lane) & 1) && s == pc;
      iso0 = ((P >> lane) & 1) && s == 0;
    }
    if constexpr (NR == 2) {
      if ((cand >> (lane + 32)) & 1) {
        const int s = O::popc(P & r1);
        k = max(k, ((s + 1) << 7) | (127 - (lane + 32)));
        el = el || (((X >> (lane + 32)) & 1) && s == pc);
        iso1 = ((P >> (lane + 32)) & 1) && s == 0;
      }
    }
    bool elo = false;
    int ko = 0;
    if constexpr (XP) {  // the root's rows all contain S = 0; a task's are in the filter
      if (per_branch && nX > 0)
        ko = outside_pivot(sl.xr, sl.xr, nX, (Word)0, P, pc, &elo);
      else if (nL > 0)
        ko = outside_pivot(sm.xl0, sl.xl, nL, S, P, pc, &elo);
    }
    if (__any_sync(MCE_FULL, el) || elo || P == 0) {
      MCE_BD(BD_OTHER);
      return;
    }
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    start_k = k;
    if (XP && (ko >> 11) > (k >> 7)) {  // an earlier neighbour covers more of P
      const int i = 2047 - (ko & 2047);
      start_row = (per_branch ? sl.xr[i] : xrow(sm.xl0, sl.xl, i));
      start_out = true;
    }
  }
  MCE_BD(BD_SETS);
  // apply_pivot_to_first_level (:204-216) / apply_pivot_to_next_level (:218-239)
  Word B = P & ~(start_out ? start_row : row_of<Word, NR>(r0, r1, 127 - (start_k & 127)));
  int depth = 0, recheck = 0, b0 = 0;  // b0: first-level branches passed
  bool want = false;
  // Leaves in bulk: a branch u of the node (Pn, Xn, Sn) with no neighbour in
  // Pn has an empty candidate set whatever its earlier siblings, so its child
  // is a leaf: the clique Sn + u is maximal iff (Xn | branches before u) has
  // no neighbour of u and no earlier-neighbour row of the root covers Sn + u.
  // All such branches are settled together from the pivot scores (one node
  // each, the same count and histogram as walking them) and leave the branch
  // set; their moves from P to X are applied when a later sibling is
  // branched (Lp, kept in the frame).  Not in the listing or op-counting
  // variants, nor for the first level of a root split over warps; with a
  // node budget the walk stops as soon as settled leaves pass it.
  // The 64-bit engine keeps its walk: the extra live values made it spill
  // more than the settled leaves saved (8.45 -> 8.77 ms on the batch).
  constexpr bool kBulk = !OPS && !LIST && NR == 1;
  Word Lp = 0;   // the current frame's settled leaves not yet moved from P to X
  Word xuni = 0; // the union of the root's earlier-neighbour rows (depth-0 leaves)
  if constexpr (kBulk) {
    if (per_branch && nX > 0) {
      Word acc = 0;
      for (int i = lane; i < nX; i += 32) acc |= sl.xr[i];
      xuni = (Word)__reduce_or_sync(MCE_FULL, (uint32_t)acc);
      if constexpr (sizeof(Word) == 8)
        xuni |= (Word)__reduce_or_sync(MCE_FULL, (uint32_t)((u64)acc >> 32)) << 32;
    }
  }
  auto take_leaves = [&](Word Bn, Word Pn, Word Xn, Word Sn) -> Word {
    Word L = (Word)__ballot_sync(MCE_FULL, iso0);
    if constexpr (NR == 2) L |= (Word)__ballot_sync(MCE_FULL, iso1) << 32;
    L &= Bn;
    if (L == 0) return 0;
    bool m0 = ((L >> lane) & 1) && ((Xn | (Bn & O::low(lane))) & r0) == 0;
    Word M = (Word)__ballot_sync(MCE_FULL, m0);
    if constexpr (NR == 2) {
      const bool m1 = ((L >> (lane + 32)) & 1) && ((Xn | (Bn & O::low(lane + 32))) & r1) == 0;
      M |= (Word)__ballot_sync(MCE_FULL, m1) << 32;
    }
    nodes += (u64)O::popc(L);
    if (M) {
      Word cover = 0;
      if (per_branch && depth == 0) {
        cover = xuni;
      } else if (nL > 0) {
        const int lb = kCompact ? sm.lb : -1;
        const Word *L0 = lb < 0 ? sm.xl0 : sl.xl + lb, *L1 = lb < 0 ? sl.xl : L0;
        Word acc = 0;
        for (int i = lane; i < nL; i += 32) {
          const Word row = i < 32 ? L0[i] : L1[i];
          if ((row & Sn) == Sn) acc |= row;
        }
        cover = (Word)__reduce_or_sync(MCE_FULL, (uint32_t)acc);
        if constexpr (sizeof(Word) == 8)
          cover |= (Word)__reduce_or_sync(MCE_FULL, (uint32_t)((u64)acc >> 32)) << 32;
      }
      M &= ~cover;
      if (M) {
        const u64 k = (u64)O::popc(M);
        cnt += k;
        const int bin = O::popc(Sn);  // clique size - 2
        if (lane == (bin & 31)) {
          if (bin < 32)
            h0 += k;
          else
            h1 += k;
        }
      }
    }
    return L;
  };
  if constexpr (kBulk) {
    if (!(SPLIT && parts > 1)) {  // a split root's first level keeps its order
      Lp = take_leaves(B, P, X, S);
      B &= ~Lp;
    }
    if (Budget && a.node_budget && nodes > a.node_budget) {  // a serving request over its budget
      if (lane == 0) atomicOr(a.err, MCE_ERR_BUDGET);
      MCE_BD(BD_OTHER);
      return;
    }
  }
  for (;;) {
    MCE_BD(BD_BRANCH);
    if (B == 0) {  // get_next_candidate found nothing: backtrack (:526-563)
      if (depth == 0) break;
      --depth;
      P = sm.stk[depth][0];
      X = sm.stk[depth][1];
      B = sm.stk[depth][2];
      S = sm.stk[depth][3];
      if constexpr (kBulk) Lp = sm.stk[depth][4];
      if constexpr (kCompact) {
        nL = sm.fln[depth];
        __syncwarp();
        if (lane == 0) sm.lb = sm.flb[depth];
        __syncwarp();
      }
      continue;
    }
    const int v = O::ctz(B);
    B &= B - 1;
    const Word vb = O::bit(v);
    const Word rv = row_of<Word, NR>(r0, r1, v);
    MCE_BD(BD_SETS);
    if constexpr (kBulk) {
      if (Lp) {  // the settled leaves before v have left P for X
        const Word mv = Lp & O::low(v);
        P &= ~mv;
        X |= mv;
        Lp &= ~mv;
      }
    }
    // populate_xl_and_cl (:321-336): child P' = P & N(v), X' = X & N(v);
    // v leaves P for X in this frame.
    const Word Pc = P & rv, Xc = X & rv, Sc = S | vb;
    P &= ~vb;
    X |= vb;
    // several warps per root: this one walks every parts-th first-level
    // branch (the others still move from P to X, as the full walk would)
    if constexpr (SPLIT)
      if (parts > 1 && depth == 0 && (b0++ % parts) != part) continue;
    ++nodes;
    if constexpr (OPS) *ops += 2 * w32 * (u64)O::popc(Pc | Xc) + 4 * w32;
    if (Budget && a.node_budget && nodes > a.node_budget) {  // a serving request over its budget
      if (lane == 0) atomicOr(a.err, MCE_ERR_BUDGET);
      break;
    }
    if (per_branch && depth == 0 && nX > 0) {  // earlier neighbours adjacent to v
      nL = xl_filter<Word>(sl.xr, nX, vb, sm.xl0, sl.xl);
      __syncwarp();
    }
    if (Pc == 0) {
      MCE_BD(BD_MAXIMAL);
      // test_maximality (:507-524): P' and X' empty and no earlier
      // neighbour of the root adjacent to the whole clique.
      if (Xc == 0) {
        bool covered = false;
        if (nL > 0) {
          const int lb = kCompact ? sm.lb : -1;
          const Word *L0 = lb < 0 ? sm.xl0 : sl.xl + lb, *L1 = lb < 0 ? sl.xl : L0;
          covered = __any_sync(MCE_FULL, lane < nL && (L0[lane] & Sc) == Sc);
          if (!covered && nL > 32) covered = xl_covers<Word>(L1, nL, Sc);
        }
        if (!covered) {
          ++cnt;
          if constexpr (LIST) reg_emit<Word, NR>(a, sm, rt.r, Sc);
          const int bin = O::popc(Sc) - 1;  // clique size - 2
          if (lane == (bin & 31)) {
            if (bin < 32)
              ++h0;
            else
              ++h1;
          }
        }
      }
      continue;
    }
    MCE_BD(BD_PIVOT);
    // select_pivot_from_P_and_Xp (:366-402): pivot over P' | X'; an X'
    // vertex adjacent to all of P' ends the path.
    const Word cand = Pc | Xc;
    const int pc = O::popc(Pc);
    int k = 0;
    uint32_t vote = 0;  // bit 0: an X' vertex covers P'; bit 1: P' is not a clique
    iso0 = iso1 = false;
    if ((cand >> lane) & 1) {
      const int s = O::popc(Pc & r0);
      k = ((s + 1) << 7) | (127 - lane);
      vote = (((Xc >> lane) & 1) && s == pc) | ((((Pc >> lane) & 1) && s != pc - 1) << 1);
      iso0 = ((Pc >> lane) & 1) && s == 0;
    }
    if constexpr (NR == 2) {
      if ((cand >> (lane + 32)) & 1) {
        const int s = O::popc(Pc & r1);
        k = max(k, ((s + 1) << 7) | (127 - (lane + 32)));
        vote |= (((Xc >> (lane + 32)) & 1) && s == pc) |
                ((((Pc >> (lane + 32)) & 1) && s != pc - 1) << 1);
        iso1 = ((Pc >> (lane + 32)) & 1) && s == 0;
      }
    }
    vote = __reduce_or_sync(MCE_FULL, vote);
    if (vote & 1u) continue;
    if (!OPS && vote == 0) {
      // P' is a clique and no X' vertex covers it: below this node the walk
      // is one path of |P'| nodes (each pivot leaves one vertex to branch
      // on; X' never covers the shrinking P') ending in S' | P', maximal
      // unless an earlier neighbour of the root covers it - the condition
      // under which the outside pivot (XP) ends the walk here instead.
      const Word Sl = Sc | Pc;
      bool covered = false;
      if (nL > 0) {
        const int lb = kCompact ? sm.lb : -1;
        const Word *L0 = lb < 0 ? sm.xl0 : sl.xl + lb, *L1 = lb < 0 ? sl.xl : L0;
        covered = __any_sync(MCE_FULL, lane < nL && (L0[lane] & Sl) == Sl);
        if (!covered && nL > 32) covered = xl_covers<Word>(L1, nL, Sl);
      }
      if (XP && covered) continue;
      nodes += (u64)pc;
      if (Budget && a.node_budget && nodes > a.node_budget) {
        if (lane == 0) atomicOr(a.err, MCE_ERR_BUDGET);
        break;
      }
      if (!covered) {
        ++cnt;
        if constexpr (LIST) reg_emit<Word, NR>(a, sm, rt.r, Sl);
        const int bin = O::popc(Sl) - 1;  // clique size - 2
        if (lane == (bin & 31)) {
          if (bin < 32)
            ++h0;
          else
            ++h1;
        }
      }
      continue;
    }
    int ko = 0;
    if constexpr (XP) {  // earlier neighbours adjacent to the whole chosen set
      if (nL > 0) {
        bool elo;
        const int lb = kCompact ? sm.lb : -1;
        const Word *L0 = lb < 0 ? sm.xl0 : sl.xl + lb, *L1 = lb < 0 ? sl.xl : L0;
        ko = outside_pivot(L0, L1, nL, Sc, Pc, pc, &elo);
        if (elo) continue;
      }
    }
    // hand the child to an idle warp (try_dequeue / do_fork_L1,
    // mce/mce_utils.cuh:872-880,1063-1113)
    if (share && pc >= a.donate_min &&
        (nodes >= a.donate_after || (a.policy && a.policy[rt.r]) || (a.level2 && depth == 0))) {
      MCE_BD(BD_QUEUE);
      if (--recheck <= 0) {  // the queue state is read every 32 candidate nodes
        want = wants_task(a.q);
        recheck = 32;
      }
      if (want) {
        const u64 w0 = (u64)(uint32_t)rt.r, w1 = (u64)Pc, w2 = (u64)Xc, w3 = (u64)Sc,
                  w4 = L2 ? (u64)XO : 0ull;
        if (q_push(a.q, [&](uint32_t k2) {
              return k2 == 0 ? w0 : k2 == 1 ? w1 : k2 == 2 ? w2 : k2 == 3 ? w3 : w4;
            })) {
          if (EV && lane == 0) warp_record(a)[2] += 1;  // opts.warp_log
          continue;
        }
        want = false;
      }
    }
    MCE_BD(BD_PIVOT);
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    MCE_BD(BD_BRANCH);
    if (lane == 0) {
      sm.stk[depth][0] = P;
      sm.stk[depth][1] = X;
      sm.stk[depth][2] = B;
      sm.stk[depth][3] = S;
      if constexpr (kBulk) sm.stk[depth][4] = Lp;
      if constexpr (kCompact) {
        sm.flb[depth] = sm.lb;
        sm.fln[depth] = nL;
      }
    }
    __syncwarp();
    ++depth;
    P = Pc;
    X = Xc;
    S = Sc;
    // apply_pivot_to_next_level (:218-239)
    if (XP && (ko >> 11) > (k >> 7)) {
      const int lb = kCompact ? sm.lb : -1;
      const Word *L0 = lb < 0 ? sm.xl0 : sl.xl + lb, *L1 = lb < 0 ? sl.xl : L0;
      B = Pc & ~xrow(L0, L1, 2047 - (ko & 2047));
    } else {
      B = Pc & ~row_of<Word, NR>(r0, r1, 127 - (k & 127));
    }
    // a long leaf-filter list keeps only the rows containing the new chosen
    // set (the reference's Xx compaction, mce/mce_utils.cuh:265-292); a
    // depth-0 branch's list already holds exactly those for depth 1
    if (kCompact && nL > 32 && depth >= (per_branch ? 2 : 1)) {
      const int lb = sm.lb, top = lb < 0 ? nL : lb + nL;
      if (top + nL <= sl.xc) {
        const Word *L0 = lb < 0 ? sm.xl0 : sl.xl + lb, *L1 = lb < 0 ? sl.xl : L0;
        nL = xl_compact<Word>(L0, L1, nL, S, sl.xl + top);
        if (lane == 0) sm.lb = top;
        __syncwarp();
      }
    }
    if constexpr (kBulk) {  // the new node's leaf branches
      Lp = take_leaves(B, P, X, S);
      B &= ~Lp;
      if (Budget && a.node_budget && nodes > a.node_budget) {
        if (lane == 0) atomicOr(a.err, MCE_ERR_BUDGET);
        break;
      }
    }
  }
  MCE_BD(BD_OTHER);
}

// L2 (-p l2): the root's units are its oriented edges (r, v), the scheme of
// mce/mce_kernel_wl.cuh:307-485 (setup_stack_original_L2_IP,
// mce/mce_utils.cuh:664-712): the unit's candidates are the triangle list
// P = N+(r) & N+(v) (block_count_and_set_tri, :151-171), its pivot is taken
// from P alone, and the root's neighbours earlier than v and adjacent to it
// are outside rows tested at the leaves only - the earlier neighbours of r
// (the rows of sl.xr containing v) and the later ones before v in the
// degeneracy order (prio, then id: include/main_support.cuh:14), passed as
// XO.  An empty triangle list counts the edge when nothing covers it.
// Units are not tree nodes (the reference counts branches inside a unit).
// `unit(P, S, XO)` searches or hands off one unit.
template <typename Word, int NR, bool LIST, typename Unit>
__device__ __forceinline__ void reg_l2_units(const BKArgs &a, const RegSmem<Word, NR> &sm,
                                             const RegSlab<Word> &sl, const RegRoot<Word> &rt,
                                             u64 &h0, u64 &cnt, Unit unit) {
  using O = WOps<Word>;
  const int lane = (int)lane_id(), d = rt.d, nX = rt.nX;
  uint32_t pk0 = 0xFFFFFFFFu, pk1 = 0xFFFFFFFFu;  // degeneracy-order key of each index
  if (lane < d) pk0 = a.prio[sm.pl[lane]];
  if (NR == 2 && lane + 32 < d) pk1 = a.prio[sm.pl[lane + 32]];
  for (int v = 0; v < d; ++v) {
    const uint32_t pv = __shfl_sync(MCE_FULL, v < 32 ? pk0 : pk1, v & 31);
    // indices later than v: larger key, or the same key and a larger id
    // (ids ascend with the index)
    Word lat = (Word)__ballot_sync(MCE_FULL, lane < d && (pk0 > pv || (pk0 == pv && lane > v)));
    if constexpr (NR == 2)
      lat |= (Word)__ballot_sync(MCE_FULL,
                                 lane + 32 < d && (pk1 > pv || (pk1 == pv && lane + 32 > v)))
             << 32;
    const Word rv = row_of<Word, NR>(rt.r0, rt.r1, v);
    const Word Pv = rv & lat, XOv = rv & ~lat, vb = O::bit(v);
    if (Pv == 0) {  // the edge {r, v}
      bool covered = XOv != 0;
      for (int i0 = 0; !covered && i0 < nX; i0 += 32) {
        const int i = i0 + lane;
        covered = __any_sync(MCE_FULL, i < nX && (sl.xr[i] & vb));
      }
      if (!covered) {
        ++cnt;
        if constexpr (LIST) reg_emit<Word, NR>(a, sm, rt.r, vb);
        if (lane == 0) ++h0;  // size 2: bin 0
      }
      continue;
    }
    unit(Pv, vb, XOv);
  }
}

// ---------------------------------------------------------------------------
// Wide engine: any d+ <= 2048, rows of W = ceil(d+/64) words in a slab.
// (mem_l2_units, after mem_tree, is the wide engine's reg_l2_units.)
// ---------------------------------------------------------------------------
struct MemSmem {
  int32_t off[32];
  int32_t beg[32];
  int32_t own[32];
};

struct Slab {
  int32_t *pl;
  u64 *rows, *stk, *xs, *xr, *hash;
  u64 *xo;       // an L2 unit's outside rows among the later neighbours (one bitmap)
  int32_t *xl;   // leaf-filter list: rows of xr (>= 0) or, -1 - i, induced row i (L2)
  uint32_t *pk;  // the later neighbours' degeneracy keys (L2)
  int32_t *pkey, *pidx;  // hash of P: vertex id (-1: empty) and its index in P
  int hcap;  // hash set entries: a power of two >= 2 * xcap
};

__host__ __device__ __forceinline__ int hash_cap(int xcap) {
  int h = 32;
  while (h < 2 * xcap) h <<= 1;
  return h;
}

// slots of the hash of P for d later neighbours: a power of two >= 2 d
__host__ __device__ __forceinline__ int p_cap(int d) {
  int h = 64;
  while (h < 2 * d) h <<= 1;
  return h;
}

__device__ __forceinline__ Slab slab_of(const BKArgs &a, int64_t gw) {
  const int D = a.dcap, WM = (a.dcap + 63) / 64, XC = a.xcap;
  u64 *base = a.slab + (size_t)gw * a.slab_words;
  Slab s;
  s.rows = base;
  s.stk = s.rows + (size_t)D * WM;
  s.xs = s.stk + (size_t)(D + 1) * 4 * WM;
  s.xr = s.xs + (size_t)32 * WM;
  s.xo = s.xr + (size_t)XC * WM;
  s.hash = s.xo + (size_t)WM;
  s.hcap = hash_cap(XC);
  s.pl = (int32_t *)(s.hash + (size_t)s.hcap);
  s.xl = s.pl + D;
  s.pk = (uint32_t *)(s.xl + XC + D);
  s.pkey = (int32_t *)(s.pk + D);
  s.pidx = s.pkey + p_cap(D);
  return s;
}

__device__ __forceinline__ uint32_t wide_slot(int32_t w, int pc) {
  return (((uint32_t)w * 0x9E3779B1u) >> 12) & (uint32_t)(pc - 1);
}

// index of w in P (hash of pc slots), or -1
__device__ __forceinline__ int wide_find(const Slab &sl, int pc, int32_t w) {
  uint32_t h = wide_slot(w, pc);
  for (;;) {
    const int32_t k = sl.pkey[h];
    if (k == w) return sl.pidx[h];
    if (k == -1) return -1;
    h = (h + 1) & (uint32_t)(pc - 1);
  }
}

struct MemRoot {
  int32_t r = -1;
  int d = 0, Wr = 0, nX = 0;
  const u64 *rows = nullptr;  // the induced rows: shared memory when d+ <= MEM_SROWS_D, else the slab
};

// Roots of the wide engine with at most this many later neighbours keep their
// induced rows (<= 2 words each) in shared memory, read at every pivot.
constexpr int MEM_SROWS_D = 128;

__device__ void mem_encode(const BKArgs &a, MemSmem &sm, const Slab &sl, int32_t r, MemRoot &rt,
                           u64 *srows = nullptr) {
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const int32_t sb = a.split[r], d = a.rp[r + 1] - sb, ub = a.rp[r], u = sb - ub;
  rt.r = r;
  rt.d = d;
  rt.nX = 0;
  if (d > a.dcap || u > a.xcap) {
    if (lane == 0) atomicOr(a.err, d > a.dcap ? MCE_ERR_DEGREE : MCE_ERR_XROWS);
    rt.d = 0;
    return;
  }
  const int Wr = (d + 63) >> 6;
  rt.Wr = Wr;
  int32_t *pl = sl.pl;
  u64 *rows = (srows && d <= MEM_SROWS_D) ? srows : sl.rows;  // srows: 2 * MEM_SROWS_D words
  rt.rows = rows;
  const int pc = p_cap(d);
  for (int i = lane; i < d; i += 32) pl[i] = a.cs[sb + i];
  for (int i = lane; i < d * Wr; i += 32) rows[i] = 0;
  for (int i = lane; i < pc; i += 32) sl.pkey[i] = -1;
  __syncwarp();
  for (int i = lane; i < d; i += 32) {  // P's ids are distinct
    const int32_t w = pl[i];
    uint32_t h = wide_slot(w, pc);
    while (atomicCAS(&sl.pkey[h], -1, w) != -1) h = (h + 1) & (uint32_t)(pc - 1);
    sl.pidx[h] = i;
  }
  __syncwarp();
  for (int c = 0; c * 32 < d; ++c) {
    const int items = min(32, d - c * 32);
    int vb = 0, vlen = 0;
    if (lane < items) {
      const int32_t v = pl[c * 32 + lane];
      vb = a.split[v];
      vlen = a.rp[v + 1] - vb;
    }
    flat_walk(a.cs, vb, vlen, sm.off, sm.beg, sm.own, [&](int t, int32_t w) {
      const int i = wide_find(sl, pc, w);
      if (i >= 0) {
        const int j = c * 32 + t;
        atomicOr(&rows[(size_t)j * Wr + (i >> 6)], 1ull << (i & 63));
        atomicOr(&rows[(size_t)i * Wr + (j >> 6)], 1ull << (j & 63));
      }
    });
    __syncwarp();
  }
  // earlier-neighbour rows: non-empty ones, distinct when one word wide
  int hc = 32;
  if (Wr == 1) {
    while (hc < 2 * u && hc < sl.hcap) hc <<= 1;
    for (int i = lane; i < hc; i += 32) sl.hash[i] = 0;
  }
  int nX = 0;
  for (int c = 0; c * 32 < u; ++c) {
    const int items = min(32, u - c * 32);
    int xb = 0, xlen = 0;
    if (lane < items) {
      const int32_t x = a.cs[ub + c * 32 + lane];
      xb = a.split[x];
      xlen = a.rp[x + 1] - xb;
    }
    for (int i = lane; i < 32 * Wr; i += 32) sl.xs[i] = 0;
    __syncwarp();
    flat_walk(a.cs, xb, xlen, sm.off, sm.beg, sm.own, [&](int t, int32_t w) {
      const int i = wide_find(sl, pc, w);
      if (i >= 0) atomicOr(&sl.xs[(size_t)t * Wr + (i >> 6)], 1ull << (i & 63));
    });
    __syncwarp();
    bool keep = false;
    if (lane < items) {
      for (int w = 0; w < Wr; ++w) keep |= sl.xs[(size_t)lane * Wr + w] != 0;
      if (keep && Wr == 1) {
        const u64 row = sl.xs[lane];
        uint32_t h = hash_word(row) & (uint32_t)(hc - 1);
        keep = false;
        for (int probe = 0; probe < hc; ++probe) {
          const u64 old = atomicCAS(&sl.hash[h], 0ull, row);
          if (old == 0) {
            keep = true;
            break;
          }
          if (old == row) break;
          h = (h + 1) & (uint32_t)(hc - 1);
        }
      }
    }
    const uint32_t mk = __ballot_sync(MCE_FULL, keep);
    if (keep) {
      const int pos = nX + __popc(mk & lt);
      for (int w = 0; w < Wr; ++w) sl.xr[(size_t)pos * Wr + w] = sl.xs[(size_t)lane * Wr + w];
    }
    nX += __popc(mk);
    __syncwarp();
  }
  rt.nX = nX;
}

// Walk the subtree under frame 0 of the slab stack (P, X, S already there).
// Whether one of the nL filtered earlier-neighbour rows contains the chosen
// set Cs (Wr words in the slab): the leaf's clique is then not maximal.
__device__ __forceinline__ bool mem_covered(const Slab &sl, int nL, int Wr, const u64 *Cs,
                                            const u64 *rows) {
  const int lane = (int)lane_id();
  for (int i0 = 0; i0 < nL; i0 += 32) {
    const int i = i0 + lane;
    bool hit = false;
    if (i < nL) {
      const int32_t k = sl.xl[i];
      const u64 *xrow = k >= 0 ? sl.xr + (size_t)k * Wr : rows + (size_t)(-1 - k) * Wr;
      hit = true;
      for (int w = 0; w < Wr && hit; ++w) hit = (xrow[w] & Cs[w]) == Cs[w];
    }
    if (__any_sync(MCE_FULL, hit)) return true;
  }
  return false;
}

// A maximal clique: the root and the set bits of Cs; bin = its size - 2.
template <bool LIST>
__device__ __forceinline__ void mem_leaf(const BKArgs &a, const Slab &sl, int32_t r, int Wr,
                                         const u64 *Cs, int bin, u64 &h0, u64 &h1, u64 &cnt) {
  const int lane = (int)lane_id();
  ++cnt;
  if constexpr (LIST) {  // record {size, root, members...}, as reg_emit
    const int sz = bin + 2;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(a.list_words, (unsigned long long)(sz + 1));
    base = __shfl_sync(MCE_FULL, base, 0);
    if (base + (unsigned long long)sz + 1 <= a.list_cap) {
      if (lane == 0) {
        a.list_buf[base] = sz;
        a.list_buf[base + 1] = r;
      }
      u64 word = lane < Wr ? Cs[lane] : 0ull;  // Wr <= 32 words
      const int c = __popcll(word);
      unsigned long long pos = base + 2 + (warp_incl_scan(c) - c);
      while (word) {
        const int b = __ffsll((long long)word) - 1;
        word &= word - 1;
        a.list_buf[pos++] = sl.pl[lane * 64 + b];
      }
    }
  }
  if (bin < 64) {
    if (lane == (bin & 31)) {
      if (bin < 32)
        ++h0;
      else
        ++h1;
    }
  } else if (lane == 0 && bin + 2 < MCE_HIST_MAX) {
    atomicAdd(&a.hist[bin + 2], 1ull);
  }
}

// OPS: the algorithmic word operations, SPLIT: several warps per root, as
// in reg_tree.
// XO (an L2 unit): sl.xo holds the unit's outside rows among the later
// neighbours (tested at the leaves like earlier-neighbour rows).
// Outside pivot of the wide engine (-i px): over the earlier-neighbour rows
// that contain the chosen set S - and, in an L2 unit, the unit's outside
// rows (sl.xo) - the best score |P & row| with the lowest row id (earlier-
// neighbour rows first).  Returns score + 1 (0: no such row) with the row in
// *row_out; *elim: one of them covers P.
__device__ __forceinline__ int mem_outside_pivot(const Slab &sl, const u64 *rows, int nX, int d,
                                                 int Wr, bool xo, const u64 *S, const u64 *P,
                                                 int pc, bool *elim, const u64 **row_out) {
  const int lane = (int)lane_id();
  int best = 0;
  uint32_t bid = 0xFFFFFFFFu;
  bool el = false;
  const int total = nX + (xo ? d : 0);
  for (int i = lane; i < total; i += 32) {
    const u64 *row;
    if (i < nX) {
      row = sl.xr + (size_t)i * Wr;
    } else {
      const int j = i - nX;
      if (!((sl.xo[j >> 6] >> (j & 63)) & 1ull)) continue;
      row = rows + (size_t)j * Wr;
    }
    bool has = true;
    int sc = 0;
    for (int w = 0; w < Wr; ++w) {
      has = has && (row[w] & S[w]) == S[w];
      sc += __popcll(row[w] & P[w]);
    }
    if (!has) continue;
    el = el || sc == pc;
    if (sc + 1 > best) {  // ids ascend within a lane: ties keep the lowest
      best = sc + 1;
      bid = (uint32_t)i;
    }
  }
  *elim = __any_sync(MCE_FULL, el);
  const int mb = (int)__reduce_max_sync(MCE_FULL, (unsigned)best);
  const uint32_t id = __reduce_min_sync(MCE_FULL, best == mb ? bid : 0xFFFFFFFFu);
  if (mb > 0)
    *row_out = (int)id < nX ? sl.xr + (size_t)id * Wr : rows + (size_t)((int)id - nX) * Wr;
  return mb;
}

// XP (-i px): pivots also from the outside rows adjacent to the whole
// chosen set, and a node one of them covers is pruned (reg_tree's rule).
template <bool Budget = false, int EV = 0, bool LIST = false, bool OPS = false,
          bool SPLIT = false, bool XP = false, bool L2 = false>
__device__ void mem_tree(const BKArgs &a, const Slab &sl, const MemRoot &rt, u64 &h0, u64 &h1,
                         u64 &nodes, u64 &cnt, Bd *bd = nullptr, u64 *ops = nullptr,
                         int part = 0, int parts = 1, bool XO = false) {
  MCE_BD(BD_PIVOT);
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const int d = rt.d, Wr = rt.Wr, nX = rt.nX;
  const u64 w32 = (u64)((d + 31) >> 5);
  const u64 *rows = rt.rows;
  const bool share = a.q.hdr != nullptr;
  u64 *F0 = sl.stk;
  // pivot of the start node
  int s_base = 0;  // chosen vertices above frame 0
  {
    int pc = 0, sc = 0;
    if (lane < Wr) {
      pc = __popcll(F0[lane]);
      sc = __popcll(F0[3 * Wr + lane]);
    }
    pc = (int)__reduce_add_sync(MCE_FULL, (unsigned)pc);
    s_base = (int)__reduce_add_sync(MCE_FULL, (unsigned)sc);
    if constexpr (OPS) {
      if (s_base == 0 && part == 0) {  // the root's first pivot: 2W per candidate
        const int cu = lane < Wr ? __popcll(F0[lane] | F0[Wr + lane]) : 0;
        *ops += 2 * w32 * (u64)__reduce_add_sync(MCE_FULL, (unsigned)cu);
      }
    }
    int k = 0;
    bool el = false;
    for (int uu = lane; uu < d; uu += 32) {
      const int uw = uu >> 6;
      const u64 ub2 = 1ull << (uu & 63);
      const bool inP = (F0[uw] & ub2) != 0, inX = (F0[Wr + uw] & ub2) != 0;
      if (!(inP || inX)) continue;
      int s = 0;
      const u64 *ru = rows + (size_t)uu * Wr;
      for (int w = 0; w < Wr; ++w) s += __popcll(F0[w] & ru[w]);
      k = max(k, ((s + 1) << 11) | (2047 - uu));
      el = el || (inX && s == pc);
    }
    const u64 *orow = nullptr;
    int mb = 0;
    bool elo = false;
    if constexpr (XP) mb = mem_outside_pivot(sl, rows, nX, d, Wr, L2 && XO, F0 + 3 * Wr, F0, pc, &elo, &orow);
    if (__any_sync(MCE_FULL, el) || elo || pc == 0) {
      MCE_BD(BD_OTHER);
      return;
    }
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    const int piv = 2047 - (k & 2047);
    const u64 *prow = (XP && mb > (k >> 11)) ? orow : rows + (size_t)piv * Wr;
    if (lane < Wr) F0[2 * Wr + lane] = F0[lane] & ~prow[lane];
    __syncwarp();
  }
  const bool per_branch = (s_base == 0);
  int nL = 0;
  if (!per_branch && nX > 0) {  // rows containing the whole chosen set
    const u64 *S0 = F0 + 3 * Wr;
    for (int i0 = 0; i0 < nX; i0 += 32) {
      const int i = i0 + lane;
      bool has = false;
      if (i < nX) {
        has = true;
        for (int w = 0; w < Wr && has; ++w) has = (sl.xr[(size_t)i * Wr + w] & S0[w]) == S0[w];
      }
      const uint32_t m2 = __ballot_sync(MCE_FULL, has);
      if (has) sl.xl[nL + __popc(m2 & lt)] = i;
      nL += __popc(m2);
    }
    __syncwarp();
  }
  if (L2 && XO) {  // an L2 unit's outside rows among the later neighbours containing S
    const u64 *S0 = F0 + 3 * Wr;
    for (int i0 = 0; i0 < d; i0 += 32) {
      const int i = i0 + lane;
      bool has = i < d && ((sl.xo[i >> 6] >> (i & 63)) & 1ull);
      for (int w = 0; w < Wr && has; ++w) has = (rows[(size_t)i * Wr + w] & S0[w]) == S0[w];
      const uint32_t m2 = __ballot_sync(MCE_FULL, has);
      if (has) sl.xl[nL + __popc(m2 & lt)] = -1 - i;
      nL += __popc(m2);
    }
    __syncwarp();
  }
  int depth = 0, recheck = 0, b0 = 0;  // b0: first-level branches passed
  bool want = false;
  for (;;) {
    MCE_BD(BD_BRANCH);
    u64 *F = sl.stk + (size_t)depth * 4 * Wr;
    u64 *Fp = F, *Fx = F + Wr, *Fb = F + 2 * Wr, *Fs = F + 3 * Wr;
    // lowest set bit of the branch set
    const u64 bw = lane < Wr ? Fb[lane] : 0ull;
    const uint32_t mk = __ballot_sync(MCE_FULL, bw != 0);
    if (!mk) {
      if (depth == 0) break;
      --depth;
      continue;
    }
    const int wl = __ffs(mk) - 1;
    const u64 word = __shfl_sync(MCE_FULL, bw, wl);
    const int v = wl * 64 + __ffsll((long long)word) - 1;
    const int vw = v >> 6;
    const u64 vbit = 1ull << (v & 63);
    MCE_BD(BD_SETS);
    if (lane == 0) {
      Fb[vw] &= ~vbit;
      Fp[vw] &= ~vbit;
      Fx[vw] |= vbit;
    }
    __syncwarp();
    // several warps per root: every parts-th first-level branch is this one's
    if constexpr (SPLIT)
      if (parts > 1 && depth == 0 && (b0++ % parts) != part) continue;
    ++nodes;
    if (Budget && a.node_budget && nodes > a.node_budget) {  // a serving request over its budget
      if (lane == 0) atomicOr(a.err, MCE_ERR_BUDGET);
      break;
    }
    u64 *C = F + 4 * Wr;
    int pc = 0;
    bool xnz = false;
    u64 pcw = 0, xcw = 0;
    if (lane < Wr) {
      const u64 rw = rows[(size_t)v * Wr + lane];
      pcw = Fp[lane] & rw;
      xcw = Fx[lane] & rw;
      C[lane] = pcw;
      C[Wr + lane] = xcw;
      C[3 * Wr + lane] = Fs[lane] | (lane == vw ? vbit : 0ull);
      pc = __popcll(pcw);
      xnz = xcw != 0;
    }
    pc = (int)__reduce_add_sync(MCE_FULL, (unsigned)pc);
    xnz = __any_sync(MCE_FULL, xnz);
    if constexpr (OPS) {
      const int cu = lane < Wr ? __popcll(pcw | xcw) : 0;
      *ops += 2 * w32 * (u64)__reduce_add_sync(MCE_FULL, (unsigned)cu) + 4 * w32;
    }
    if (per_branch && depth == 0 && nX > 0) {
      nL = 0;
      for (int i0 = 0; i0 < nX; i0 += 32) {
        const int i = i0 + lane;
        const bool has = i < nX && (sl.xr[(size_t)i * Wr + vw] & vbit);
        const uint32_t m2 = __ballot_sync(MCE_FULL, has);
        if (has) sl.xl[nL + __popc(m2 & lt)] = i;
        nL += __popc(m2);
      }
    }
    __syncwarp();
    if (pc == 0) {
      MCE_BD(BD_MAXIMAL);
      const u64 *Cs = C + 3 * Wr;
      if (!xnz && !mem_covered(sl, nL, Wr, Cs, rows))
        mem_leaf<LIST>(a, sl, rt.r, Wr, Cs, s_base + depth, h0, h1, cnt);
      continue;
    }
    MCE_BD(BD_PIVOT);
    int k = 0;
    bool el = false, nc = false;  // nc: a vertex of P' misses another one
    if (Wr <= 2) {  // P' and X' words from the lanes that made them, no frame loads
      const u64 p0 = __shfl_sync(MCE_FULL, pcw, 0), p1 = __shfl_sync(MCE_FULL, pcw, 1);
      const u64 x0 = __shfl_sync(MCE_FULL, xcw, 0), x1 = __shfl_sync(MCE_FULL, xcw, 1);
      for (int uu = lane; uu < d; uu += 32) {
        const int sh = uu & 63;
        const bool inP = (((uu < 64 ? p0 : p1) >> sh) & 1ull) != 0;
        const bool inX = (((uu < 64 ? x0 : x1) >> sh) & 1ull) != 0;
        if (!(inP || inX)) continue;
        const u64 *ru = rows + (size_t)uu * Wr;
        int s = __popcll(p0 & ru[0]);
        if (Wr == 2) s += __popcll(p1 & ru[1]);
        k = max(k, ((s + 1) << 11) | (2047 - uu));
        el = el || (inX && s == pc);
        nc = nc || (inP && s != pc - 1);
      }
    } else {
      for (int uu = lane; uu < d; uu += 32) {
        const int uw = uu >> 6;
        const u64 ub2 = 1ull << (uu & 63);
        const bool inP = (C[uw] & ub2) != 0, inX = (C[Wr + uw] & ub2) != 0;
        if (!(inP || inX)) continue;
        int s = 0;
        const u64 *ru = rows + (size_t)uu * Wr;
        for (int w = 0; w < Wr; ++w) s += __popcll(C[w] & ru[w]);
        k = max(k, ((s + 1) << 11) | (2047 - uu));
        el = el || (inX && s == pc);
        nc = nc || (inP && s != pc - 1);
      }
    }
    const uint32_t vote = __reduce_or_sync(MCE_FULL, (el ? 1u : 0u) | (nc ? 2u : 0u));
    if (vote & 1u) continue;
    if (!OPS && vote == 0) {
      // P' is a clique and no X' vertex covers it: one path of |P'| nodes
      // below ends in S' | P' (the register engine's shortcut); the union
      // goes into the child's unused branch words.  With -i px an outside
      // row covering the union would have ended the path here.
      u64 *Cl = C + 2 * Wr;
      if (lane < Wr) Cl[lane] = C[3 * Wr + lane] | C[lane];
      __syncwarp();
      const bool cov = mem_covered(sl, nL, Wr, Cl, rows);
      if (XP && cov) continue;
      nodes += (u64)pc;
      if (Budget && a.node_budget && nodes > a.node_budget) {
        if (lane == 0) atomicOr(a.err, MCE_ERR_BUDGET);
        break;
      }
      if (!cov) mem_leaf<LIST>(a, sl, rt.r, Wr, Cl, s_base + depth + pc, h0, h1, cnt);
      continue;
    }
    const u64 *orow = nullptr;
    int mbo = 0;
    if constexpr (XP) {  // outside rows adjacent to the whole chosen set
      bool elo = false;
      mbo = mem_outside_pivot(sl, rows, nX, d, Wr, L2 && XO, C + 3 * Wr, C, pc, &elo, &orow);
      if (elo) continue;
    }
    if (share && pc >= a.donate_min &&
        (nodes >= a.donate_after || (a.policy && a.policy[rt.r]) || (a.level2 && depth == 0)) &&
        (--recheck <= 0 ? (recheck = 32, want = wants_task(a.q)) : want)) {
      MCE_BD(BD_QUEUE);
      const int WM = (a.dcap + 63) >> 6;
      const u64 *Cp = C, *Cx = C + Wr, *Cs = C + 3 * Wr;
      if (q_push(a.q, [&](uint32_t k2) -> u64 {
            if (k2 == 0) return (u64)(uint32_t)rt.r;
            const uint32_t part = (k2 - 1) / WM, w = (k2 - 1) % WM;
            if ((int)w >= Wr) return 0ull;
            return part == 0 ? Cp[w] : part == 1 ? Cx[w] : part == 2 ? Cs[w] : (L2 && XO ? sl.xo[w] : 0ull);
          })) {
        if (EV && lane == 0) warp_record(a)[2] += 1;  // opts.warp_log
        continue;
      }
      want = false;
    }
    MCE_BD(BD_PIVOT);
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    const int up = 2047 - (k & 2047);
    MCE_BD(BD_BRANCH);
    const u64 *prow = (XP && mbo > (k >> 11)) ? orow : rows + (size_t)up * Wr;
    if (lane < Wr) C[2 * Wr + lane] = C[lane] & ~prow[lane];
    __syncwarp();
    ++depth;
  }
  MCE_BD(BD_OTHER);
}

// L2 units of a wide root (see reg_l2_units): frame 0 gets the unit's P
// (the triangle list), X = 0 and S = {v}; sl.xo its outside rows among the
// later neighbours.  `unit(xo_any)` searches or hands off the unit.
template <bool LIST, typename Unit>
__device__ __forceinline__ void mem_l2_units(const BKArgs &a, const Slab &sl, const MemRoot &rt,
                                             u64 &h0, u64 &h1, u64 &cnt, Unit unit) {
  const int lane = (int)lane_id(), d = rt.d, Wr = rt.Wr, nX = rt.nX;
  const u64 *rows = rt.rows;
  for (int i = lane; i < d; i += 32) sl.pk[i] = a.prio[sl.pl[i]];
  __syncwarp();
  for (int v = 0; v < d; ++v) {
    const uint32_t pv = sl.pk[v];
    u64 lat = 0;  // lane w < Wr: word w of the indices later than v
    for (int c = 0; c * 32 < d; ++c) {
      const int i = c * 32 + lane;
      const bool later = i < d && (sl.pk[i] > pv || (sl.pk[i] == pv && i > v));
      const uint32_t m = __ballot_sync(MCE_FULL, later);
      if (lane == (c >> 1)) lat |= (u64)m << (32 * (c & 1));
    }
    u64 pw = 0, xw = 0;
    if (lane < Wr) {
      const u64 rw = rows[(size_t)v * Wr + lane];
      pw = rw & lat;
      xw = rw & ~lat;
      sl.stk[lane] = pw;
      sl.stk[Wr + lane] = 0;
      sl.stk[3 * Wr + lane] = (lane == (v >> 6)) ? 1ull << (v & 63) : 0ull;
      sl.xo[lane] = xw;
    }
    const bool tri = __any_sync(MCE_FULL, pw != 0), xo_any = __any_sync(MCE_FULL, xw != 0);
    __syncwarp();
    if (!tri) {  // the edge {r, v}: maximal unless an outside row contains v
      bool covered = xo_any;
      for (int i0 = 0; !covered && i0 < nX; i0 += 32) {
        const int i = i0 + lane;
        covered = __any_sync(MCE_FULL,
                             i < nX && ((sl.xr[(size_t)i * Wr + (v >> 6)] >> (v & 63)) & 1ull));
      }
      if (!covered) mem_leaf<LIST>(a, sl, rt.r, Wr, sl.stk + 3 * Wr, 0, h0, h1, cnt);  // size 2
      continue;
    }
    unit(xo_any);
  }
}

}  // namespace
}  // namespace mce
