// Per-root Bron-Kerbosch search with Tomita pivoting, one warp per root.
//
// Replaces the block-per-root kernels mce_kernel_l1_ip_{nowl,wl}
// (mce/mce_kernel_nowl.cuh:9-109, mce/mce_kernel_wl.cuh:9-154) and the
// helpers they call in mce/mce_utils.cuh.  The search rules are the
// reference's (cited inline); the execution model is not:
//  - a warp, not a 128/256-thread block, owns a root, so a tree step costs
//    a few warp instructions instead of several __syncthreads;
//  - the induced subgraph of the root's later neighbours lives in registers
//    (lane i holds adjacency row i, and row i+32 for the 64-bit engine) or,
//    for wide roots, in a per-warp slab, instead of per-block global arrays;
//  - the pivot is the candidate u maximising popc(P & N(u)), found with one
//    __reduce_max_sync over (score, -index) keys: every lane scores its own
//    row(s) in parallel;
//  - the DFS stack is an explicit array of (P, X, branch set, chosen set)
//    frames in shared memory (register engine) or the slab (wide engine);
//  - earlier neighbours of the root (the reference's Xx list, tested with a
//    binary search per tree node, mce/mce_utils.cuh:265-292) are encoded once
//    per root as bitmaps over the root's later neighbours, duplicates
//    dropped; a leaf is maximal only if none of them contains the clique;
//  - load balance: a warp about to descend into a child with many candidates
//    hands the child to the device task queue instead while other warps are
//    idle (queue.cuh), the counterpart of the reference's worker list.
// Tie-breaking: the pivot with the lowest index among the best scores, so
// per-root tree sizes are deterministic and independent of who walks them.
#include <climits>
#include <cstring>

#include "common.cuh"
#include "engine.cuh"
#include "kernels.h"
#include "queue.cuh"

namespace mce {

__global__ void queue_init_kernel(QueueView q) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q.cap; i += gridDim.x * blockDim.x)
    q.seq[i] = i;
}

namespace {

// Blocks per SM: the 32-bit engine runs 6 (48 warps: more warps hide the
// encode's memory latency better than the registers they give up), the
// 64-bit engine 4.
// EV (opts.warp_log): 0 none, 1 per-warp load and donations, 2 plus the
// per-phase cycle breakdown.
// OPS (opts.count_ops): the variant that sums the algorithmic word
// operations of every walk (reg_tree / mem_tree), run outside timed calls.
// SPLIT: the variant for several warps per root (opts.warps_per_root > 1);
// the others keep no state for it.  STAGE (opts.stage_lists): the encode's
// lists are staged in shared memory by 1-D bulk copies (flat_walk_staged).
// L2 (-p l2): the edge-rooted variant.
template <typename Word, int NR, int EV = 0, bool LIST = false, bool XP = false, bool OPS = false,
          bool SPLIT = false, bool STAGE = false, bool L2 = false>
__global__ void __launch_bounds__(REG_BLOCK, (NR == 1 && sizeof(Word) == 4) ? 6 : (NR == 2 ? 4 : 1))
    bk_reg_kernel(BKArgs a, int cls) {
  __shared__ RegSmem<Word, NR> sm_all[REG_BLOCK / 32];
  RegSmem<Word, NR> &sm = sm_all[threadIdx.x >> 5];
  const int lane = (int)lane_id();
  if constexpr (STAGE) stage_init();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const RegSlab<Word> sl = reg_slab<Word>(a, gw);
  const uint32_t beg = a.shape->cls_off[cls], end = a.shape->cls_off[cls + 1];
  const bool share = a.q.hdr != nullptr;
  u64 h0 = 0, h1 = 0, nodes = 0, ops = 0;
  RegRoot<Word> rt;
  Bd bdv, *bd = &bdv;
  if constexpr (EV == 2) bdv.start();
  if (share && lane == 0) atomicAdd(&a.q.hdr->work, 1u);
  // units of work: (root, part) pairs, the parts of a root fetched one
  // after the other so that different warps take them
  const uint32_t parts = SPLIT && a.parts > 1 ? (uint32_t)a.parts : 1u;
  const uint32_t units = (end - beg) * parts;
  for (;;) {
    uint32_t i0 = 0;
    if (lane == 0) i0 = atomicAdd(&a.fetch[cls], (uint32_t)REG_CHUNK);
    i0 = __shfl_sync(MCE_FULL, i0, 0);
    if (i0 >= units) break;
    for (int k = 0; k < REG_CHUNK; ++k) {
      const uint32_t u = i0 + k;
      if (u >= units) break;
      const int32_t r = a.roots[beg + u / parts];
      MCE_BD(BD_ENCODE);
      if (parts == 1 || r != rt.r) reg_encode<Word, NR, STAGE>(a, sm, sl, r, rt);
      MCE_BD(BD_OTHER);
      u64 nd = 0, cnt = 0, op = 0;
      if constexpr (L2) {  // -p l2: the root's edges are the units
        reg_l2_units<Word, NR, LIST>(a, sm, sl, rt, h0, cnt, [&](Word Pv, Word Sv, Word XOv) {
          if (share && q_wants(a.q)) {  // offered to idle warps at once
            const u64 w0 = (u64)(uint32_t)rt.r, w1 = (u64)Pv, w3 = (u64)Sv, w4 = (u64)XOv;
            if (q_push(a.q, [&](uint32_t k2) {
                  return k2 == 0 ? w0 : k2 == 1 ? w1 : k2 == 2 ? 0ull : k2 == 3 ? w3 : w4;
                })) {
              if (EV && lane == 0) warp_record(a)[2] += 1;
              return;
            }
          }
          reg_tree<Word, NR, false, EV, LIST, XP, OPS, SPLIT, true>(a, sm, sl, rt, Pv, (Word)0, Sv,
                                                                    h0, h1, nd, cnt, bd, &op, 0, 1,
                                                                    XOv);
        });
      } else {
        reg_tree<Word, NR, false, EV, LIST, XP, OPS, SPLIT>(a, sm, sl, rt, WOps<Word>::low(rt.d),
                                                            (Word)0, (Word)0, h0, h1, nd, cnt, bd,
                                                            &op, (int)(u % parts), (int)parts);
      }
      nodes += nd;
      root_done(a, r, nd, cnt);
      if constexpr (OPS) {
        ops += op;
        root_ops_done(a, r, op);
      }
    }
  }
  if (share) {
    if (lane == 0) {
      atomicSub(&a.q.hdr->work, 1u);
      atomicAdd(&a.q.hdr->epoch, 1u);
    }
    u64 t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0;
    MCE_BD(BD_QUEUE);
    idle_phase(
        a,
        [&](uint32_t k, u64 w) {  // lane k receives word k
          if (k == 0) t0 = w;
          if (k == 1) t1 = w;
          if (k == 2) t2 = w;
          if (k == 3) t3 = w;
          if (k == 4) t4 = w;
        },
        [&]() {
          // word k of the task arrived on lane k
          const int32_t r = (int32_t)__shfl_sync(MCE_FULL, t0, 0);
          const Word P = (Word)__shfl_sync(MCE_FULL, t1, 1);
          const Word X = (Word)__shfl_sync(MCE_FULL, t2, 2);
          const Word S = (Word)__shfl_sync(MCE_FULL, t3, 3);
          const Word XO = L2 ? (Word)__shfl_sync(MCE_FULL, t4, 4) : (Word)0;  // L2 unit's outside rows
          MCE_BD(BD_ENCODE);
          if (r != rt.r) reg_encode<Word, NR, STAGE>(a, sm, sl, r, rt);
          u64 nd = 0, cnt = 0, op = 0;
          reg_tree<Word, NR, false, EV, LIST, XP, OPS, false, L2>(a, sm, sl, rt, P, X, S, h0, h1, nd,
                                                                  cnt, bd, &op, 0, 1, XO);
          nodes += nd;
          root_done(a, r, nd, cnt);
          if constexpr (OPS) {
            ops += op;
            root_ops_done(a, r, op);
          }
          MCE_BD(BD_QUEUE);
        });
  }
  MCE_BD(BD_OTHER);
  if (h0) atomicAdd(&a.hist[lane + 2], h0);
  if (h1) atomicAdd(&a.hist[lane + 34], h1);
  if (lane == 0 && nodes) atomicAdd(a.nodes, nodes);  // warp-uniform count
  if (OPS && lane == 0 && ops) atomicAdd(a.ops, ops);
  if (EV && lane == 0) {  // opts.warp_log
    u64 *w = warp_record(a);
    w[0] = sm_id();
    w[1] = nodes;
    if constexpr (EV == 2)
      for (int i = 0; i < 7; ++i) w[3 + i] = bdv.acc[i];
  }
}

// The wide engine at 4 blocks per SM (96 registers) or, with
// opts.wide_blocks = 8, at 8 (64 registers): more warps pay on graphs whose
// wide roots have large shared subtrees (R-MAT), fewer on many small ones.
template <int EV = 0, int MINB = 1, bool LIST = false, bool OPS = false, bool SPLIT = false,
          bool XP = false, bool L2 = false>
__global__ void __launch_bounds__(MEM_BLOCK, MINB) bk_mem_kernel(BKArgs a, int cls) {
  __shared__ MemSmem sm_all[MEM_BLOCK / 32];
  __shared__ u64 srows_all[MEM_BLOCK / 32][2 * MEM_SROWS_D];
  MemSmem &sm = sm_all[threadIdx.x >> 5];
  u64 *srows = srows_all[threadIdx.x >> 5];
  const int lane = (int)lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const Slab sl = slab_of(a, gw);
  const uint32_t beg = a.shape->cls_off[cls], end = a.shape->cls_off[cls + 1];
  const bool share = a.q.hdr != nullptr;
  u64 h0 = 0, h1 = 0, nodes = 0, ops = 0;
  MemRoot rt;
  Bd bdv, *bd = &bdv;
  if constexpr (EV == 2) bdv.start();
  if (share && lane == 0) atomicAdd(&a.q.hdr->work, 1u);
  const uint32_t parts = SPLIT && a.parts > 1 ? (uint32_t)a.parts : 1u;  // warps per root
  const uint32_t units = (end - beg) * parts;
  for (;;) {
    uint32_t i0 = 0;
    if (lane == 0) i0 = atomicAdd(&a.fetch[cls], 1u);
    i0 = __shfl_sync(MCE_FULL, i0, 0);
    if (i0 >= units) break;
    const int32_t r = a.roots[beg + i0 / parts];
    MCE_BD(BD_ENCODE);
    if (parts == 1 || r != rt.r) mem_encode(a, sm, sl, r, rt, srows);
    MCE_BD(BD_OTHER);
    if (rt.d == 0) continue;
    const int Wr = rt.Wr;
    u64 nd = 0, cnt = 0, op = 0;
    if constexpr (L2) {  // -p l2: the root's edges are the units
      const int WM = (a.dcap + 63) >> 6;
      mem_l2_units<LIST>(a, sl, rt, h0, h1, cnt, [&](bool xo_any) {
        if (share && q_wants(a.q)) {  // offered to idle warps at once
          const u64 *F0 = sl.stk;
          if (q_push(a.q, [&](uint32_t k2) -> u64 {
                if (k2 == 0) return (u64)(uint32_t)r;
                const uint32_t part = (k2 - 1) / WM, w = (k2 - 1) % WM;
                if ((int)w >= Wr) return 0ull;
                return part == 0 ? F0[w] : part == 1 ? 0ull : part == 2 ? F0[3 * Wr + w] : sl.xo[w];
              })) {
            if (EV && lane == 0) warp_record(a)[2] += 1;
            return;
          }
        }
        mem_tree<false, EV, LIST, OPS, SPLIT, XP, true>(a, sl, rt, h0, h1, nd, cnt, bd, &op, 0, 1,
                                                        xo_any);
      });
    } else {
      if (lane < Wr) {  // root frame: P = all of N+(r), X = 0, S = 0
        const u64 all = (lane == Wr - 1 && (rt.d & 63)) ? ((1ull << (rt.d & 63)) - 1ull) : ~0ull;
        sl.stk[lane] = all;
        sl.stk[Wr + lane] = 0;
        sl.stk[3 * Wr + lane] = 0;
      }
      __syncwarp();
      mem_tree<false, EV, LIST, OPS, SPLIT, XP>(a, sl, rt, h0, h1, nd, cnt, bd, &op, (int)(i0 % parts),
                                            (int)parts);
    }
    nodes += nd;
    root_done(a, r, nd, cnt);
    if constexpr (OPS) {
      ops += op;
      root_ops_done(a, r, op);
    }
  }
  if (share) {
    if (lane == 0) {
      atomicSub(&a.q.hdr->work, 1u);
      atomicAdd(&a.q.hdr->epoch, 1u);
    }
    const int WM = (a.dcap + 63) >> 6;
    int32_t task_root = -1;
    MCE_BD(BD_QUEUE);
    idle_phase(
        a,
        [&](uint32_t k, u64 w) {
          if (k == 0) {
            task_root = (int32_t)w;  // lane 0 reads word 0
          } else {
            const uint32_t part = (k - 1) / WM, ww = (k - 1) % WM;
            sl.xs[part * WM + ww] = w;  // staged; moved to frame 0 after encode
          }
        },
        [&]() {
          const int32_t r = __shfl_sync(MCE_FULL, task_root, 0);
          __syncwarp();
          // the staging area is rewritten by mem_encode: keep the task first
          u64 tp = 0, tx = 0, ts = 0, to = 0;
          if (lane < WM) {
            tp = sl.xs[lane];
            tx = sl.xs[WM + lane];
            ts = sl.xs[2 * WM + lane];
            to = sl.xs[3 * WM + lane];  // an L2 unit's outside rows (0 otherwise)
          }
          __syncwarp();
          MCE_BD(BD_ENCODE);
          if (r != rt.r) mem_encode(a, sm, sl, r, rt, srows);
          MCE_BD(BD_QUEUE);
          if (rt.d == 0) return;
          const int Wr = rt.Wr;
          if (lane < Wr) {
            sl.stk[lane] = tp;
            sl.stk[Wr + lane] = tx;
            sl.stk[3 * Wr + lane] = ts;
            sl.xo[lane] = to;
          }
          const bool xo_any = __any_sync(MCE_FULL, lane < Wr && to != 0);
          __syncwarp();
          u64 nd = 0, cnt = 0, op = 0;
          mem_tree<false, EV, LIST, OPS, false, XP, L2>(a, sl, rt, h0, h1, nd, cnt, bd, &op, 0, 1,
                                                        xo_any);
          nodes += nd;
          root_done(a, r, nd, cnt);
          if constexpr (OPS) {
            ops += op;
            root_ops_done(a, r, op);
          }
          MCE_BD(BD_QUEUE);
        });
  }
  MCE_BD(BD_OTHER);
  if (h0) atomicAdd(&a.hist[lane + 2], h0);
  if (h1) atomicAdd(&a.hist[lane + 34], h1);
  if (lane == 0 && nodes) atomicAdd(a.nodes, nodes);  // warp-uniform count
  if (OPS && lane == 0 && ops) atomicAdd(a.ops, ops);
  if (EV && lane == 0) {  // opts.warp_log
    u64 *w = warp_record(a);
    w[0] = sm_id();
    w[1] = nodes;
    if constexpr (EV == 2)
      for (int i = 0; i < 7; ++i) w[3 + i] = bdv.acc[i];
  }
}

// ---------------------------------------------------------------------------
// Hub rows: the earlier-neighbour rows of roots with d- > HUB_XMIN, built
// before the search by many warps at once (the root's own warp would walk
// thousands of later lists one window at a time, a chain of dependent
// loads that leaves the rest of its class idle at the end).
// ---------------------------------------------------------------------------
constexpr int HUB_BLOCK = 256;
constexpr int HUB_FETCH = 4;  // 32-row chunks a warp of hub_rows_kernel takes at a time

// off[j] = sum over k < j of hub k's earlier degree rounded up to 32; one
// block of HUB_OFF_BLOCK threads walks the list in tiles of HUB_OFF_PER
// hubs per thread (their offsets gathered together), scanning each tile.
constexpr int HUB_OFF_BLOCK = 1024, HUB_OFF_PER = 8;
__global__ void __launch_bounds__(HUB_OFF_BLOCK) hub_offsets_kernel(
    const int32_t *__restrict__ rp, const int32_t *__restrict__ split,
    const int32_t *__restrict__ hub_list, uint32_t cnt, int64_t *__restrict__ off,
    int32_t *__restrict__ nx) {
  __shared__ long long wsum[HUB_OFF_BLOCK / 32];
  __shared__ long long carry;
  const int lane = (int)lane_id(), wid = (int)(threadIdx.x >> 5);
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < cnt; base += HUB_OFF_BLOCK * HUB_OFF_PER) {
    const uint32_t j0 = base + threadIdx.x * HUB_OFF_PER;
    long long v[HUB_OFF_PER];
    long long mine = 0;
#pragma unroll
    for (int k = 0; k < HUB_OFF_PER; ++k) {
      v[k] = 0;
      if (j0 + k < cnt) {
        const int32_t r = hub_list[j0 + k];
        v[k] = (long long)(((uint32_t)(split[r] - rp[r]) + 31u) & ~31u);
      }
      mine += v[k];
    }
    long long x = mine;  // inclusive scan of the threads' sums in the warp
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(MCE_FULL, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    long long before = carry + x - mine;
    for (int w = 0; w < wid; ++w) before += wsum[w];
#pragma unroll
    for (int k = 0; k < HUB_OFF_PER; ++k) {
      if (j0 + k < cnt) {
        off[j0 + k] = (int64_t)before;
        nx[j0 + k] = -1;
      }
      before += v[k];
    }
    __syncthreads();
    if (threadIdx.x == HUB_OFF_BLOCK - 1) carry = before;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    off[cnt] = (int64_t)carry;
    off[cnt + 1] = 0;  // hub_rows_kernel's chunk counter
  }
}

struct HubSmem {
  int32_t hkey[256];  // hash of the hub's later list (<= 64 ids): vertex id (-1: empty) ...
  uint8_t hidx[256];  // ... and its index in the list
  u64 xs[32];         // the rows of the current 32 earlier neighbours
  int32_t off[32], beg[32], own[64];  // flattened-walk scratch (two windows)
};

// flat_walk (engine.cuh) two windows at a time: the two elements of a lane
// are loaded together, so a warp keeps two reads of the lists in flight.
template <typename F>
__device__ __forceinline__ void flat_walk2(const int32_t *__restrict__ cs, int32_t b, int len,
                                           int32_t *off_sm, int32_t *beg_sm, int32_t *own_sm,
                                           F f) {
  const int lane = (int)lane_id();
  const int incl = warp_incl_scan(len);
  const int T = __shfl_sync(MCE_FULL, incl, 31);
  const int off = incl - len;
  off_sm[lane] = off;
  beg_sm[lane] = b;
  int carry = 0;
  for (int e0 = 0; e0 < T; e0 += 64) {
    const bool stA = len > 0 && off >= e0 && off < e0 + 32;
    const bool stB = len > 0 && off >= e0 + 32 && off < e0 + 64;
    if (stA) own_sm[off - e0] = lane;
    if (stB) own_sm[off - e0] = lane;  // 32 .. 63: window B
    const uint32_t mA = __reduce_or_sync(MCE_FULL, stA ? 1u << (off - e0) : 0u);
    const uint32_t mB = __reduce_or_sync(MCE_FULL, stB ? 1u << (off - e0 - 32) : 0u);
    __syncwarp();
    const uint32_t keep = 0xFFFFFFFFu >> (31 - lane);
    const uint32_t bA = mA & keep, bB = mB & keep;
    const int tA = bA ? own_sm[31 - __clz(bA)] : carry;
    const int cA = __shfl_sync(MCE_FULL, tA, 31);
    const int tB = bB ? own_sm[32 + 31 - __clz(bB)] : cA;
    carry = __shfl_sync(MCE_FULL, tB, 31);
    const int eA = e0 + lane, eB = e0 + 32 + lane;
    int32_t wA = -1, wB = -1;
    if (eA < T) wA = cs[beg_sm[tA] + (eA - off_sm[tA])];
    if (eB < T) wB = cs[beg_sm[tB] + (eB - off_sm[tB])];
    if (eA < T) f(tA, wA);
    if (eB < T) f(tB, wB);
    __syncwarp();
  }
}

__device__ __forceinline__ uint32_t hub_slot(int32_t w) { return ((uint32_t)w * 0x9E3779B1u) >> 24; }

// Warps fetch HUB_FETCH 32-row chunks at a time from a counter (off[cnt + 1],
// zeroed by hub_offsets_kernel), so a warp whose chunks walk long lists takes
// fewer; the hash of a hub's later list (d+ <= 64) is rebuilt when a warp's
// chunks move on to the next hub (a warp's chunks only move forward).
__global__ void __launch_bounds__(HUB_BLOCK) hub_rows_kernel(
    const int32_t *__restrict__ rp, const int32_t *__restrict__ split,
    const int32_t *__restrict__ cs, const int32_t *__restrict__ hub_list, uint32_t cnt,
    const int64_t *__restrict__ off, int64_t chunks, unsigned long long *__restrict__ rows,
    unsigned long long *next) {
  __shared__ HubSmem sm_all[HUB_BLOCK / 32];
  HubSmem &sm = sm_all[threadIdx.x >> 5];
  const int lane = (int)lane_id();
  int32_t cur = -1;  // hub whose hash is built
  uint32_t j = 0;
  int64_t c = 0, c1 = 0;
  for (;;) {
    if (c == c1) {
      unsigned long long f = 0;
      if (lane == 0) f = atomicAdd(next, (unsigned long long)HUB_FETCH);
      c = (int64_t)__shfl_sync(MCE_FULL, f, 0);
      if (c >= chunks) break;
      c1 = min(chunks, c + HUB_FETCH);
    }
    const int64_t row0 = 32 * c++;
    if (cur < 0 || row0 >= off[j + 1]) {  // first chunk, or the next hub: last j with off[j] <= row0
      uint32_t lo = 0, hi = cnt - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= row0) lo = mid; else hi = mid - 1;
      }
      j = lo;
      cur = hub_list[j];
      const int32_t sb = split[cur], d = rp[cur + 1] - sb;
      for (int i = lane; i < 256; i += 32) sm.hkey[i] = -1;
      __syncwarp();
      for (int i = lane; i < d; i += 32) {  // the later list's ids are distinct
        const int32_t w = cs[sb + i];
        uint32_t h = hub_slot(w);
        while (atomicCAS(&sm.hkey[h], -1, w) != -1) h = (h + 1) & 255u;
        sm.hidx[h] = (uint8_t)i;
      }
      __syncwarp();
    }
    const int32_t ub = rp[cur], u = split[cur] - ub;
    const int64_t i0 = row0 - off[j];
    const int items = (int)min((int64_t)32, (int64_t)u - i0);
    int xb = 0, xlen = 0;
    if (lane < items) {
      const int32_t x = cs[ub + i0 + lane];
      xb = split[x];
      xlen = rp[x + 1] - xb;
    }
    sm.xs[lane] = 0;
    __syncwarp();
    flat_walk2(cs, xb, xlen, sm.off, sm.beg, sm.own, [&](int t, int32_t w) {
      uint32_t h = hub_slot(w);
      for (;;) {
        const int32_t k = sm.hkey[h];
        if (k == w) {
          atomicOr(&sm.xs[t], 1ull << sm.hidx[h]);
          break;
        }
        if (k == -1) break;
        h = (h + 1) & 255u;
      }
    });
    __syncwarp();
    rows[row0 + lane] = sm.xs[lane];  // lanes past the hub's list write its zero padding
    __syncwarp();
  }
}

}  // namespace


namespace {
__global__ void hub_index_kernel(const int32_t *__restrict__ list, uint32_t cnt, int32_t *hub_of) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x)
    hub_of[list[i]] = (int32_t)i;
}
}  // namespace

int hub_index_launch(const int32_t *list, uint32_t cnt, int32_t *hub_of, cudaStream_t s,
                     int *launches) {
  if (cnt == 0) return MCE_OK;
  hub_index_kernel<<<(cnt + 255) / 256 < 1184 ? (cnt + 255) / 256 : 1184, 256, 0, s>>>(list, cnt,
                                                                                   hub_of);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return MCE_OK;
}

int hub_rows_launch(const int32_t *rp, const int32_t *split, const int32_t *cs,
                    const int32_t *hub_list, uint32_t cnt, int64_t total_rows, int64_t *off,
                    int32_t *nx, unsigned long long *rows, int sms, cudaStream_t s,
                    int *launches) {
  if (cnt == 0) return MCE_OK;
  hub_offsets_kernel<<<1, HUB_OFF_BLOCK, 0, s>>>(rp, split, hub_list, cnt, off, nx);
  MCE_CUDA(cudaGetLastError());
  const int64_t chunks = total_rows / 32;
  int64_t blocks = ((chunks + 7) / 8 + 0);  // up to one chunk per warp
  const int64_t cap = (int64_t)sms * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  hub_rows_kernel<<<(unsigned)blocks, HUB_BLOCK, 0, s>>>(
      rp, split, cs, hub_list, cnt, off, chunks, rows,
      reinterpret_cast<unsigned long long *>(off + cnt + 1));
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 2;
  return MCE_OK;
}

size_t bk_slab_words(int cls, int dcap, int xcap, int rxcap) {
  if (cls == CLS_R32 || cls == CLS_R64) return 4 * (size_t)rxcap;  // hash, rows, leaf list
  const size_t WM = (size_t)(dcap + 63) / 64;
  size_t w = (size_t)dcap * WM + (size_t)(dcap + 1) * 4 * WM + 32 * WM + (size_t)xcap * WM;
  w += WM;                                          // xo (an L2 unit's outside rows)
  w += (size_t)hash_cap(xcap);                      // hash set (one-word rows)
  w += (3 * (size_t)dcap + (size_t)xcap + 1) / 2 + 1;  // pl, xl (xcap + dcap) and pk (int32)
  w += (size_t)p_cap(dcap);                         // hash of P: keys and indices (int32)
  w = w > 3 * WM + 1 ? w : 3 * WM + 1;
  return (w + 31) & ~(size_t)31;                    // 256-byte aligned slabs
}

uint32_t bk_task_words(int cls, int dcap) {
  if (cls == CLS_R32 || cls == CLS_R64) return 5;  // root, P, X, chosen set, L2 outside rows
  return 1 + 4 * (uint32_t)((dcap + 63) / 64);     // the same, W words each
}

int bk_warps_for_class(int cls, int sms, int wide_blocks, int *warps, int *block, int *smem) {
  int per_sm = 0;
  if (cls == CLS_R32 || cls == CLS_R64) {
    *block = REG_BLOCK;
    *smem = 0;
    if (cls == CLS_R32)
      MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bk_reg_kernel<uint32_t, 1>, REG_BLOCK, 0));
    else
      MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bk_reg_kernel<u64, 2>, REG_BLOCK, 0));
    if (per_sm < 1) per_sm = 1;
    *warps = sms * per_sm * (REG_BLOCK / 32);
  } else {
    *block = MEM_BLOCK;
    *smem = 0;
    // the variant's resident blocks per SM (its registers decide), at most 4 or 8
    if (wide_blocks == 8)
      MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bk_mem_kernel<0, 8>, MEM_BLOCK, 0));
    else
      MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bk_mem_kernel<>, MEM_BLOCK, 0));
    const int cap = wide_blocks == 8 ? 8 : 4;
    if (per_sm > cap) per_sm = cap;
    if (per_sm < 1) per_sm = 1;
    *warps = sms * per_sm * (MEM_BLOCK / 32);
  }
  return MCE_OK;
}

namespace {

// One engine-class launch of the variant <EV, LIST, XP, OPS, SPLIT, STAGE, L2>.
template <int EV, bool LIST, bool XP, bool OPS, bool SPLIT, bool STAGE, bool L2>
int launch_cls(int cls, int word_bits, const BKArgs &a, int grid, int block, int smem,
               cudaStream_t s) {
  if (cls == CLS_R32 && word_bits == 64)
    bk_reg_kernel<u64, 1, EV, LIST, XP, OPS, SPLIT, false, L2><<<grid, block, smem, s>>>(a, cls);
  else if (cls == CLS_R32)
    bk_reg_kernel<uint32_t, 1, EV, LIST, XP, OPS, SPLIT, STAGE, L2><<<grid, block, smem, s>>>(a, cls);
  else if (cls == CLS_R64)
    bk_reg_kernel<u64, 2, EV, LIST, XP, OPS, SPLIT, false, L2><<<grid, block, smem, s>>>(a, cls);
  else if (cls == CLS_MEM && a.wide8 && EV == 0)
    bk_mem_kernel<EV, 8, LIST, OPS, SPLIT, XP, L2><<<grid, block, smem, s>>>(a, cls);
  else if (cls == CLS_MEM)
    bk_mem_kernel<EV, 1, LIST, OPS, SPLIT, XP, L2><<<grid, block, smem, s>>>(a, cls);
  else
    return MCE_EINVAL;
  MCE_CUDA(cudaGetLastError());
  return MCE_OK;
}

}  // namespace

// The variant a call needs: listing, the evaluation logs (per-warp load, and
// cycles), the word-op count, several warps per root, -i px, staged lists,
// L2 units.  Modes that do not combine: the evaluation and listing variants
// run with one warp per root and IP pivots; the word-op count with IP and L1.
int bk_launch(int cls, int word_bits, const BKArgs &a, int grid, int block, int smem,
              cudaStream_t s, int *launches) {
  if (grid <= 0) return MCE_OK;
  const int ev = a.warp_log == nullptr ? 0 : (a.warp_cycles ? 2 : 1);
  const bool xp = a.x_pivot != 0, split = a.parts > 1;
  int rc;
  if (a.level2) {
    if (a.list_buf)
      rc = launch_cls<0, true, false, false, false, false, true>(cls, word_bits, a, grid, block, smem, s);
    else if (ev == 2)
      rc = launch_cls<2, false, false, false, false, false, true>(cls, word_bits, a, grid, block, smem, s);
    else if (ev == 1)
      rc = launch_cls<1, false, false, false, false, false, true>(cls, word_bits, a, grid, block, smem, s);
    else if (xp)
      rc = launch_cls<0, false, true, false, false, false, true>(cls, word_bits, a, grid, block, smem, s);
    else
      rc = launch_cls<0, false, false, false, false, false, true>(cls, word_bits, a, grid, block, smem, s);
  } else if (a.list_buf) {
    rc = launch_cls<0, true, false, false, false, false, false>(cls, word_bits, a, grid, block, smem, s);
  } else if (a.count_ops) {
    rc = launch_cls<0, false, false, true, true, false, false>(cls, word_bits, a, grid, block, smem, s);
  } else if (ev == 2) {
    rc = launch_cls<2, false, false, false, false, false, false>(cls, word_bits, a, grid, block, smem, s);
  } else if (ev == 1) {
    rc = launch_cls<1, false, false, false, false, false, false>(cls, word_bits, a, grid, block, smem, s);
  } else if (split) {
    if (xp)
      rc = launch_cls<0, false, true, false, true, false, false>(cls, word_bits, a, grid, block, smem, s);
    else
      rc = launch_cls<0, false, false, false, true, false, false>(cls, word_bits, a, grid, block, smem, s);
  } else if (xp) {
    rc = launch_cls<0, false, true, false, false, false, false>(cls, word_bits, a, grid, block, smem, s);
  } else if (a.stage) {
    rc = launch_cls<0, false, false, false, false, true, false>(cls, word_bits, a, grid, block, smem, s);
  } else {
    rc = launch_cls<0, false, false, false, false, false, false>(cls, word_bits, a, grid, block, smem, s);
  }
  if (rc == MCE_OK && launches) *launches += 1;
  return rc;
}

int queue_launch_init(const QueueView &q, cudaStream_t s, int *launches) {
  MCE_CUDA(cudaMemsetAsync(q.hdr, 0, sizeof(QueueHdr), s));
  queue_init_kernel<<<(q.cap + 255) / 256, 256, 0, s>>>(q);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return MCE_OK;
}

// ===========================================================================
// Allocation-free search entry point.
//
// For callers that cannot allocate device memory: processes whose GPU memory
// is owned entirely by another allocator (a framework's caching allocator
// that has reserved the device), and latency-critical loops in which
// cudaMalloc's implicit device-wide synchronisation is not acceptable.  The
// caller passes an oriented graph, a root list and a histogram, all already
// in device memory; the search runs the 32-wide register engine with its
// per-warp scratch in the file-scope array below, which every GPU that loads
// this library holds until the process exits.
//
// Every call resolves the array's device address on the current device with
// cudaGetSymbolAddress, checks the root ids against the vertex count before
// any read at them, and synchronises its stream twice (the root check, the
// status) before it returns.  Every call shares
// the array and clears the part that must start at zero, so calls whose work
// overlaps on the GPU race with each other: serialise them (one stream, or
// events).
// ===========================================================================
namespace {

constexpr size_t NOALLOC_CTL_BYTES = 1024;  // ShapeInfo, fetch counters, status, nodes
constexpr size_t NOALLOC_SLAB_WORDS = 2 * REG_XCAP;  // u64 words per warp: 4 x REG_XCAP u32 words
static_assert(MCE_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size");

static __device__ __align__(256) unsigned long long g_noalloc_scratch[MCE_NOALLOC_SCRATCH_BYTES / 8];

struct NoallocCtl {
  ShapeInfo shape;
  uint32_t fetch[8];
  uint32_t err[4];
  unsigned long long nodes[4];
};
static_assert(sizeof(NoallocCtl) <= NOALLOC_CTL_BYTES, "control block");

// The host-side name g_noalloc_scratch is not a device address; the address
// of the current device's copy is looked up on every call (cheap next to the
// call's two stream synchronisations), so there is no host-side cache to
// guard between threads or to go stale after a device reset.
int noalloc_scratch(unsigned long long **out) {
  void *p = nullptr;
  MCE_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  *out = (unsigned long long *)p;
  return MCE_OK;
}

// Every root id must lie in [0, n) - tested before anything is read at that
// id (bit 2 of err[0]) - and fit the 32-wide engine: 1..32 later and
// <= REG_XCAP earlier neighbours (bit 1).
__global__ void noalloc_check_kernel(const int32_t *rp, const int32_t *split, int64_t n,
                                     const int32_t *roots, uint32_t num_roots, NoallocCtl *ctl) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    ctl->shape.cls_off[CLS_R32] = 0;
    ctl->shape.cls_off[CLS_R32 + 1] = num_roots;
  }
  if (i >= num_roots) return;
  const int32_t r = roots[i];
  if (r < 0 || (int64_t)r >= n) {
    atomicOr(&ctl->err[0], 2u);
    return;
  }
  const int32_t dplus = rp[r + 1] - split[r], dminus = split[r] - rp[r];
  if (dplus < 1 || dplus > 32 || dminus > REG_XCAP) atomicOr(&ctl->err[0], 1u);
}

}  // namespace

extern "C" int mce_count_oriented_noalloc(const int32_t *d_row_ptr, const int32_t *d_split,
                                          const int32_t *d_col_split, int64_t n,
                                          const int32_t *d_roots, int64_t num_roots,
                                          uint64_t *d_hist, void *stream) {
  if (num_roots < 0 || n < 0 || !d_hist ||
      (num_roots > 0 && (!d_row_ptr || !d_split || !d_col_split || !d_roots)))
    return MCE_EINVAL;
  if (num_roots >= ((int64_t)1 << 31) || n >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  int dev = 0, sms = 0, per_sm = 0;
  MCE_CUDA(cudaGetDevice(&dev));
  unsigned long long *base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  NoallocCtl *ctl = (NoallocCtl *)base;
  MCE_CUDA(cudaMemsetAsync(ctl, 0, NOALLOC_CTL_BYTES, s));
  const uint32_t nr = (uint32_t)num_roots;
  noalloc_check_kernel<<<(nr + 255) / 256 + 1, 256, 0, s>>>(d_row_ptr, d_split, n, d_roots, nr,
                                                             ctl);
  MCE_CUDA(cudaGetLastError());
  uint32_t err = 0;
  MCE_CUDA(cudaMemcpyAsync(&err, &ctl->err[0], sizeof(err), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  if (err & 2u) return MCE_EINVAL;
  if (err) return MCE_ELIMIT;
  MCE_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(uint64_t) * MCE_HIST_MAX, s));
  if (nr == 0) {
    MCE_CUDA(cudaStreamSynchronize(s));
    return MCE_OK;
  }
  // as many whole blocks of warps as the occupancy, the roots and the array allow
  MCE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bk_reg_kernel<uint32_t, 1>,
                                                         REG_BLOCK, 0));
  const int wpb = REG_BLOCK / 32;
  const int64_t slab_warps =
      (int64_t)((MCE_NOALLOC_SCRATCH_BYTES - NOALLOC_CTL_BYTES) / (NOALLOC_SLAB_WORDS * 8));
  int64_t blocks = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  blocks = blocks < slab_warps / wpb ? blocks : slab_warps / wpb;
  const int64_t want = ((int64_t)nr + REG_CHUNK * wpb - 1) / (REG_CHUNK * wpb);
  if (want < blocks) blocks = want;
  BKArgs a;
  memset(&a, 0, sizeof(a));
  a.rp = d_row_ptr;
  a.split = d_split;
  a.cs = d_col_split;
  a.roots = d_roots;
  a.shape = &ctl->shape;
  a.fetch = ctl->fetch;
  a.hist = (unsigned long long *)d_hist;
  a.nodes = ctl->nodes;
  a.err = &ctl->err[1];
  a.slab = base + NOALLOC_CTL_BYTES / 8;
  a.slab_words = NOALLOC_SLAB_WORDS;
  a.dcap = 32;
  a.xcap = REG_XCAP;
  a.rxcap = REG_XCAP;
  bk_reg_kernel<uint32_t, 1><<<(unsigned)blocks, REG_BLOCK, 0, s>>>(a, CLS_R32);
  MCE_CUDA(cudaGetLastError());
  MCE_CUDA(cudaMemcpyAsync(&err, &ctl->err[1], sizeof(err), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  return err ? MCE_ELIMIT : MCE_OK;
}

}  // namespace mce
