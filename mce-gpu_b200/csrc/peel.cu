// Degeneracy order by synchronous k-core peeling: one cooperative launch.
//
// Replaces graph::SingleGPU_Kcore::findKcoreIncremental_async
// (include/kcore.cuh:233-316), which drives every peel round from the host
// with several launches and a cudaDeviceSynchronize + scalar read-backs per
// round.  Here all levels and rounds run inside one persistent kernel whose
// blocks meet at a bounded grid barrier between phases; the host launches
// once and reads nothing until the end.
//
// Semantics kept from the reference (so priorities are bit-identical):
//  - at level k, round 0 is every remaining vertex of remaining degree k
//    (filter_window + filter_with_random_append, include/kcore.cuh:21-48);
//  - removing a round lowers neighbour degrees; a neighbour whose degree
//    falls from k+1 to k joins the next round (process_degree, :80-95);
//  - rounds are numbered over all levels; priority[v] = v's round number,
//    and the round that empties the graph is not processed, so its vertices
//    keep priority = m (:258, :276);
//  - a level with no vertex of degree k runs no round (the scan below jumps
//    straight to the smallest remaining degree, which numbers rounds the
//    same way).
// Decrements of a vertex that is already removed or queued are skipped;
// they cannot change any round's membership.
#include <climits>

#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace mce {

struct PeelCtl {
  GridBarrier bar;
  uint32_t err;
  uint32_t fcnt[3];    // light frontier sizes, one slot per phase mod 3
  unsigned long long hpack[3];  // heavy frontier: (count << 32) | 32-edge chunks
  uint32_t acnt[3];    // alive-list sizes, one slot per scan mod 3
  uint32_t amin[3];    // min degree over the alive list written by a scan
  int32_t degeneracy;
  uint32_t rounds;
  uint32_t levels;
  // state handed back by a solo section (written by block 0, read by all)
  uint32_t solo_q, solo_cnt, solo_priority, solo_rounds;
  int64_t solo_todo;
  int32_t solo_degen;
  uint32_t solo_sections;
  unsigned long long t_scan, t_round, t_wait;  // ns seen by block 0 (diagnostics)
  uint32_t seg_next;   // batches: next graph to peel
  uint32_t seg_part[MAX_BATCH_PARTS];  // ... the same per part of a batch still arriving
  uint32_t seg_mid_next;       // the same for the middle and small graphs' launches
  uint32_t seg_mid_part[MAX_BATCH_PARTS];
  uint32_t seg_small_next;
  uint32_t seg_small_part[MAX_BATCH_PARTS];
};

namespace {

constexpr int PEEL_BLOCK = 512;
// A frontier of at most solo_max vertices is peeled by block 0 alone, round
// after round with __syncthreads between them, for up to SOLO_ROUNDS rounds
// (well inside the other blocks' barrier wait limit).
constexpr uint32_t SOLO_ROUNDS = 65536;
// A frontier vertex with more neighbours than this is "heavy": it is stored
// from the back of the frontier buffer, its first chunk number goes to the
// slot's chunk-base array, and the round spreads all heavy chunks (32 edges
// each) over every warp, so no single warp serialises a hub while the rest
// of the grid waits at the next barrier.  One 64-bit atomic hands out both
// the slot and the chunk base, so bases increase with the slot.
constexpr int32_t HEAVY_DEG = 256;
// Light frontier vertices a warp takes at a time in a large frontier.
constexpr int PEEL_GROUP = 8;

// A warp's staging buffer for the next frontier: appends gather here and
// reach the list STAGE at a time, one atomic on its counter per flush
// instead of one per 32-edge window (the counter is shared by the grid).
constexpr uint32_t STAGE = 256;
struct Stage {
  int32_t *buf;  // STAGE entries of shared memory, one buffer per warp
  uint32_t n;    // warp-uniform fill
};

__device__ __forceinline__ void stage_flush(Stage &st, int32_t *list, uint32_t *cnt) {
  if (!st.n) return;
  const uint32_t lane = lane_id();
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(cnt, st.n);
  base = __shfl_sync(MCE_FULL, base, 0);
  for (uint32_t i = lane; i < st.n; i += 32) list[base + i] = st.buf[i];
  __syncwarp();
  st.n = 0;
}

__device__ __forceinline__ void stage_append(Stage &st, bool pred, int32_t val, int32_t *list,
                                             uint32_t *cnt) {
  const uint32_t mask = __ballot_sync(MCE_FULL, pred);
  if (!mask) return;
  const uint32_t k = __popc(mask);
  if (st.n + k > STAGE) stage_flush(st, list, cnt);
  if (pred) st.buf[st.n + __popc(mask & ((1u << lane_id()) - 1u))] = val;
  __syncwarp();
  st.n += k;
}

// Block-aggregated appends to two lists (one atomic per list per block);
// every thread of the block must call it.
__device__ __forceinline__ void block_append2(bool p1, int32_t v1, int32_t *l1, uint32_t *c1,
                                              bool p2, int32_t v2, int32_t *l2, uint32_t *c2) {
  __shared__ uint32_t w1[PEEL_BLOCK / 32], w2[PEEL_BLOCK / 32], base1, base2;
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t m1 = __ballot_sync(MCE_FULL, p1), m2 = __ballot_sync(MCE_FULL, p2);
  if (lane == 0) {
    w1[wid] = __popc(m1);
    w2[wid] = __popc(m2);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t a = 0, b = 0;
    for (uint32_t w = 0; w < nw; ++w) {
      const uint32_t x = w1[w], y = w2[w];
      w1[w] = a;
      w2[w] = b;
      a += x;
      b += y;
    }
    base1 = a ? atomicAdd(c1, a) : 0;
    base2 = b ? atomicAdd(c2, b) : 0;
  }
  __syncthreads();
  if (p1) l1[base1 + w1[wid] + __popc(m1 & lt)] = v1;
  if (p2) l2[base2 + w2[wid] + __popc(m2 & lt)] = v2;
  __syncthreads();  // the shared counters are reused by the next call
}

// Append a heavy vertex: slot k at list[cap - 1 - k], first chunk at base[k].
__device__ __forceinline__ void heavy_append(bool pred, int32_t v, int32_t degv, int32_t *list,
                                             int32_t *base, int64_t cap,
                                             unsigned long long *pack) {
  if (!pred) return;
  const unsigned long long chunks = (unsigned long long)((degv + 31) / 32);
  const unsigned long long old = atomicAdd(pack, (1ull << 32) | chunks);
  const uint32_t slot = (uint32_t)(old >> 32);
  list[cap - 1 - (int64_t)slot] = v;
  base[slot] = (int32_t)(uint32_t)old;
}

__device__ __forceinline__ unsigned long long ld_volatile64(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}

__device__ __forceinline__ uint32_t frontier_size(const PeelCtl *ctl, int slot) {
  return ld_volatile(&ctl->fcnt[slot]) + (uint32_t)(ld_volatile64(&ctl->hpack[slot]) >> 32);
}

// Lower the degree of neighbour col[j] of a vertex being removed; true if it
// falls to `level` (it then joins the next round).
__device__ __forceinline__ bool peel_edge(int32_t j, int32_t e, int32_t level,
                                          const int32_t *__restrict__ col, int32_t *deg,
                                          int32_t *core, int32_t &u) {
  u = 0;
  if (j >= e) return false;
  u = col[j];
  if (ld_volatile((const uint32_t *)&core[u]) != 0xFFFFFFFFu) return false;
  const int32_t old = atomicSub(&deg[u], 1);
  if (old != level + 1) return false;
  core[u] = level;
  return true;
}

// One peel round (phase q) over the frontier in slot q % 3, executed by the
// threads [t0, t0 + nt) (the whole grid, or block 0 alone): set the round's
// priority, lower the neighbours' degrees and append every neighbour whose
// degree falls to `level` to the frontier in slot (q + 1) % 3.
__device__ __forceinline__ void peel_round(uint32_t q, int32_t level, uint32_t priority,
                                           int64_t t0, int64_t nt, int64_t cap,
                                           const int32_t *__restrict__ rp,
                                           const int32_t *__restrict__ col, int32_t *deg,
                                           int32_t *core, uint32_t *prio, int32_t *const *fr,
                                           int32_t *const *hb, PeelCtl *ctl, int32_t *stage) {
  const uint32_t lane = lane_id();
  Stage st{stage, 0};
  const int fn = (q + 1) % 3;
  if (t0 == 0) {
    ctl->fcnt[(q + 2) % 3] = 0;
    ctl->hpack[(q + 2) % 3] = 0;
  }
  const uint32_t lc = ld_volatile(&ctl->fcnt[q % 3]);
  const unsigned long long hp = ld_volatile64(&ctl->hpack[q % 3]);
  const uint32_t hc = (uint32_t)(hp >> 32), hch = (uint32_t)hp;
  const int32_t *Fc = fr[q % 3], *HB = hb[q % 3];
  int32_t *Fn = fr[fn], *HBn = hb[fn];
  for (int64_t i = t0; i < lc; i += nt) prio[Fc[i]] = priority;
  for (int64_t i = t0; i < hc; i += nt) prio[Fc[cap - 1 - i]] = priority;
  auto push = [&](bool p, int32_t u) {
    int32_t du = 0;
    if (p) du = rp[u + 1] - rp[u];
    const bool heavy = p && du > HEAVY_DEG;
    stage_append(st, p && !heavy, u, Fn, &ctl->fcnt[fn]);
    heavy_append(heavy, u, du, Fn, HBn, cap, &ctl->hpack[fn]);
  };
  // light vertices: a warp each; in a frontier with at least PEEL_GROUP of
  // them per warp, a warp takes PEEL_GROUP at a time and keeps the loads
  // and degree updates of their first windows in flight together (one chain
  // of dependent accesses per group instead of one per vertex)
  const int64_t nwarp = nt >> 5;
  if (lc >= (int64_t)PEEL_GROUP * nwarp) {
    constexpr int R = PEEL_GROUP;
    const int64_t groups = (lc + R - 1) / R;
    for (int64_t gi = t0 >> 5; gi < groups; gi += nwarp) {
      const int64_t i0 = gi * R;
      const int rows = lc - i0 < R ? (int)(lc - i0) : R;
      int32_t v = 0, b = 0, e = 0;
      if ((int)lane < rows) {
        v = Fc[i0 + lane];
        b = rp[v];
        e = rp[v + 1];
      }
      int32_t U[R];
      bool live[R];
#pragma unroll
      for (int k = 0; k < R; ++k) {  // every row's first window
        const int32_t j = __shfl_sync(MCE_FULL, b, k) + (int32_t)lane;
        const bool in = k < rows && j < __shfl_sync(MCE_FULL, e, k);
        U[k] = in ? col[j] : 0;
        live[k] = in;
      }
#pragma unroll
      for (int k = 0; k < R; ++k)
        live[k] = live[k] && ld_volatile((const uint32_t *)&core[U[k]]) == 0xFFFFFFFFu;
      int32_t old[R];
#pragma unroll
      for (int k = 0; k < R; ++k) old[k] = live[k] ? atomicSub(&deg[U[k]], 1) : 0;
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const bool p = live[k] && old[k] == level + 1;
        if (p) core[U[k]] = level;
        push(p, U[k]);
      }
      for (int k = 0; k < rows; ++k) {  // the rest of rows longer than a window
        const int32_t bk = __shfl_sync(MCE_FULL, b, k), ek = __shfl_sync(MCE_FULL, e, k);
        for (int32_t j0 = bk + 32; j0 < ek; j0 += 32) {
          int32_t u;
          const bool p = peel_edge(j0 + (int32_t)lane, ek, level, col, deg, core, u);
          push(p, u);
        }
      }
    }
  } else {
    for (int64_t i = t0 >> 5; i < lc; i += nwarp) {
      const int32_t v = Fc[i];
      const int32_t b = rp[v], e = rp[v + 1];
      for (int32_t j0 = b; j0 < e; j0 += 32) {
        int32_t u;
        const bool p = peel_edge(j0 + (int32_t)lane, e, level, col, deg, core, u);
        push(p, u);
      }
    }
  }
  // heavy vertices: chunk c belongs to the last slot whose base is <= c
  for (int64_t c = t0 >> 5; c < hch; c += nt >> 5) {
    int lo = 0, hi = (int)hc;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (HB[mid] <= (int32_t)c)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int h = lo - 1;
    const int32_t v = Fc[cap - 1 - h];
    const int32_t e = rp[v + 1];
    const int32_t j = rp[v] + ((int32_t)c - HB[h]) * 32 + (int32_t)lane;
    int32_t u;
    const bool p = peel_edge(j, e, level, col, deg, core, u);
    push(p, u);
  }
  stage_flush(st, Fn, &ctl->fcnt[fn]);
}

__global__ void __launch_bounds__(PEEL_BLOCK)
    peel_kernel(int32_t n, uint32_t m, const int32_t *__restrict__ rp,
                const int32_t *__restrict__ col, int32_t *deg, int32_t *core, uint32_t *prio,
                int32_t *alistA, int32_t *alistB, int32_t *front0, int32_t *front1,
                int32_t *front2, int32_t *hb0, int32_t *hb1, int32_t *hb2, PeelCtl *ctl,
                uint64_t limit_ns, uint32_t solo_max) {
  __shared__ int32_t stage_all[PEEL_BLOCK / 32][STAGE];
  int32_t *const stage = stage_all[threadIdx.x >> 5];
  const uint32_t nblocks = gridDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
  const uint32_t lane = lane_id();
  int32_t *const fr[3] = {front0, front1, front2};
  int32_t *const hb[3] = {hb0, hb1, hb2};
  int32_t *alist[2] = {alistA, alistB};

  for (int64_t v = tid; v < n; v += nthr) {
    deg[v] = rp[v + 1] - rp[v];
    core[v] = -1;
    prio[v] = m;
    alistA[v] = (int32_t)v;
  }
  if (tid == 0) {  // phase/scan 0 reads acnt[0]; every other counter starts at 0
    ctl->fcnt[0] = ctl->fcnt[1] = ctl->fcnt[2] = 0;
    ctl->hpack[0] = ctl->hpack[1] = ctl->hpack[2] = 0;
    ctl->acnt[0] = (uint32_t)n;
    ctl->acnt[1] = ctl->acnt[2] = 0;
    ctl->amin[0] = ctl->amin[1] = ctl->amin[2] = 0xFFFFFFFFu;
  }
  if (!grid_sync(&ctl->bar, nblocks, &ctl->err, limit_ns)) return;

  // phase timers of block 0 (diagnostics only)
  unsigned long long t_ts = 0, t_tr = 0, t_w = 0, mark = tid == 0 ? globaltimer_ns() : 0;
  auto tick = [&](unsigned long long &acc) {
    if (tid == 0) {
      const unsigned long long now = globaltimer_ns();
      acc += now - mark;
      mark = now;
    }
  };
  int64_t todo = n;
  int32_t level = 0, degen = 0;
  uint32_t priority = 0, rounds = 0, levels = 0;
  // Phases (scans and rounds) are numbered q = 0, 1, 2, ...  Phase q appends
  // its output frontier to buffer/counter slot (q + 1) % 3 and resets slot
  // (q + 2) % 3; after barrier q every thread reads slot (q + 1) % 3.  A
  // slot is reset two phases after it was read, so a slow reader can never
  // see a counter that another block has already started to refill.  Scans
  // are numbered s the same way for the alive-list counters (3 slots) and
  // buffers (2 slots).
  uint32_t q = 0, s = 0;
  while (todo > 0) {
    // ---- scan: split the alive list into {deg == level} and {deg > level}
    const uint32_t nalive = ld_volatile(&ctl->acnt[s % 3]);
    const int32_t *A = alist[s & 1];
    int32_t *A2 = alist[(s + 1) & 1];
    const int fo = (q + 1) % 3, ao = (s + 1) % 3;
    int32_t *F = fr[fo];
    if (tid == 0) {
      ctl->acnt[(s + 2) % 3] = 0;
      ctl->amin[(s + 2) % 3] = 0xFFFFFFFFu;
      ctl->fcnt[(q + 2) % 3] = 0;
      ctl->hpack[(q + 2) % 3] = 0;
    }
    {
      uint32_t mymin = 0xFFFFFFFFu;
      // block-strided so that every thread of a block runs the same number
      // of iterations: appends are aggregated per block (one atomic each)
      const int64_t bs = blockDim.x;
      const int64_t lim = ((int64_t)nalive + bs - 1) / bs * bs;
      for (int64_t i = tid; i < lim; i += nthr) {
        int32_t v = 0, d = 0;
        bool live = false;
        if (i < nalive) {
          v = A[i];
          live = ld_volatile((const uint32_t *)&core[v]) == 0xFFFFFFFFu;
          d = deg[v];
        }
        const bool inF = live && d == level;
        const bool keep = live && d > level;
        if (inF) core[v] = level;
        const int32_t dv = inF ? rp[v + 1] - rp[v] : 0;
        const bool heavy = inF && dv > HEAVY_DEG;
        block_append2(inF && !heavy, v, F, &ctl->fcnt[fo], keep, v, A2, &ctl->acnt[ao]);
        heavy_append(heavy, v, dv, F, hb[fo], (int64_t)n + 1, &ctl->hpack[fo]);
        if (keep) mymin = min(mymin, (uint32_t)d);
      }
      mymin = __reduce_min_sync(MCE_FULL, mymin);
      if (lane == 0 && mymin != 0xFFFFFFFFu) atomicMin(&ctl->amin[ao], mymin);
    }
    tick(t_ts);
    if (!grid_sync(&ctl->bar, nblocks, &ctl->err, limit_ns)) return;
    tick(t_w);
    ++q;
    ++s;
    uint32_t cnt = frontier_size(ctl, q % 3);
    if (cnt == 0) {
      // no vertex of degree `level` remains: jump to the smallest degree
      // (a rescan at that level always finds the vertex that attains it)
      const uint32_t mn = ld_volatile(&ctl->amin[s % 3]);
      if (mn == 0xFFFFFFFFu || (int32_t)mn <= level) {
        if (tid == 0) atomicOr(&ctl->err, MCE_ERR_QUEUE);  // inconsistent state: stop
        break;
      }
      level = (int32_t)mn;
      continue;
    }
    ++levels;
    // ---- rounds of this level: phase q reads frontier q % 3
    while (cnt > 0) {
      degen = level;
      todo -= cnt;
      if (todo == 0) break;  // the final round keeps priority = m
      if (cnt <= solo_max) {
        // Small frontier: block 0 peels consecutive rounds alone.  The first
        // barrier lets every block read `cnt` before block 0 recycles slots.
        tick(t_tr);
        if (!grid_sync(&ctl->bar, nblocks, &ctl->err, limit_ns)) return;
        tick(t_w);
        if (blockIdx.x == 0) {
          uint32_t it = 0;
          for (;;) {
            peel_round(q, level, priority, threadIdx.x, blockDim.x, (int64_t)n + 1, rp, col,
                       deg, core, prio, fr, hb, ctl, stage);
            __syncthreads();
            ++q;
            cnt = frontier_size(ctl, q % 3);
            ++priority;
            ++rounds;
            if (cnt == 0 || cnt > solo_max || ++it >= SOLO_ROUNDS) break;  // cnt not yet counted
            degen = level;
            todo -= cnt;
            if (todo == 0) break;  // the final round keeps priority = m
            __syncthreads();       // every thread has read cnt before slots rotate
          }
          if (threadIdx.x == 0) {
            ctl->solo_q = q;
            ctl->solo_cnt = cnt;
            ctl->solo_priority = priority;
            ctl->solo_rounds = rounds;
            ctl->solo_todo = todo;
            ctl->solo_degen = degen;
            ++ctl->solo_sections;
          }
        }
        tick(t_tr);
        if (!grid_sync(&ctl->bar, nblocks, &ctl->err, limit_ns)) return;
        tick(t_w);
        q = ld_volatile(&ctl->solo_q);
        cnt = ld_volatile(&ctl->solo_cnt);
        priority = ld_volatile(&ctl->solo_priority);
        rounds = ld_volatile(&ctl->solo_rounds);
        todo = *(volatile int64_t *)&ctl->solo_todo;
        degen = *(volatile int32_t *)&ctl->solo_degen;
        if (todo == 0) break;
        continue;
      }
      peel_round(q, level, priority, tid, nthr, (int64_t)n + 1, rp, col, deg, core, prio, fr, hb,
                 ctl, stage);
      tick(t_tr);
      if (!grid_sync(&ctl->bar, nblocks, &ctl->err, limit_ns)) return;
      tick(t_w);
      ++q;
      cnt = frontier_size(ctl, q % 3);
      ++priority;
      ++rounds;
    }
    if (todo == 0) break;
    ++level;
  }
  if (tid == 0) {
    ctl->degeneracy = degen;
    ctl->t_scan = t_ts;
    ctl->t_round = t_tr;
    ctl->t_wait = t_w;
    ctl->rounds = rounds;
    ctl->levels = levels;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Batches: one block peels one graph of the disjoint union at a time.
//
// The graphs of a batch share no edge, so each can be peeled alone; a block
// runs a graph's synchronous rounds with __syncthreads between them instead
// of grid barriers, and blocks take graphs largest first.  Rounds are
// numbered per graph and a graph's final round keeps priority m_g (its own
// arc count): each graph gets the numbering the reference gives it when it
// is the whole input.  Orientation only compares vertices of one graph.
// ---------------------------------------------------------------------------
namespace {

// 16 warps per graph: on the 4,096-graph batch the per-graph peel took
// 5.6 ms with 256 threads, 3.6 ms with 512 and 5.0 ms with 1,024 (its length
// is the round chain of the largest graphs; more threads shorten each round,
// fewer resident blocks leave fewer graphs running at once).
constexpr int SEG_BLOCK = 512;

struct SegShared {
  int32_t todo, level, minv, fcnt, ncnt;
  uint32_t g;
};

// Graphs of at most SEG_SMEM_N vertices keep their remaining degrees (16-bit
// halves of 32-bit words, decremented by one atomic on the word: a degree
// never falls below zero, so no borrow reaches the other half) and their
// core numbers (16-bit, -1 while unpeeled) in shared memory: the rounds'
// decrements and tests stay on the SM.  Their frontiers hold local ids.
constexpr int SEG_SMEM_N = 16384;

__device__ __forceinline__ int sdeg_get(const uint32_t *w, int i) {
  return (int)((w[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu);
}
__device__ __forceinline__ int sdeg_dec(uint32_t *w, int i) {  // returns the old degree
  const uint32_t sh = (uint32_t)(i & 1) * 16u;
  return (int)((atomicSub(&w[i >> 1], 1u << sh) >> sh) & 0xFFFFu);
}

// One graph (local vertices 0..n-1 = union vertices vb..vb+n-1) with its
// state in shared memory; the rounds and their numbering are those of the
// global-memory path below.
__device__ void peel_graph_smem(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                int32_t *core, uint32_t *prio, int32_t *F0, int32_t *G0,
                                int64_t vb, int n, uint32_t mg, uint32_t *sdeg, int16_t *score,
                                SegShared &sh, PeelCtl *ctl) {
  const int lane = (int)lane_id(), w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = threadIdx.x; 2 * k < n; k += blockDim.x) {
    const int64_t v = vb + 2 * k;
    const uint32_t d0 = (uint32_t)(rp[v + 1] - rp[v]);
    const uint32_t d1 = 2 * k + 1 < n ? (uint32_t)(rp[v + 2] - rp[v + 1]) : 0u;
    sdeg[k] = d0 | (d1 << 16);
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    score[i] = -1;
    prio[vb + i] = mg;
  }
  if (threadIdx.x == 0) {
    sh.todo = n;
    sh.level = 0;
  }
  __syncthreads();
  uint32_t priority = 0;
  int last_level = -1;
  while (sh.todo > 0) {
    const int level = sh.level;
    __syncthreads();
    if (threadIdx.x == 0) {
      sh.fcnt = 0;
      sh.minv = INT_MAX;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      if (score[i] == -1) {
        const int d = sdeg_get(sdeg, i);
        if (d <= level) {  // == level: a remaining vertex never has less
          score[i] = (int16_t)level;
          F0[atomicAdd(&sh.fcnt, 1)] = i;
        } else {
          atomicMin(&sh.minv, d);
        }
      }
    }
    __syncthreads();
    if (sh.fcnt == 0) {  // no vertex at this level: go to the lowest remaining degree
      __syncthreads();
      if (threadIdx.x == 0) sh.level = sh.minv;
      __syncthreads();
      continue;
    }
    int32_t *F = F0, *Gq = G0;
    for (;;) {
      const int cnt = sh.fcnt;
      __syncthreads();
      if (cnt == 0) break;
      last_level = level;
      if (threadIdx.x == 0) {
        sh.todo -= cnt;
        sh.ncnt = 0;
      }
      __syncthreads();
      if (sh.todo == 0) break;  // the final round keeps priority m_g
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) prio[vb + F[i]] = priority;
      for (int i = w; i < cnt; i += nw) {
        const int64_t v = vb + F[i];
        for (int32_t j = rp[v] + lane; j < rp[v + 1]; j += 32) {
          const int u = (int)(col[j] - vb);
          if ((unsigned)u >= (unsigned)n) continue;  // not this graph's vertex (invalid input)
          if (*(volatile int16_t *)&score[u] == -1) {
            const int old = sdeg_dec(sdeg, u);
            if (old == level + 1) {
              score[u] = (int16_t)level;
              Gq[atomicAdd(&sh.ncnt, 1)] = u;
            }
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) sh.fcnt = sh.ncnt;
      int32_t *t = F;
      F = Gq;
      Gq = t;
      ++priority;
      __syncthreads();
    }
    if (threadIdx.x == 0) sh.level = level + 1;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) core[vb + i] = score[i];
  if (threadIdx.x == 0) {
    atomicMax(&ctl->rounds, priority);
    atomicMax(&ctl->degeneracy, last_level < 0 ? 0 : last_level);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(SEG_BLOCK)
    peel_segments_kernel(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                         int32_t *deg, int32_t *core, uint32_t *prio, int32_t *fa, int32_t *fb,
                         const int64_t *__restrict__ vtx_off, const int64_t *__restrict__ arc_off,
                         const int32_t *__restrict__ order, int32_t G, PeelCtl *ctl,
                         uint32_t *next, int smem_n) {
  __shared__ SegShared sh;
  extern __shared__ uint32_t seg_dyn[];  // smem_n / 2 degree words, then smem_n cores
  uint32_t *sdeg = seg_dyn;
  int16_t *score = (int16_t *)(seg_dyn + smem_n / 2);
  const int lane = (int)lane_id(), w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) sh.g = atomicAdd(next, 1u);  // next graph, largest first
    __syncthreads();
    const uint32_t gi = sh.g;
    if (gi >= (uint32_t)G) break;
    const int32_t gr = order[gi];
    const int64_t vb = vtx_off[gr] - gr, n = vtx_off[gr + 1] - vtx_off[gr] - 1;
    const uint32_t mg = (uint32_t)(arc_off[gr + 1] - arc_off[gr]);
    if (n <= smem_n) {
      peel_graph_smem(rp, col, core, prio, fa + vb, fb + vb, vb, (int)n, mg, sdeg, score, sh, ctl);
      continue;
    }
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
      const int64_t v = vb + i;
      deg[v] = rp[v + 1] - rp[v];
      core[v] = -1;
      prio[v] = mg;
    }
    if (threadIdx.x == 0) {
      sh.todo = (int32_t)n;
      sh.level = 0;
    }
    __syncthreads();
    int32_t *F0 = fa + vb, *G0 = fb + vb;  // this graph's slice of the frontier buffers
    uint32_t priority = 0;
    int last_level = -1;
    while (sh.todo > 0) {
      const int level = sh.level;
      __syncthreads();
      if (threadIdx.x == 0) {
        sh.fcnt = 0;
        sh.minv = INT_MAX;
      }
      __syncthreads();
      for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const int64_t v = vb + i;
        if (core[v] == -1) {
          if (deg[v] <= level) {  // == level: a remaining vertex never has less
            core[v] = level;
            F0[atomicAdd(&sh.fcnt, 1)] = (int32_t)v;
          } else {
            atomicMin(&sh.minv, deg[v]);
          }
        }
      }
      __syncthreads();
      if (sh.fcnt == 0) {  // no vertex at this level: go to the lowest remaining degree
        __syncthreads();
        if (threadIdx.x == 0) sh.level = sh.minv;
        __syncthreads();
        continue;
      }
      int32_t *F = F0, *Gq = G0;
      for (;;) {
        const int cnt = sh.fcnt;
        __syncthreads();
        if (cnt == 0) break;
        last_level = level;
        if (threadIdx.x == 0) {
          sh.todo -= cnt;
          sh.ncnt = 0;
        }
        __syncthreads();
        if (sh.todo == 0) break;  // the final round keeps priority m_g
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) prio[F[i]] = priority;
        for (int i = w; i < cnt; i += nw) {
          const int32_t v = F[i];
          for (int32_t j = rp[v] + lane; j < rp[v + 1]; j += 32) {
            const int32_t u = col[j];
            if (*(volatile int32_t *)&core[u] == -1) {
              const int old = atomicSub(&deg[u], 1);
              if (old == level + 1) {
                core[u] = level;
                Gq[atomicAdd(&sh.ncnt, 1)] = u;
              }
            }
          }
        }
        __syncthreads();
        if (threadIdx.x == 0) sh.fcnt = sh.ncnt;
        int32_t *t = F;
        F = Gq;
        Gq = t;
        ++priority;
        __syncthreads();
      }
      if (threadIdx.x == 0) sh.level = level + 1;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      atomicMax(&ctl->rounds, priority);
      atomicMax(&ctl->degeneracy, last_level < 0 ? 0 : last_level);
    }
    __syncthreads();
  }
}

}  // namespace

// 128 threads per small graph (at most PEEL_SMALL_N vertices) and 256 per
// middle one (at most PEEL_MID_N): blocks that need 8 or 32 KB of shared
// memory, so many more of them fit on an SM than of the 512-thread blocks
// with room for 16,384 vertices.
constexpr int SEG_SMALL_BLOCK = 128, SEG_MID_BLOCK = 256;

int peel_segments_launch(const PeelArgs &a, const int64_t *vtx_off, const int64_t *arc_off,
                         const int32_t *order, int32_t G, int32_t g_big, int32_t g_mid,
                         cudaStream_t s, const PeelSide &ps, int *launches, int part,
                         int64_t max_n) {
  int dev = 0, sms = 0;
  MCE_CUDA(cudaGetDevice(&dev));
  MCE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // set on every call: the attribute belongs to the current device
  MCE_CUDA(cudaFuncSetAttribute(peel_segments_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SEG_SMEM_N * 4));
  if (part >= MAX_BATCH_PARTS) return MCE_EINVAL;
  if (g_big < 0 || g_mid < 0 || g_big + g_mid > G) return MCE_EINVAL;
  PeelCtl *ctl = (PeelCtl *)a.ctl;
  if (part < 0) MCE_CUDA(cudaMemsetAsync(ctl, 0, sizeof(PeelCtl), s));
  // one launch: `cnt` graphs of order[first..], blocks of `threads`, shared
  // state for graphs of up to `nmax` vertices
  auto launch = [&](int32_t first, int32_t cnt, int threads, int64_t nmax, uint32_t *next,
                    cudaStream_t st) -> int {
    if (cnt <= 0) return MCE_OK;
    const int smem_n = nmax <= 0 ? 0 : (int)((std::min<int64_t>(nmax, SEG_SMEM_N) + 1) & ~1);
    const size_t smem = (size_t)smem_n * 4;  // 2 bytes of degree + 2 of core per vertex
    int per_sm = 0;
    MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, peel_segments_kernel, threads,
                                                           smem));
    if (per_sm < 1) return MCE_ECUDA;
    int blocks = sms * per_sm;
    if (blocks > cnt) blocks = cnt;
    peel_segments_kernel<<<blocks, threads, smem, st>>>(a.rp, a.col, a.deg, a.core, a.prio,
                                                        a.front0, a.front1, vtx_off, arc_off,
                                                        order + first, cnt, ctl, next, smem_n);
    MCE_CUDA(cudaGetLastError());
    if (launches) *launches += 1;
    return MCE_OK;
  };
  const bool p0 = part < 0;
  const int32_t g_small = G - g_big - g_mid;
  const bool fork = ps.side[0] && ps.side[1] && ps.fork && ps.join[0] && ps.join[1] &&
                    (g_mid > 0 || g_small > 0);
  if (fork) {
    MCE_CUDA(cudaEventRecord(ps.fork, s));
    MCE_CUDA(cudaStreamWaitEvent(ps.side[0], ps.fork, 0));
    MCE_CUDA(cudaStreamWaitEvent(ps.side[1], ps.fork, 0));
  }
  int rc = launch(0, g_big, SEG_BLOCK, max_n, p0 ? &ctl->seg_next : &ctl->seg_part[part], s);
  if (rc) return rc;
  rc = launch(g_big, g_mid, SEG_MID_BLOCK, std::min<int64_t>(max_n, PEEL_MID_N),
              p0 ? &ctl->seg_mid_next : &ctl->seg_mid_part[part], fork ? ps.side[0] : s);
  if (rc) return rc;
  rc = launch(g_big + g_mid, g_small, SEG_SMALL_BLOCK, std::min<int64_t>(max_n, PEEL_SMALL_N),
              p0 ? &ctl->seg_small_next : &ctl->seg_small_part[part], fork ? ps.side[1] : s);
  if (rc) return rc;
  if (fork) {
    MCE_CUDA(cudaEventRecord(ps.join[0], ps.side[0]));
    MCE_CUDA(cudaEventRecord(ps.join[1], ps.side[1]));
    MCE_CUDA(cudaStreamWaitEvent(s, ps.join[0], 0));
    MCE_CUDA(cudaStreamWaitEvent(s, ps.join[1], 0));
  }
  return MCE_OK;
}

size_t peel_ctl_bytes() { return sizeof(PeelCtl); }

int peel_launch(const PeelArgs &a, cudaStream_t s, int *launches) {
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  MCE_CUDA(cudaGetDevice(&dev));
  MCE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MCE_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return MCE_ENODEV;
  MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, peel_kernel, PEEL_BLOCK, 0));
  if (per_sm < 1) return MCE_ECUDA;
  per_sm = per_sm > 2 ? 2 : per_sm;
  int32_t n = (int32_t)a.n;
  uint32_t m = (uint32_t)a.m;
  PeelCtl *ctl = (PeelCtl *)a.ctl;
  MCE_CUDA(cudaMemsetAsync(ctl, 0, sizeof(PeelCtl), s));
  uint64_t limit = a.wait_limit_ns;
  uint32_t solo_max = a.solo_max;
  void *args[] = {(void *)&n,        (void *)&m,        (void *)&a.rp,     (void *)&a.col,
                  (void *)&a.deg,    (void *)&a.core,   (void *)&a.prio,   (void *)&a.alistA,
                  (void *)&a.alistB, (void *)&a.front0, (void *)&a.front1, (void *)&a.front2,
                  (void *)&a.hb0,    (void *)&a.hb1,    (void *)&a.hb2,
                  (void *)&ctl,      (void *)&limit,    (void *)&solo_max};
  MCE_CUDA(cudaLaunchCooperativeKernel((void *)peel_kernel, dim3(sms * per_sm), dim3(PEEL_BLOCK),
                                       args, 0, s));
  if (launches) *launches += 1;
  return MCE_OK;
}

int peel_read(const void *ctl_dev, int32_t *degeneracy, uint32_t *err, uint32_t *rounds,
              uint32_t *solo_sections, cudaStream_t s, double *phase_ms) {
  PeelCtl h;
  MCE_CUDA(cudaMemcpyAsync(&h, ctl_dev, sizeof(PeelCtl), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  if (degeneracy) *degeneracy = h.degeneracy;
  if (err) *err = h.err;
  if (rounds) *rounds = h.rounds;
  if (solo_sections) *solo_sections = h.solo_sections;
  if (phase_ms) {
    phase_ms[0] = h.t_scan * 1e-6;
    phase_ms[1] = h.t_round * 1e-6;
    phase_ms[2] = h.t_wait * 1e-6;
  }
  return MCE_OK;
}

}  // namespace mce
