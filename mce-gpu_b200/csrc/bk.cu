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
#include "kernels.h"
#include "queue.cuh"

namespace mce {

__global__ void queue_init_kernel(QueueView q) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q.cap; i += gridDim.x * blockDim.x)
    q.seq[i] = i;
}

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
constexpr int REG_CHUNK = 4;    // roots fetched per atomic by the register engine

__device__ __forceinline__ int warp_incl_scan(int x) {
  const int lane = (int)lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(MCE_FULL, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// index t of the chunk item owning flattened element e: the last t with
// off[t] <= e (off is the exclusive prefix of the items' list lengths).
__device__ __forceinline__ int chunk_owner(const int32_t *off, int e) {
  int lo = 0, hi = 32;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= e)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo - 1;
}

__device__ __forceinline__ int lower_bound_g(const int32_t *a, int n, int32_t key) {
  int lo = 0, len = n;
  while (len > 0) {
    const int half = len >> 1;
    const bool right = a[lo + half] < key;
    lo = right ? lo + half + 1 : lo;
    len = right ? len - half - 1 : half;
  }
  return lo;
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

// Per-root outputs shared by donor and takers: accumulate.
__device__ __forceinline__ void root_done(const BKArgs &a, int32_t r, u64 nodes, u64 cnt) {
  if (lane_id() != 0) return;
  if (a.root_nodes && nodes) atomicAdd(&a.root_nodes[r], nodes);
  if (a.root_count && cnt) atomicAdd(&a.root_count[r], cnt);
  if (a.graph_count && cnt) atomicAdd(&a.graph_count[a.graph_of[r]], cnt);
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
  Word stk[32 * NR + 1][4]; // DFS frames: P, X, branch set, chosen set
  int32_t pl[32 * NR];      // the root's later neighbours (sorted ids), padded
  int32_t off[32];          // chunk prefix offsets
  int32_t beg[32];          // chunk list starts
};

// Per-warp slab of the register engine, in Words: a hash set used while the
// earlier-neighbour rows are built (2 * REG_XCAP), the distinct rows
// (REG_XCAP) and the rows adjacent to the current branch (REG_XCAP).
template <typename Word>
struct RegSlab {
  Word *hash, *xr, *xl;
};

template <typename Word>
__device__ __forceinline__ RegSlab<Word> reg_slab(const BKArgs &a, int64_t gw) {
  Word *base = (Word *)(a.slab + (size_t)gw * a.slab_words);
  RegSlab<Word> s;
  s.hash = base;
  s.xr = base + 2 * REG_XCAP;
  s.xl = s.xr + REG_XCAP;
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

template <typename Word, int NR>
__device__ void reg_encode(const BKArgs &a, RegSmem<Word, NR> &sm, const RegSlab<Word> &sl,
                           int32_t r, RegRoot<Word> &rt) {
  using O = WOps<Word>;
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const int32_t sb = a.split[r], d = a.rp[r + 1] - sb, ub = a.rp[r], u = sb - ub;

  // setup_stack_original_L1_IP (mce/mce_utils.cuh:565-611): P = N+(r)
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int i = lane + 32 * k;
    sm.pl[i] = i < d ? a.cs[sb + i] : INT_MAX;
    sm.rows[i] = 0;
  }
  __syncwarp();

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
    const int incl = warp_incl_scan(vlen);
    const int T = __shfl_sync(MCE_FULL, incl, 31);
    sm.off[lane] = incl - vlen;
    sm.beg[lane] = vb;
    __syncwarp();
    for (int e = lane; e < T; e += 32) {
      const int t = chunk_owner(sm.off, e);
      const int32_t w = a.cs[sm.beg[t] + (e - sm.off[t])];
      const int i = lower_bound_g(sm.pl, 32 * NR, w);
      if (i < d && sm.pl[i] == w) {
        const int j = c * 32 + t;
        atomicOr(&sm.rows[j], O::bit(i));
        atomicOr(&sm.rows[i], O::bit(j));
      }
    }
    __syncwarp();
  }
  rt.r0 = sm.rows[lane];
  rt.r1 = 0;
  if constexpr (NR == 2) rt.r1 = sm.rows[lane + 32];

  // Earlier neighbours x of r: row(x) = N(x) & P, kept once per distinct
  // non-empty value; x is earlier than every vertex of P, so N(x) & P lies
  // in N+(x).
  int nX = 0;
  if (u > 0) {
    int hc = 32;
    while (hc < 2 * u && hc < 2 * REG_XCAP) hc <<= 1;
    for (int i = lane; i < hc; i += 32) sl.hash[i] = 0;
    __syncwarp();
    for (int c = 0; c * 32 < u; ++c) {
      const int items = min(32, u - c * 32);
      int xb = 0, xlen = 0;
      if (lane < items) {
        const int32_t x = a.cs[ub + c * 32 + lane];
        xb = a.split[x];
        xlen = a.rp[x + 1] - xb;
      }
      sm.xs[lane] = 0;
      const int incl = warp_incl_scan(xlen);
      const int T = __shfl_sync(MCE_FULL, incl, 31);
      sm.off[lane] = incl - xlen;
      sm.beg[lane] = xb;
      __syncwarp();
      for (int e = lane; e < T; e += 32) {
        const int t = chunk_owner(sm.off, e);
        const int32_t w = a.cs[sm.beg[t] + (e - sm.off[t])];
        const int i = lower_bound_g(sm.pl, 32 * NR, w);
        if (i < d && sm.pl[i] == w) atomicOr(&sm.xs[t], O::bit(i));
      }
      __syncwarp();
      const Word row = sm.xs[lane];
      bool fresh = false;
      if (lane < items && row != 0) {
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
  }
  rt.r = r;
  rt.d = d;
  rt.nX = nX;
}

// Walk the subtree under node (P, X, S) of root rt.r.  For the root itself
// S = 0; for a task S holds the vertices chosen above the node.
template <typename Word, int NR>
__device__ void reg_tree(const BKArgs &a, RegSmem<Word, NR> &sm, const RegSlab<Word> &sl,
                         const RegRoot<Word> &rt, Word P, Word X, Word S, u64 &h0, u64 &h1,
                         u64 &nodes, u64 &cnt) {
  using O = WOps<Word>;
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const Word r0 = rt.r0, r1 = rt.r1;
  const int nX = rt.nX;
  const bool share = a.q.hdr != nullptr;
  // pivot of the start node (select_pivot_from_P / _and_Xp, mce/mce_utils.cuh:338-402)
  int start_k = 0;
  {
    const Word cand = P | X;
    const int pc = O::popc(P);
    int k = 0;
    bool el = false;
    if ((cand >> lane) & 1) {
      const int s = O::popc(P & r0);
      k = ((s + 1) << 7) | (127 - lane);
      el = ((X >> lane) & 1) && s == pc;
    }
    if constexpr (NR == 2) {
      if ((cand >> (lane + 32)) & 1) {
        const int s = O::popc(P & r1);
        k = max(k, ((s + 1) << 7) | (127 - (lane + 32)));
        el = el || (((X >> (lane + 32)) & 1) && s == pc);
      }
    }
    if (__any_sync(MCE_FULL, el) || P == 0) return;
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    start_k = k;
  }
  // apply_pivot_to_first_level (:204-216) / apply_pivot_to_next_level (:218-239)
  Word B = P & ~row_of<Word, NR>(r0, r1, 127 - (start_k & 127));
  // Leaf filter: for the root it is rebuilt at every depth-0 branch (rows
  // adjacent to that branch vertex); for a task it is built once (rows
  // containing the whole chosen set).
  const bool per_branch = (S == 0);
  int nL = 0;
  if (!per_branch && nX > 0) {
    for (int i0 = 0; i0 < nX; i0 += 32) {
      const int i = i0 + lane;
      const Word row = i < nX ? sl.xr[i] : (Word)0;
      const bool has = i < nX && (row & S) == S;
      const uint32_t mk = __ballot_sync(MCE_FULL, has);
      if (has) sl.xl[nL + __popc(mk & lt)] = row;
      nL += __popc(mk);
    }
    __syncwarp();
  }
  int depth = 0, recheck = 0;
  bool want = false;
  for (;;) {
    if (B == 0) {  // get_next_candidate found nothing: backtrack (:526-563)
      if (depth == 0) break;
      --depth;
      P = sm.stk[depth][0];
      X = sm.stk[depth][1];
      B = sm.stk[depth][2];
      S = sm.stk[depth][3];
      continue;
    }
    const int v = O::ctz(B);
    B &= B - 1;
    const Word vb = O::bit(v);
    const Word rv = row_of<Word, NR>(r0, r1, v);
    // populate_xl_and_cl (:321-336): child P' = P & N(v), X' = X & N(v);
    // v leaves P for X in this frame.
    const Word Pc = P & rv, Xc = X & rv, Sc = S | vb;
    P &= ~vb;
    X |= vb;
    ++nodes;
    if (per_branch && depth == 0 && nX > 0) {  // earlier neighbours adjacent to v
      nL = 0;
      for (int i0 = 0; i0 < nX; i0 += 32) {
        const int i = i0 + lane;
        const Word row = i < nX ? sl.xr[i] : (Word)0;
        const bool has = (row & vb) != 0;
        const uint32_t mk = __ballot_sync(MCE_FULL, has);
        if (has) sl.xl[nL + __popc(mk & lt)] = row;
        nL += __popc(mk);
      }
      __syncwarp();
    }
    if (Pc == 0) {
      // test_maximality (:507-524): P' and X' empty and no earlier
      // neighbour of the root adjacent to the whole clique.
      if (Xc == 0) {
        bool covered = false;
        for (int i0 = 0; i0 < nL; i0 += 32) {
          const int i = i0 + lane;
          const bool hit = i < nL && (sl.xl[i] & Sc) == Sc;
          if (__any_sync(MCE_FULL, hit)) {
            covered = true;
            break;
          }
        }
        if (!covered) {
          ++cnt;
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
    // select_pivot_from_P_and_Xp (:366-402): pivot over P' | X'; an X'
    // vertex adjacent to all of P' ends the path.
    const Word cand = Pc | Xc;
    const int pc = O::popc(Pc);
    int k = 0;
    bool el = false;
    if ((cand >> lane) & 1) {
      const int s = O::popc(Pc & r0);
      k = ((s + 1) << 7) | (127 - lane);
      el = ((Xc >> lane) & 1) && s == pc;
    }
    if constexpr (NR == 2) {
      if ((cand >> (lane + 32)) & 1) {
        const int s = O::popc(Pc & r1);
        k = max(k, ((s + 1) << 7) | (127 - (lane + 32)));
        el = el || (((Xc >> (lane + 32)) & 1) && s == pc);
      }
    }
    if (__any_sync(MCE_FULL, el)) continue;
    // hand the child to an idle warp (try_dequeue / do_fork_L1,
    // mce/mce_utils.cuh:872-880,1063-1113)
    if (share && pc >= a.donate_min &&
        (nodes >= a.donate_after || (a.policy && a.policy[rt.r]))) {
      if (--recheck <= 0) {  // the queue state is read every 32 candidate nodes
        want = wants_task(a.q);
        recheck = 32;
      }
      if (want) {
        const u64 w0 = (u64)(uint32_t)rt.r, w1 = (u64)Pc, w2 = (u64)Xc, w3 = (u64)Sc;
        if (q_push(a.q, [&](uint32_t k2) { return k2 == 0 ? w0 : k2 == 1 ? w1 : k2 == 2 ? w2 : w3; }))
          continue;
        want = false;
      }
    }
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    if (lane == 0) {
      sm.stk[depth][0] = P;
      sm.stk[depth][1] = X;
      sm.stk[depth][2] = B;
      sm.stk[depth][3] = S;
    }
    __syncwarp();
    ++depth;
    P = Pc;
    X = Xc;
    S = Sc;
    // apply_pivot_to_next_level (:218-239)
    B = Pc & ~row_of<Word, NR>(r0, r1, 127 - (k & 127));
  }
}

template <typename Word, int NR>
__global__ void __launch_bounds__(REG_BLOCK) bk_reg_kernel(BKArgs a, int cls) {
  __shared__ RegSmem<Word, NR> sm_all[REG_BLOCK / 32];
  RegSmem<Word, NR> &sm = sm_all[threadIdx.x >> 5];
  const int lane = (int)lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const RegSlab<Word> sl = reg_slab<Word>(a, gw);
  const uint32_t beg = a.shape->cls_off[cls], end = a.shape->cls_off[cls + 1];
  const bool share = a.q.hdr != nullptr;
  u64 h0 = 0, h1 = 0, nodes = 0;
  RegRoot<Word> rt;
  if (share && lane == 0) atomicAdd(&a.q.hdr->work, 1u);
  for (;;) {
    uint32_t i0 = 0;
    if (lane == 0) i0 = atomicAdd(&a.fetch[cls], (uint32_t)REG_CHUNK);
    i0 = __shfl_sync(MCE_FULL, i0, 0);
    if (i0 >= end - beg) break;
    for (int k = 0; k < REG_CHUNK; ++k) {
      const uint32_t idx = beg + i0 + k;
      if (idx >= end) break;
      const int32_t r = a.roots[idx];
      reg_encode<Word, NR>(a, sm, sl, r, rt);
      u64 nd = 0, cnt = 0;
      reg_tree<Word, NR>(a, sm, sl, rt, WOps<Word>::low(rt.d), (Word)0, (Word)0, h0, h1, nd, cnt);
      nodes += nd;
      root_done(a, r, nd, cnt);
    }
  }
  if (share) {
    if (lane == 0) {
      atomicSub(&a.q.hdr->work, 1u);
      atomicAdd(&a.q.hdr->epoch, 1u);
    }
    u64 t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    idle_phase(
        a,
        [&](uint32_t k, u64 w) {  // lane k receives word k
          if (k == 0) t0 = w;
          if (k == 1) t1 = w;
          if (k == 2) t2 = w;
          if (k == 3) t3 = w;
        },
        [&]() {
          // word k of the task arrived on lane k
          const int32_t r = (int32_t)__shfl_sync(MCE_FULL, t0, 0);
          const Word P = (Word)__shfl_sync(MCE_FULL, t1, 1);
          const Word X = (Word)__shfl_sync(MCE_FULL, t2, 2);
          const Word S = (Word)__shfl_sync(MCE_FULL, t3, 3);
          if (r != rt.r) reg_encode<Word, NR>(a, sm, sl, r, rt);
          u64 nd = 0, cnt = 0;
          reg_tree<Word, NR>(a, sm, sl, rt, P, X, S, h0, h1, nd, cnt);
          nodes += nd;
          root_done(a, r, nd, cnt);
        });
  }
  if (h0) atomicAdd(&a.hist[lane + 2], h0);
  if (h1) atomicAdd(&a.hist[lane + 34], h1);
  if (lane == 0 && nodes) atomicAdd(a.nodes, nodes);  // warp-uniform count
}

// ---------------------------------------------------------------------------
// Wide engine: any d+ <= 2048, rows of W = ceil(d+/64) words in a slab.
// ---------------------------------------------------------------------------
struct MemSmem {
  int32_t off[32];
  int32_t beg[32];
};

struct Slab {
  int32_t *pl;
  u64 *rows, *stk, *xs, *xr, *hash;
  int32_t *xl;
  int hcap;  // hash set entries: a power of two >= 2 * xcap
};

__host__ __device__ __forceinline__ int hash_cap(int xcap) {
  int h = 32;
  while (h < 2 * xcap) h <<= 1;
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
  s.hash = s.xr + (size_t)XC * WM;
  s.hcap = hash_cap(XC);
  s.pl = (int32_t *)(s.hash + (size_t)s.hcap);
  s.xl = s.pl + D;
  return s;
}

struct MemRoot {
  int32_t r = -1;
  int d = 0, Wr = 0, nX = 0;
};

__device__ void mem_encode(const BKArgs &a, MemSmem &sm, const Slab &sl, int32_t r, MemRoot &rt) {
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
  u64 *rows = sl.rows;
  for (int i = lane; i < d; i += 32) pl[i] = a.cs[sb + i];
  for (int i = lane; i < d * Wr; i += 32) rows[i] = 0;
  __syncwarp();
  for (int c = 0; c * 32 < d; ++c) {
    const int items = min(32, d - c * 32);
    int vb = 0, vlen = 0;
    if (lane < items) {
      const int32_t v = pl[c * 32 + lane];
      vb = a.split[v];
      vlen = a.rp[v + 1] - vb;
    }
    const int incl = warp_incl_scan(vlen);
    const int T = __shfl_sync(MCE_FULL, incl, 31);
    sm.off[lane] = incl - vlen;
    sm.beg[lane] = vb;
    __syncwarp();
    for (int e = lane; e < T; e += 32) {
      const int t = chunk_owner(sm.off, e);
      const int32_t w = a.cs[sm.beg[t] + (e - sm.off[t])];
      const int i = lower_bound_g(pl, d, w);
      if (i < d && pl[i] == w) {
        const int j = c * 32 + t;
        atomicOr(&rows[(size_t)j * Wr + (i >> 6)], 1ull << (i & 63));
        atomicOr(&rows[(size_t)i * Wr + (j >> 6)], 1ull << (j & 63));
      }
    }
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
    const int incl = warp_incl_scan(xlen);
    const int T = __shfl_sync(MCE_FULL, incl, 31);
    sm.off[lane] = incl - xlen;
    sm.beg[lane] = xb;
    __syncwarp();
    for (int e = lane; e < T; e += 32) {
      const int t = chunk_owner(sm.off, e);
      const int32_t w = a.cs[sm.beg[t] + (e - sm.off[t])];
      const int i = lower_bound_g(pl, d, w);
      if (i < d && pl[i] == w) atomicOr(&sl.xs[(size_t)t * Wr + (i >> 6)], 1ull << (i & 63));
    }
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
__device__ void mem_tree(const BKArgs &a, const Slab &sl, const MemRoot &rt, u64 &h0, u64 &h1,
                         u64 &nodes, u64 &cnt) {
  const int lane = (int)lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const int d = rt.d, Wr = rt.Wr, nX = rt.nX;
  const u64 *rows = sl.rows;
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
    if (__any_sync(MCE_FULL, el) || pc == 0) return;
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    const int piv = 2047 - (k & 2047);
    if (lane < Wr) F0[2 * Wr + lane] = F0[lane] & ~rows[(size_t)piv * Wr + lane];
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
  int depth = 0, recheck = 0;
  bool want = false;
  for (;;) {
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
    if (lane == 0) {
      Fb[vw] &= ~vbit;
      Fp[vw] &= ~vbit;
      Fx[vw] |= vbit;
    }
    __syncwarp();
    ++nodes;
    u64 *C = F + 4 * Wr;
    int pc = 0;
    bool xnz = false;
    if (lane < Wr) {
      const u64 rw = rows[(size_t)v * Wr + lane];
      const u64 pcw = Fp[lane] & rw, xcw = Fx[lane] & rw;
      C[lane] = pcw;
      C[Wr + lane] = xcw;
      C[3 * Wr + lane] = Fs[lane] | (lane == vw ? vbit : 0ull);
      pc = __popcll(pcw);
      xnz = xcw != 0;
    }
    pc = (int)__reduce_add_sync(MCE_FULL, (unsigned)pc);
    xnz = __any_sync(MCE_FULL, xnz);
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
      if (!xnz) {
        const u64 *Cs = C + 3 * Wr;
        bool covered = false;
        for (int i0 = 0; i0 < nL; i0 += 32) {
          const int i = i0 + lane;
          bool hit = false;
          if (i < nL) {
            const u64 *xrow = sl.xr + (size_t)sl.xl[i] * Wr;
            hit = true;
            for (int w = 0; w < Wr && hit; ++w) hit = (xrow[w] & Cs[w]) == Cs[w];
          }
          if (__any_sync(MCE_FULL, hit)) {
            covered = true;
            break;
          }
        }
        if (!covered) {
          ++cnt;
          const int bin = s_base + depth;  // clique size - 2
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
      }
      continue;
    }
    int k = 0;
    bool el = false;
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
    }
    if (__any_sync(MCE_FULL, el)) continue;
    if (share && pc >= a.donate_min &&
        (nodes >= a.donate_after || (a.policy && a.policy[rt.r])) &&
        (--recheck <= 0 ? (recheck = 32, want = wants_task(a.q)) : want)) {
      const int WM = (a.dcap + 63) >> 6;
      const u64 *Cp = C, *Cx = C + Wr, *Cs = C + 3 * Wr;
      if (q_push(a.q, [&](uint32_t k2) -> u64 {
            if (k2 == 0) return (u64)(uint32_t)rt.r;
            const uint32_t part = (k2 - 1) / WM, w = (k2 - 1) % WM;
            if ((int)w >= Wr) return 0ull;
            return part == 0 ? Cp[w] : part == 1 ? Cx[w] : Cs[w];
          }))
        continue;
      want = false;
    }
    k = (int)__reduce_max_sync(MCE_FULL, (unsigned)k);
    const int up = 2047 - (k & 2047);
    if (lane < Wr) C[2 * Wr + lane] = C[lane] & ~rows[(size_t)up * Wr + lane];
    __syncwarp();
    ++depth;
  }
}

__global__ void __launch_bounds__(MEM_BLOCK) bk_mem_kernel(BKArgs a, int cls) {
  __shared__ MemSmem sm_all[MEM_BLOCK / 32];
  MemSmem &sm = sm_all[threadIdx.x >> 5];
  const int lane = (int)lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const Slab sl = slab_of(a, gw);
  const uint32_t beg = a.shape->cls_off[cls], end = a.shape->cls_off[cls + 1];
  const bool share = a.q.hdr != nullptr;
  u64 h0 = 0, h1 = 0, nodes = 0;
  MemRoot rt;
  if (share && lane == 0) atomicAdd(&a.q.hdr->work, 1u);
  for (;;) {
    uint32_t i0 = 0;
    if (lane == 0) i0 = atomicAdd(&a.fetch[cls], 1u);
    i0 = __shfl_sync(MCE_FULL, i0, 0);
    if (i0 >= end - beg) break;
    const int32_t r = a.roots[beg + i0];
    mem_encode(a, sm, sl, r, rt);
    if (rt.d == 0) continue;
    const int Wr = rt.Wr;
    if (lane < Wr) {  // root frame: P = all of N+(r), X = 0, S = 0
      const u64 all = (lane == Wr - 1 && (rt.d & 63)) ? ((1ull << (rt.d & 63)) - 1ull) : ~0ull;
      sl.stk[lane] = all;
      sl.stk[Wr + lane] = 0;
      sl.stk[3 * Wr + lane] = 0;
    }
    __syncwarp();
    u64 nd = 0, cnt = 0;
    mem_tree(a, sl, rt, h0, h1, nd, cnt);
    nodes += nd;
    root_done(a, r, nd, cnt);
  }
  if (share) {
    if (lane == 0) {
      atomicSub(&a.q.hdr->work, 1u);
      atomicAdd(&a.q.hdr->epoch, 1u);
    }
    const int WM = (a.dcap + 63) >> 6;
    int32_t task_root = -1;
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
          u64 tp = 0, tx = 0, ts = 0;
          if (lane < WM) {
            tp = sl.xs[lane];
            tx = sl.xs[WM + lane];
            ts = sl.xs[2 * WM + lane];
          }
          __syncwarp();
          if (r != rt.r) mem_encode(a, sm, sl, r, rt);
          if (rt.d == 0) return;
          const int Wr = rt.Wr;
          if (lane < Wr) {
            sl.stk[lane] = tp;
            sl.stk[Wr + lane] = tx;
            sl.stk[3 * Wr + lane] = ts;
          }
          __syncwarp();
          u64 nd = 0, cnt = 0;
          mem_tree(a, sl, rt, h0, h1, nd, cnt);
          nodes += nd;
          root_done(a, r, nd, cnt);
        });
  }
  if (h0) atomicAdd(&a.hist[lane + 2], h0);
  if (h1) atomicAdd(&a.hist[lane + 34], h1);
  if (lane == 0 && nodes) atomicAdd(a.nodes, nodes);  // warp-uniform count
}

}  // namespace

size_t bk_slab_words(int cls, int dcap, int xcap) {
  if (cls == CLS_R32 || cls == CLS_R64) return 4 * (size_t)REG_XCAP;  // hash, rows, leaf list
  const size_t WM = (size_t)(dcap + 63) / 64;
  size_t w = (size_t)dcap * WM + (size_t)(dcap + 1) * 4 * WM + 32 * WM + (size_t)xcap * WM;
  w += (size_t)hash_cap(xcap);                      // hash set (one-word rows)
  w += ((size_t)dcap + (size_t)xcap + 1) / 2 + 1;  // pl and xl (int32)
  w = w > 3 * WM + 1 ? w : 3 * WM + 1;
  return (w + 31) & ~(size_t)31;                    // 256-byte aligned slabs
}

uint32_t bk_task_words(int cls, int dcap) {
  if (cls == CLS_R32 || cls == CLS_R64) return 4;
  return 1 + 3 * (uint32_t)((dcap + 63) / 64);
}

int bk_warps_for_class(int cls, int sms, int *warps, int *block, int *smem) {
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
    per_sm = 4;
    *warps = sms * per_sm * (MEM_BLOCK / 32);
  }
  return MCE_OK;
}

int bk_launch(int cls, int word_bits, const BKArgs &a, int grid, int block, int smem,
              cudaStream_t s, int *launches) {
  if (grid <= 0) return MCE_OK;
  switch (cls) {
    case CLS_R32:
      if (word_bits == 64)
        bk_reg_kernel<u64, 1><<<grid, block, smem, s>>>(a, cls);
      else
        bk_reg_kernel<uint32_t, 1><<<grid, block, smem, s>>>(a, cls);
      break;
    case CLS_R64:
      bk_reg_kernel<u64, 2><<<grid, block, smem, s>>>(a, cls);
      break;
    case CLS_MEM:
      bk_mem_kernel<<<grid, block, smem, s>>>(a, cls);
      break;
    default:
      return MCE_EINVAL;
  }
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return MCE_OK;
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
// Set-up: the first call on a device (with that device current) resolves the
// array's device address with cudaGetSymbolAddress and caches it; make that
// first call before any stream capture.  Every call shares the array and
// clears the part that must start at zero, so calls whose work overlaps on
// the GPU race with each other: serialise them (one stream, or events).
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

constexpr int NOALLOC_MAX_DEVICES = 64;
unsigned long long *g_noalloc_addr[NOALLOC_MAX_DEVICES];  // host cache of device addresses
bool g_noalloc_ready[NOALLOC_MAX_DEVICES];

int noalloc_scratch(int dev, unsigned long long **out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return MCE_ELIMIT;
  if (!g_noalloc_ready[dev]) {
    // the host-side name g_noalloc_scratch is not a device address: resolve it
    void *p = nullptr;
    MCE_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = (unsigned long long *)p;
    g_noalloc_ready[dev] = true;
  }
  *out = g_noalloc_addr[dev];
  return MCE_OK;
}

// Every root must fit the 32-wide engine: 1..32 later and <= REG_XCAP
// earlier neighbours.  A root outside those limits sets err[0].
__global__ void noalloc_check_kernel(const int32_t *rp, const int32_t *split,
                                     const int32_t *roots, uint32_t num_roots, NoallocCtl *ctl) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    ctl->shape.cls_off[CLS_R32] = 0;
    ctl->shape.cls_off[CLS_R32 + 1] = num_roots;
  }
  if (i >= num_roots) return;
  const int32_t r = roots[i];
  const int32_t dplus = rp[r + 1] - split[r], dminus = split[r] - rp[r];
  if (dplus < 1 || dplus > 32 || dminus > REG_XCAP) atomicOr(&ctl->err[0], MCE_ERR_DEGREE);
}

}  // namespace

extern "C" int mce_count_oriented_noalloc(const int32_t *d_row_ptr, const int32_t *d_split,
                                          const int32_t *d_col_split, const int32_t *d_roots,
                                          int64_t num_roots, uint64_t *d_hist, void *stream) {
  if (num_roots < 0 || !d_hist ||
      (num_roots > 0 && (!d_row_ptr || !d_split || !d_col_split || !d_roots)))
    return MCE_EINVAL;
  if (num_roots >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  int dev = 0, sms = 0, per_sm = 0;
  MCE_CUDA(cudaGetDevice(&dev));
  unsigned long long *base = nullptr;
  int rc = noalloc_scratch(dev, &base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  NoallocCtl *ctl = (NoallocCtl *)base;
  MCE_CUDA(cudaMemsetAsync(ctl, 0, NOALLOC_CTL_BYTES, s));
  MCE_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(uint64_t) * MCE_HIST_MAX, s));
  const uint32_t nr = (uint32_t)num_roots;
  noalloc_check_kernel<<<(nr + 255) / 256 + 1, 256, 0, s>>>(d_row_ptr, d_split, d_roots, nr, ctl);
  MCE_CUDA(cudaGetLastError());
  uint32_t err = 0;
  MCE_CUDA(cudaMemcpyAsync(&err, &ctl->err[0], sizeof(err), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  if (err) return MCE_ELIMIT;
  if (nr == 0) return MCE_OK;
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
  bk_reg_kernel<uint32_t, 1><<<(unsigned)blocks, REG_BLOCK, 0, s>>>(a, CLS_R32);
  MCE_CUDA(cudaGetLastError());
  MCE_CUDA(cudaMemcpyAsync(&err, &ctl->err[1], sizeof(err), cudaMemcpyDeviceToHost, s));
  MCE_CUDA(cudaStreamSynchronize(s));
  return err ? MCE_ELIMIT : MCE_OK;
}

}  // namespace mce
