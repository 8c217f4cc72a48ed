// Orientation: split every CSR row into [earlier | later] neighbours.
//
// Replaces set_priority / split_pointer / two CUB scans / split_data
// (include/main_support.cuh:6-84, driven from src/main.cu:102-146) and the
// max-degree reductions getNodeDegree_kernel / getSplitDegree_kernel
// (mce/mce.cuh:25-59) with one kernel.  A warp takes ORIENT_ROWS
// consecutive rows at a time and keeps their loads in flight together: one
// load of their offsets and priorities, then the col window of every short
// row (at most 32 arcs), then the prio gather of every such window, so a
// group costs one chain of dependent loads instead of one chain per row.  A
// short row is split in one pass with ballot ranks; a longer row is walked
// twice (count the earlier neighbours, then write; the second read hits
// L1/L2).  The same pass classifies the group's vertices as roots for the
// search engines and writes their sort keys.
//
// Orientation rule (include/main_support.cuh:14): u is later than v iff
// prio[v] == prio[u] ? v < u : prio[v] < prio[u].
#include <cub/cub.cuh>

#include "common.cuh"
#include "kernels.h"

namespace mce {

namespace {

constexpr int ORIENT_BLOCK = 256;
constexpr int ORIENT_WARPS = ORIENT_BLOCK / 32;
constexpr int ORIENT_ROWS = 8;   // rows a warp has in flight
constexpr int ORIENT_FETCH = 4;  // groups a warp takes at a time
// Rows longer than this go to orient_long_kernel (a block per row): one warp
// walking a hub row of 10^5 arcs twice would set the kernel's end.
constexpr int ORIENT_LONG = 512;

__device__ __forceinline__ uint32_t classify(uint32_t dplus, uint32_t dminus) {
  if (dplus == 0) return CLS_NONE;
  if (dplus > MCE_MAX_LATER_DEGREE) return CLS_BIG;
  if (dminus <= (uint32_t)REG_XCAP_MAX) {
    if (dplus <= 32) return CLS_R32;
    if (dplus <= 64) return CLS_R64;
  }
  return CLS_MEM;
}

__device__ __forceinline__ bool is_later(uint32_t pv, int32_t v, uint32_t pu, int32_t u) {
  return pv == pu ? v < u : pv < pu;
}

// A row of more than 32 arcs: count its earlier neighbours, then write
// earlier ones from b and later ones from b + count.  Returns the count.
__device__ int32_t split_long_row(const OrientArgs &a, int32_t v, uint32_t pv, int32_t b,
                                  int32_t e, uint32_t lane) {
  const uint32_t lt = (1u << lane) - 1u;
  int32_t cntE = 0;
  for (int32_t j0 = b; j0 < e; j0 += 32) {
    const int32_t j = j0 + (int32_t)lane;
    bool earlier = false;
    if (j < e) {
      const int32_t u = a.col[j];
      earlier = !is_later(pv, v, a.prio[u], u);
    }
    cntE += __popc(__ballot_sync(MCE_FULL, earlier));
  }
  int32_t eo = b, lo = b + cntE;
  for (int32_t j0 = b; j0 < e; j0 += 32) {
    const int32_t j = j0 + (int32_t)lane;
    const bool valid = j < e;
    bool later = false;
    int32_t u = 0;
    if (valid) {
      u = a.col[j];
      later = is_later(pv, v, a.prio[u], u);
    }
    const uint32_t mL = __ballot_sync(MCE_FULL, valid && later);
    const uint32_t mE = __ballot_sync(MCE_FULL, valid && !later);
    if (valid) a.cs[later ? lo + __popc(mL & lt) : eo + __popc(mE & lt)] = u;
    eo += __popc(mE);
    lo += __popc(mL);
  }
  return cntE;
}

// Vertex v with row [b, e) and cntE earlier neighbours: its split point,
// engine class and sort key, and its entry in the hub list.  Returns the class.
__device__ __forceinline__ uint32_t finish_vertex(const OrientArgs &a, int32_t v, int32_t b,
                                                  int32_t e, int32_t cntE, uint32_t &dplus,
                                                  uint32_t &dminus) {
  const int32_t sp = b + cntE;
  a.split[v] = sp;
  dplus = (uint32_t)(e - sp);
  dminus = (uint32_t)cntE;
  const uint32_t cls = classify(dplus, dminus);
  uint32_t key = cls;
  if (a.cost) {
    float c = a.cost[v];
    c = c < 0.f ? 0.f : (c > 268435455.f ? 268435455.f : c);
    key = (cls << 28) | (0x0FFFFFFFu - (uint32_t)c);
  }
  a.keys_in[v] = key;
  a.vals_in[v] = v;
  if (a.hub_of) {
    int32_t hi = -1;
    if ((cls == CLS_R32 || cls == CLS_R64) && dminus > (uint32_t)HUB_XMIN) {
      hi = (int32_t)atomicAdd(&a.shape->hub_cnt, 1u);
      a.hub_list[hi] = v;
      atomicAdd(&a.shape->hub_rows, (unsigned long long)((dminus + 31u) & ~31u));
      if (cls == CLS_R32) atomicAdd(&a.shape->hub_r32, 1u);
    }
    a.hub_of[v] = hi;
  }
  return cls;
}

__global__ void __launch_bounds__(ORIENT_BLOCK, 6) orient_kernel(OrientArgs a) {
  constexpr int R = ORIENT_ROWS;
  __shared__ uint32_t s_cls[8];
  __shared__ uint32_t s_maxd, s_maxdm, s_maxdeg, s_maxdr;
  if (threadIdx.x < 8) s_cls[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_maxd = s_maxdm = s_maxdeg = s_maxdr = 0;
  __syncthreads();
  const uint32_t lane = lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t groups = (uint32_t)((a.n - a.v0 + R - 1) / R);
  uint32_t ccnt = 0;  // lane c < NCLS: roots of class c seen by this warp
  uint32_t maxd = 0, maxdm = 0, maxdr = 0, maxdeg = 0;
  // groups are fetched ORIENT_FETCH at a time: a warp that meets a long row
  // takes fewer, so the block's warps end together
  uint32_t g0 = 0, gq = ORIENT_FETCH;
  for (;;) {
    if (gq == ORIENT_FETCH) {
      if (lane == 0) g0 = atomicAdd(a.next, (uint32_t)ORIENT_FETCH);
      g0 = __shfl_sync(MCE_FULL, g0, 0);
      gq = 0;
    }
    const uint32_t gi = g0 + gq++;
    if (gi >= groups) break;
    const int64_t vb = a.v0 + (int64_t)gi * R;
    const int rows = a.n - vb < R ? (int)(a.n - vb) : R;
    // lane k <= rows: rp[vb + k]; lane k < rows: prio[vb + k]
    const int32_t ro = (int)lane <= rows ? a.rp[vb + lane] : 0;
    const uint32_t pl = (int)lane < rows ? a.prio[vb + lane] : 0u;
    // lane k + 1 holds row k's end; rows past the group are empty
    auto row_b = [&](int k) { return __shfl_sync(MCE_FULL, ro, k); };
    auto row_e = [&](int k) { return k < rows ? __shfl_sync(MCE_FULL, ro, k + 1) : row_b(k); };
    int32_t U[R];
    uint32_t PU[R];
    // every short row's window, then every window's priorities
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int32_t b = row_b(k), e = row_e(k), j = b + (int32_t)lane;
      U[k] = (e - b <= 32 && j < e) ? a.col[j] : -1;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) PU[k] = U[k] >= 0 ? a.prio[U[k]] : 0u;
    int32_t mycntE = 0;  // lane k: earlier neighbours of row k
#pragma unroll
    for (int k = 0; k < R; ++k) {
      if (k >= rows) break;
      const int32_t v = (int32_t)(vb + k);
      const uint32_t pv = __shfl_sync(MCE_FULL, pl, k);
      const int32_t b = row_b(k), e = row_e(k);
      int32_t cntE;
      if (e - b <= 32) {
        const bool valid = U[k] >= 0;
        const bool later = valid && is_later(pv, v, PU[k], U[k]);
        const uint32_t mL = __ballot_sync(MCE_FULL, later);
        const uint32_t mE = __ballot_sync(MCE_FULL, valid && !later);
        cntE = __popc(mE);
        if (valid) a.cs[later ? b + cntE + __popc(mL & lt) : b + __popc(mE & lt)] = U[k];
      } else if (e - b <= ORIENT_LONG) {
        cntE = split_long_row(a, v, pv, b, e, lane);
      } else {  // left to orient_long_kernel, with its vertex's summary
        cntE = -1;
        if (lane == 0) a.long_list[atomicAdd(a.next + 1, 1u)] = v;
      }
      if ((int)lane == k) mycntE = cntE;
    }
    // the group's vertices, lane k for row k: split point, class, sort key
    const bool has = (int)lane < rows && mycntE >= 0;
    const int32_t e_own = __shfl_down_sync(MCE_FULL, ro, 1);  // rp[vb + lane + 1]
    uint32_t cls = CLS_NONE, dplus = 0, dminus = 0, deg = 0;
    if (has) {
      cls = finish_vertex(a, (int32_t)(vb + lane), ro, e_own, mycntE, dplus, dminus);
      deg = (uint32_t)(e_own - ro);
    }
#pragma unroll
    for (uint32_t c = 0; c < (uint32_t)NCLS; ++c) {
      const uint32_t nc = __popc(__ballot_sync(MCE_FULL, has && cls == c));
      if (lane == c) ccnt += nc;
    }
    maxd = max(maxd, cls != CLS_NONE ? dplus : 0u);
    if (cls == CLS_MEM) maxdm = max(maxdm, dminus);
    if (cls == CLS_R32 || cls == CLS_R64) maxdr = max(maxdr, dminus);
    maxdeg = max(maxdeg, deg);
  }
  if (lane < (uint32_t)NCLS && ccnt) atomicAdd(&s_cls[lane], ccnt);
  maxd = __reduce_max_sync(MCE_FULL, maxd);
  maxdm = __reduce_max_sync(MCE_FULL, maxdm);
  maxdr = __reduce_max_sync(MCE_FULL, maxdr);
  maxdeg = __reduce_max_sync(MCE_FULL, maxdeg);
  if (lane == 0) {
    atomicMax(&s_maxd, maxd);
    atomicMax(&s_maxdm, maxdm);
    atomicMax(&s_maxdr, maxdr);
    atomicMax(&s_maxdeg, maxdeg);
  }
  __syncthreads();
  if (threadIdx.x < NCLS && s_cls[threadIdx.x]) atomicAdd(&a.shape->cls_cnt[threadIdx.x], s_cls[threadIdx.x]);
  if (threadIdx.x == 0) {
    atomicMax(&a.shape->max_dplus, s_maxd);
    atomicMax(&a.shape->max_dminus_mem, s_maxdm);
    atomicMax(&a.shape->max_deg, s_maxdeg);
    atomicMax(&a.shape->max_dminus_reg, s_maxdr);
  }
}

// The rows orient_kernel left (more than ORIENT_LONG arcs), a block per row:
// the block counts the row's earlier neighbours (ORIENT_UNROLL loads in
// flight per thread), then writes the row in tiles of ORIENT_UNROLL x
// ORIENT_BLOCK arcs (ballot ranks within a warp, the warps' counts scanned in
// shared memory, one barrier pair per tile), then settles its vertex's
// summary with global atomics (these rows are few).
constexpr int ORIENT_UNROLL = 4;
__global__ void __launch_bounds__(ORIENT_BLOCK) orient_long_kernel(OrientArgs a) {
  constexpr int U = ORIENT_UNROLL, TILE = U * ORIENT_BLOCK;
  __shared__ int32_t s_e[U][ORIENT_WARPS], s_l[U][ORIENT_WARPS];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t count = *(volatile const uint32_t *)(a.next + 1);
  for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
    const int32_t v = a.long_list[i];
    const int32_t b = a.rp[v], e = a.rp[v + 1];
    const uint32_t pv = a.prio[v];
    int32_t mine = 0;
    for (int32_t t0 = b; t0 < e; t0 += TILE) {
      int32_t u[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int32_t j = t0 + k * ORIENT_BLOCK + (int32_t)threadIdx.x;
        u[k] = j < e ? a.col[j] : -1;
      }
#pragma unroll
      for (int k = 0; k < U; ++k)
        if (u[k] >= 0) mine += !is_later(pv, v, a.prio[u[k]], u[k]);
    }
    mine = (int32_t)__reduce_add_sync(MCE_FULL, (uint32_t)mine);
    if (lane == 0) s_e[0][w] = mine;
    __syncthreads();
    int32_t cntE = 0;
    for (int k = 0; k < ORIENT_WARPS; ++k) cntE += s_e[0][k];
    __syncthreads();
    int32_t eo = b, lo = b + cntE;
    for (int32_t t0 = b; t0 < e; t0 += TILE) {
      int32_t u[U];
      uint32_t mL[U], mE[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int32_t j = t0 + k * ORIENT_BLOCK + (int32_t)threadIdx.x;
        u[k] = j < e ? a.col[j] : -1;
      }
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const bool valid = u[k] >= 0;
        const bool later = valid && is_later(pv, v, a.prio[u[k]], u[k]);
        mL[k] = __ballot_sync(MCE_FULL, later);
        mE[k] = __ballot_sync(MCE_FULL, valid && !later);
        if (lane == 0) {
          s_e[k][w] = __popc(mE[k]);
          s_l[k][w] = __popc(mL[k]);
        }
      }
      __syncthreads();
      // arcs of sub-tile k, warp w come after every (k', w') before them
      int32_t pe = 0, pl = 0;
#pragma unroll
      for (int k = 0; k < U; ++k) {
        for (int ww = 0; ww < ORIENT_WARPS; ++ww) {
          if (ww == (int)w && u[k] >= 0) {
            const bool later = (mL[k] >> lane) & 1u;
            a.cs[later ? lo + pl + __popc(mL[k] & lt) : eo + pe + __popc(mE[k] & lt)] = u[k];
          }
          pe += s_e[k][ww];
          pl += s_l[k][ww];
        }
      }
      eo += pe;
      lo += pl;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      uint32_t dplus, dminus;
      const uint32_t cls = finish_vertex(a, v, b, e, cntE, dplus, dminus);
      atomicAdd(&a.shape->cls_cnt[cls], 1u);
      if (cls != CLS_NONE) atomicMax(&a.shape->max_dplus, dplus);
      if (cls == CLS_MEM) atomicMax(&a.shape->max_dminus_mem, dminus);
      if (cls == CLS_R32 || cls == CLS_R64) atomicMax(&a.shape->max_dminus_reg, dminus);
      atomicMax(&a.shape->max_deg, (uint32_t)(e - b));
    }
  }
}

__global__ void class_offsets_kernel(ShapeInfo *sh) {
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int c = 0; c < NCLS; ++c) {
      sh->cls_off[c] = acc;
      acc += sh->cls_cnt[c];
    }
    for (int c = NCLS; c < 9; ++c) sh->cls_off[c] = acc;
  }
}

}  // namespace

int orient_launch(const OrientArgs &a, cudaStream_t s, int *launches) {
  int dev = 0, sms = 0;
  MCE_CUDA(cudaGetDevice(&dev));
  MCE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (!a.keep_shape) MCE_CUDA(cudaMemsetAsync(a.shape, 0, sizeof(ShapeInfo), s));
  if (a.n <= a.v0) return MCE_OK;
  if (!a.next || !a.long_list) return MCE_EINVAL;
  MCE_CUDA(cudaMemsetAsync(a.next, 0, 2 * sizeof(uint32_t), s));
  const int64_t groups = (a.n - a.v0 + ORIENT_ROWS - 1) / ORIENT_ROWS;  // a warp per group
  int64_t blocks = (groups + ORIENT_WARPS - 1) / ORIENT_WARPS;
  // one wave of resident blocks striding over the groups: a block's warps
  // meet at its final barrier once, not once per wave
  int per_sm = 0;
  MCE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, orient_kernel, ORIENT_BLOCK, 0));
  const int64_t cap = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  if (blocks > cap) blocks = cap;
  orient_kernel<<<(unsigned)blocks, ORIENT_BLOCK, 0, s>>>(a);
  MCE_CUDA(cudaGetLastError());
  // the long rows it left, if any (at most m / ORIENT_LONG of them)
  orient_long_kernel<<<(unsigned)sms * 4, ORIENT_BLOCK, 0, s>>>(a);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 2;
  return MCE_OK;
}

int roots_sort(int64_t n, const uint32_t *keys_in, uint32_t *keys_out, const int32_t *vals_in,
               int32_t *vals_out, int end_bit, void **temp, size_t *temp_bytes,
               ShapeInfo *shape, cudaStream_t s, int *launches) {
  if (n > 0) {
    size_t need = 0;
    MCE_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, keys_in, keys_out, vals_in,
                                             vals_out, (int)n, 0, end_bit, s));
    if (need > *temp_bytes) {
      if (*temp) MCE_CUDA(cudaFree(*temp));
      *temp = nullptr;
      *temp_bytes = 0;
      MCE_CUDA(cudaMalloc(temp, need));
      *temp_bytes = need;
    }
    size_t have = *temp_bytes;
    MCE_CUDA(cub::DeviceRadixSort::SortPairs(*temp, have, keys_in, keys_out, vals_in, vals_out,
                                             (int)n, 0, end_bit, s));
  }
  class_offsets_kernel<<<1, 32, 0, s>>>(shape);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return MCE_OK;
}

}  // namespace mce
