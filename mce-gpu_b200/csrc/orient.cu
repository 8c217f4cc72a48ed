// Orientation: split every CSR row into [earlier | later] neighbours.
//
// Replaces set_priority / split_pointer / two CUB scans / split_data
// (include/main_support.cuh:6-84, driven from src/main.cu:102-146) and the
// max-degree reductions getNodeDegree_kernel / getSplitDegree_kernel
// (mce/mce.cuh:25-59) with one kernel: a warp owns a row, reads it twice
// (the second pass hits L2) and writes each neighbour once, compacting with
// ballot ranks instead of a block-wide scan.  The same pass classifies the
// row's vertex as a root for one of the search engines and writes its sort
// key, so no separate pass over the vertices is needed.
//
// Orientation rule (include/main_support.cuh:14): u is later than v iff
// prio[v] == prio[u] ? v < u : prio[v] < prio[u].
#include <cub/cub.cuh>

#include "common.cuh"
#include "kernels.h"

namespace mce {

namespace {

constexpr int ORIENT_BLOCK = 256;

__device__ __forceinline__ uint32_t classify(uint32_t dplus, uint32_t dminus) {
  if (dplus == 0) return CLS_NONE;
  if (dplus > MCE_MAX_LATER_DEGREE) return CLS_BIG;
  if (dminus <= (uint32_t)REG_XCAP_MAX) {
    if (dplus <= 32) return CLS_R32;
    if (dplus <= 64) return CLS_R64;
  }
  return CLS_MEM;
}

__global__ void __launch_bounds__(ORIENT_BLOCK) orient_kernel(OrientArgs a) {
  __shared__ uint32_t s_cls[8];
  __shared__ uint32_t s_maxd, s_maxdm, s_maxdeg, s_maxdr;
  if (threadIdx.x < 8) s_cls[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_maxd = s_maxdm = s_maxdeg = s_maxdr = 0;
  __syncthreads();
  const uint32_t lane = lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t vv = a.v0 + gwarp; vv < a.n; vv += nwarps) {
    const int32_t v = (int32_t)vv;
    const int32_t b = a.rp[v], e = a.rp[v + 1];
    const uint32_t pv = a.prio[v];
    int32_t cntE = 0;
    if (e - b <= 32) {  // the whole row in one window: one gather, one pass
      const int32_t j = b + (int32_t)lane;
      const bool valid = j < e;
      bool later = false;
      int32_t u = 0;
      if (valid) {
        u = a.col[j];
        const uint32_t pu = a.prio[u];
        later = pv == pu ? v < u : pv < pu;
      }
      const uint32_t mL = __ballot_sync(MCE_FULL, valid && later);
      const uint32_t mE = __ballot_sync(MCE_FULL, valid && !later);
      cntE = __popc(mE);
      if (valid) a.cs[later ? b + cntE + __popc(mL & lt) : b + __popc(mE & lt)] = u;
    } else {
      for (int32_t j0 = b; j0 < e; j0 += 32) {
        const int32_t j = j0 + (int32_t)lane;
        bool earlier = false;
        if (j < e) {
          const int32_t u = a.col[j];
          const uint32_t pu = a.prio[u];
          earlier = !(pv == pu ? v < u : pv < pu);
        }
        cntE += __popc(__ballot_sync(MCE_FULL, earlier));
      }
      int32_t eo = b, lo = b + cntE;
      for (int32_t j0 = b; j0 < e; j0 += 32) {
        const int32_t j = j0 + (int32_t)lane;
        bool later = false, valid = j < e;
        int32_t u = 0;
        if (valid) {
          u = a.col[j];
          const uint32_t pu = a.prio[u];
          later = pv == pu ? v < u : pv < pu;
        }
        const uint32_t mL = __ballot_sync(MCE_FULL, valid && later);
        const uint32_t mE = __ballot_sync(MCE_FULL, valid && !later);
        if (valid) {
          if (later)
            a.cs[lo + __popc(mL & lt)] = u;
          else
            a.cs[eo + __popc(mE & lt)] = u;
        }
        eo += __popc(mE);
        lo += __popc(mL);
      }
    }
    const int32_t sp = b + cntE;
    if (lane == 0) {
      a.split[v] = sp;
      const uint32_t dplus = (uint32_t)(e - sp), dminus = (uint32_t)cntE;
      const uint32_t cls = classify(dplus, dminus);
      uint32_t key = cls;
      if (a.cost) {
        float c = a.cost[v];
        c = c < 0.f ? 0.f : (c > 268435455.f ? 268435455.f : c);
        key = (cls << 28) | (0x0FFFFFFFu - (uint32_t)c);
      }
      a.keys_in[v] = key;
      a.vals_in[v] = v;
      atomicAdd(&s_cls[cls], 1u);
      if (cls != CLS_NONE) atomicMax(&s_maxd, dplus);
      if (cls == CLS_MEM) atomicMax(&s_maxdm, dminus);
      if (cls == CLS_R32 || cls == CLS_R64) atomicMax(&s_maxdr, dminus);
      if (a.hub_of) {
        int32_t hi = -1;
        if ((cls == CLS_R32 || cls == CLS_R64) && dminus > (uint32_t)HUB_XMIN) {
          hi = (int32_t)atomicAdd(&a.shape->hub_cnt, 1u);
          a.hub_list[hi] = v;
          atomicAdd(&a.shape->hub_rows, (unsigned long long)((dminus + 31u) & ~31u));
        }
        a.hub_of[v] = hi;
      }
      atomicMax(&s_maxdeg, (uint32_t)(e - b));
    }
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
  const int64_t warps_needed = a.n - a.v0;
  int64_t blocks = (warps_needed + (ORIENT_BLOCK / 32) - 1) / (ORIENT_BLOCK / 32);
  const int64_t cap = (int64_t)sms * 8 * 4;  // enough resident warps to cover latency
  if (blocks > cap) blocks = cap;
  orient_kernel<<<(unsigned)blocks, ORIENT_BLOCK, 0, s>>>(a);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
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
