// Shared device/host helpers for the B200 kernels of libmce.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mce.h"

#define MCE_FULL 0xFFFFFFFFu

// Status bits the kernels set in a device word the host reads after a call.
#define MCE_ERR_WAIT_TIMEOUT 0x1u   // a bounded wait (grid barrier, queue) ran out
#define MCE_ERR_DEPTH 0x2u          // search depth above the stack capacity
#define MCE_ERR_XROWS 0x4u          // earlier-neighbour rows above the slab capacity
#define MCE_ERR_DEGREE 0x8u         // later degree above the engine's width
#define MCE_ERR_QUEUE 0x10u         // task queue misuse
#define MCE_ERR_BUDGET 0x20u        // a search passed its node budget (serving)
#define MCE_ERR_ARCS 0x40u          // an ego graph above the arena's arc capacity (serving)

// Check a CUDA call; on failure record it and return MCE_ECUDA from the caller.
#define MCE_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      mce::set_last_cuda_error(e_, #call, __FILE__, __LINE__);                \
      return e_ == cudaErrorMemoryAllocation ? MCE_ENOMEM : MCE_ECUDA;        \
    }                                                                         \
  } while (0)

namespace mce {

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);

// nanoseconds since an arbitrary epoch (the GPU's global timer)
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) {
  return *(const volatile uint32_t *)p;
}

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}

// Grid-wide barrier for a kernel whose blocks are all resident (launched with
// cudaLaunchCooperativeKernel, which refuses a grid that cannot be).  Bounded:
// if the other blocks do not arrive within `limit_ns`, the flag `err` gets
// MCE_ERR_WAIT_TIMEOUT and the function returns false so the caller can stop.
struct GridBarrier {
  uint32_t count;
  uint32_t gen;
};

__device__ __forceinline__ bool grid_sync(GridBarrier *b, uint32_t nblocks, uint32_t *err,
                                          uint64_t limit_ns) {
  __syncthreads();
  __shared__ uint32_t ok;
  if (threadIdx.x == 0) {
    ok = 1;
    const uint32_t g = ld_volatile(&b->gen);
    __threadfence();
    const uint32_t arrived = atomicAdd(&b->count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      const uint64_t t0 = globaltimer_ns();
      uint32_t ns = 32;
      while (ld_volatile(&b->gen) == g) {
        if (ld_volatile(err) & MCE_ERR_WAIT_TIMEOUT) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > limit_ns) {
          atomicOr(err, MCE_ERR_WAIT_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// ---- 1-D bulk copies global -> shared through an mbarrier (the TMA unit's
// untiled form; no multicast, this GPU's memory only).  Source, destination
// and size must be multiples of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t arrivals) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic accesses of shared memory before its
// later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// One probe of the phase with parity `parity`: true once it has completed.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase: false (and MCE_ERR_WAIT_TIMEOUT in *err) if
// it has not completed within limit_ns.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity, uint32_t *err,
                                          uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > limit_ns) {
      atomicOr(err, MCE_ERR_WAIT_TIMEOUT);
      return false;
    }
  }
  return true;
}

// Binary search in a sorted int array: index of key in [lo, hi) or -1.
__device__ __forceinline__ int32_t bsearch_idx(const int32_t *a, int32_t lo, int32_t hi,
                                               int32_t key) {
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    const int32_t v = a[mid];
    if (v == key) return mid;
    if (v < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return -1;
}

// Branch-free lower bound over a small sorted array (length n <= 2^k).
__device__ __forceinline__ int32_t lower_bound_small(const int32_t *a, int32_t n, int32_t key) {
  int32_t lo = 0, len = n;
  while (len > 0) {
    const int32_t half = len >> 1;
    const bool right = a[lo + half] < key;
    lo = right ? lo + half + 1 : lo;
    len = right ? len - half - 1 : half;
  }
  return lo;
}

}  // namespace mce
