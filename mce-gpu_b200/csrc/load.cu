// .bel loader that builds the CSR on the device.
//
// Replaces graph::read_bel + CSRCOO::from_edgelist (include/fileop.h:81-129,
// include/csrcoo.cuh:41-81) for graphs that are read straight into a device
// handle.  The file is streamed through two pinned staging buffers (the read
// of chunk k+1 overlaps the copy and decode of chunk k); on the device each
// 24-byte record (dst, src, 0) is narrowed to int32 dst (the CSR's column
// array) and src (scratch), then one pass checks the order and builds the
// row offsets from the boundaries between sources.  The same checks as the
// host reader: ids below 2^31, records sorted by (src, dst) without
// duplicates, no self-loops, every destination below n = max src + 1.
#include <sys/stat.h>

#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "kernels.h"

namespace mce {

int graph_adopt(int32_t device, int64_t n, int64_t m, struct ::mce_graph **out, int32_t **rp,
                int32_t **col, int32_t **scratch, cudaStream_t *own);

namespace {

constexpr uint32_t BEL_RANGE = 1u, BEL_ORDER = 2u, BEL_LOOP = 4u, BEL_DST = 8u;
constexpr int64_t BEL_CHUNK = 1 << 21;  // records per staging buffer (48 MiB)

__global__ void bel_decode_kernel(const unsigned long long *__restrict__ raw, int64_t count,
                                  int64_t base, int32_t *__restrict__ src,
                                  int32_t *__restrict__ dst, uint32_t *flags) {
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long d = raw[3 * i], s = raw[3 * i + 1];
    bad |= (s >> 31) != 0 || (d >> 31) != 0;
    src[base + i] = (int32_t)s;
    dst[base + i] = (int32_t)d;
  }
  if (__any_sync(MCE_FULL, bad) && lane_id() == 0) atomicOr(flags, BEL_RANGE);
}

// Checks record i against record i-1 and writes row_ptr[v] = i for every
// vertex v whose row starts at i: src[i-1] < v <= src[i] (v <= n for i = m).
__global__ void bel_rows_kernel(const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                                int64_t m, int64_t n, int32_t *rp, uint32_t *flags) {
  uint32_t f = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t prev = i > 0 ? (int64_t)src[i - 1] : -1;
    int64_t cur = n;
    if (i < m) {
      cur = src[i];
      const int32_t d = dst[i];
      if (cur == d) f |= BEL_LOOP;
      if (d >= n) f |= BEL_DST;
      if (i > 0 && (cur < prev || (cur == prev && d <= dst[i - 1]))) f |= BEL_ORDER;
    }
    for (int64_t v = prev + 1; v <= cur && v <= n; ++v) rp[v] = (int32_t)i;
  }
  const unsigned fw = __reduce_or_sync(MCE_FULL, f);
  if (fw && lane_id() == 0) atomicOr(flags, fw);
}

}  // namespace
}  // namespace mce

using namespace mce;

extern "C" int mce_bel_load(const char *path, int32_t device, void *stream, mce_graph_t *out) {
  if (!path || !out) return MCE_EINVAL;
  *out = nullptr;
  struct stat st;
  if (stat(path, &st) != 0) return MCE_EIO;
  if (st.st_size % 24 != 0) return MCE_EFORMAT;
  const int64_t m = (int64_t)(st.st_size / 24);
  if (m >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return MCE_EIO;
  int64_t n = 0;
  if (m > 0) {  // n = max src + 1 = the last record's src (rows are sorted; checked below)
    unsigned long long last[3];
    if (std::fseek(fp, (long)(st.st_size - 24), SEEK_SET) != 0 || std::fread(last, 24, 1, fp) != 1 ||
        std::fseek(fp, 0, SEEK_SET) != 0) {
      std::fclose(fp);
      return MCE_EIO;
    }
    if (last[1] >> 31) {
      std::fclose(fp);
      return MCE_EFORMAT;
    }
    n = (int64_t)last[1] + 1;
  }
  mce_graph *g = nullptr;
  int32_t *rp = nullptr, *col = nullptr, *src = nullptr;
  cudaStream_t own = nullptr;
  int rc = graph_adopt(device, n, m, &g, &rp, &col, &src, &own);
  if (rc) {
    std::fclose(fp);
    return rc;
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : own;
  const int64_t chunk = m < BEL_CHUNK ? (m > 0 ? m : 1) : BEL_CHUNK;
  unsigned long long *host[2] = {nullptr, nullptr}, *raw[2] = {nullptr, nullptr};
  uint32_t *flags = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int sms = 0;
  auto cleanup = [&]() {
    for (int b = 0; b < 2; ++b) {
      if (host[b]) cudaFreeHost(host[b]);
      if (raw[b]) cudaFree(raw[b]);
      if (ev[b]) cudaEventDestroy(ev[b]);
    }
    if (flags) cudaFree(flags);
    std::fclose(fp);
  };
  for (int b = 0; b < 2 && rc == MCE_OK; ++b)
    if (cudaHostAlloc((void **)&host[b], 24 * (size_t)chunk, cudaHostAllocDefault) != cudaSuccess ||
        cudaMalloc((void **)&raw[b], 24 * (size_t)chunk) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming) != cudaSuccess)
      rc = MCE_ENOMEM;
  if (rc == MCE_OK && (cudaMalloc((void **)&flags, 4) != cudaSuccess ||
                       cudaMemsetAsync(flags, 0, 4, s) != cudaSuccess ||
                       cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) !=
                           cudaSuccess))
    rc = MCE_ECUDA;
  for (int64_t base = 0, k = 0; rc == MCE_OK && base < m; base += chunk, ++k) {
    const int b = (int)(k & 1);
    const int64_t cnt = m - base < chunk ? m - base : chunk;
    if (k >= 2 && cudaEventSynchronize(ev[b]) != cudaSuccess) {  // buffer b is free again
      rc = MCE_ECUDA;
      break;
    }
    if (std::fread(host[b], 24, (size_t)cnt, fp) != (size_t)cnt) {
      rc = MCE_EIO;
      break;
    }
    if (cudaMemcpyAsync(raw[b], host[b], 24 * (size_t)cnt, cudaMemcpyHostToDevice, s) !=
        cudaSuccess) {
      rc = MCE_ECUDA;
      break;
    }
    bel_decode_kernel<<<sms * 4, 256, 0, s>>>(raw[b], cnt, base, src, col, flags);
    if (cudaGetLastError() != cudaSuccess || cudaEventRecord(ev[b], s) != cudaSuccess)
      rc = MCE_ECUDA;
  }
  uint32_t fl = 0;
  if (rc == MCE_OK) {
    bel_rows_kernel<<<sms * 4, 256, 0, s>>>(src, col, m, n, rp, flags);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&fl, flags, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      rc = MCE_ECUDA;
  }
  if (rc == MCE_OK && fl) rc = MCE_EFORMAT;
  cleanup();
  if (rc) {
    mce_graph_free(g);
    return rc;
  }
  *out = g;
  return MCE_OK;
}
