// Text edge list -> sorted, deduplicated arcs on the device.
//
// Replaces graph::convert_to_bel (include/fileop.h:13-79), which reads the
// text with fscanf/sscanf, pushes both directions of every edge into a
// std::vector, sorts it on one host thread and writes the .bel records.
// Here the file streams through two pinned staging buffers into one device
// buffer; one thread per 16-byte segment finds the line starts in its
// segment (a byte after '\n', or offset 0) and parses every line that starts
// with a digit the way sscanf("%llu %llu") does; a line yields an edge when
// both numbers parse and differ.  A count pass sizes the arc array exactly,
// an emit pass appends the arcs (both directions, ids narrowed to 32 bits as
// T(src) does in the reference), a radix sort over only the key bits in use
// and a unique pass give the .bel order.  The result is either written as a
// .bel file (24-byte records dst, src, 0, through two pinned buffers) or
// turned into a device CSR in place of mce_bel_load.
//
// Line semantics shared with the host converter (host/bel.cpp): the parse
// sees at most the first 65,535 bytes of a line (its fgets buffer); '\n'
// ends a line and a NUL byte ends its parse; an empty line is skipped.
// Number syntax follows strtoull, which sscanf's %llu uses: optional sign,
// decimal digits, ULLONG_MAX on overflow, a '-' negates modulo 2^64.
#include <sys/stat.h>

#include <cooperative_groups.h>
#include <cub/cub.cuh>
#include <cstdio>

#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace mce {

int graph_adopt(int32_t device, int64_t n, int64_t m, struct ::mce_graph **out, int32_t **rp,
                int32_t **col, int32_t **scratch, cudaStream_t *own);

namespace {

constexpr int64_t TX_CHUNK = 64ll << 20;    // text bytes per staging buffer
constexpr int64_t TX_LINE_MAX = 65535;      // bytes of a line the parse reads
constexpr int64_t TX_REC_CHUNK = 1ll << 21;  // .bel records per output buffer (48 MiB)

struct TxCtl {
  unsigned long long edges;     // lines that gave an edge
  unsigned long long max_id;    // max over both numbers, before narrowing
  uint32_t max_id32;            // max over both numbers, after narrowing
  uint32_t loops;               // CSR build: arcs whose narrowed ends are equal
  unsigned long long emitted;   // arcs written by the emit pass
};

__device__ __forceinline__ bool tx_digit(uint32_t c) { return c - '0' < 10u; }
// isspace() in the C locale without '\n', which ends the line
__device__ __forceinline__ bool tx_space(uint32_t c) {
  return c == ' ' || c == '\t' || c == '\v' || c == '\f' || c == '\r';
}

// One %llu conversion at t[p..lim): leading blanks, optional sign, decimal
// digits.  Returns false (no conversion) when no digit follows.
__device__ bool tx_number(const uint8_t *__restrict__ t, int64_t &p, int64_t lim,
                          unsigned long long &v) {
  while (p < lim && tx_space(t[p])) ++p;
  bool neg = false;
  if (p < lim && (t[p] == '+' || t[p] == '-')) {
    neg = t[p] == '-';
    ++p;
  }
  if (p >= lim || !tx_digit(t[p])) return false;
  unsigned long long x = 0;
  bool over = false;
  for (; p < lim && tx_digit(t[p]); ++p) {
    const unsigned dig = t[p] - '0';
    if (x > (~0ull - dig) / 10ull) over = true;
    else if (!over) x = x * 10ull + dig;
  }
  v = over ? ~0ull : (neg ? 0ull - x : x);
  return true;
}

// sscanf(line, "%llu %llu", &s, &d) == 2 && s != d for the line at p
__device__ __forceinline__ bool tx_edge(const uint8_t *__restrict__ t, int64_t p, int64_t size,
                                        unsigned long long &s, unsigned long long &d) {
  const int64_t lim = min(size, p + TX_LINE_MAX);
  return tx_number(t, p, lim, s) && tx_number(t, p, lim, d) && s != d;
}

// bit j set: offset 16*seg + j starts a line and holds a digit
__device__ __forceinline__ uint32_t tx_starts(const uint8_t *__restrict__ t, int64_t seg,
                                              int64_t size) {
  const uint4 w = reinterpret_cast<const uint4 *>(t)[seg];
  const uint32_t words[4] = {w.x, w.y, w.z, w.w};
  uint32_t prev = seg ? t[16 * seg - 1] : '\n';
  uint32_t mask = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t c = (words[j >> 2] >> (8 * (j & 3))) & 0xffu;
    if (prev == '\n' && tx_digit(c)) mask |= 1u << j;
    prev = c;
  }
  const int64_t left = size - 16 * seg;  // bytes of the segment inside the file
  if (left < 16) mask &= (1u << left) - 1u;
  return mask;
}

__global__ void tx_count_kernel(const uint8_t *__restrict__ t, int64_t size, TxCtl *ctl) {
  unsigned long long cnt = 0, mx = 0;
  uint32_t mx32 = 0;
  const int64_t nseg = (size + 15) / 16;
  for (int64_t seg = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; seg < nseg;
       seg += (int64_t)gridDim.x * blockDim.x) {
    for (uint32_t mask = tx_starts(t, seg, size); mask; mask &= mask - 1) {
      unsigned long long s, d;
      if (tx_edge(t, 16 * seg + __ffs(mask) - 1, size, s, d)) {
        ++cnt;
        mx = max(mx, max(s, d));
        mx32 = max(mx32, max((uint32_t)s, (uint32_t)d));
      }
    }
  }
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(MCE_FULL, cnt, o);
    mx = max(mx, __shfl_xor_sync(MCE_FULL, mx, o));
  }
  mx32 = __reduce_max_sync(MCE_FULL, mx32);
  if (lane_id() == 0 && cnt) {
    atomicAdd(&ctl->edges, cnt);
    atomicMax(&ctl->max_id, mx);
    atomicMax(&ctl->max_id32, mx32);
  }
}

// Appends both arcs of every edge as (src << b) | dst; the order of the
// appends does not matter (a sort follows).  `cap` bounds the writes.
__global__ void tx_emit_kernel(const uint8_t *__restrict__ t, int64_t size, int b,
                               unsigned long long *__restrict__ keys, unsigned long long cap,
                               TxCtl *ctl) {
  const int64_t nseg = (size + 15) / 16;
  for (int64_t seg = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; seg < nseg;
       seg += (int64_t)gridDim.x * blockDim.x) {
    for (uint32_t mask = tx_starts(t, seg, size); mask; mask &= mask - 1) {
      unsigned long long s, d;
      if (!tx_edge(t, 16 * seg + __ffs(mask) - 1, size, s, d)) continue;
      cg::coalesced_group grp = cg::coalesced_threads();
      unsigned long long base = 0;
      if (grp.thread_rank() == 0) base = atomicAdd(&ctl->emitted, 2ull * grp.size());
      base = grp.shfl(base, 0) + 2ull * grp.thread_rank();
      const unsigned long long s32 = (uint32_t)s, d32 = (uint32_t)d;
      if (base + 1 < cap) {
        keys[base] = (s32 << b) | d32;
        keys[base + 1] = (d32 << b) | s32;
      }
    }
  }
}

// .bel records (dst, src, 0) of keys[base, base + cnt)
__global__ void tx_records_kernel(const unsigned long long *__restrict__ keys, int64_t base,
                                  int64_t cnt, int b, unsigned long long *__restrict__ rec) {
  const unsigned long long lo = (1ull << b) - 1ull;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[base + i];
    rec[3 * i] = k & lo;
    rec[3 * i + 1] = k >> b;
    rec[3 * i + 2] = 0;
  }
}

// CSR of the sorted unique keys: col[i] = dst, row_ptr[v] = first arc of v.
// Two ids that differ only above bit 31 narrow to a self-loop, which the
// .bel reader rejects; it is counted in ctl->loops.
__global__ void tx_csr_kernel(const unsigned long long *__restrict__ keys, int64_t m, int64_t n,
                              int b, int32_t *__restrict__ rp, int32_t *__restrict__ col,
                              TxCtl *ctl) {
  const unsigned long long lo = (1ull << b) - 1ull;
  bool loop = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t prev = i > 0 ? (int64_t)(keys[i - 1] >> b) : -1;
    int64_t cur = n;
    if (i < m) {
      cur = (int64_t)(keys[i] >> b);
      col[i] = (int32_t)(keys[i] & lo);
      loop |= (keys[i] & lo) == (unsigned long long)cur;
    }
    for (int64_t v = prev + 1; v <= cur && v <= n; ++v) rp[v] = (int32_t)i;
  }
  if (__any_sync(MCE_FULL, loop) && lane_id() == 0) atomicAdd(&ctl->loops, 1u);
}

// Device buffers and staging of one conversion; the destructor waits for
// the stream and frees them, on every exit path.
struct TxRun {
  int sms = 0;
  cudaStream_t s = nullptr, own = nullptr;
  uint8_t *text = nullptr;
  unsigned long long *keys[2] = {nullptr, nullptr}, *rec = nullptr;
  void *temp = nullptr;
  TxCtl *ctl = nullptr;
  int64_t *nsel = nullptr;
  void *host[2] = {nullptr, nullptr};
  size_t host_bytes = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~TxRun() {
    if (s) cudaStreamSynchronize(s);
    cudaFree(text);
    cudaFree(keys[0]);
    cudaFree(keys[1]);
    cudaFree(rec);
    cudaFree(temp);
    cudaFree(ctl);
    cudaFree(nsel);
    for (int i = 0; i < 2; ++i) {
      if (host[i]) cudaFreeHost(host[i]);
      if (ev[i]) cudaEventDestroy(ev[i]);
    }
    if (own) cudaStreamDestroy(own);
  }
};

// two pinned buffers of at least `bytes` (the stream is idle when they grow)
int tx_staging(TxRun &r, size_t bytes) {
  if (r.host_bytes < bytes) {
    MCE_CUDA(cudaStreamSynchronize(r.s));
    for (int i = 0; i < 2; ++i) {
      if (r.host[i]) cudaFreeHost(r.host[i]);
      r.host[i] = nullptr;
    }
    r.host_bytes = 0;
    for (int i = 0; i < 2; ++i) MCE_CUDA(cudaHostAlloc(&r.host[i], bytes, cudaHostAllocDefault));
    r.host_bytes = bytes;
  }
  for (int i = 0; i < 2; ++i)
    if (!r.ev[i]) MCE_CUDA(cudaEventCreateWithFlags(&r.ev[i], cudaEventDisableTiming));
  return MCE_OK;
}

// Reads the text into r.text (zero-padded to 16 bytes) and leaves the
// sorted unique keys in *keys_out; *m_out arcs, b bits per id.
int tx_arcs(TxRun &r, const char *path, unsigned long long **keys_out, int64_t *m_out, int *b_out,
            TxCtl *ctl_out) {
  struct stat st;
  if (stat(path, &st) != 0) return MCE_EIO;
  const int64_t size = (int64_t)st.st_size;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return MCE_EIO;
  const int64_t padded = (size + 16) / 16 * 16;  // at least one zero byte after the text
  int rc = MCE_OK;
  auto fail = [&](int code) {
    std::fclose(fp);
    return code;
  };
  if (cudaMalloc(&r.text, (size_t)padded) != cudaSuccess) return fail(MCE_ENOMEM);
  if (cudaMemsetAsync(r.text + (padded - 16), 0, 16, r.s) != cudaSuccess) return fail(MCE_ECUDA);
  const int64_t chunk = size < TX_CHUNK ? (size > 0 ? size : 1) : TX_CHUNK;
  if ((rc = tx_staging(r, (size_t)chunk))) return fail(rc);
  for (int64_t base = 0, k = 0; base < size; base += chunk, ++k) {
    const int b = (int)(k & 1);
    const int64_t cnt = size - base < chunk ? size - base : chunk;
    if (k >= 2 && cudaEventSynchronize(r.ev[b]) != cudaSuccess) return fail(MCE_ECUDA);
    if (std::fread(r.host[b], 1, (size_t)cnt, fp) != (size_t)cnt) return fail(MCE_EIO);
    if (cudaMemcpyAsync(r.text + base, r.host[b], (size_t)cnt, cudaMemcpyHostToDevice, r.s) !=
            cudaSuccess ||
        cudaEventRecord(r.ev[b], r.s) != cudaSuccess)
      return fail(MCE_ECUDA);
  }
  std::fclose(fp);
  MCE_CUDA(cudaMalloc(&r.ctl, sizeof(TxCtl)));
  MCE_CUDA(cudaMemsetAsync(r.ctl, 0, sizeof(TxCtl), r.s));
  const int grid = r.sms * 8;
  tx_count_kernel<<<grid, 256, 0, r.s>>>(r.text, size, r.ctl);
  MCE_CUDA(cudaGetLastError());
  TxCtl h;
  MCE_CUDA(cudaMemcpyAsync(&h, r.ctl, sizeof(TxCtl), cudaMemcpyDeviceToHost, r.s));
  MCE_CUDA(cudaStreamSynchronize(r.s));
  *ctl_out = h;
  const int64_t arcs = 2 * (int64_t)h.edges;
  const int b = h.max_id32 ? 32 - __builtin_clz(h.max_id32) : 1;
  *b_out = b;
  if (arcs == 0) {
    *keys_out = nullptr;
    *m_out = 0;
    return MCE_OK;
  }
  for (int i = 0; i < 2; ++i)
    if (cudaMalloc(&r.keys[i], (size_t)arcs * 8) != cudaSuccess) return MCE_ENOMEM;
  tx_emit_kernel<<<grid, 256, 0, r.s>>>(r.text, size, b, r.keys[0], (unsigned long long)arcs,
                                        r.ctl);
  MCE_CUDA(cudaGetLastError());
  TxCtl h2;
  MCE_CUDA(cudaMemcpyAsync(&h2, r.ctl, sizeof(TxCtl), cudaMemcpyDeviceToHost, r.s));
  MCE_CUDA(cudaStreamSynchronize(r.s));
  if ((int64_t)h2.emitted != arcs) return MCE_ESTATE;  // the two passes disagree
  MCE_CUDA(cudaFree(r.text));
  r.text = nullptr;
  cub::DoubleBuffer<unsigned long long> db(r.keys[0], r.keys[1]);
  size_t sort_bytes = 0, uniq_bytes = 0;
  MCE_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, db, arcs, 0, 2 * b, r.s));
  MCE_CUDA(cub::DeviceSelect::Unique(nullptr, uniq_bytes, r.keys[0], r.keys[1], (int64_t *)nullptr,
                                     arcs, r.s));
  MCE_CUDA(cudaMalloc(&r.temp, sort_bytes > uniq_bytes ? sort_bytes : uniq_bytes));
  MCE_CUDA(cudaMalloc(&r.nsel, sizeof(int64_t)));
  MCE_CUDA(cub::DeviceRadixSort::SortKeys(r.temp, sort_bytes, db, arcs, 0, 2 * b, r.s));
  unsigned long long *sorted = db.Current(), *uniq = db.Alternate();
  MCE_CUDA(cub::DeviceSelect::Unique(r.temp, uniq_bytes, sorted, uniq, r.nsel, arcs, r.s));
  int64_t m = 0;
  MCE_CUDA(cudaMemcpyAsync(&m, r.nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, r.s));
  MCE_CUDA(cudaStreamSynchronize(r.s));
  *keys_out = uniq;
  *m_out = m;
  return MCE_OK;
}

// the caller's stream, or a stream of the run's own
int tx_begin(TxRun &r, int32_t device, void *stream) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return MCE_ENODEV;
  if (device < 0 || device >= count) return MCE_EINVAL;
  MCE_CUDA(cudaSetDevice(device));
  MCE_CUDA(cudaDeviceGetAttribute(&r.sms, cudaDevAttrMultiProcessorCount, device));
  if (stream) {
    r.s = (cudaStream_t)stream;
  } else {
    MCE_CUDA(cudaStreamCreateWithFlags(&r.own, cudaStreamNonBlocking));
    r.s = r.own;
  }
  return MCE_OK;
}

// .bel records of keys[0, m) into an open file; chunk k+1 is decoded and
// copied while the host writes chunk k
int tx_write_bel(TxRun &r, const unsigned long long *keys, int64_t m, int b, FILE *w) {
  if (m == 0) return MCE_OK;
  const int64_t chunk = m < TX_REC_CHUNK ? m : TX_REC_CHUNK;
  int rc = tx_staging(r, 24 * (size_t)chunk);
  if (rc) return rc;
  MCE_CUDA(cudaMalloc(&r.rec, 24 * (size_t)chunk));
  const int64_t nchunks = (m + chunk - 1) / chunk;
  auto count_of = [&](int64_t k) { return m - k * chunk < chunk ? m - k * chunk : chunk; };
  auto enqueue = [&](int64_t k) -> int {
    const int64_t cnt = count_of(k);
    tx_records_kernel<<<r.sms * 4, 256, 0, r.s>>>(keys, k * chunk, cnt, b, r.rec);
    MCE_CUDA(cudaGetLastError());
    MCE_CUDA(cudaMemcpyAsync(r.host[k & 1], r.rec, 24 * (size_t)cnt, cudaMemcpyDeviceToHost, r.s));
    MCE_CUDA(cudaEventRecord(r.ev[k & 1], r.s));
    return MCE_OK;
  };
  if ((rc = enqueue(0))) return rc;
  for (int64_t k = 0; k < nchunks; ++k) {
    if (k + 1 < nchunks && (rc = enqueue(k + 1))) return rc;
    MCE_CUDA(cudaEventSynchronize(r.ev[k & 1]));
    const size_t cnt = (size_t)count_of(k);
    if (std::fwrite(r.host[k & 1], 24, cnt, w) != cnt) return MCE_EIO;
  }
  return MCE_OK;
}

}  // namespace
}  // namespace mce

using namespace mce;

extern "C" int mce_convert_to_bel_device(const char *txt_path, const char *bel_path,
                                         int32_t device, void *stream, int64_t *n_out,
                                         int64_t *undirected_edges_out) {
  if (!txt_path || !bel_path) return MCE_EINVAL;
  TxRun r;
  int rc = tx_begin(r, device, stream);
  if (rc) return rc;
  unsigned long long *keys = nullptr;
  int64_t m = 0;
  int b = 1;
  TxCtl ctl;
  if ((rc = tx_arcs(r, txt_path, &keys, &m, &b, &ctl))) return rc;
  FILE *w = std::fopen(bel_path, "wb");
  if (!w) return MCE_EIO;
  rc = tx_write_bel(r, keys, m, b, w);
  if (std::fclose(w) != 0 && rc == MCE_OK) rc = MCE_EIO;
  if (rc) return rc;
  // the two numbers graph::convert_to_bel prints (include/fileop.h:78)
  if (n_out) *n_out = ctl.edges ? (int64_t)(ctl.max_id + 1ull) : 1;
  if (undirected_edges_out) *undirected_edges_out = m / 2;
  return MCE_OK;
}

extern "C" int mce_text_load(const char *txt_path, int32_t device, void *stream,
                             mce_graph_t *out) {
  if (!txt_path || !out) return MCE_EINVAL;
  *out = nullptr;
  TxRun r;
  int rc = tx_begin(r, device, stream);
  if (rc) return rc;
  unsigned long long *keys = nullptr;
  int64_t m = 0;
  int b = 1;
  TxCtl ctl;
  if ((rc = tx_arcs(r, txt_path, &keys, &m, &b, &ctl))) return rc;
  int64_t n = 0;
  if (m > 0) {
    unsigned long long last = 0;
    MCE_CUDA(cudaMemcpyAsync(&last, keys + (m - 1), 8, cudaMemcpyDeviceToHost, r.s));
    MCE_CUDA(cudaStreamSynchronize(r.s));
    n = (int64_t)(last >> b) + 1;  // max source + 1, as the .bel reader sets it
  }
  mce_graph *g = nullptr;
  int32_t *rp = nullptr, *col = nullptr, *scratch = nullptr;
  cudaStream_t gs = nullptr;
  if ((rc = graph_adopt(device, n, m, &g, &rp, &col, &scratch, &gs))) return rc;
  uint32_t loops = 0;
  tx_csr_kernel<<<r.sms * 4, 256, 0, r.s>>>(keys, m, n, b, rp, col, r.ctl);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&loops, &r.ctl->loops, 4, cudaMemcpyDeviceToHost, r.s) != cudaSuccess ||
      cudaStreamSynchronize(r.s) != cudaSuccess) {
    mce_graph_free(g);
    return MCE_ECUDA;
  }
  if (loops) {
    mce_graph_free(g);
    return MCE_EFORMAT;
  }
  *out = g;
  return MCE_OK;
}
