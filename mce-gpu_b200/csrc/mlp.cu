// Learned root scheduling: per-root features and a small cost MLP.
//
// The reference schedules roots in vertex-id order and balances load only
// by donating branches at run time (mce/mce_kernel_wl.cuh:37,
// mce/mce_utils.cuh:1063-1113); its only static choice is per-graph (the
// L1+IP vs L1+IPX rule of thumb on max degree / degeneracy, table.py:127).
// Here a network predicts the search-tree size of every root from eight
// features, and the prediction orders roots longest-first and decides which
// roots may hand subtrees to idle warps.  The count never depends on it.
//
// Network: 8 -> 64 -> 64 -> 1, ReLU, FP16 weights, FP32 accumulation and
// FP32 master weights for training.  Target: log2(1 + search-tree nodes).
// Kernels (all this project's): features, forward (inference), one fused
// forward+backward pass per minibatch with block-level gradient reduction,
// and Adam.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "kernels.h"

namespace mce {

namespace {

constexpr int F = MLP_IN, H = MLP_HIDDEN;
// parameter offsets (floats / halves)
constexpr int O_W1 = 0, O_B1 = O_W1 + H * F, O_W2 = O_B1 + H, O_B2 = O_W2 + H * H, O_W3 = O_B2 + H,
              O_B3 = O_W3 + H, NPARAM = O_B3 + 1;
static_assert(NPARAM == MLP_PARAMS, "parameter layout");

__device__ __forceinline__ float lg(float x) { return log2f(1.0f + x); }

// ---------------------------------------------------------------------------
// Features of root r (one warp): degrees, core number, density of the
// subgraph induced by the later neighbours (on the first FEAT_CAP of them),
// its largest degree and the number of first-level branches that degree
// leaves (|P| - max |P & N(u)|: the popcount of P at depth 1 after the
// pivot).  Non-roots get zeros.
// ---------------------------------------------------------------------------
constexpr int FEAT_CAP = 64;
// Roots with fewer later neighbours have trees too small to be worth
// scheduling: their features stay zero and the model is not run on them.
constexpr int FEAT_MIN = MLP_MIN_LATER;

// The roots with at least FEAT_MIN later neighbours (warp-aggregated append;
// their order does not matter).
__global__ void cand_list_kernel(int64_t n, const int32_t *__restrict__ rp,
                                 const int32_t *__restrict__ split, int32_t *list,
                                 uint32_t *count, int min_later) {
  const int lane = (int)lane_id();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v - lane < n; v += stride) {
    const bool c = v < n && rp[v + 1] - split[v] >= min_later;
    const uint32_t mk = __ballot_sync(MCE_FULL, c);
    if (!mk) continue;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(count, (uint32_t)__popc(mk));
    base = __shfl_sync(MCE_FULL, base, 0);
    if (c) list[base + __popc(mk & ((1u << lane) - 1u))] = (int32_t)v;
  }
}

// Features of the listed roots, one warp each.  The later lists of the
// first d later neighbours are walked flattened over the lanes, each element
// tested against a hash of those neighbours' ids.
__global__ void features_kernel(const int32_t *__restrict__ list, const uint32_t *count,
                                const int32_t *__restrict__ rp, const int32_t *__restrict__ split,
                                const int32_t *__restrict__ cs, const int32_t *__restrict__ core,
                                float *__restrict__ out) {
  __shared__ int32_t s_p[8][FEAT_CAP];
  __shared__ int32_t s_deg[8][FEAT_CAP];
  __shared__ int32_t s_key[8][2 * FEAT_CAP];
  __shared__ uint8_t s_idx[8][2 * FEAT_CAP];
  __shared__ int32_t s_off[8][32], s_beg[8][32], s_own[8][32];
  const int lane = (int)lane_id(), wib = threadIdx.x >> 5;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t cnt = (int64_t)*count;
  auto slot = [](int32_t w) { return ((uint32_t)w * 0x9E3779B1u) >> 25; };  // 128 slots
  for (int64_t t = gw; t < cnt; t += nw) {
    const int32_t v = list[t];
    const int32_t sb = split[v], dp = rp[v + 1] - sb, dm = sb - rp[v];
    float *o = out + (size_t)v * F;
    const int d = dp < FEAT_CAP ? dp : FEAT_CAP;
    for (int i = lane; i < FEAT_CAP; i += 32) {
      s_p[wib][i] = i < d ? cs[sb + i] : 0x7FFFFFFF;
      s_deg[wib][i] = 0;
    }
    for (int i = lane; i < 2 * FEAT_CAP; i += 32) s_key[wib][i] = -1;
    __syncwarp();
    for (int i = lane; i < d; i += 32) {  // the ids are distinct
      const int32_t w = s_p[wib][i];
      uint32_t h = slot(w);
      while (atomicCAS(&s_key[wib][h], -1, w) != -1) h = (h + 1) & (2 * FEAT_CAP - 1);
      s_idx[wib][h] = (uint8_t)i;
    }
    __syncwarp();
    // induced edges among the first d later neighbours; later-list mass
    long long mass = 0;
    int edges = 0;
    for (int c = 0; c * 32 < d; ++c) {
      const int items = min(32, d - c * 32);
      int ub = 0, ulen = 0;
      if (lane < items) {
        const int32_t u = s_p[wib][c * 32 + lane];
        ub = split[u];
        ulen = rp[u + 1] - ub;
      }
      mass += ulen;
      flat_walk(cs, ub, ulen, s_off[wib], s_beg[wib], s_own[wib], [&](int tt, int32_t w) {
        uint32_t h = slot(w);
        for (;;) {
          const int32_t k = s_key[wib][h];
          if (k == w) {
            ++edges;
            atomicAdd(&s_deg[wib][c * 32 + tt], 1);
            atomicAdd(&s_deg[wib][s_idx[wib][h]], 1);
            break;
          }
          if (k == -1) break;
          h = (h + 1) & (2 * FEAT_CAP - 1);
        }
      });
    }
    __syncwarp();
    edges = __reduce_add_sync(MCE_FULL, edges);
    for (int o2 = 16; o2; o2 >>= 1) mass += __shfl_xor_sync(MCE_FULL, mass, o2);
    int mx = 0;
    for (int j = lane; j < d; j += 32) mx = max(mx, s_deg[wib][j]);
    mx = __reduce_max_sync(MCE_FULL, mx);
    __syncwarp();
    if (lane == 0) {
      const float pairs = 0.5f * (float)d * (float)(d - 1);
      o[0] = lg((float)dp);
      o[1] = lg((float)dm);
      o[2] = lg((float)core[v]);
      o[3] = lg((float)(rp[v + 1] - rp[v]));
      o[4] = pairs > 0 ? (float)edges / pairs : 0.f;
      o[5] = lg((float)(d - mx));
      o[6] = lg((float)mass);
      o[7] = lg((float)mx);
    }
  }
}

// ---------------------------------------------------------------------------
// Inference: one thread per sample; FP16 weights staged to shared memory as
// floats, FP32 accumulation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mlp_eval(const float *w, const float *x) {
  float h1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float a = w[O_B1 + j];
#pragma unroll
    for (int i = 0; i < F; ++i) a = fmaf(w[O_W1 + j * F + i], x[i], a);
    h1[j] = a > 0.f ? a : 0.f;
  }
  float out = w[O_B3];
  for (int k = 0; k < H; ++k) {
    float a = w[O_B2 + k];
#pragma unroll
    for (int j = 0; j < H; ++j) a = fmaf(w[O_W2 + k * H + j], h1[j], a);
    out = fmaf(w[O_W3 + k], a > 0.f ? a : 0.f, out);
  }
  return out;
}

// idx null: out[t] for rows t < count of X; else out[idx[t]] for t < *idx_count
// (the candidate list), the other entries of out untouched.
__global__ void mlp_forward_kernel(const __half *__restrict__ wh, const float *__restrict__ X,
                                   const int32_t *__restrict__ idx, const uint32_t *idx_count,
                                   int64_t count, float *__restrict__ out) {
  __shared__ float w[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) w[i] = __half2float(wh[i]);
  __syncthreads();
  if (idx) count = (int64_t)*idx_count;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = idx ? idx[t] : t;
    float x[F];
#pragma unroll
    for (int i = 0; i < F; ++i) x[i] = X[(size_t)s * F + i];
    out[s] = x[0] > 0.f ? mlp_eval(w, x) : 0.f;  // all-zero features: not a candidate
  }
}

// ---------------------------------------------------------------------------
// Training: forward + backward of up to TB samples per block; activations
// in shared memory; the block's gradient is a sum over its samples, added
// to the global FP32 gradient with one atomic per parameter.
// Loss: mean over the minibatch of (out - y)^2.
// ---------------------------------------------------------------------------
constexpr int TB = 128;
// rows padded by one float so that thread t's row starts in bank t % 32
constexpr int HP = H + 1, FP = F + 1;

__global__ void __launch_bounds__(TB) mlp_train_kernel(const __half *__restrict__ wh,
                                                       const float *__restrict__ X,
                                                       const float *__restrict__ Y,
                                                       const int32_t *__restrict__ idx,
                                                       int64_t begin, int64_t end, float inv_b,
                                                       float *__restrict__ grad,
                                                       float *__restrict__ loss) {
  extern __shared__ float sm[];
  float *w = sm;                       // NPARAM
  float *xs = w + NPARAM;              // TB x FP
  float *h1 = xs + TB * FP;            // TB x HP  post-ReLU layer 1 (> 0 marks active units)
  float *h2 = h1 + TB * HP;            // TB x HP  post-ReLU layer 2
  float *d2 = h2 + TB * HP;            // TB x HP  dL/d(pre-activation of layer 2)
  float *d1 = d2 + TB * HP;            // TB x HP  dL/d(pre-activation of layer 1)
  float *dout = d1 + TB * HP;          // TB
  const int t = threadIdx.x;
  for (int i = t; i < NPARAM; i += TB) w[i] = __half2float(wh[i]);
  const int64_t s0 = begin + (int64_t)blockIdx.x * TB;
  const int nb = (int)min((int64_t)TB, end - s0);
  if (nb <= 0) return;
  __syncthreads();
  float l = 0.f;
  if (t < nb) {
    const int64_t s = idx ? idx[s0 + t] : s0 + t;
    float x[F];
#pragma unroll
    for (int i = 0; i < F; ++i) {
      x[i] = X[(size_t)s * F + i];
      xs[t * FP + i] = x[i];
    }
    for (int j = 0; j < H; ++j) {
      float a = w[O_B1 + j];
#pragma unroll
      for (int i = 0; i < F; ++i) a = fmaf(w[O_W1 + j * F + i], x[i], a);
      h1[t * HP + j] = a > 0.f ? a : 0.f;
    }
    float out = w[O_B3];
    for (int k = 0; k < H; ++k) {
      float a = w[O_B2 + k];
      for (int j = 0; j < H; ++j) a = fmaf(w[O_W2 + k * H + j], h1[t * HP + j], a);
      a = a > 0.f ? a : 0.f;
      h2[t * HP + k] = a;
      out = fmaf(w[O_W3 + k], a, out);
    }
    const float e = out - Y[s];
    l = e * e;
    const float g = 2.f * e * inv_b;
    dout[t] = g;
    for (int k = 0; k < H; ++k) d2[t * HP + k] = h2[t * HP + k] > 0.f ? g * w[O_W3 + k] : 0.f;
    for (int j = 0; j < H; ++j) {
      float a = 0.f;
      if (h1[t * HP + j] > 0.f)
        for (int k = 0; k < H; ++k) a = fmaf(w[O_W2 + k * H + j], d2[t * HP + k], a);
      d1[t * HP + j] = a;
    }
  }
  __syncthreads();
  // gradient sums over the block's samples, one parameter per thread-iteration
  for (int p = t; p < NPARAM; p += TB) {
    float acc = 0.f;
    if (p < O_B1) {  // W1[j][i] = sum_b d1[b][j] x[b][i]
      const int j = p / F, i = p % F;
      for (int b = 0; b < nb; ++b) acc = fmaf(d1[b * HP + j], xs[b * FP + i], acc);
    } else if (p < O_W2) {  // b1[j]
      const int j = p - O_B1;
      for (int b = 0; b < nb; ++b) acc += d1[b * HP + j];
    } else if (p < O_B2) {  // W2[k][j] = sum_b d2[b][k] h1[b][j]
      const int q = p - O_W2, k = q / H, j = q % H;
      for (int b = 0; b < nb; ++b) acc = fmaf(d2[b * HP + k], h1[b * HP + j], acc);
    } else if (p < O_W3) {  // b2[k]
      const int k = p - O_B2;
      for (int b = 0; b < nb; ++b) acc += d2[b * HP + k];
    } else if (p < O_B3) {  // W3[k] = sum_b dout[b] h2[b][k]
      const int k = p - O_W3;
      for (int b = 0; b < nb; ++b) acc = fmaf(dout[b], h2[b * HP + k], acc);
    } else {  // b3
      for (int b = 0; b < nb; ++b) acc += dout[b];
    }
    atomicAdd(&grad[p], acc);
  }
  // loss sum (mean taken by the host)
  float ls = l;
  for (int o = 16; o; o >>= 1) ls += __shfl_xor_sync(MCE_FULL, ls, o);
  if ((t & 31) == 0) atomicAdd(loss, ls);
}

// Adam on FP32 master weights; refreshes the FP16 copy and clears the gradient.
__global__ void adam_kernel(float *__restrict__ master, __half *__restrict__ wh,
                            float *__restrict__ grad, float *__restrict__ m1,
                            float *__restrict__ m2, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  const float g = grad[p];
  const float a = b1 * m1[p] + (1.f - b1) * g;
  const float b = b2 * m2[p] + (1.f - b2) * g * g;
  m1[p] = a;
  m2[p] = b;
  const float upd = lr * (a / c1) / (sqrtf(b / c2) + eps);
  const float w = master[p] - upd;
  master[p] = w;
  wh[p] = __float2half_rn(w);
  grad[p] = 0.f;
}

// Sort key: class in the top 4 bits; then roots whose cost reaches `heavy`,
// larger first; every other root keeps the key 0x0FFFFFFF, so the stable
// sort leaves them in vertex order (neighbouring roots share adjacency
// lists, and in a batch each graph stays together in L2).
// With a model, roots with at least cost_min later neighbours take its
// prediction and the others the degree heuristic.
__global__ void rekey_kernel(int64_t n, uint32_t *keys, const float *__restrict__ cost,
                             const int32_t *__restrict__ rp, const int32_t *__restrict__ split,
                             uint8_t *policy, float heavy_cost, float share_cost, int cost_min,
                             const int32_t *__restrict__ hub_of) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t cls = keys[v] & 0xF;
    const int32_t dpi = rp[v + 1] - split[v];
    const bool learned = cost && dpi >= cost_min;
    float c;
    if (learned) {
      c = cost[v];
    } else {  // degree heuristic: trees grow with the later degree
      const float dp = (float)dpi;
      c = dp >= 16.f ? log2f(1.f + dp * dp * log2f(2.f + (float)(split[v] - rp[v]))) : 0.f;
    }
    c = c < 0.f ? 0.f : (c > 63.f ? 63.f : c);
    const bool heavy = c >= heavy_cost;
    const uint32_t q = heavy ? (uint32_t)(c * (float)(1 << 22)) : 0u;  // < 2^28
    if (hub_of)  // hubs first within the class, then the cost in 27 bits
      keys[v] = (cls << 28) | ((hub_of[v] < 0 ? 1u : 0u) << 27) | (0x07FFFFFFu - (q >> 1));
    else
      keys[v] = (cls << 28) | (0x0FFFFFFFu - q);
    if (policy) policy[v] = learned && c >= share_cost ? 1 : 0;
  }
}

}  // namespace

int features_launch(int64_t n, const int32_t *rp, const int32_t *split, const int32_t *cs,
                    const int32_t *core, float *out, int32_t *cand, uint32_t *cand_count, int sms,
                    cudaStream_t s, int *launches, int min_later) {
  if (n == 0) return MCE_OK;
  MCE_CUDA(cudaMemsetAsync(cand_count, 0, sizeof(uint32_t), s));
  cand_list_kernel<<<sms * 8, 256, 0, s>>>(n, rp, split, cand, cand_count,
                                           min_later > 0 ? min_later : FEAT_MIN);
  MCE_CUDA(cudaGetLastError());
  features_kernel<<<sms * 8, 256, 0, s>>>(cand, cand_count, rp, split, cs, core, out);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 2;
  return MCE_OK;
}

int mlp_forward_launch(const void *wh, const float *X, const int32_t *idx, const uint32_t *idx_count,
                       int64_t count, float *out, int sms, cudaStream_t s, int *launches) {
  if (count == 0) return MCE_OK;
  int64_t blocks = (count + 127) / 128;
  if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
  mlp_forward_kernel<<<(unsigned)blocks, 128, 0, s>>>((const __half *)wh, X, idx, idx_count, count,
                                                       out);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return MCE_OK;
}

size_t mlp_train_smem() { return sizeof(float) * (NPARAM + TB * FP + 4 * TB * HP + TB); }

int mlp_grad_launch(const void *wh, const float *X, const float *Y, const int32_t *idx,
                    int64_t begin, int64_t end, float *grad, float *loss, cudaStream_t s) {
  const int64_t cnt = end - begin;
  if (cnt <= 0) return MCE_OK;
  // set on every call: the attribute belongs to the current device, and a
  // cached flag would be shared by every device and host thread
  MCE_CUDA(cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)mlp_train_smem()));
  mlp_train_kernel<<<(unsigned)((cnt + TB - 1) / TB), TB, mlp_train_smem(), s>>>(
      (const __half *)wh, X, Y, idx, begin, end, 1.0f / (float)cnt, grad, loss);
  MCE_CUDA(cudaGetLastError());
  return MCE_OK;
}

int mlp_adam_launch(float *master, void *wh, float *grad, float *m1, float *m2, float lr,
                    int step, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
  adam_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(master, (__half *)wh, grad, m1, m2, lr, b1, b2,
                                                   1e-8f, c1, c2);
  MCE_CUDA(cudaGetLastError());
  return MCE_OK;
}

int rekey_launch(int64_t n, uint32_t *keys, const float *cost, const int32_t *rp,
                 const int32_t *split, uint8_t *policy, float heavy_cost, float share_cost,
                 int sms, cudaStream_t s, int *launches, int cost_min, const int32_t *hub_of) {
  if (n == 0) return MCE_OK;
  rekey_kernel<<<sms * 8, 256, 0, s>>>(n, keys, cost, rp, split, policy, heavy_cost, share_cost,
                                       cost_min, hub_of);
  MCE_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return MCE_OK;
}

}  // namespace mce
