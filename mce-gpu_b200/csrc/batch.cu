// Batched graphs: rebase a concatenation of per-graph CSRs into one
// disjoint-union CSR on the device.
//
// The reference runs one graph per process (src/main.cu); a batch of
// thousands of small graphs there means thousands of runs.  Here the batch
// is uploaded as concatenated local CSRs (graph g: rows
// row_ptr[vtx_off[g] .. vtx_off[g+1]), arcs col[arc_off[g] .. arc_off[g+1]),
// local ids) and turned into one graph whose vertex v of graph g has global
// id vbase[g] + v, vbase[g] = vtx_off[g] - g.  Peeling and search then run
// once over all graphs; graph_of[] routes each root's count to its graph.
// Both kernels are one pass over their array (HBM-bound).
#include "common.cuh"
#include "kernels.h"

namespace mce {

namespace {

// last g with off[g] <= i, for off ascending over g = 0 .. G
__device__ __forceinline__ int32_t owner(const int64_t *off, int32_t G, int64_t i) {
  int32_t lo = 0, hi = G + 1;
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (off[mid] <= i)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo - 1;
}

// Rows [row0, row1) of the upload; rp[vend] = rp_end closes the last one.
__global__ void batch_rows_kernel(const int32_t *rp_local, const int64_t *vtx_off,
                                  const int64_t *arc_off, int32_t G, int64_t row0, int64_t row1,
                                  int32_t *rp, int32_t *graph_of, int64_t vend, int32_t rp_end) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = row0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < row1; i += stride) {
    const int32_t g = owner(vtx_off, G, i);
    const int64_t k = i - vtx_off[g];
    if (i + 1 == vtx_off[g + 1]) continue;  // the closing offset of graph g
    const int64_t v = vtx_off[g] - g + k;
    rp[v] = (int32_t)(arc_off[g] + rp_local[i]);
    graph_of[v] = g;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) rp[vend] = rp_end;
}

__global__ void batch_cols_kernel(const int32_t *col_local, const int64_t *vtx_off,
                                  const int64_t *arc_off, int32_t G, int64_t arc0, int64_t arc1,
                                  int32_t *col) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = arc0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < arc1; j += stride) {
    const int32_t g = owner(arc_off, G, j);
    col[j] = (int32_t)(col_local[j] + (vtx_off[g] - g));
  }
}

}  // namespace

int batch_rebase_part_launch(const int32_t *rp_local, const int32_t *col_local,
                             const int64_t *vtx_off, const int64_t *arc_off, int32_t G,
                             int64_t row0, int64_t row1, int64_t arc0, int64_t arc1, int64_t vend,
                             int32_t rp_end, int32_t *rp, int32_t *col, int32_t *graph_of, int sms,
                             cudaStream_t s, int *launches) {
  const int blocks = sms * 8;
  batch_rows_kernel<<<blocks, 256, 0, s>>>(rp_local, vtx_off, arc_off, G, row0, row1, rp, graph_of,
                                           vend, rp_end);
  MCE_CUDA(cudaGetLastError());
  if (arc1 > arc0) {
    batch_cols_kernel<<<blocks, 256, 0, s>>>(col_local, vtx_off, arc_off, G, arc0, arc1, col);
    MCE_CUDA(cudaGetLastError());
  }
  if (launches) *launches += arc1 > arc0 ? 2 : 1;
  return MCE_OK;
}

int batch_rebase_launch(const int32_t *rp_local, const int32_t *col_local,
                        const int64_t *vtx_off, const int64_t *arc_off, int32_t G, int64_t n,
                        int64_t m, int32_t *rp, int32_t *col, int32_t *graph_of, int sms,
                        cudaStream_t s, int *launches) {
  return batch_rebase_part_launch(rp_local, col_local, vtx_off, arc_off, G, 0, n + G, 0, m, n,
                                  (int32_t)m, rp, col, graph_of, sms, s, launches);
}

}  // namespace mce
