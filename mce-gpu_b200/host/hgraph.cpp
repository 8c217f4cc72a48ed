// Host CSR graphs: normalisation, validation, union, relabelling, ego nets.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <unordered_map>
#include <unordered_set>

#include "../../include/mce_gen.h"
#include "host.h"

namespace mce {

int hgraph_alloc(mce_hgraph_t *g, int64_t n, int64_t m, int32_t num_graphs) {
  std::memset(g, 0, sizeof(*g));
  g->n = n;
  g->m = m;
  g->num_graphs = num_graphs;
  g->row_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(n + num_graphs));
  g->col = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  g->vtx_offsets = (int64_t *)std::malloc(sizeof(int64_t) * (size_t)(num_graphs + 1));
  g->arc_offsets = (int64_t *)std::malloc(sizeof(int64_t) * (size_t)(num_graphs + 1));
  if (!g->row_ptr || !g->col || !g->vtx_offsets || !g->arc_offsets) {
    mce_hgraph_free(g);
    return MCE_ENOMEM;
  }
  if (num_graphs == 1) {
    g->vtx_offsets[0] = 0;
    g->vtx_offsets[1] = n + 1;
    g->arc_offsets[0] = 0;
    g->arc_offsets[1] = m;
  }
  return MCE_OK;
}

std::vector<int64_t> sample_distinct(Rng &rng, int64_t n, int64_t k) {
  if (k > n) k = n;
  std::unordered_set<int64_t> chosen;
  chosen.reserve((size_t)k * 2);
  for (int64_t j = n - k; j < n; ++j) {
    int64_t t = (int64_t)rng.below((uint64_t)(j + 1));
    if (chosen.count(t))
      chosen.insert(j);
    else
      chosen.insert(t);
  }
  std::vector<int64_t> out(chosen.begin(), chosen.end());
  std::sort(out.begin(), out.end());
  return out;
}

// Counting sort by source, then per-row sort + unique.  Deterministic: the
// scatter order inside a row does not matter because every row is sorted.
int build_csr(const std::vector<std::pair<int64_t, int64_t>> &pairs, int64_t n,
              mce_hgraph_t *out) {
  const int64_t E = (int64_t)pairs.size();
  for (int64_t i = 0; i < E; ++i) {
    if (pairs[i].first < 0 || pairs[i].second < 0) return MCE_EINVAL;
    n = std::max(n, std::max(pairs[i].first, pairs[i].second) + 1);
  }
  if (n >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  std::vector<std::atomic<int64_t>> deg((size_t)n);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < n; ++v) deg[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < E; ++i) {
    const int64_t u = pairs[i].first, v = pairs[i].second;
    if (u == v) continue;
    deg[u].fetch_add(1, std::memory_order_relaxed);
    deg[v].fetch_add(1, std::memory_order_relaxed);
  }
  std::vector<int64_t> off((size_t)n + 1);
  off[0] = 0;
  for (int64_t v = 0; v < n; ++v) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
  const int64_t M0 = off[n];
  std::vector<int32_t> tmp((size_t)(M0 > 0 ? M0 : 1));
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < n; ++v) deg[v].store(off[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < E; ++i) {
    const int64_t u = pairs[i].first, v = pairs[i].second;
    if (u == v) continue;
    tmp[deg[u].fetch_add(1, std::memory_order_relaxed)] = (int32_t)v;
    tmp[deg[v].fetch_add(1, std::memory_order_relaxed)] = (int32_t)u;
  }
  std::vector<int64_t> uniq((size_t)n + 1);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < n; ++v) {
    int32_t *b = tmp.data() + off[v], *e = tmp.data() + off[v + 1];
    std::sort(b, e);
    uniq[v] = std::unique(b, e) - b;
  }
  int64_t M = 0;
  for (int64_t v = 0; v < n; ++v) M += uniq[v];
  if (M >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  int rc = hgraph_alloc(out, n, M, 1);
  if (rc) return rc;
  int64_t acc = 0;
  for (int64_t v = 0; v < n; ++v) {
    out->row_ptr[v] = (int32_t)acc;
    acc += uniq[v];
  }
  out->row_ptr[n] = (int32_t)acc;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < n; ++v)
    std::memcpy(out->col + out->row_ptr[v], tmp.data() + off[v], sizeof(int32_t) * uniq[v]);
  return MCE_OK;
}

}  // namespace mce

using namespace mce;

extern "C" void mce_hgraph_free(mce_hgraph_t *g) {
  if (!g) return;
  std::free(g->row_ptr);
  std::free(g->col);
  std::free(g->vtx_offsets);
  std::free(g->arc_offsets);
  std::memset(g, 0, sizeof(*g));
}

extern "C" int mce_hgraph_from_edges(const int64_t *src, const int64_t *dst, int64_t count,
                                     int64_t n_hint, mce_hgraph_t *out) {
  if (!out || count < 0 || (count > 0 && (!src || !dst))) return MCE_EINVAL;
  std::vector<std::pair<int64_t, int64_t>> pairs((size_t)count);
  for (int64_t i = 0; i < count; ++i) pairs[i] = {src[i], dst[i]};
  return build_csr(pairs, n_hint < 0 ? 0 : n_hint, out);
}

extern "C" int mce_csr_validate(const int32_t *row_ptr, const int32_t *col, int64_t n,
                                int64_t m) {
  if (n < 0 || m < 0 || (!row_ptr && n > 0)) return MCE_EINVAL;
  if (n == 0) return m == 0 ? MCE_OK : MCE_EFORMAT;
  if (row_ptr[0] != 0 || row_ptr[n] != m) return MCE_EFORMAT;
  std::atomic<int> bad(0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < n; ++v) {
    const int64_t b = row_ptr[v], e = row_ptr[v + 1];
    if (e < b) {
      bad = 1;
      continue;
    }
    for (int64_t j = b; j < e; ++j) {
      const int32_t u = col[j];
      if (u < 0 || u >= n || u == v || (j > b && col[j - 1] >= u)) {
        bad = 1;
        break;
      }
      // symmetry: v must appear in u's row
      if (!std::binary_search(col + row_ptr[u], col + row_ptr[u + 1], (int32_t)v)) {
        bad = 1;
        break;
      }
    }
  }
  return bad ? MCE_EFORMAT : MCE_OK;
}

extern "C" int mce_gen_permute(const mce_hgraph_t *in, uint64_t seed, mce_hgraph_t *out) {
  if (!in || !out || in->num_graphs != 1) return MCE_EINVAL;
  const int64_t n = in->n;
  std::vector<int64_t> perm((size_t)n);
  for (int64_t i = 0; i < n; ++i) perm[i] = i;
  Rng rng(seed, 0x5045524dull);
  for (int64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[(int64_t)rng.below(i + 1)]);
  std::vector<std::pair<int64_t, int64_t>> pairs;
  pairs.reserve((size_t)(in->m / 2));
  for (int64_t v = 0; v < n; ++v)
    for (int64_t j = in->row_ptr[v]; j < in->row_ptr[v + 1]; ++j)
      if (v < in->col[j]) pairs.push_back({perm[v], perm[in->col[j]]});
  return build_csr(pairs, n, out);
}

extern "C" int mce_hgraph_union(const mce_hgraph_t *b, mce_hgraph_t *out) {
  if (!b || !out || b->num_graphs < 1) return MCE_EINVAL;
  const int32_t G = b->num_graphs;
  const int64_t n = b->n, m = b->m;
  if (m >= ((int64_t)1 << 31) || n >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  int rc = hgraph_alloc(out, n, m, 1);
  if (rc) return rc;
  int64_t vbase = 0;
  for (int32_t g = 0; g < G; ++g) {
    const int64_t rb = b->vtx_offsets[g], ng = b->vtx_offsets[g + 1] - rb - 1;
    const int64_t ab = b->arc_offsets[g];
    for (int64_t v = 0; v < ng; ++v) {
      out->row_ptr[vbase + v] = (int32_t)(ab + b->row_ptr[rb + v]);
      for (int64_t j = b->row_ptr[rb + v]; j < b->row_ptr[rb + v + 1]; ++j)
        out->col[ab + j] = (int32_t)(vbase + b->col[ab + j]);
    }
    vbase += ng;
  }
  out->row_ptr[n] = (int32_t)m;
  return MCE_OK;
}

extern "C" int mce_ego_subgraph(const int32_t *row_ptr, const int32_t *col, int64_t n,
                                int64_t seed_vertex, int64_t cap, mce_hgraph_t *out,
                                int32_t *vertex_map_out) {
  if (!row_ptr || !col || !out || seed_vertex < 0 || seed_vertex >= n || cap < 1)
    return MCE_EINVAL;
  std::vector<int32_t> verts;
  verts.push_back((int32_t)seed_vertex);
  std::unordered_set<int32_t> in;
  in.insert((int32_t)seed_vertex);
  for (int64_t j = row_ptr[seed_vertex]; j < row_ptr[seed_vertex + 1] && (int64_t)verts.size() < cap; ++j)
    if (in.insert(col[j]).second) verts.push_back(col[j]);
  const size_t k1 = verts.size();
  for (size_t i = 1; i < k1 && (int64_t)verts.size() < cap; ++i) {  // 2-hop, discovery order
    const int32_t u = verts[i];
    for (int64_t j = row_ptr[u]; j < row_ptr[u + 1] && (int64_t)verts.size() < cap; ++j)
      if (in.insert(col[j]).second) verts.push_back(col[j]);
  }
  std::sort(verts.begin(), verts.end());
  // relabel
  std::unordered_map<int32_t, int64_t> id;
  id.reserve(verts.size() * 2);
  for (size_t i = 0; i < verts.size(); ++i) id[verts[i]] = (int64_t)i;
  std::vector<std::pair<int64_t, int64_t>> pairs;
  for (size_t i = 0; i < verts.size(); ++i) {
    const int32_t u = verts[i];
    for (int64_t j = row_ptr[u]; j < row_ptr[u + 1]; ++j) {
      auto it = id.find(col[j]);
      if (it != id.end() && (int64_t)i < it->second) pairs.push_back({(int64_t)i, it->second});
    }
  }
  if (vertex_map_out)
    for (size_t i = 0; i < verts.size(); ++i) vertex_map_out[i] = verts[i];
  return build_csr(pairs, (int64_t)verts.size(), out);
}
