// Seeded synthetic graph generators (stand-ins for the downloaded datasets).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/mce_gen.h"
#include "host.h"

using namespace mce;

namespace {

void add_clique(std::vector<std::pair<int64_t, int64_t>> &pairs, const std::vector<int64_t> &vs) {
  for (size_t i = 0; i < vs.size(); ++i)
    for (size_t j = i + 1; j < vs.size(); ++j) pairs.push_back({vs[i], vs[j]});
}

}  // namespace

extern "C" int mce_gen_er(int64_t n, double p, uint64_t seed, int32_t planted,
                          int32_t clique_min, int32_t clique_max, mce_hgraph_t *out) {
  if (!out || n < 0 || p < 0 || p > 1 || planted < 0 || clique_min < 1 ||
      clique_max < clique_min)
    return MCE_EINVAL;
  Rng rng(seed, 0x4552ull);
  std::vector<std::pair<int64_t, int64_t>> pairs;
  // Geometric skipping over the pairs (v, w), w < v, in row-major order
  // (Batagelj & Brandes 2005, "Efficient generation of large random networks").
  if (p > 0 && n > 1) {
    if (p >= 1) {
      for (int64_t v = 1; v < n; ++v)
        for (int64_t w = 0; w < v; ++w) pairs.push_back({v, w});
    } else {
      const double lp = std::log1p(-p);
      int64_t v = 1, w = -1;
      while (v < n) {
        const double r = rng.uniform();
        w += 1 + (int64_t)std::floor(std::log1p(-r) / lp);
        while (w >= v && v < n) {
          w -= v;
          ++v;
        }
        if (v < n) pairs.push_back({v, w});
      }
    }
  }
  for (int32_t k = 0; k < planted; ++k) {
    const int64_t s = rng.range(clique_min, clique_max);
    add_clique(pairs, sample_distinct(rng, n, s));
  }
  return build_csr(pairs, n, out);
}

extern "C" int mce_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                            uint64_t seed, mce_hgraph_t *out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 ||
      a + b + c > 1)
    return MCE_EINVAL;
  const int64_t n = (int64_t)1 << scale;
  const int64_t E = (int64_t)edge_factor * n;
  // integer thresholds on 32-bit draws
  const uint64_t ta = (uint64_t)(a * 4294967296.0);
  const uint64_t tab = (uint64_t)((a + b) * 4294967296.0);
  const uint64_t tabc = (uint64_t)((a + b + c) * 4294967296.0);
  std::vector<std::pair<int64_t, int64_t>> pairs((size_t)E);
  const int64_t chunk = (int64_t)1 << 16;
  const int64_t nchunks = (E + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t ch = 0; ch < nchunks; ++ch) {
    Rng rng(seed, 0x524d4154ull + (uint64_t)ch);  // one stream per chunk
    const int64_t lo = ch * chunk, hi = std::min(E, lo + chunk);
    for (int64_t e = lo; e < hi; ++e) {
      int64_t u = 0, v = 0;
      uint64_t bits = 0;
      int avail = 0;
      for (int l = 0; l < scale; ++l) {
        if (avail == 0) {
          bits = rng.next();
          avail = 2;
        }
        const uint64_t r = bits & 0xFFFFFFFFull;
        bits >>= 32;
        --avail;
        int ub, vb;
        if (r < ta) {
          ub = 0; vb = 0;
        } else if (r < tab) {
          ub = 0; vb = 1;
        } else if (r < tabc) {
          ub = 1; vb = 0;
        } else {
          ub = 1; vb = 1;
        }
        u = (u << 1) | ub;
        v = (v << 1) | vb;
      }
      pairs[e] = {u, v};
    }
  }
  return build_csr(pairs, n, out);
}

extern "C" int mce_gen_ba(int64_t n, int32_t m, uint64_t seed, int32_t planted,
                          int32_t clique_min, int32_t clique_max, mce_hgraph_t *out) {
  if (!out || m < 1 || n < m + 1 || planted < 0 || clique_min < 1 || clique_max < clique_min)
    return MCE_EINVAL;
  Rng rng(seed, 0x4241ull);
  std::vector<std::pair<int64_t, int64_t>> pairs;
  pairs.reserve((size_t)(n * m + (int64_t)planted * clique_max * clique_max / 2));
  std::vector<int32_t> ends;  // every edge endpoint once per edge: sampling ~ degree
  ends.reserve((size_t)(2 * n * m));
  for (int64_t u = 0; u <= m; ++u)
    for (int64_t v = u + 1; v <= m; ++v) {
      pairs.push_back({u, v});
      ends.push_back((int32_t)u);
      ends.push_back((int32_t)v);
    }
  std::vector<int32_t> tgt((size_t)m);
  for (int64_t t = m + 1; t < n; ++t) {
    int k = 0;
    while (k < m) {
      const int32_t x = ends[rng.below(ends.size())];
      bool dup = false;
      for (int i = 0; i < k; ++i) dup |= (tgt[i] == x);
      if (!dup) tgt[k++] = x;
    }
    for (int i = 0; i < m; ++i) {
      pairs.push_back({t, tgt[i]});
      ends.push_back((int32_t)t);
      ends.push_back(tgt[i]);
    }
  }
  if (planted > 0) {
    const int64_t pool_n =
        std::min<int64_t>(n, std::max<int64_t>(clique_max, (int64_t)planted * (clique_min + clique_max) / 4));
    const std::vector<int64_t> pool = sample_distinct(rng, n, pool_n);
    for (int32_t k = 0; k < planted; ++k) {
      const int64_t s = std::min<int64_t>(rng.range(clique_min, clique_max), pool_n);
      std::vector<int64_t> idx = sample_distinct(rng, pool_n, s), vs;
      for (int64_t i : idx) vs.push_back(pool[i]);
      add_clique(pairs, vs);
    }
  }
  return build_csr(pairs, n, out);
}

namespace {

// One Chung-Lu graph by edge sampling: both endpoints of each of
// round(n * mean / 2) samples are drawn with probability proportional to
// w_j = (j + 1)^(-1 / (gamma - 1)); loops and repeats are then removed.
int chung_lu_one(Rng &rng, int64_t n, double gamma, double mean, int32_t planted,
                 int32_t cmin, int32_t cmax, mce_hgraph_t *out) {
  const double alpha = 1.0 / (gamma - 1.0);
  std::vector<double> cdf((size_t)n);
  double acc = 0;
  for (int64_t j = 0; j < n; ++j) {
    acc += std::pow((double)(j + 1), -alpha);
    cdf[j] = acc;
  }
  const int64_t samples = (int64_t)std::llround((double)n * mean / 2.0);
  std::vector<std::pair<int64_t, int64_t>> pairs;
  pairs.reserve((size_t)samples + (size_t)planted * cmax * cmax / 2);
  auto draw = [&]() -> int64_t {
    const double r = rng.uniform() * acc;
    int64_t j = std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin();
    return j < n ? j : n - 1;
  };
  for (int64_t e = 0; e < samples; ++e) {
    const int64_t u = draw(), v = draw();
    pairs.push_back({u, v});
  }
  for (int32_t k = 0; k < planted; ++k) {
    const int64_t s = std::min<int64_t>(rng.range(cmin, cmax), n);
    add_clique(pairs, sample_distinct(rng, n, s));
  }
  return build_csr(pairs, n, out);
}

}  // namespace

extern "C" int mce_gen_chung_lu_batch(int32_t num_graphs, int64_t n_min, int64_t n_max,
                                      double gamma, double deg_min, double deg_max,
                                      int32_t max_planted, int32_t clique_min,
                                      int32_t clique_max, uint64_t seed, mce_hgraph_t *out) {
  if (!out || num_graphs < 1 || n_min < 1 || n_max < n_min || gamma <= 1 || deg_min < 0 ||
      deg_max < deg_min || max_planted < 0 || clique_min < 1 || clique_max < clique_min)
    return MCE_EINVAL;
  std::vector<mce_hgraph_t> gs((size_t)num_graphs);
  std::vector<int> rcs((size_t)num_graphs, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int32_t g = 0; g < num_graphs; ++g) {
    Rng rng(seed, 0x434cull * 1000003ull + (uint64_t)g);
    const double ln = std::log((double)n_min), lx = std::log((double)n_max);
    int64_t n = (int64_t)std::llround(std::exp(ln + (lx - ln) * rng.uniform()));
    n = std::min(std::max(n, n_min), n_max);
    const double mean = deg_min + (deg_max - deg_min) * rng.uniform();
    const int32_t planted = (int32_t)rng.range(0, max_planted);
    rcs[g] = chung_lu_one(rng, n, gamma, mean, planted, clique_min, clique_max, &gs[g]);
  }
  for (int32_t g = 0; g < num_graphs; ++g)
    if (rcs[g]) {
      for (auto &x : gs) mce_hgraph_free(&x);
      return rcs[g];
    }
  int64_t N = 0, M = 0;
  for (auto &x : gs) {
    N += x.n;
    M += x.m;
  }
  if (M >= ((int64_t)1 << 31)) {
    for (auto &x : gs) mce_hgraph_free(&x);
    return MCE_ELIMIT;
  }
  int rc = hgraph_alloc(out, N, M, num_graphs);
  if (rc) {
    for (auto &x : gs) mce_hgraph_free(&x);
    return rc;
  }
  int64_t vo = 0, ao = 0;
  for (int32_t g = 0; g < num_graphs; ++g) {
    out->vtx_offsets[g] = vo;
    out->arc_offsets[g] = ao;
    std::memcpy(out->row_ptr + vo, gs[g].row_ptr, sizeof(int32_t) * (size_t)(gs[g].n + 1));
    std::memcpy(out->col + ao, gs[g].col, sizeof(int32_t) * (size_t)gs[g].m);
    vo += gs[g].n + 1;
    ao += gs[g].m;
    mce_hgraph_free(&gs[g]);
  }
  out->vtx_offsets[num_graphs] = vo;
  out->arc_offsets[num_graphs] = ao;
  return MCE_OK;
}
