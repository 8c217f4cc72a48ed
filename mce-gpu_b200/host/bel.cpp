// .bel binary edge lists: reader, writer and the text -> .bel converter.
//
// Record layout (graph::convert_to_bel, include/fileop.h:62-71): three
// little-endian u64 per arc - dst, src, 0 - both directions of every edge,
// sorted by (src, dst).  The reader follows graph::read_bel
// (include/fileop.h:81-129): m = file size / 24, src at byte 8, dst at
// byte 0; and CSRCOO::from_edgelist (include/csrcoo.cuh:41-81): rows must be
// sorted by src, n = max src + 1, empty rows are filled.
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host.h"

using namespace mce;

extern "C" int mce_bel_read(const char *path, mce_hgraph_t *out) {
  if (!path || !out) return MCE_EINVAL;
  struct stat st;
  if (stat(path, &st) != 0) return MCE_EIO;
  if (st.st_size % 24 != 0) return MCE_EFORMAT;
  const int64_t m = (int64_t)(st.st_size / 24);
  if (m >= ((int64_t)1 << 31)) return MCE_ELIMIT;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return MCE_EIO;
  std::vector<int32_t> src((size_t)m), dst((size_t)m);
  const size_t shard = 1 << 16;
  std::vector<uint64_t> buf(3 * shard);
  int64_t got = 0;
  int rc = MCE_OK;
  while (got < m) {
    const size_t want = (size_t)std::min<int64_t>((int64_t)shard, m - got);
    if (std::fread(buf.data(), 24, want, fp) != want) {
      rc = MCE_EIO;
      break;
    }
    for (size_t i = 0; i < want; ++i) {
      const uint64_t d = buf[3 * i], s = buf[3 * i + 1];
      if (s >= ((uint64_t)1 << 31) || d >= ((uint64_t)1 << 31)) {
        rc = MCE_EFORMAT;
        break;
      }
      src[got + i] = (int32_t)s;
      dst[got + i] = (int32_t)d;
    }
    if (rc) break;
    got += (int64_t)want;
  }
  std::fclose(fp);
  if (rc) return rc;
  // sorted by (src, dst), strictly (no duplicate records), no self-loops
  for (int64_t i = 0; i < m; ++i) {
    if (src[i] == dst[i]) return MCE_EFORMAT;
    if (i > 0 && (src[i] < src[i - 1] || (src[i] == src[i - 1] && dst[i] <= dst[i - 1])))
      return MCE_EFORMAT;
  }
  const int64_t n = m ? (int64_t)src[m - 1] + 1 : 0;
  for (int64_t i = 0; i < m; ++i)
    if (dst[i] >= n) return MCE_EFORMAT;  // an arc whose reverse cannot exist
  rc = hgraph_alloc(out, n, m, 1);
  if (rc) return rc;
  int64_t j = 0;
  for (int64_t v = 0; v < n; ++v) {
    out->row_ptr[v] = (int32_t)j;
    while (j < m && src[j] == v) ++j;
  }
  out->row_ptr[n] = (int32_t)m;
  if (m) std::memcpy(out->col, dst.data(), sizeof(int32_t) * (size_t)m);
  return MCE_OK;
}

extern "C" int mce_bel_write(const char *path, const mce_hgraph_t *g) {
  if (!path || !g || g->num_graphs != 1) return MCE_EINVAL;
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return MCE_EIO;
  const size_t shard = 1 << 16;
  std::vector<uint64_t> buf(3 * shard);
  size_t k = 0;
  int rc = MCE_OK;
  for (int64_t v = 0; v < g->n && rc == MCE_OK; ++v)
    for (int64_t j = g->row_ptr[v]; j < g->row_ptr[v + 1]; ++j) {
      buf[3 * k] = (uint64_t)g->col[j];
      buf[3 * k + 1] = (uint64_t)v;
      buf[3 * k + 2] = 0;
      if (++k == shard) {
        if (std::fwrite(buf.data(), 24, k, fp) != k) rc = MCE_EIO;
        k = 0;
      }
    }
  if (rc == MCE_OK && k && std::fwrite(buf.data(), 24, k, fp) != k) rc = MCE_EIO;
  if (std::fclose(fp) != 0 && rc == MCE_OK) rc = MCE_EIO;
  return rc;
}

// graph::convert_to_bel (include/fileop.h:13-79).  The parse sees the
// first 65,535 bytes of each line (a NUL byte ends it earlier), the window
// the device converter uses too.  One deviation: an empty line is skipped
// here; the reference's fscanf("%[^\n]%*c") loop never advances past it.
extern "C" int mce_convert_to_bel(const char *txt_path, const char *bel_path, int64_t *n_out,
                                  int64_t *undirected_edges_out) {
  if (!txt_path || !bel_path) return MCE_EINVAL;
  FILE *fp = std::fopen(txt_path, "r");
  if (!fp) return MCE_EIO;
  std::vector<std::pair<uint32_t, uint32_t>> edges;
  unsigned long long maxnode = 0;
  bool any = false;
  char *line = nullptr;
  size_t cap = 0;
  ssize_t len;
  while ((len = getline(&line, &cap, fp)) != -1) {
    if (len > 65535) line[65535] = '\0';
    if (!std::isdigit((unsigned char)line[0])) continue;
    unsigned long long s = 0, d = 0;
    if (std::sscanf(line, "%llu %llu", &s, &d) == 2 && s != d) {
      // ids narrowed to 32 bits, as T(src) does in the reference
      edges.push_back({(uint32_t)s, (uint32_t)d});
      edges.push_back({(uint32_t)d, (uint32_t)s});
      maxnode = std::max({maxnode, s, d});
      any = true;
    }
  }
  std::free(line);
  std::fclose(fp);
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  FILE *w = std::fopen(bel_path, "wb");
  if (!w) return MCE_EIO;
  const size_t shard = 1 << 16;
  std::vector<uint64_t> buf(3 * shard);
  size_t k = 0;
  int rc = MCE_OK;
  for (size_t i = 0; i < edges.size() && rc == MCE_OK; ++i) {
    buf[3 * k] = edges[i].second;
    buf[3 * k + 1] = edges[i].first;
    buf[3 * k + 2] = 0;
    if (++k == shard) {
      if (std::fwrite(buf.data(), 24, k, w) != k) rc = MCE_EIO;
      k = 0;
    }
  }
  if (rc == MCE_OK && k && std::fwrite(buf.data(), 24, k, w) != k) rc = MCE_EIO;
  if (std::fclose(w) != 0 && rc == MCE_OK) rc = MCE_EIO;
  if (n_out) *n_out = any ? (int64_t)maxnode + 1 : 1;
  if (undirected_edges_out) *undirected_edges_out = (int64_t)edges.size() / 2;
  return rc;
}
