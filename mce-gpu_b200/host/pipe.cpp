// Pipelined counting of a batch that lives in host memory.
//
// No counterpart in the reference, which reads one graph per run.  The
// batch is cut into `parts` runs of consecutive graphs of about equal arc
// counts; two device batches take the parts in turn, each on its own
// stream, so the host-to-device copy of part k + 1 runs on a copy engine
// while part k is counted.  Built on the public batch entry points only.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/mce.h"

struct mce_pipe {
  int32_t device = 0, parts = 1;
  mce_batch_t h[2] = {nullptr, nullptr};
  std::vector<int64_t> vo[2], ao[2];  // the parts' rebased offsets (alive while copies run)
};

namespace {

// graph index where each part starts, parts + 1 entries
std::vector<int32_t> cut(const int64_t *ao, int32_t G, int32_t parts) {
  std::vector<int32_t> at(1, 0);
  const int64_t m = ao[G];
  for (int32_t p = 1; p < parts; ++p) {
    const int64_t want = m * p / parts;
    int32_t g = (int32_t)(std::lower_bound(ao, ao + G + 1, want) - ao);
    g = std::max(g, at.back() + 1);
    if (g >= G) break;
    at.push_back(g);
  }
  at.push_back(G);
  return at;
}

// queue the copy of graphs [g0, g1) into handle slot k (async on its stream
// once the handle exists)
int submit(mce_pipe *p, int k, const int32_t *row_ptr, const int32_t *col, const int64_t *vo,
           const int64_t *ao, int32_t g0, int32_t g1) {
  const int32_t G = g1 - g0;
  std::vector<int64_t> &v = p->vo[k], &a = p->ao[k];
  v.resize((size_t)G + 1);
  a.resize((size_t)G + 1);
  for (int32_t i = 0; i <= G; ++i) {
    v[(size_t)i] = vo[g0 + i] - vo[g0];
    a[(size_t)i] = ao[g0 + i] - ao[g0];
  }
  const int32_t *rp = row_ptr + vo[g0];
  const int32_t *cl = col + ao[g0];
  if (!p->h[k]) return mce_batch_upload(rp, cl, v.data(), a.data(), G, p->device, nullptr, &p->h[k]);
  return mce_batch_reload(p->h[k], rp, cl, v.data(), a.data(), G, nullptr);
}

}  // namespace

extern "C" int mce_pipe_create(int32_t device, int32_t parts, mce_pipe_t *out) {
  if (!out || parts < 1 || parts > 1024) return MCE_EINVAL;
  mce_pipe *p = new mce_pipe();
  p->device = device;
  p->parts = parts;
  *out = p;
  return MCE_OK;
}

extern "C" int mce_pipe_count(mce_pipe_t p, const int32_t *row_ptr, const int32_t *col,
                              const int64_t *vtx_offsets, const int64_t *arc_offsets,
                              int32_t num_graphs, const mce_opts_t *opts,
                              uint64_t *per_graph_total, uint64_t *total, uint64_t *hist) {
  if (!p || !row_ptr || !vtx_offsets || !arc_offsets || num_graphs < 1 || !per_graph_total ||
      !total)
    return MCE_EINVAL;
  mce_opts_t o;
  if (opts) {
    o = *opts;
  } else {
    mce_opts_default(&o);
    o.cuda_graph = 1;
  }
  o.stream = nullptr;  // each device batch on its own stream: copies overlap counts
  const std::vector<int32_t> at = cut(arc_offsets, num_graphs, p->parts);
  const int P = (int)at.size() - 1;
  *total = 0;
  if (hist) std::memset(hist, 0, sizeof(uint64_t) * MCE_HIST_MAX);
  std::vector<uint64_t> h(MCE_HIST_MAX);
  int rc = submit(p, 0, row_ptr, col, vtx_offsets, arc_offsets, at[0], at[1]);
  if (!rc && P > 1) rc = submit(p, 1, row_ptr, col, vtx_offsets, arc_offsets, at[1], at[2]);
  for (int k = 0; k < P && !rc; ++k) {
    uint64_t t = 0;
    rc = mce_batch_count(p->h[k & 1], &o, per_graph_total + at[k], &t, hist ? h.data() : nullptr,
                         nullptr);
    if (rc) break;
    *total += t;
    if (hist)
      for (int s = 0; s < MCE_HIST_MAX; ++s) hist[s] += h[(size_t)s];
    if (k + 2 < P)  // this handle is free again: queue part k + 2 behind part k + 1's count
      rc = submit(p, k & 1, row_ptr, col, vtx_offsets, arc_offsets, at[k + 2], at[k + 3]);
  }
  return rc;
}

extern "C" int mce_pipe_free(mce_pipe_t p) {
  if (!p) return MCE_EINVAL;
  for (auto &h : p->h)
    if (h) mce_batch_free(h);
  delete p;
  return MCE_OK;
}
