// Autotuner: per graph-shape class, the search settings that ran fastest.
//
// No counterpart in the reference, whose only per-graph choice is the
// L1+IP / L1+IPX rule of thumb of its evaluation script (table.py:127).
// A shape class buckets a graph (or a batch's disjoint union) by
// floor(log2) of its vertex count, mean degree and degeneracy, plus the
// batch size for batches.  Tuning walks the knobs one at a time (donation
// gate, donation threshold, bitmap word width of narrow roots, single-block
// peeling of small frontiers, blocks per SM of the wide engine, pivots from
// the root's earlier neighbours (-i px); subtree
// sharing itself stays as given, since
// without it one heavy root can run for minutes), times each value with
// the device timers of mce_count / mce_batch_count, keeps a value only when
// it is at least 2% faster, and checks that every trial returns the same
// count.  Then, bucket by bucket - the engine classes of the roots, by
// bitmap width: d+ <= 32, 33..64, wider - it walks that bucket's warps per
// root, donation threshold and donation gate, scored by the bucket's own
// launch time (the classes run one after the other, so a bucket's settings
// do not move the others' times).  The winners are stored in a text table:
// one line per shape class and one per bucket of it ("<class>:b32",
// ":b64", ":wide"); later runs of the same class read them back without
// trials.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mce.h"

namespace mce {
int graph_shape(const struct ::mce_graph *g, int64_t *n, int64_t *m);
struct ::mce_graph *batch_union(struct ::mce_batch *b, int32_t *num_graphs);
}  // namespace mce

namespace {

struct Knobs {
  int32_t worker_list, donate_after, donate_threshold, bitmap_width, peel_solo_max, wide_blocks,
      x_pivot;
};

// the library's defaults, written out so that a table entry is explicit
Knobs resolved(const mce_opts_t &o) {
  Knobs k;
  k.worker_list = o.worker_list ? o.worker_list : MCE_WL_ON;
  k.donate_after = o.donate_after > 0 ? o.donate_after : 256;
  k.donate_threshold = o.donate_threshold > 0 ? o.donate_threshold : 10;
  k.bitmap_width = o.bitmap_width ? o.bitmap_width : 32;
  k.peel_solo_max = o.peel_solo_max > 0 ? o.peel_solo_max : -1;
  k.wide_blocks = o.wide_blocks ? o.wide_blocks : 4;
  k.x_pivot = o.x_pivot ? 1 : 0;
  return k;
}

void apply(const Knobs &k, mce_opts_t *o) {
  o->worker_list = k.worker_list;
  o->donate_after = k.donate_after;
  o->donate_threshold = k.donate_threshold;
  o->bitmap_width = k.bitmap_width;
  o->peel_solo_max = k.peel_solo_max;
  o->wide_blocks = k.wide_blocks;
  o->x_pivot = k.x_pivot;
}

int ilog2(double x) { return x < 1.0 ? 0 : (int)std::floor(std::log2(x)); }

// per bucket (engine class): 0 = the global value
struct Bucket {
  int32_t warps = 0, threshold = 0, after = 0;
  double best_ms = 0, default_ms = 0;
  bool present = false;
};

struct Entry {
  Knobs k;
  double best_ms, default_ms;
  Bucket b[3];
};

const char *kBucketName[3] = {"b32", "b64", "wide"};

void apply_buckets(const Bucket *b, mce_opts_t *o) {
  for (int c = 0; c < 3; ++c) {
    o->bucket_warps_per_root[c] = b[c].present ? b[c].warps : 0;
    o->bucket_donate_threshold[c] = b[c].present ? b[c].threshold : 0;
    o->bucket_donate_after[c] = b[c].present ? b[c].after : 0;
  }
}

const char *kHeader =
    "# mce autotune table v4: class worker_list donate_after donate_threshold bitmap_width "
    "peel_solo_max wide_blocks x_pivot best_ms default_ms\n"
    "# and per bucket of roots: class:bucket warps_per_root donate_threshold donate_after "
    "bucket_best_ms bucket_default_ms";

// v3 lines have 10 fields; v2 lines (9, no x_pivot) read as x_pivot 0 and
// v1 lines (8, no wide_blocks either) as wide_blocks 4
bool read_table(const char *path, std::map<std::string, Entry> *t) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    std::string key;
    std::vector<double> v;
    double x;
    ss >> key;
    while (ss >> x) v.push_back(x);
    const size_t colon = key.find(':');
    if (colon != std::string::npos) {  // a bucket line
      if (v.size() != 5) continue;
      const std::string cls = key.substr(0, colon), bk = key.substr(colon + 1);
      for (int c = 0; c < 3; ++c)
        if (bk == kBucketName[c]) {
          Bucket &b = (*t)[cls].b[c];
          b.warps = (int32_t)v[0];
          b.threshold = (int32_t)v[1];
          b.after = (int32_t)v[2];
          b.best_ms = v[3];
          b.default_ms = v[4];
          b.present = true;
        }
      continue;
    }
    if (v.size() < 7 || v.size() > 9) continue;
    const size_t knobs = v.size() - 2;  // 5, 6 or 7
    Entry e;
    e.k.worker_list = (int32_t)v[0];
    e.k.donate_after = (int32_t)v[1];
    e.k.donate_threshold = (int32_t)v[2];
    e.k.bitmap_width = (int32_t)v[3];
    e.k.peel_solo_max = (int32_t)v[4];
    e.k.wide_blocks = knobs >= 6 ? (int32_t)v[5] : 4;
    e.k.x_pivot = knobs >= 7 ? (int32_t)v[6] : 0;
    e.best_ms = v[knobs];
    e.default_ms = v[knobs + 1];
    Entry &dst = (*t)[key];  // keeps bucket lines read before it
    dst.k = e.k;
    dst.best_ms = e.best_ms;
    dst.default_ms = e.default_ms;
  }
  return true;
}

int write_table(const char *path, const std::map<std::string, Entry> &t) {
  const std::string tmp = std::string(path) + ".tmp";
  FILE *f = std::fopen(tmp.c_str(), "w");
  if (!f) return MCE_EIO;
  std::fprintf(f, "%s\n", kHeader);
  for (const auto &kv : t) {
    const Entry &e = kv.second;
    std::fprintf(f, "%s %d %d %d %d %d %d %d %.4f %.4f\n", kv.first.c_str(), e.k.worker_list,
                 e.k.donate_after, e.k.donate_threshold, e.k.bitmap_width, e.k.peel_solo_max,
                 e.k.wide_blocks, e.k.x_pivot, e.best_ms, e.default_ms);
    for (int c = 0; c < 3; ++c)
      if (e.b[c].present)
        std::fprintf(f, "%s:%s %d %d %d %.4f %.4f\n", kv.first.c_str(), kBucketName[c],
                     e.b[c].warps, e.b[c].threshold, e.b[c].after, e.b[c].best_ms,
                     e.b[c].default_ms);
  }
  if (std::fclose(f) != 0 || std::rename(tmp.c_str(), path) != 0) return MCE_EIO;
  return MCE_OK;
}

int shape_key(struct ::mce_graph *g, int32_t num_graphs, char *key, size_t len) {
  int64_t n = 0, m = 0;
  int rc = mce::graph_shape(g, &n, &m);
  if (rc) return rc;
  int32_t dg = 0;
  if ((rc = mce_degeneracy(g, nullptr, nullptr, &dg))) return rc;
  char buf[64];
  const int a = ilog2(n > 0 ? (double)m / (double)n : 0.0);
  if (num_graphs > 0)
    std::snprintf(buf, sizeof(buf), "b%d-n%d-a%d-k%d", ilog2(num_graphs), ilog2((double)n), a,
                  ilog2(dg));
  else
    std::snprintf(buf, sizeof(buf), "n%d-a%d-k%d", ilog2((double)n), a, ilog2(dg));
  if (std::strlen(buf) + 1 > len) return MCE_EINVAL;
  std::strcpy(key, buf);
  return MCE_OK;
}

// Run(opts, &ms, &total, class_ms[3]) -> status
template <typename Run>
int tune(const char *key, const mce_opts_t &base, const char *table_path, int32_t reps,
         int32_t force, Run run, mce_tune_result_t *out) {
  std::memset(out, 0, sizeof(*out));
  std::snprintf(out->key, sizeof(out->key), "%s", key);
  std::map<std::string, Entry> table;
  if (table_path) read_table(table_path, &table);
  out->best = base;
  if (!force && table.count(key) && table[key].best_ms > 0) {
    const Entry &e = table[key];
    apply(e.k, &out->best);
    apply_buckets(e.b, &out->best);
    out->best_ms = e.best_ms;
    out->default_ms = e.default_ms;
    out->from_table = 1;
    return MCE_OK;
  }
  if (reps < 1) reps = 1;
  uint64_t want = 0;
  bool have = false;
  // best of `reps` calls: total and per-class device times
  auto timed_opts = [&](const mce_opts_t &o, double *ms, double *cls) -> int {
    double best = 1e300;
    for (int c = 0; c < 3; ++c) cls[c] = 1e300;
    for (int r = 0; r < reps; ++r) {
      double t = 0, cm[3] = {0, 0, 0};
      uint64_t total = 0;
      const int rc = run(o, &t, &total, cm);
      if (rc) return rc;
      if (have && total != want) return MCE_ESTATE;  // a setting changed the count
      want = total;
      have = true;
      best = std::min(best, t);
      for (int c = 0; c < 3; ++c) cls[c] = std::min(cls[c], cm[c]);
      ++out->trials_run;
    }
    *ms = best;
    return MCE_OK;
  };
  auto timed = [&](const Knobs &k, double *ms) -> int {
    mce_opts_t o = base;
    apply(k, &o);
    double cls[3];
    return timed_opts(o, ms, cls);
  };
  Knobs cur = resolved(base);
  double cur_ms = 0;
  int rc = timed(cur, &cur_ms);
  if (rc) return rc;
  out->default_ms = cur_ms;
  struct Axis {
    int32_t Knobs::*field;
    std::vector<int32_t> values;
  };
  const Axis axes[] = {
      {&Knobs::donate_after, {64, 256, 1024}},
      {&Knobs::donate_threshold, {6, 10, 16}},
      {&Knobs::bitmap_width, {32, 64}},
      {&Knobs::peel_solo_max, {-1, 64}},
      {&Knobs::wide_blocks, {4, 8}},
      {&Knobs::x_pivot, {0, 1}},
  };
  for (const Axis &ax : axes) {
    if (cur.worker_list == MCE_WL_OFF &&
        (ax.field == &Knobs::donate_after || ax.field == &Knobs::donate_threshold))
      continue;  // no sharing: the donation knobs do nothing
    Knobs best = cur;
    double best_ms = cur_ms;
    for (int32_t v : ax.values) {
      if (v == cur.*(ax.field)) continue;
      Knobs k = cur;
      k.*(ax.field) = v;
      double ms = 0;
      if ((rc = timed(k, &ms))) return rc;
      if (ms < best_ms * 0.98) {
        best = k;
        best_ms = ms;
      }
    }
    cur = best;
    cur_ms = best_ms;
  }
  // per bucket: warps per root, donation threshold and gate, each scored by
  // the bucket's own launch time
  Entry ent{cur, cur_ms, out->default_ms, {}};
  mce_opts_t o = base;
  apply(cur, &o);
  double tot_ms = 0, cls_ms[3];
  if ((rc = timed_opts(o, &tot_ms, cls_ms))) return rc;
  const bool wl = cur.worker_list != MCE_WL_OFF;
  for (int c = 0; c < 3; ++c) {
    if (!(cls_ms[c] > 0 && cls_ms[c] < 1e299)) continue;  // no roots in this bucket
    Bucket b;
    b.warps = 1;
    b.threshold = cur.donate_threshold;
    b.after = cur.donate_after;
    b.default_ms = b.best_ms = cls_ms[c];
    b.present = true;
    struct BAxis {
      int32_t Bucket::*field;
      std::vector<int32_t> values;
      bool donation;
    };
    const BAxis baxes[] = {{&Bucket::warps, {1, 2, 4}, false},
                           {&Bucket::threshold, {6, 10, 16}, true},
                           {&Bucket::after, {64, 256, 1024}, true}};
    for (const BAxis &ax : baxes) {
      if (ax.donation && !wl) continue;
      Bucket best = b;
      for (int32_t v : ax.values) {
        if (v == b.*(ax.field)) continue;
        Bucket t = b;
        t.*(ax.field) = v;
        mce_opts_t ot = o;
        Bucket all[3];
        for (int k = 0; k < 3; ++k) all[k] = ent.b[k];
        all[c] = t;
        apply_buckets(all, &ot);
        double ms = 0, cm[3];
        if ((rc = timed_opts(ot, &ms, cm))) return rc;
        if (cm[c] < best.best_ms * 0.98) {
          best = t;
          best.best_ms = cm[c];
        }
      }
      b = best;
    }
    ent.b[c] = b;
  }
  apply(cur, &out->best);
  apply_buckets(ent.b, &out->best);
  {  // the whole call with every bucket's winner
    double cm[3];
    if ((rc = timed_opts(out->best, &cur_ms, cm))) return rc;
  }
  ent.best_ms = cur_ms;
  out->best_ms = cur_ms;
  if (table_path) {
    table[key] = ent;
    if ((rc = write_table(table_path, table))) return rc;
  }
  return MCE_OK;
}

}  // namespace

extern "C" int mce_shape_key(mce_graph_t g, char *key_out, size_t len) {
  if (!g || !key_out) return MCE_EINVAL;
  return shape_key(g, 0, key_out, len);
}

extern "C" int mce_batch_shape_key(mce_batch_t b, char *key_out, size_t len) {
  if (!b || !key_out) return MCE_EINVAL;
  int32_t G = 0;
  struct ::mce_graph *g = mce::batch_union(b, &G);
  return shape_key(g, G, key_out, len);
}

extern "C" int mce_tune_lookup(const char *table_path, const char *key, mce_opts_t *inout) {
  if (!table_path || !key || !inout) return MCE_EINVAL;
  std::map<std::string, Entry> t;
  if (!read_table(table_path, &t)) return MCE_EIO;
  auto it = t.find(key);
  if (it == t.end() || !(it->second.best_ms > 0)) return MCE_ESTATE;
  apply(it->second.k, inout);
  apply_buckets(it->second.b, inout);
  return MCE_OK;
}

extern "C" int mce_autotune(mce_graph_t g, const mce_opts_t *base, const char *table_path,
                            int32_t reps, int32_t force, mce_tune_result_t *out) {
  if (!g || !out) return MCE_EINVAL;
  mce_opts_t b;
  if (base)
    b = *base;
  else
    mce_opts_default(&b);
  char key[48];
  int rc = mce_shape_key(g, key, sizeof(key));
  if (rc) return rc;
  return tune(key, b, table_path, reps, force,
              [&](const mce_opts_t &o, double *ms, uint64_t *total, double *cls) {
                mce_stats_t st;
                const int r = mce_count(g, &o, total, nullptr, &st);
                *ms = st.total_ms;
                for (int c = 0; c < 3; ++c) cls[c] = st.class_ms[c];
                return r;
              },
              out);
}

extern "C" int mce_batch_autotune(mce_batch_t bt, const mce_opts_t *base, const char *table_path,
                                  int32_t reps, int32_t force, mce_tune_result_t *out) {
  if (!bt || !out) return MCE_EINVAL;
  mce_opts_t b;
  if (base) {
    b = *base;
  } else {
    mce_opts_default(&b);
    b.cuda_graph = 1;
  }
  char key[48];
  int rc = mce_batch_shape_key(bt, key, sizeof(key));
  if (rc) return rc;
  int32_t G = 0;
  mce::batch_union(bt, &G);
  std::vector<uint64_t> per((size_t)std::max(G, 1));
  return tune(key, b, table_path, reps, force,
              [&](const mce_opts_t &o, double *ms, uint64_t *total, double *cls) {
                mce_stats_t st;
                const int r = mce_batch_count(bt, &o, per.data(), total, nullptr, &st);
                *ms = st.total_ms;
                for (int c = 0; c < 3; ++c) cls[c] = st.class_ms[c];
                return r;
              },
              out);
}
