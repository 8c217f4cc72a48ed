// parallel_mce_on_gpus: the command-line drop-in, a thin client of libmce.so.
//
// Options and output follow the reference's CLI (include/config.h:141-291,
// src/main.cu:18-187) so that its experiment scripts (run.py, table.py)
// parse this program's stdout unchanged:
//   Degeneracy ordering time: %f s / count time %f s /
//   Found N maximal cliques in total. / Parallelization Scheme = ... etc.
// Errors in the options print to stderr and exit(0), as the reference does;
// a failing library call prints its message and exits 1.
#include <getopt.h>
#include <sys/time.h>
#include <time.h>

#include <cctype>
#include <cstdarg>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mce.h"

namespace {

enum Task { TASK_UNKNOWN, TASK_CONVERT, TASK_MCE, TASK_LB, TASK_BD, TASK_DONOR };

struct Config {
  std::string src, dst;
  Task task = TASK_UNKNOWN;
  int level = 0, induced = 0, wl = 0;
  std::vector<int> gpus;
  int bitmap_width = 0, sched = MCE_SCHED_PLAIN;
  bool print_hist = false;
};

// Log(info, ...) of include/logger.h:4-42: colour, [HH:MM:SS], message.
void log_info(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
void log_info(const char *fmt, ...) {
  std::printf("\033[1;32m");
  time_t raw;
  time(&raw);
  struct tm *ti = localtime(&raw);
  std::printf("[%02d:%02d:%02d] ", ti->tm_hour, ti->tm_min, ti->tm_sec);
  va_list ap;
  va_start(ap, fmt);
  std::vprintf(fmt, ap);
  va_end(ap);
  std::printf("\n\033[0m");
}

[[noreturn]] void fail(const char *what, int rc) {
  std::fprintf(stderr, "\033[1;31m%s failed: %s (%d)\033[0m\n", what, mce_strerror(rc), rc);
  std::exit(1);
}

void usage() {
  std::fprintf(stderr,
               "\nUsage:  ./parallel_mce_on_gpus [options]"
               "\n"
               "\nOptions:"
               "\n    -g <Src graph FileName>       Name of file with source graph"
               "\n    -r <Dst graph FileName>       Name of file with destination graph only for conversion"
               "\n    -d <Device Id(s)>             GPU Device Id(s) separated by commas without spaces"
               "\n    -m <Main Task>                Name of the task to perform <convert: graph conversion, mce, mce-lb-eval: load balance evaluation, mce-bd-eval: breakdown evaluation, mce-donor-eval: donation evaluation>"
               "\n    -p <Parallelization Scheme>   Level of subtrees to parallelize <l1: first level, l2: second level>"
               "\n    -i <Induced Subgraphs Scheme> Building induced subgraphs from which sets <p: P only, px: P and X>"
               "\n    -w <Worker List Scheme>       Use worker list to achieve load balance or not <nowl: No worker list, wl: Use worker list>"
               "\n    -h                            Help"
               "\n    --bitmap-width <32|64>        Word width of 32-wide induced-subgraph rows (default: auto)"
               "\n    --sched <plain|degree|learned> Root scheduling (default: plain)"
               "\n    --hist                        Print the clique-size histogram"
               "\n"
               "\n");
}

// parseDevice (include/config.h:112-127): every run of digits is an id.
std::vector<int> parse_devices(const std::string &s) {
  std::vector<int> res;
  for (size_t i = 0; i < s.size(); ++i) {
    if (!std::isdigit((unsigned char)s[i])) continue;
    int cur = 0;
    size_t j = i;
    while (j < s.size() && std::isdigit((unsigned char)s[j])) cur = cur * 10 + (s[j++] - '0');
    res.push_back(cur);
    i = j;
  }
  return res;
}

Config parse_args(int argc, char **argv) {
  Config c;
  static const struct option longopts[] = {{"bitmap-width", required_argument, nullptr, 1},
                                           {"sched", required_argument, nullptr, 2},
                                           {"hist", no_argument, nullptr, 3},
                                           {nullptr, 0, nullptr, 0}};
  int opt;
  while ((opt = getopt_long(argc, argv, "g:r:d:m:p:i:w:h", longopts, nullptr)) >= 0) {
    const std::string a = optarg ? optarg : "";
    switch (opt) {
      case 'g': c.src = a; break;
      case 'r': c.dst = a; break;
      case 'd': c.gpus = parse_devices(a); break;
      case 'm':
        if (a == "convert") c.task = TASK_CONVERT;
        else if (a == "mce") c.task = TASK_MCE;
        else if (a == "mce-lb-eval") c.task = TASK_LB;
        else if (a == "mce-bd-eval") c.task = TASK_BD;
        else if (a == "mce-donor-eval") c.task = TASK_DONOR;
        else {
          std::fprintf(stderr, "Unrecognized -m option (Main Task): %s\n", a.c_str());
          std::exit(0);
        }
        break;
      case 'p':
        if (a == "l1") c.level = MCE_LEVEL_L1;
        else if (a == "l2") c.level = MCE_LEVEL_L2;
        else {
          std::fprintf(stderr, "Unrecognized -p option (Parallelization Scheme): %s\n", a.c_str());
          std::exit(0);
        }
        break;
      case 'i':
        if (a == "p") c.induced = MCE_INDUCED_P;
        else if (a == "px") c.induced = MCE_INDUCED_PX;
        else {
          std::fprintf(stderr, "Unrecognized -i option (Induced Subgraphs Scheme): %s\n", a.c_str());
          std::exit(0);
        }
        break;
      case 'w':
        if (a == "nowl") c.wl = MCE_WL_OFF;
        else if (a == "wl") c.wl = MCE_WL_ON;
        else {
          std::fprintf(stderr, "Unrecognized -w option (Worker List Scheme): %s\n", a.c_str());
          std::exit(0);
        }
        break;
      case 'h': usage(); std::exit(0);
      case 1: c.bitmap_width = std::atoi(a.c_str()); break;
      case 2:
        c.sched = a == "degree" ? MCE_SCHED_DEGREE : a == "learned" ? MCE_SCHED_LEARNED : MCE_SCHED_PLAIN;
        break;
      case 3: c.print_hist = true; break;
      default:
        std::fprintf(stderr, "\nUnrecognized option!\n");
        usage();
        std::exit(0);
    }
  }
  auto need = [](bool ok, const char *msg) {
    if (!ok) {
      std::fprintf(stderr, "%s\n", msg);
      std::exit(0);
    }
  };
  if (c.task == TASK_UNKNOWN) {
    std::fprintf(stderr, "Must specify -m option (Main Task)\n");
    usage();
    std::exit(0);
  }
  need(!c.src.empty(), "Must specify -g option (Src graph FileName)");
  if (c.task == TASK_CONVERT) {
    need(!c.dst.empty(), "Must specify -r option (Dst graph FileName)");
    return c;
  }
  need(!c.gpus.empty(), "Must specify -d option (Device Ids)");
  need(c.level != 0, "Must specify -p option (Parallelization Scheme)");
  need(c.induced != 0, "Must specify -i option (Induced Subgraphs Scheme)");
  need(c.wl != 0, "Must specify -w option (Worker List Scheme)");
  need(!(c.task == TASK_BD && c.wl == MCE_WL_OFF), "No breakdown for kernels without worker list");
  need(!(c.task == TASK_DONOR && c.wl == MCE_WL_OFF), "No donoation for kernels without worker list");
  need(c.task == TASK_MCE || c.gpus.size() == 1,
       "Must use only one GPU to evaluate load balance, time breakdown or donation");
  return c;
}

const char *task_name(Task t) {
  switch (t) {
    case TASK_CONVERT: return "convert";
    case TASK_MCE: return "mce";
    case TASK_LB: return "mce-lb-eval";
    case TASK_BD: return "mce-bd-eval";
    case TASK_DONOR: return "mce-donor-eval";
    default: return "unknown";
  }
}

void print_config(const Config &c) {
  std::printf("    Main Task = %s\n", task_name(c.task));
  std::printf("    Source Graph = %s\n", c.src.c_str());
  if (c.task == TASK_CONVERT) {
    std::printf("    Destination Graph = %s\n", c.dst.c_str());
  } else {
    std::printf("    Parallelization Scheme = %s trees\n", c.level == MCE_LEVEL_L1 ? "L1" : "L2");
    std::printf("    Induced Subgraphs Scheme = %s\n", c.induced == MCE_INDUCED_P ? "IP" : "IPX");
    std::printf("    Worker List Scheme = %s\n", c.wl == MCE_WL_ON ? "Worker List" : "No Worker List");
    std::string ids;
    for (size_t i = 0; i < c.gpus.size(); ++i) ids += (i ? "," : "") + std::to_string(c.gpus[i]);
    std::printf("    Device ID(s) = %s\n", ids.c_str());
  }
  std::printf("-----------------------------\n");
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char **argv) {
  Config c = parse_args(argc, argv);
  std::printf("\033[0m");
  std::printf("Welcome ---------------------\n");
  print_config(c);

  if (c.task == TASK_CONVERT) {
    // on the first device when there is one; the host converter (the
    // reference's own path, include/fileop.h:13-79) writes the same file
    int64_t n = 0, e = 0;
    int rc = mce_convert_to_bel_device(c.src.c_str(), c.dst.c_str(), c.gpus.empty() ? 0 : c.gpus[0],
                                       nullptr, &n, &e);
    if (rc == MCE_ENODEV) rc = mce_convert_to_bel(c.src.c_str(), c.dst.c_str(), &n, &e);
    if (rc) fail("convert", rc);
    std::printf("n = %lld and m = %lld\n", (long long)n, (long long)e);
    return 0;
  }
  if (c.gpus.size() > 1)
    std::fprintf(stderr, "warning: this build runs on one GPU; using device %d\n", c.gpus[0]);

  double t0 = now_s();
  mce_hgraph_t hg;
  std::memset(&hg, 0, sizeof(hg));
  int rc = mce_bel_read(c.src.c_str(), &hg);
  if (rc) fail("read_bel", rc);
  log_info("Read graph time: %f s", now_s() - t0);
  log_info("n = %u and m = %u", (unsigned)hg.n, (unsigned)hg.m);

  t0 = now_s();
  mce_graph_t g = nullptr;
  rc = mce_graph_upload(hg.row_ptr, hg.col, hg.n, hg.m, c.gpus[0], nullptr, &g);
  if (rc) fail("upload", rc);
  log_info("Transfer Time: %f s", now_s() - t0);

  mce_opts_t o;
  mce_opts_default(&o);
  o.level = c.level;
  o.induced = c.induced;
  o.worker_list = c.wl;
  o.bitmap_width = c.bitmap_width;
  o.sched = c.sched;
  o.warp_log = (c.task == TASK_LB || c.task == TASK_DONOR) ? 1 : c.task == TASK_BD ? 2 : 0;
  uint64_t total = 0;
  std::vector<uint64_t> hist(MCE_HIST_MAX, 0);
  mce_stats_t st;
  std::memset(&st, 0, sizeof(st));
  rc = mce_count(g, &o, &total, hist.data(), &st);
  if (rc) fail("count", rc);
  std::printf("Max Core = %d\n", st.degeneracy);
  log_info("Degeneracy ordering time: %f s", st.peel_ms / 1e3);
  log_info("CSR Recreation time: %f s", st.orient_ms / 1e3);
  if (o.warp_log) {
    // per-unit load lines as the reference's evaluation kernels print them
    // (mce/mce.cuh:385-390); the unit here is a search warp
    int64_t k = 0;
    rc = mce_warp_log(g, nullptr, nullptr, nullptr, nullptr, 0, &k);
    std::vector<uint32_t> sm((size_t)k);
    std::vector<uint64_t> nodes((size_t)k), don((size_t)k), cyc(7 * (size_t)k);
    if (!rc) rc = mce_warp_log(g, sm.data(), nodes.data(), don.data(), cyc.data(), k, &k);
    if (rc) fail("warp_log", rc);
    if (c.task == TASK_BD) {
      std::printf("OTHER, BUILDING INDUCED SUBGRAPHS, WORKER LIST, SELECTING PIVOTS, SET "
                  "OPERATIONS, TESTING MAXIMALITY, BRANCHING AND BACKTRACKING\n");
      for (int64_t i = 0; i < k; ++i) {
        const uint64_t *r = &cyc[7 * (size_t)i];
        std::printf("%llu, %llu, %llu, %llu, %llu, %llu, %llu\n", (unsigned long long)r[0],
                    (unsigned long long)r[1], (unsigned long long)r[2], (unsigned long long)r[3],
                    (unsigned long long)r[4], (unsigned long long)r[5], (unsigned long long)r[6]);
      }
    } else {
      std::printf(c.task == TASK_LB ? "BLOCK ID, SM ID, Number of traversed nodes\n"
                                    : "BLOCK ID, SM ID, Number of donations\n");
      for (int64_t i = 0; i < k; ++i)
        std::printf("%lld, %u, %llu\n", (long long)i, sm[(size_t)i],
                    (unsigned long long)(c.task == TASK_LB ? nodes[(size_t)i] : don[(size_t)i]));
    }
  }
  std::printf("Finished Launching Instance 0.\n");
  log_info("count time %f s", st.count_ms / 1e3);
  std::printf("Instance 0 found %llu maximal cliques.\n", (unsigned long long)total);
  std::printf("Found %llu maximal cliques in total.\n", (unsigned long long)total);
  if (c.print_hist)
    for (int s = 0; s < MCE_HIST_MAX; ++s)
      if (hist[s]) std::printf("size %d: %llu\n", s, (unsigned long long)hist[s]);
  mce_graph_free(g);
  mce_hgraph_free(&hg);
  std::printf("Done ...\n");
  return 0;
}
