// hybrid_main.cpp -- the hybrid_sssp / hybrid_bfs / hybrid_cc / hybrid_pr command-line
// drop-ins (reference: samples/hybrid_*/main.cu + include/utils/app_skeleton.h flags,
// batch loops samples/hybrid_sssp/hybrid_sssp.cu:357-674, hybrid_cc.cu, hybrid_pr.cu),
// built on the C ABI of libdycg. The algorithm comes from the program name (or -algo).
// Log lines keep the reference's tags so its smoke scripts can parse them.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/dycg.h"

namespace {

std::map<std::string, std::string> g_flags;

std::string flag(const std::string &k, const std::string &dflt) {
  auto it = g_flags.find(k);
  return it == g_flags.end() ? dflt : it->second;
}
long long flag_i(const std::string &k, long long d) {
  auto s = flag(k, "");
  return s.empty() ? d : std::atoll(s.c_str());
}
double flag_f(const std::string &k, double d) {
  auto s = flag(k, "");
  return s.empty() ? d : std::atof(s.c_str());
}
bool flag_b(const std::string &k, bool d) {
  auto s = flag(k, "");
  if (s.empty()) return d;
  return s == "1" || s == "true" || s == "True" || s == "yes";
}

// gflags spellings: -f=v, --f=v, -f v, and bare boolean -f.
void parse(int argc, char **argv) {
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a.size() < 2 || a[0] != '-') continue;
    size_t s = a.find_first_not_of('-');
    std::string body = a.substr(s);
    size_t eq = body.find('=');
    if (eq != std::string::npos) {
      g_flags[body.substr(0, eq)] = body.substr(eq + 1);
    } else if (i + 1 < argc && argv[i + 1][0] != '-') {
      g_flags[body] = argv[++i];
    } else {
      g_flags[body] = "true";
    }
  }
}

struct Updates {
  std::vector<std::pair<uint32_t, uint32_t>> sizes;  // (adds, dels)
  std::vector<dycg_edge> adds, dels;
};

// include/framework/Loader.h:30-101: per-snapshot "adds dels" lines; all 'a'
// records in file order feed the adds, all 'd' records the deletions.
bool read_updates(const std::string &upd, const std::string &sizes, Updates &U) {
  std::ifstream fs(sizes);
  if (!fs) return false;
  std::string line;
  while (std::getline(fs, line)) {
    std::istringstream ss(line);
    uint32_t a = 0, d = 0;
    if (ss >> a >> d) U.sizes.push_back({a, d});
  }
  std::ifstream fu(upd);
  if (!fu) return false;
  while (std::getline(fu, line)) {
    std::istringstream ss(line);
    std::string t;
    uint32_t u, v, w = 1;
    if (!(ss >> t >> u >> v)) continue;
    if (!(ss >> w)) w = 1;
    dycg_edge e{u, v, w};
    if (t == "a") U.adds.push_back(e);
    else if (t == "d") U.dels.push_back(e);
  }
  return true;
}

// Binary stream "DYCGUPD1": sizes (adds, dels) per snapshot, then per snapshot
// its deletions followed by its insertions (12-byte records).
bool read_updates_binary(const std::string &path, Updates &U) {
  std::ifstream f(path, std::ios::binary);
  char magic[8];
  uint64_t hdr[3];
  if (!f.read(magic, 8) || std::memcmp(magic, "DYCGUPD1", 8) != 0) return false;
  if (!f.read(reinterpret_cast<char *>(hdr), sizeof hdr)) return false;
  std::vector<uint32_t> sz(hdr[0] * 2);
  if (!f.read(reinterpret_cast<char *>(sz.data()), sz.size() * 4)) return false;
  for (uint64_t b = 0; b < hdr[0]; b++) {
    U.sizes.push_back({sz[2 * b], sz[2 * b + 1]});
    std::vector<dycg_edge> d(sz[2 * b + 1]), a(sz[2 * b]);
    if (!d.empty() && !f.read(reinterpret_cast<char *>(d.data()), d.size() * 12)) return false;
    if (!a.empty() && !f.read(reinterpret_cast<char *>(a.data()), a.size() * 12)) return false;
    U.dels.insert(U.dels.end(), d.begin(), d.end());
    U.adds.insert(U.adds.end(), a.begin(), a.end());
  }
  return true;
}

uint64_t distance_checksum(const std::vector<uint32_t> &d) {
  // samples/hybrid_sssp/hybrid_sssp.cu:335-347
  uint64_t c = 1469598103934665603ull;
  for (uint64_t v = 0; v < d.size(); v++) {
    if (d[v] == DYCG_INFINITY) continue;
    c ^= v + 0x9e3779b97f4a7c15ull + ((uint64_t)d[v] << 6) + ((uint64_t)d[v] >> 2);
    c *= 1099511628211ull;
  }
  return c;
}

uint64_t parent_checksum(const std::vector<uint32_t> &d, const std::vector<uint32_t> &p) {
  // samples/hybrid_sssp/hybrid_sssp.cu:622-637
  uint64_t c = 1099511628211ull;
  for (uint64_t v = 0; v < d.size(); v++) {
    if (d[v] == DYCG_INFINITY) continue;
    c ^= v + 0x517cc1b727220a95ull + ((uint64_t)p[v] << 7) + ((uint64_t)p[v] >> 3);
    c *= 1469598103934665603ull;
  }
  return c;
}

struct Csr {
  std::vector<uint64_t> off;
  std::vector<uint32_t> dst, w;
};

bool export_csr(dycg_engine *e, uint32_t n, Csr &g) {
  dycg_graph_info gi;
  if (dycg_graph_info_get(e, &gi)) return false;
  g.off.assign(n + 1ull, 0);
  g.dst.assign(gi.live_edges + 1, 0);
  g.w.assign(gi.live_edges + 1, 0);
  return dycg_export_csr(e, g.off.data(), g.dst.data(), g.w.data()) == DYCG_OK;
}

uint32_t rule_w(uint32_t algo, uint32_t u, uint32_t v) {
  if (algo == DYCG_ALGO_BFS) return 1;
  if (algo == DYCG_ALGO_CC) return 0;
  return (uint32_t)(((uint64_t)u + v) % 128 + 1);
}

// CheckBellmanRelaxed (samples/hybrid_sssp/hybrid_sssp.cu:228-281): no edge
// relaxes further and every reachable vertex has a tight in-edge.
void bellman(const Csr &g, uint32_t algo, uint32_t source, const std::vector<uint32_t> &d,
             uint64_t &relax, uint64_t &missing) {
  const uint32_t n = (uint32_t)d.size();
  std::vector<uint8_t> tight(n, 0);
  if (algo != DYCG_ALGO_CC && source < n) tight[source] = 1;
  relax = 0;
  for (uint32_t u = 0; u < n; u++) {
    if (algo == DYCG_ALGO_CC && d[u] == u) tight[u] = 1;
    if (d[u] == DYCG_INFINITY) continue;
    for (uint64_t e = g.off[u]; e < g.off[u + 1]; e++) {
      const uint32_t v = g.dst[e];
      const uint64_t c = (uint64_t)d[u] + rule_w(algo, u, v);
      if (d[v] != DYCG_INFINITY && c == d[v]) tight[v] = 1;
      if (c < d[v]) relax++;
    }
  }
  missing = 0;
  for (uint32_t v = 0; v < n; v++)
    if (d[v] != DYCG_INFINITY && !tight[v]) missing++;
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

int fail(dycg_engine *e, const char *what, int rc) {
  char buf[512] = {0};
  if (e) dycg_last_error(e, buf, sizeof buf);
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, buf);
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  parse(argc, argv);
  std::string prog = argv[0];
  prog = prog.substr(prog.find_last_of('/') + 1);
  std::string algo_s = flag("algo", "");
  if (algo_s.empty()) {
    size_t p = prog.find("hybrid_");
    algo_s = p == std::string::npos ? "sssp" : prog.substr(p + 7);
  }
  uint32_t algo = algo_s == "bfs" ? DYCG_ALGO_BFS
                  : algo_s == "cc" ? DYCG_ALGO_CC
                  : algo_s == "pr" ? DYCG_ALGO_PR
                                   : DYCG_ALGO_SSSP;
  const char *TAG = algo == DYCG_ALGO_BFS ? "BFS" : algo == DYCG_ALGO_CC ? "CC"
                    : algo == DYCG_ALGO_PR ? "PR" : "SSSP";
  const std::string graphfile = flag("graphfile", "");
  if (graphfile.empty()) {
    std::fprintf(stderr, "usage: %s -graphfile=G [-updatefile=U -update_size=S] [flags]\n",
                 prog.c_str());
    return 2;
  }
  dycg_options o;
  dycg_options_default(&o);
  o.algo = algo;
  o.source = (uint32_t)std::max(0LL, flag_i("source_node", 0));
  o.segments = (uint32_t)std::max(1LL, flag_i("SEGMENT", 1));
  const long long cache = flag_i("cache", 0);
  // include/framework/graph_datum.cuh:164-176: -cache selects an edge capacity
  static const uint64_t cap_edges[5] = {0, 268435455ull, 536870921ull, 805306365ull,
                                        1073741824ull};
  uint64_t budget = cache >= 0 && cache <= 4 ? cap_edges[cache] * 4ull : 0;
  if (flag("hbm_graph_budget_mb", "") != "") budget = (uint64_t)flag_i("hbm_graph_budget_mb", 0) << 20;
  o.hbm_graph_budget_bytes = budget;
  o.cache_policy = budget ? DYCG_CACHE_HOTNESS : DYCG_CACHE_NONE;
  o.epsilon = (float)flag_f("error", 1e-6);
  o.max_rounds = (uint32_t)flag_i("pr_max_rounds", 100);
  o.device = 0;
  dycg_engine *e = nullptr;
  int rc = dycg_create(&o, &e);
  if (rc) return fail(nullptr, "dycg_create", rc);
  const std::string fmt = flag("format", "market_big");
  rc = fmt == "binary" ? dycg_load_graph_binary(e, graphfile.c_str())
                       : dycg_load_graph_file(e, graphfile.c_str(), 0, 0);
  if (rc) return fail(e, "load graph", rc);
  dycg_graph_info gi;
  dycg_graph_info_get(e, &gi);
  const uint32_t n = (uint32_t)gi.nodes;
  if (o.source >= n) o.source = n - 1;
  std::printf("[%s-LOAD] nodes=%u edges=%llu host_bytes=%llu cache_slots=%llu\n", TAG, n,
              (unsigned long long)gi.live_edges, (unsigned long long)gi.host_bytes,
              (unsigned long long)gi.cache_slots);
  double t0 = now_ms();
  rc = dycg_init(e);
  if (rc) return fail(e, "init", rc);
  std::printf("[%s-INITIAL] compute_ms=%.3f\n", TAG, now_ms() - t0);

  Updates U;
  const std::string updfile = flag("updatefile", ""), sizefile = flag("update_size", "");
  const bool upd_bin = flag("update_format", "") == "binary";
  if (!updfile.empty() && upd_bin && !read_updates_binary(updfile, U)) {
    std::fprintf(stderr, "cannot read binary update file\n");
    return 1;
  }
  if (!updfile.empty() && !upd_bin && !read_updates(updfile, sizefile, U)) {
    std::fprintf(stderr, "cannot read update files\n");
    return 1;
  }
  const long long max_b = flag_i(algo_s + "_max_batches", 10);
  const size_t nb = std::min<size_t>(U.sizes.size(), (size_t)std::max(0LL, max_b));
  const bool check = flag_b("check", true);
  std::vector<uint32_t> val(n), par(n);
  size_t ia = 0, id = 0;
  bool ok_all = true;
  auto do_check = [&](const char *stage, size_t b) {
    if (algo == DYCG_ALGO_PR) return;
    dycg_gather(e, val.data(), par.data());
    Csr g;
    export_csr(e, n, g);
    uint64_t relax = 0, missing = 0;
    bellman(g, algo, o.source, val, relax, missing);
    const bool ok = relax == 0 && missing == 0 &&
                    (algo == DYCG_ALGO_CC || val[o.source] == 0);
    ok_all &= ok;
    if (algo == DYCG_ALGO_CC)
      std::printf("[CC-%s-CHECK][batch %zu] %s errors=%llu label_checksum=%llu\n", stage, b,
                  ok ? "passed" : "failed", (unsigned long long)(relax + missing),
                  (unsigned long long)distance_checksum(val));
    else
      std::printf("[%s-%s-CHECK][batch %zu] %s source_ok=%d relaxable_edges=%llu "
                  "missing_tight_witnesses=%llu distance_checksum=%llu\n",
                  TAG, stage, b, ok ? "passed" : "failed", val[o.source] == 0 ? 1 : 0,
                  (unsigned long long)relax, (unsigned long long)missing,
                  (unsigned long long)distance_checksum(val));
  };
  for (size_t b = 0; b < nb; b++) {
    const uint32_t na = U.sizes[b].first, nd = U.sizes[b].second;
    if (ia + na > U.adds.size() || id + nd > U.dels.size()) {
      std::fprintf(stderr, "update file ended before batch %zu\n", b);
      return 1;
    }
    dycg_batch_stats sd{}, sa{}, sc{};
    double t = now_ms();
    if (algo == DYCG_ALGO_PR) {
      rc = dycg_apply_batch(e, U.dels.data() + id, nd, U.adds.data() + ia, na, &sa);
      if (rc) return fail(e, "batch", rc);
      const double ms = now_ms() - t;
      std::printf("[PR-BATCH] batch=%zu touched_sources=%llu rounds=%llu\n", b,
                  (unsigned long long)sa.touched_sources, (unsigned long long)sa.waves);
      std::printf("[P0-TIMER][PR][batch %zu] total_batch: %.3f ms\n", b, ms);
    } else {
      rc = dycg_delete_edges(e, U.dels.data() + id, nd, &sd);
      if (rc) return fail(e, "delete", rc);
      double ms = now_ms() - t;
      if (check) do_check("DELETE-STAGE", b);
      t = now_ms();
      rc = dycg_insert_edges(e, U.adds.data() + ia, na, &sa);
      if (rc) return fail(e, "insert", rc);
      rc = dycg_cache_maintenance(e, &sc);
      if (rc) return fail(e, "cache", rc);
      ms += now_ms() - t;
      std::printf("[P0-ATTR][%s][batch %zu] deletion=%.3f add=%.3f cache=%.3f affected=%llu "
                  "missing_deletes=%llu\n",
                  TAG, b, sd.ms_total, sa.ms_total, sc.ms_cache, (unsigned long long)sd.affected,
                  (unsigned long long)sd.missing_deletes);
      std::printf("[P0-TIMER][%s][batch %zu] total_batch: %.3f ms\n", TAG, b, ms);
      if (check) do_check("BATCH", b);
    }
    ia += na;
    id += nd;
  }
  const std::string out = flag("output", "");
  if (algo == DYCG_ALGO_PR) {
    std::vector<float> x(n), r(n);
    dycg_gather_ranks(e, x.data(), r.data());
    std::printf("[PR-FINAL] vertices=%u batches=%zu\n", n, nb);
    if (!out.empty()) {
      FILE *f = std::fopen(out.c_str(), "w");
      for (uint32_t v = 0; f && v < n; v++) std::fprintf(f, "%u %.9g %.9g\n", v, x[v], r[v]);
      if (f) std::fclose(f);
    }
  } else {
    dycg_gather(e, val.data(), par.data());
    uint64_t reach = 0;
    for (uint32_t v = 0; v < n; v++) reach += val[v] != DYCG_INFINITY;
    const bool print_ck = flag_b(algo_s + "_print_checksum", false);
    std::printf("[%s-FINAL-CHECK] final_reachable=%llu checksum=%s\n", TAG,
                (unsigned long long)reach, print_ck ? "enabled" : "disabled");
    if (print_ck)
      std::printf("[%s-FINAL-CHECK] distance_checksum=%llu parent_checksum=%llu\n", TAG,
                  (unsigned long long)distance_checksum(val),
                  (unsigned long long)parent_checksum(val, par));
    if (!out.empty()) {
      FILE *f = std::fopen(out.c_str(), "w");
      for (uint32_t v = 0; f && v < n; v++)
        std::fprintf(f, "%u %u %u %u\n", v, val[v], par[v], val[v]);
      if (f) std::fclose(f);
    }
  }
  dycg_destroy(e);
  return ok_all ? 0 : 3;
}
