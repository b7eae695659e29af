// gem — command-line drop-in for the reference's `GEM` executable
// (in-core/src/main.cu:23-275, out-of-core/src/main.cu:412-460), built on the
// C-ABI of libgem only.
//
//   gem -q <query file | directory of Q_<id>.in> -d <data graph> [-t N] [-g GPU]
//       [--eviction POLICY] [--ooc] [--budget-gb X] [--mode count|hash]
//       [--count-u32] [--time-cap-ms N] [--ooc-part-kib N] [--ooc-stream auto|always|never]
//
// Output lines follow the reference: per-phase "… time: <us> us" lines, two
// "Join Time" lines, "=== Final Results ===" and
// "Relaxed Query ET <32-bit edge set>: <count> matches", one line per
// relaxed query at -t T (default 2, like the reference; -t 0 is exact
// matching of the query alone).  The reference
// prints the count through a uint32_t (in-core/src/main.cu:233); this tool
// prints the exact u64 unless --count-u32 asks for the reference's truncation.
// A directory runs every Q_<id>.in in id order in one context and ends with
// the reference's "=== Batch Summary ===" block (out-of-core/src/main.cu
// :334-410); a failing query is reported and the batch continues.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dirent.h>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "gem.h"

namespace {

struct Args {
  std::string query, data, eviction = "lru", mode = "count";
  int gpu = 0;
  int threshold = 2;  // the reference's default (in-core/src/main.cu:31)
  bool ooc = false, u32 = false;
  double budget_gb = 0;
  unsigned time_cap_ms = 0;
  unsigned ooc_part_kib = 0;  // out-of-core adjacency partition (0 = library default)
  unsigned ooc_stream = 0;    // 0 auto, 1 always, 2 never
};

void usage() {
  std::fprintf(stderr,
               "usage: gem -q <query file|dir> -d <data graph> [-t 0..10] [-g GPU] [--eviction P]\n"
               "           [--ooc] [--budget-gb X] [--mode count|hash] [--count-u32] [--time-cap-ms N]\n"
               "           [--ooc-part-kib N] [--ooc-stream auto|always|never]\n");
}

bool parse(int argc, char **argv, Args &a) {
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto need = [&](const char *what) -> const char * {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "ERROR: %s needs a value\n", what);
        return nullptr;
      }
      return argv[++i];
    };
    const char *v = nullptr;
    if (s == "-q" || s == "--query") {
      if (!(v = need("-q"))) return false;
      a.query = v;
    } else if (s == "-d" || s == "--data") {
      if (!(v = need("-d"))) return false;
      a.data = v;
    } else if (s == "-g" || s == "--gpu") {
      if (!(v = need("-g"))) return false;
      a.gpu = std::atoi(v);
    } else if (s == "-t" || s == "--threshold") {
      if (!(v = need("-t"))) return false;
      a.threshold = std::atoi(v);
      if (a.threshold < 0 || a.threshold > 10) {
        std::fprintf(stderr, "ERROR: --threshold must be in [0, 10]\n");
        return false;
      }
    } else if (s == "--eviction") {
      if (!(v = need("--eviction"))) return false;
      a.eviction = v;
    } else if (s == "--ooc") {
      a.ooc = true;
    } else if (s == "--budget-gb") {
      if (!(v = need("--budget-gb"))) return false;
      a.budget_gb = std::atof(v);
    } else if (s == "--mode") {
      if (!(v = need("--mode"))) return false;
      a.mode = v;
    } else if (s == "--count-u32") {
      a.u32 = true;
    } else if (s == "--time-cap-ms") {
      if (!(v = need("--time-cap-ms"))) return false;
      a.time_cap_ms = (unsigned)std::atoi(v);
    } else if (s == "--ooc-part-kib") {
      if (!(v = need("--ooc-part-kib"))) return false;
      a.ooc_part_kib = (unsigned)std::atoi(v);
    } else if (s == "--ooc-stream") {
      if (!(v = need("--ooc-stream"))) return false;
      const std::string m = v;
      if (m == "auto") a.ooc_stream = 0;
      else if (m == "always") a.ooc_stream = 1;
      else if (m == "never") a.ooc_stream = 2;
      else {
        std::fprintf(stderr, "ERROR: --ooc-stream must be auto, always or never\n");
        return false;
      }
    } else if (s == "-h" || s == "--help") {
      return false;
    } else {
      std::fprintf(stderr, "ERROR: unknown option %s\n", s.c_str());
      return false;
    }
  }
  if (a.query.empty() || a.data.empty()) {
    std::fprintf(stderr, "ERROR: -q and -d are required\n");
    return false;
  }
  return true;
}

// Parses Q_<id>.in / q-<id>.in / <id>.in like the reference's tryParseQueryId.
bool query_id(const std::string &name, unsigned &id) {
  std::string stem = name;
  size_t dot = stem.rfind('.');
  if (dot != std::string::npos) stem = stem.substr(0, dot);
  size_t p = 0;
  if (p < stem.size() && (stem[p] == 'Q' || stem[p] == 'q')) ++p;
  if (p < stem.size() && (stem[p] == '_' || stem[p] == '-')) ++p;
  if (p >= stem.size()) return false;
  unsigned long v = 0;
  for (size_t i = p; i < stem.size(); ++i) {
    if (!std::isdigit((unsigned char)stem[i])) return false;
    v = v * 10 + (unsigned)(stem[i] - '0');
    if (v > 0xFFFFFFFFul) return false;
  }
  id = (unsigned)v;
  return true;
}

struct Job {
  unsigned id;
  std::string path, file;
};

int run_one(gem_ctx *ctx, const Job &job, const Args &a) {
  uint32_t nv = 0, ne = 0;
  std::vector<uint32_t> lab(GEM_MAX_QV), edges(2 * GEM_MAX_QE);
  gem_status st = gem_query_read_text(job.path.c_str(), &nv, &ne, lab.data(), edges.data());
  if (st != GEM_OK) {
    std::fprintf(stderr, "ERROR: cannot read query %s: %s\n", job.path.c_str(), gem_strerror(st));
    return 1;
  }
  gem_query q{nv, ne, lab.data(), edges.data()};
  const int mode = a.mode == "hash" ? GEM_MODE_HASH : GEM_MODE_COUNT;
  // the relaxed queries (only q itself at -t 0), counted in one batch
  const uint32_t cap = 1u << 16;
  std::vector<uint64_t> ets(cap);
  std::vector<gem_result> rs(cap);
  uint32_t nrq = 0;
  if (a.threshold == 0) {
    st = gem_query_run(ctx, &q, 0, mode, nullptr, 0, &rs[0]);
    ets[0] = ne >= 64 ? ~0ull : (1ull << ne) - 1ull;
    nrq = 1;
  } else {
    st = gem_relaxed_run(ctx, &q, (uint32_t)a.threshold, mode, cap, ets.data(), rs.data(), &nrq);
  }
  if (st != GEM_OK) {
    std::fprintf(stderr, "ERROR: query %s: %s (%s)\n", job.path.c_str(), gem_strerror(st), gem_last_error(ctx));
    return st == GEM_ERR_LIMIT ? 3 : 2;
  }
  const gem_result &r = rs[0];
  std::printf("Filter time: %lld us\n", (long long)(r.ms[GEM_PH_FILTER] * 1000.0f));
  std::printf("Build Hash Table time: %lld us\n", (long long)(r.ms[GEM_PH_INDEX] * 1000.0f));
  std::printf("initVertexTries time: %d us\n", 0);
  std::printf("construct time: %lld us\n", (long long)(r.ms[GEM_PH_TABLES] * 1000.0f));
  std::printf("Join Time: %lld us\n", (long long)(r.ms[GEM_PH_JOIN] * 1000.0f));
  std::printf("Join Time: %lld ms\n", (long long)(r.ms[GEM_PH_JOIN]));
  std::printf("\n=== Final Results ===\n");
  for (uint32_t i = 0; i < nrq; ++i) {
    char bits[33];
    for (int b = 0; b < 32; ++b) bits[31 - b] = ((ets[i] >> b) & 1u) ? '1' : '0';
    bits[32] = 0;
    if (a.u32)
      std::printf("Relaxed Query ET %s: %u matches\n", bits, (unsigned)(uint32_t)rs[i].count);
    else
      std::printf("Relaxed Query ET %s: %llu matches\n", bits, (unsigned long long)rs[i].count);
    if (mode == GEM_MODE_HASH) std::printf("Embedding hash: %016llx\n", (unsigned long long)rs[i].emb_hash);
  }
  std::printf("\n");
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  Args a;
  if (!parse(argc, argv, a)) {
    usage();
    return 1;
  }
  std::vector<Job> jobs;
  bool is_dir = false;
  struct stat sb;
  if (stat(a.query.c_str(), &sb) != 0) {
    std::fprintf(stderr, "ERROR: Query path is not a file or directory: %s\n", a.query.c_str());
    return 1;
  }
  if (S_ISDIR(sb.st_mode)) {
    is_dir = true;
    DIR *d = opendir(a.query.c_str());
    if (!d) return 1;
    std::vector<unsigned> seen;
    while (dirent *e = readdir(d)) {
      std::string f = e->d_name;
      if (f.size() < 4 || f.substr(f.size() - 3) != ".in") continue;
      unsigned id;
      if (!query_id(f, id)) {
        std::fprintf(stderr, "ERROR: Query file does not match expected pattern Q_<id>.in: %s\n", f.c_str());
        closedir(d);
        return 1;
      }
      if (std::find(seen.begin(), seen.end(), id) != seen.end()) {
        std::fprintf(stderr, "ERROR: Duplicate query id %u in directory: %s\n", id, a.query.c_str());
        closedir(d);
        return 1;
      }
      seen.push_back(id);
      jobs.push_back({id, a.query + "/" + f, f});
    }
    closedir(d);
    std::sort(jobs.begin(), jobs.end(), [](const Job &x, const Job &y) { return x.id < y.id; });
    if (jobs.empty()) {
      std::fprintf(stderr, "ERROR: No query graphs found in: %s\n", a.query.c_str());
      return 1;
    }
  } else {
    unsigned id = 0;
    std::string f = a.query.substr(a.query.find_last_of('/') == std::string::npos ? 0 : a.query.find_last_of('/') + 1);
    if (!query_id(f, id)) id = 0;
    jobs.push_back({id, a.query, f});
  }
  gem_hgraph *hg = nullptr;
  gem_status st = gem_hgraph_read_text(a.data.c_str(), &hg);
  if (st != GEM_OK) {
    std::fprintf(stderr, "ERROR: cannot read data graph %s: %s\n", a.data.c_str(), gem_strerror(st));
    return 1;
  }
  gem_opts o;
  std::memset(&o, 0, sizeof o);
  o.device = a.gpu;
  o.device_budget_bytes = (uint64_t)(a.budget_gb * (1ull << 30));
  o.ooc = a.ooc ? 1 : 0;
  o.time_cap_ms = a.time_cap_ms;
  o.ooc_part_kib = a.ooc_part_kib;
  o.ooc_stream = a.ooc_stream;
  gem_ctx *ctx = nullptr;
  st = gem_ctx_create(&o, &ctx);
  if (st == GEM_OK) st = gem_ctx_load_graph(ctx, hg);
  if (st != GEM_OK) {
    std::fprintf(stderr, "ERROR: device setup failed: %s (%s)\n", gem_strerror(st), ctx ? gem_last_error(ctx) : "");
    gem_hgraph_destroy(hg);
    if (ctx) gem_ctx_destroy(ctx);
    return 2;
  }
  int rc = 0;
  if (!is_dir) {
    rc = run_one(ctx, jobs[0], a);
  } else {
    int ok = 0;
    std::vector<std::pair<Job, int>> failed;
    for (const Job &j : jobs) {
      std::printf("%u\n", j.id);
      std::fflush(stdout);
      int r = run_one(ctx, j, a);
      if (r == 0) {
        ++ok;
      } else {
        failed.push_back({j, r});
        std::printf("[batch-fail] query %u file=%s exit=%d continuing\n", j.id, j.file.c_str(), r);
      }
    }
    std::printf("=== Batch Summary ===\n");
    std::printf("success=%d failed=%zu\n", ok, failed.size());
    for (auto &f : failed) std::printf("[failed] query %u file=%s exit=%d\n", f.first.id, f.first.file.c_str(), f.second);
  }
  gem_ctx_destroy(ctx);
  gem_hgraph_destroy(hg);
  return rc;
}
