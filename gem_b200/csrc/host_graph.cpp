// Host-side graph construction: R-MAT generation, label assignment, the t/v/e
// text format and random-walk query extraction.
//
// The text reader replaces readGraphToCPUStandard
// (in-core/lib/io/src/io.cu:45-220).  Differences, all deliberate: vertex
// lines may come in any order (the reference derives offsets from the running
// sum of declared degrees, so it needs ascending vertex lines), declared
// degrees are checked against the edges, adjacency lists are sorted (the
// reference keeps file order, which is sorted only for lexicographically
// sorted edge lines), and labels keep their values (the reference remaps query
// labels to first-seen order and data labels absent from the query to one
// sentinel; label equality, the only thing the matcher uses, is the same).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <memory>
#include <omp.h>

#include "gem_internal.h"

void gem_hgraph::refresh_stats() {
  max_label_plus1 = 0;
  max_degree = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    max_label_plus1 = std::max(max_label_plus1, lab[v] + 1);
    max_degree = std::max<uint32_t>(max_degree, (uint32_t)(off[v + 1] - off[v]));
  }
}

namespace gem {

void radix_sort_u64(std::vector<uint64_t> &keys, uint32_t bits) {
  const size_t n = keys.size();
  if (n < 2) return;
  const int RB = 11, R = 1 << RB;
  std::vector<uint64_t> tmp(n);
  int nt = omp_get_max_threads();
  std::vector<size_t> hist((size_t)nt * R);
  for (uint32_t shift = 0; shift < bits; shift += RB) {
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
    {
      int t = omp_get_thread_num();
      size_t lo = n * t / nt, hi = n * (t + 1) / nt;
      size_t *h = &hist[(size_t)t * R];
      for (size_t i = lo; i < hi; ++i) h[(keys[i] >> shift) & (R - 1)]++;
#pragma omp barrier
#pragma omp single
      {
        size_t sum = 0;
        for (int d = 0; d < R; ++d)
          for (int tt = 0; tt < nt; ++tt) {
            size_t c = hist[(size_t)tt * R + d];
            hist[(size_t)tt * R + d] = sum;
            sum += c;
          }
      }
      for (size_t i = lo; i < hi; ++i) {
        uint64_t k = keys[i];
        tmp[h[(k >> shift) & (R - 1)]++] = k;
      }
    }
    keys.swap(tmp);
  }
}

gem_status make_host_query(const gem_query *q, HostQuery &out, std::string &err) {
  if (!q) { err = "null query"; return GEM_ERR_ARG; }
  if (q->nv == 0 || q->nv > GEM_MAX_QV) {
    err = "query vertex count must be in 1.." + std::to_string(GEM_MAX_QV);
    return q->nv == 0 ? GEM_ERR_ARG : GEM_ERR_LIMIT;
  }
  if (q->ne > GEM_MAX_QE) { err = "too many query edges"; return GEM_ERR_LIMIT; }
  if (!q->labels || (q->ne && !q->edges)) { err = "null query arrays"; return GEM_ERR_ARG; }
  out.nv = q->nv;
  out.ne = q->ne;
  for (uint32_t u = 0; u < q->nv; ++u) { out.lab[u] = q->labels[u]; out.adj[u] = 0; }
  out.edges.assign(q->edges, q->edges + 2 * (size_t)q->ne);
  for (uint32_t e = 0; e < q->ne; ++e) {
    uint32_t a = q->edges[2 * e], b = q->edges[2 * e + 1];
    if (a >= q->nv || b >= q->nv) { err = "query edge endpoint out of range"; return GEM_ERR_ARG; }
    if (a == b) { err = "query self loop"; return GEM_ERR_ARG; }
    if (out.adj[a] & (1u << b)) { err = "duplicate query edge"; return GEM_ERR_ARG; }
    out.adj[a] |= 1u << b;
    out.adj[b] |= 1u << a;
  }
  // connectivity
  uint32_t seen = 1u, frontier = 1u;
  while (frontier) {
    uint32_t nxt = 0;
    for (uint32_t u = 0; u < q->nv; ++u)
      if (frontier & (1u << u)) nxt |= out.adj[u];
    nxt &= ~seen;
    seen |= nxt;
    frontier = nxt;
  }
  uint32_t all = q->nv == 32 ? 0xFFFFFFFFu : ((1u << q->nv) - 1);
  if (seen != all) { err = "query graph is not connected"; return GEM_ERR_ARG; }
  return GEM_OK;
}

}  // namespace gem

using namespace gem;

// Builds a symmetric CSR with sorted adjacency from canonical (lo, hi) keys
// packed as lo << sh | hi (sorted, unique, lo < hi).
static void csr_from_sorted_pairs(gem_hgraph &g, std::vector<uint64_t> &keys, uint32_t sh) {
  const uint64_t mask = (1ull << sh) - 1;
  const uint32_t nv = g.nv;
  const size_t m = keys.size();
  // Transposed copy (hi, lo), sorted: gives every vertex its lower neighbours.
  std::vector<uint64_t> tk(m);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < m; ++i) tk[i] = ((keys[i] & mask) << sh) | (keys[i] >> sh);
  radix_sort_u64(tk, 2 * sh);
  auto first_of = [&](const std::vector<uint64_t> &k, uint32_t v) -> size_t {
    return (size_t)(std::lower_bound(k.begin(), k.end(), (uint64_t)v << sh) - k.begin());
  };
  std::vector<uint64_t> up(nv + 1), lo(nv + 1);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v <= (int64_t)nv; ++v) {
    up[v] = first_of(keys, (uint32_t)v);
    lo[v] = first_of(tk, (uint32_t)v);
  }
  g.off.assign(nv + 1, 0);
  for (uint32_t v = 0; v < nv; ++v)
    g.off[v + 1] = g.off[v] + (up[v + 1] - up[v]) + (lo[v + 1] - lo[v]);
  g.nbr.resize(g.off[nv]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < (int64_t)nv; ++v) {
    uint64_t p = g.off[v];
    for (size_t i = lo[v]; i < lo[v + 1]; ++i) g.nbr[p++] = (uint32_t)(tk[i] & mask);
    for (size_t i = up[v]; i < up[v + 1]; ++i) g.nbr[p++] = (uint32_t)(keys[i] & mask);
  }
}

extern "C" {

gem_status gem_hgraph_create(uint32_t nv, const uint64_t *offsets, const uint32_t *nbrs,
                             const uint32_t *labels, gem_hgraph **out) {
  if (!out || !offsets || !labels || (offsets[nv] && !nbrs)) return GEM_ERR_ARG;
  *out = nullptr;
  if (offsets[0] != 0) return GEM_ERR_ARG;
  for (uint32_t v = 0; v < nv; ++v)
    if (offsets[v + 1] < offsets[v]) return GEM_ERR_ARG;
  std::unique_ptr<gem_hgraph> g(new gem_hgraph());
  g->nv = nv;
  g->off.assign(offsets, offsets + nv + 1);
  g->nbr.assign(nbrs, nbrs + offsets[nv]);
  g->lab.assign(labels, labels + nv);
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < (int64_t)nv; ++v) {
    for (uint64_t i = g->off[v]; i < g->off[v + 1]; ++i) {
      uint32_t w = g->nbr[i];
      if (w >= nv || w == (uint32_t)v || (i > g->off[v] && g->nbr[i - 1] >= w)) { bad = 1; break; }
      // reverse arc present
      const uint32_t *b = g->nbr.data() + g->off[w], *e = g->nbr.data() + g->off[w + 1];
      if (!std::binary_search(b, e, (uint32_t)v)) { bad = 1; break; }
    }
  }
  if (bad) return GEM_ERR_ARG;
  g->refresh_stats();
  *out = g.release();
  return GEM_OK;
}

gem_status gem_hgraph_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                           uint64_t seed, gem_hgraph **out) {
  if (!out || scale == 0 || scale > 31 || edge_factor == 0) return GEM_ERR_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return GEM_ERR_ARG;
  *out = nullptr;
  const uint32_t nv = 1u << scale;
  const uint64_t m = (uint64_t)edge_factor << scale;
  const uint64_t ta = (uint64_t)(a * 9007199254740992.0);
  const uint64_t tb = (uint64_t)((a + b) * 9007199254740992.0);
  const uint64_t tc = (uint64_t)((a + b + c) * 9007199254740992.0);
  const uint32_t sh = scale;
  std::vector<uint64_t> keys(m);
  const uint64_t drop = ~0ull;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i) {
    uint64_t s = rng_at(seed, (uint64_t)i);
    uint32_t src = 0, dst = 0;
    for (uint32_t lvl = 0; lvl < scale; ++lvl) {
      s = mix64(s);
      uint64_t r = s >> 11;
      uint32_t bs = 0, bd = 0;
      if (r < ta) {
      } else if (r < tb) {
        bd = 1;
      } else if (r < tc) {
        bs = 1;
      } else {
        bs = 1;
        bd = 1;
      }
      src = (src << 1) | bs;
      dst = (dst << 1) | bd;
    }
    if (src == dst) {
      keys[i] = drop;
    } else {
      uint32_t lo = std::min(src, dst), hi = std::max(src, dst);
      keys[i] = ((uint64_t)lo << sh) | hi;
    }
  }
  radix_sort_u64(keys, 2 * sh + (2 * sh < 64 ? 1 : 0));  // drop marker sorts last
  // unique + strip drop markers
  size_t w = 0;
  for (size_t i = 0; i < keys.size(); ++i) {
    if (keys[i] == drop) break;
    if (w == 0 || keys[w - 1] != keys[i]) keys[w++] = keys[i];
  }
  keys.resize(w);
  keys.shrink_to_fit();
  std::unique_ptr<gem_hgraph> g(new gem_hgraph());
  g->nv = nv;
  csr_from_sorted_pairs(*g, keys, sh);
  g->lab.assign(nv, 0);
  g->refresh_stats();
  *out = g.release();
  return GEM_OK;
}

gem_status gem_hgraph_set_labels(gem_hgraph *g, uint32_t nlabels, double zipf_s, uint64_t seed) {
  if (!g || nlabels == 0 || zipf_s < 0) return GEM_ERR_ARG;
  std::vector<double> cdf(nlabels);
  double tot = 0;
  for (uint32_t l = 0; l < nlabels; ++l) {
    tot += zipf_s == 0 ? 1.0 : std::pow((double)(l + 1), -zipf_s);
    cdf[l] = tot;
  }
  for (auto &x : cdf) x /= tot;
  cdf[nlabels - 1] = 1.0;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)g->nv; ++v) {
    double u = u01(rng_at(seed, (uint64_t)v));
    uint32_t l = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
    g->lab[v] = std::min(l, nlabels - 1);
  }
  g->refresh_stats();
  return GEM_OK;
}

gem_status gem_hgraph_info(const gem_hgraph *g, uint32_t *nv, uint64_t *n_arcs,
                           uint32_t *max_label_plus1, uint32_t *max_degree) {
  if (!g) return GEM_ERR_ARG;
  if (nv) *nv = g->nv;
  if (n_arcs) *n_arcs = g->n_arcs();
  if (max_label_plus1) *max_label_plus1 = g->max_label_plus1;
  if (max_degree) *max_degree = g->max_degree;
  return GEM_OK;
}

gem_status gem_hgraph_view(const gem_hgraph *g, const uint64_t **offsets, const uint32_t **nbrs,
                           const uint32_t **labels) {
  if (!g) return GEM_ERR_ARG;
  if (offsets) *offsets = g->off.data();
  if (nbrs) *nbrs = g->nbr.data();
  if (labels) *labels = g->lab.data();
  return GEM_OK;
}

void gem_hgraph_destroy(gem_hgraph *g) { delete g; }

}  // extern "C"

// ------------------------------------------------------------------------
// Text format
// ------------------------------------------------------------------------
namespace {

struct TextFile {
  std::vector<char> buf;
  size_t pos = 0;
  bool load(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) { std::fclose(f); return false; }
    buf.resize((size_t)n + 1);
    size_t r = std::fread(buf.data(), 1, (size_t)n, f);
    std::fclose(f);
    buf.resize(r);
    buf.push_back('\0');
    return true;
  }
  void skip_ws() {
    while (pos < buf.size() && (buf[pos] == ' ' || buf[pos] == '\t' || buf[pos] == '\n' || buf[pos] == '\r')) ++pos;
  }
  int next_tag() {  // returns tag char or 0 at EOF
    skip_ws();
    if (pos >= buf.size() || buf[pos] == '\0') return 0;
    return buf[pos++];
  }
  bool next_uint(uint64_t &x) {
    skip_ws();
    if (pos >= buf.size() || buf[pos] < '0' || buf[pos] > '9') return false;
    x = 0;
    while (pos < buf.size() && buf[pos] >= '0' && buf[pos] <= '9') x = x * 10 + (uint64_t)(buf[pos++] - '0');
    return true;
  }
};

struct TextGraph {
  uint64_t nv = 0, ne = 0;
  std::vector<uint32_t> lab, deg;
  std::vector<uint32_t> edges;  // 2*ne in file order
};

gem_status parse_text(const char *path, TextGraph &tg, uint64_t max_nv) {
  TextFile f;
  if (!path || !f.load(path)) return GEM_ERR_IO;
  if (f.next_tag() != 't') return GEM_ERR_IO;
  if (!f.next_uint(tg.nv) || !f.next_uint(tg.ne)) return GEM_ERR_IO;
  if (tg.nv > max_nv || tg.nv > 0xFFFFFFF0ull) return GEM_ERR_LIMIT;
  tg.lab.assign(tg.nv, 0);
  tg.deg.assign(tg.nv, 0);
  std::vector<uint8_t> seen(tg.nv, 0);
  tg.edges.clear();
  tg.edges.reserve(2 * tg.ne);
  uint64_t nvl = 0;
  for (;;) {
    int t = f.next_tag();
    if (t == 0) break;
    uint64_t a, b, c;
    if (t == 'v') {
      if (!f.next_uint(a) || !f.next_uint(b) || !f.next_uint(c)) return GEM_ERR_IO;
      if (a >= tg.nv || seen[a] || b > 0xFFFFFFFFull || c > 0xFFFFFFFFull) return GEM_ERR_IO;
      seen[a] = 1;
      tg.lab[a] = (uint32_t)b;
      tg.deg[a] = (uint32_t)c;
      ++nvl;
    } else if (t == 'e') {
      if (!f.next_uint(a) || !f.next_uint(b)) return GEM_ERR_IO;
      if (a >= tg.nv || b >= tg.nv) return GEM_ERR_IO;
      // optional edge label (some t/v/e dialects): ignore a third integer on the line
      size_t save = f.pos;
      while (f.pos < f.buf.size() && (f.buf[f.pos] == ' ' || f.buf[f.pos] == '\t')) ++f.pos;
      if (f.pos < f.buf.size() && f.buf[f.pos] >= '0' && f.buf[f.pos] <= '9') {
        f.next_uint(c);
      } else {
        f.pos = save;
      }
      tg.edges.push_back((uint32_t)a);
      tg.edges.push_back((uint32_t)b);
    } else {
      return GEM_ERR_IO;
    }
  }
  if (nvl != tg.nv || tg.edges.size() != 2 * tg.ne) return GEM_ERR_IO;
  return GEM_OK;
}

}  // namespace

extern "C" {

gem_status gem_hgraph_read_text(const char *path, gem_hgraph **out) {
  if (!out) return GEM_ERR_ARG;
  *out = nullptr;
  TextGraph tg;
  gem_status st = parse_text(path, tg, 0xFFFFFFF0ull);
  if (st != GEM_OK) return st;
  const uint32_t nv = (uint32_t)tg.nv;
  std::unique_ptr<gem_hgraph> g(new gem_hgraph());
  g->nv = nv;
  g->lab = std::move(tg.lab);
  g->off.assign((size_t)nv + 1, 0);
  for (uint64_t e = 0; e < tg.ne; ++e) {
    uint32_t a = tg.edges[2 * e], b = tg.edges[2 * e + 1];
    if (a == b) return GEM_ERR_IO;
    g->off[a + 1]++;
    g->off[b + 1]++;
  }
  for (uint32_t v = 0; v < nv; ++v) {
    if (g->off[v + 1] != tg.deg[v]) return GEM_ERR_IO;  // declared degree mismatch
    g->off[v + 1] += g->off[v];
  }
  g->nbr.resize(g->off[nv]);
  std::vector<uint64_t> cur(g->off.begin(), g->off.end() - 1);
  for (uint64_t e = 0; e < tg.ne; ++e) {
    uint32_t a = tg.edges[2 * e], b = tg.edges[2 * e + 1];
    g->nbr[cur[a]++] = b;
    g->nbr[cur[b]++] = a;
  }
  bool dup = false;
#pragma omp parallel for schedule(dynamic, 4096) reduction(|| : dup)
  for (int64_t v = 0; v < (int64_t)nv; ++v) {
    auto b = g->nbr.begin() + g->off[v], e = g->nbr.begin() + g->off[v + 1];
    std::sort(b, e);
    if (std::adjacent_find(b, e) != e) dup = true;
  }
  if (dup) return GEM_ERR_IO;
  g->refresh_stats();
  *out = g.release();
  return GEM_OK;
}

gem_status gem_hgraph_write_text(const gem_hgraph *g, const char *path) {
  if (!g || !path) return GEM_ERR_ARG;
  FILE *f = std::fopen(path, "wb");
  if (!f) return GEM_ERR_IO;
  std::vector<char> buf;
  buf.reserve(1 << 22);
  auto flush = [&]() {
    if (!buf.empty()) std::fwrite(buf.data(), 1, buf.size(), f);
    buf.clear();
  };
  char line[96];
  int n = std::snprintf(line, sizeof line, "t %u %llu\n", g->nv, (unsigned long long)(g->n_arcs() / 2));
  buf.insert(buf.end(), line, line + n);
  for (uint32_t v = 0; v < g->nv; ++v) {
    n = std::snprintf(line, sizeof line, "v %u %u %llu\n", v, g->lab[v],
                      (unsigned long long)(g->off[v + 1] - g->off[v]));
    buf.insert(buf.end(), line, line + n);
    if (buf.size() > (1u << 22)) flush();
  }
  for (uint32_t v = 0; v < g->nv; ++v) {
    for (uint64_t i = g->off[v]; i < g->off[v + 1]; ++i) {
      if (g->nbr[i] <= v) continue;
      n = std::snprintf(line, sizeof line, "e %u %u\n", v, g->nbr[i]);
      buf.insert(buf.end(), line, line + n);
    }
    if (buf.size() > (1u << 22)) flush();
  }
  flush();
  bool ok = std::fclose(f) == 0;
  return ok ? GEM_OK : GEM_ERR_IO;
}

gem_status gem_query_read_text(const char *path, uint32_t *nv, uint32_t *ne, uint32_t *labels,
                               uint32_t *edges) {
  if (!nv || !ne || !labels || !edges) return GEM_ERR_ARG;
  TextGraph tg;
  gem_status st = parse_text(path, tg, GEM_MAX_QV);
  if (st != GEM_OK) return st;
  if (tg.ne > GEM_MAX_QE) return GEM_ERR_LIMIT;
  std::vector<uint32_t> d(tg.nv, 0);
  for (uint64_t e = 0; e < tg.ne; ++e) {
    d[tg.edges[2 * e]]++;
    d[tg.edges[2 * e + 1]]++;
  }
  for (uint64_t v = 0; v < tg.nv; ++v)
    if (d[v] != tg.deg[v]) return GEM_ERR_IO;
  *nv = (uint32_t)tg.nv;
  *ne = (uint32_t)tg.ne;
  for (uint64_t v = 0; v < tg.nv; ++v) labels[v] = tg.lab[v];
  for (uint64_t i = 0; i < 2 * tg.ne; ++i) edges[i] = tg.edges[i];
  return GEM_OK;
}

gem_status gem_query_write_text(const gem_query *q, const char *path) {
  if (!q || !path || !q->labels || (q->ne && !q->edges)) return GEM_ERR_ARG;
  FILE *f = std::fopen(path, "wb");
  if (!f) return GEM_ERR_IO;
  std::vector<uint32_t> d(q->nv, 0);
  for (uint32_t e = 0; e < q->ne; ++e) {
    if (q->edges[2 * e] >= q->nv || q->edges[2 * e + 1] >= q->nv) { std::fclose(f); return GEM_ERR_ARG; }
    d[q->edges[2 * e]]++;
    d[q->edges[2 * e + 1]]++;
  }
  std::fprintf(f, "t %u %u\n", q->nv, q->ne);
  for (uint32_t v = 0; v < q->nv; ++v) std::fprintf(f, "v %u %u %u\n", v, q->labels[v], d[v]);
  for (uint32_t e = 0; e < q->ne; ++e) std::fprintf(f, "e %u %u\n", q->edges[2 * e], q->edges[2 * e + 1]);
  return std::fclose(f) == 0 ? GEM_OK : GEM_ERR_IO;
}

// ------------------------------------------------------------------------
// Random-walk queries
// ------------------------------------------------------------------------
gem_status gem_gen_queries(const gem_hgraph *g, uint32_t k, int density, uint32_t count,
                           uint64_t seed, uint32_t max_e, uint32_t *ne_out, uint32_t *labels_out,
                           uint32_t *edges_out) {
  if (!g || k == 0 || k > GEM_MAX_QV || !ne_out || !labels_out || !edges_out) return GEM_ERR_ARG;
  if (density < 0 || density > 2) return GEM_ERR_ARG;
  if (g->nv == 0 || g->n_arcs() == 0) return GEM_ERR_ARG;
  if (k > g->nv) return GEM_ERR_ARG;
  const uint32_t max_tries = 4096;
  std::atomic<int> fail{0};
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t qi = 0; qi < (int64_t)count; ++qi) {
    uint64_t stream = mix64(seed) ^ mix64((uint64_t)qi + 0x51ull);
    uint64_t draw = 0;
    auto next = [&]() { return rng_at(stream, draw++); };
    std::vector<uint32_t> best_vis;
    std::vector<std::pair<uint32_t, uint32_t>> best_tree;
    bool done = false;
    for (uint32_t attempt = 0; attempt < max_tries && !done; ++attempt) {
      // start vertex with degree >= 1
      uint32_t s;
      do { s = (uint32_t)(next() % g->nv); } while (g->off[s + 1] == g->off[s]);
      std::vector<uint32_t> vis{s};
      std::vector<std::pair<uint32_t, uint32_t>> tree;  // first-visit edges (local ids)
      uint32_t cur = s, cur_local = 0;
      uint64_t steps = 0, step_cap = 64ull * k + 256;
      while (vis.size() < k && steps < step_cap) {
        ++steps;
        uint64_t d = g->off[cur + 1] - g->off[cur];
        uint32_t nx = g->nbr[g->off[cur] + next() % d];
        auto it = std::find(vis.begin(), vis.end(), nx);
        uint32_t nx_local;
        if (it == vis.end()) {
          nx_local = (uint32_t)vis.size();
          vis.push_back(nx);
          tree.emplace_back(cur_local, nx_local);
        } else {
          nx_local = (uint32_t)(it - vis.begin());
        }
        cur = nx;
        cur_local = nx_local;
      }
      if (vis.size() < k) continue;
      // induced edges
      uint32_t m = 0;
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = i + 1; j < k; ++j) {
          const uint32_t *b = g->nbr.data() + g->off[vis[i]], *e = g->nbr.data() + g->off[vis[i] + 1];
          if (std::binary_search(b, e, vis[j])) ++m;
        }
      bool dense = 2.0 * m / k > 3.0;
      bool ok = density == 0 || (density == 1 && !dense) || (density == 2 && dense);
      if (best_vis.empty()) { best_vis = vis; best_tree = tree; }
      if (ok) { best_vis = vis; best_tree = tree; done = true; }
    }
    if (best_vis.empty()) { fail = 1; continue; }
    const std::vector<uint32_t> &vis = best_vis;
    // emit edges: induced edges, or for an unsatisfied sparse request the
    // walk tree plus induced edges in (i, j) order while avg degree <= 3
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    std::vector<uint8_t> has((size_t)k * k, 0);
    if (done || density != 1) {
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = i + 1; j < k; ++j) {
          const uint32_t *b = g->nbr.data() + g->off[vis[i]], *e = g->nbr.data() + g->off[vis[i] + 1];
          if (std::binary_search(b, e, vis[j])) edges.emplace_back(i, j);
        }
    } else {
      for (auto &t : best_tree) {
        uint32_t i = std::min(t.first, t.second), j = std::max(t.first, t.second);
        has[(size_t)i * k + j] = 1;
        edges.emplace_back(i, j);
      }
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = i + 1; j < k; ++j) {
          if (has[(size_t)i * k + j]) continue;
          if (2.0 * (edges.size() + 1) / k > 3.0) { i = k; break; }
          const uint32_t *b = g->nbr.data() + g->off[vis[i]], *e = g->nbr.data() + g->off[vis[i] + 1];
          if (std::binary_search(b, e, vis[j])) edges.emplace_back(i, j);
        }
      std::sort(edges.begin(), edges.end());
    }
    if (edges.size() > max_e) { fail = 2; continue; }
    ne_out[qi] = (uint32_t)edges.size();
    for (uint32_t i = 0; i < k; ++i) labels_out[(size_t)qi * k + i] = g->lab[vis[i]];
    for (size_t e = 0; e < edges.size(); ++e) {
      edges_out[(size_t)qi * 2 * max_e + 2 * e] = edges[e].first;
      edges_out[(size_t)qi * 2 * max_e + 2 * e + 1] = edges[e].second;
    }
  }
  if (fail == 2) return GEM_ERR_OVERFLOW;
  if (fail) return GEM_ERR_LIMIT;
  return GEM_OK;
}

uint64_t gem_embedding_hash(const uint32_t *f, uint32_t nv) {
  uint64_t s = 0;
  for (uint32_t u = 0; u < nv; ++u) s += mix64((uint64_t)f[u] | ((uint64_t)u << 32));
  return mix64(s);
}

}  // extern "C"
