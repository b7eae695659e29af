// Relaxed ("similarity") matching: the relaxed queries of a query at a
// threshold, each counted exactly as a query of its own.
//
// The reference (in-core/lib/plan/src/relax.cpp:84-142) starts from the full
// edge set and removes one edge at a time, breadth first, up to `threshold`
// removals, keeping every edge set whose edges still connect all query
// vertices and expanding no spanning tree further; its lattice then shares
// intermediate results between the relaxed queries and prints one count per
// relaxed query (in-core/src/main.cu:229-236).  Every connected spanning
// subset with at most `threshold` edges removed is reached that way (remove
// the missing edges in any order: every intermediate set contains the subset,
// so it stays connected and is not yet a tree), so the relaxed queries are
// exactly those subsets.  Here they are enumerated the same way and counted
// in one wave whose filter rows are the original query's at the threshold
// (the reference's slack filter), so the relaxed queries share candidate
// lists and edge tables; the join counts each on its own.
#include <algorithm>
#include <cstring>
#include <queue>
#include <unordered_set>
#include <vector>

#include "../../include/gem.h"
#include "gem_internal.h"

namespace gem {

// True when the edges in `keep` connect all of q's vertices.
static bool spans(const HostQuery &q, uint64_t keep) {
  uint32_t adj[GEM_MAX_QV] = {};
  for (uint32_t j = 0; j < q.ne; ++j)
    if ((keep >> j) & 1u) {
      const uint32_t u = q.edges[2 * j], v = q.edges[2 * j + 1];
      adj[u] |= 1u << v;
      adj[v] |= 1u << u;
    }
  const uint32_t all = q.nv >= 32 ? 0xFFFFFFFFu : (1u << q.nv) - 1u;
  uint32_t seen = 1u, frontier = 1u;
  while (frontier) {
    uint32_t next = 0;
    for (uint32_t f = frontier; f; f &= f - 1) next |= adj[__builtin_ctz(f)];
    next &= ~seen;
    seen |= next;
    frontier = next;
  }
  return seen == all;
}

// The relaxed edge sets of q (bit j = q's edge j kept), fewest edges removed
// first, then by mask descending.  GEM_ERR_LIMIT when q has more than 64
// edges or when more than `cap` sets exist (out then holds cap + 1 of them).
gem_status relaxed_sets(const HostQuery &q, uint32_t threshold, uint32_t cap, std::vector<uint64_t> &out) {
  out.clear();
  if (q.ne > 64) return GEM_ERR_LIMIT;
  const uint64_t full = q.ne == 64 ? ~0ull : (1ull << q.ne) - 1ull;
  std::unordered_set<uint64_t> seen{full};
  std::queue<std::pair<uint64_t, uint32_t>> bfs;
  bfs.push({full, 0});
  out.push_back(full);
  while (!bfs.empty()) {
    const auto [cur, removed] = bfs.front();
    bfs.pop();
    if (removed >= threshold) continue;
    if ((uint32_t)__builtin_popcountll(cur) + 1 <= q.nv) continue;  // a spanning tree: nothing to remove
    for (uint32_t j = 0; j < q.ne; ++j) {
      if (!((cur >> j) & 1u)) continue;
      const uint64_t next = cur & ~(1ull << j);
      if (!seen.insert(next).second) continue;
      if (!spans(q, next)) continue;
      out.push_back(next);
      if (out.size() > cap) return GEM_ERR_LIMIT;
      bfs.push({next, removed + 1});
    }
  }
  std::sort(out.begin(), out.end(), [](uint64_t x, uint64_t y) {
    const int px = __builtin_popcountll(x), py = __builtin_popcountll(y);
    return px != py ? px > py : x > y;
  });
  return GEM_OK;
}

}  // namespace gem

using namespace gem;

extern "C" gem_status gem_relaxed_sets(const gem_query *q, uint32_t threshold, uint32_t cap, uint64_t *ets,
                                       uint32_t *n_out) {
  if (!q || !n_out || (cap && !ets)) return GEM_ERR_ARG;
  HostQuery hq;
  std::string err;
  gem_status st = make_host_query(q, hq, err);
  if (st != GEM_OK) return st;
  std::vector<uint64_t> sets;
  st = relaxed_sets(hq, threshold, cap, sets);
  *n_out = (uint32_t)sets.size();
  if (st != GEM_OK) return st;
  std::memcpy(ets, sets.data(), sets.size() * sizeof(uint64_t));
  return GEM_OK;
}

extern "C" gem_status gem_relaxed_run(gem_ctx *ctx, const gem_query *q, uint32_t threshold, int mode, uint32_t cap,
                                      uint64_t *ets, gem_result *res, uint32_t *n_out) {
  if (!ctx || !q || !n_out || (cap && (!ets || !res))) return GEM_ERR_ARG;
  HostQuery hq;
  std::string err;
  gem_status st = make_host_query(q, hq, err);
  if (st != GEM_OK) return st;
  std::vector<uint64_t> sets;
  st = relaxed_sets(hq, threshold, cap, sets);
  *n_out = (uint32_t)sets.size();
  if (st != GEM_OK) return st;
  // each relaxed query keeps q's vertices and labels and the edges of its set, in q's order
  std::vector<std::vector<uint32_t>> edges(sets.size());
  std::vector<gem_query> rq(sets.size());
  for (size_t i = 0; i < sets.size(); ++i) {
    for (uint32_t j = 0; j < hq.ne; ++j)
      if ((sets[i] >> j) & 1u) {
        edges[i].push_back(hq.edges[2 * j]);
        edges[i].push_back(hq.edges[2 * j + 1]);
      }
    rq[i] = gem_query{q->nv, (uint32_t)(edges[i].size() / 2), q->labels, edges[i].data()};
    ets[i] = sets[i];
  }
  // one wave on q's filter rows at the threshold (shared candidate lists and
  // tables); a plain batch when that wave does not fit the device budget
  std::vector<HostQuery> hr(rq.size());
  for (size_t i = 0; i < rq.size(); ++i) {
    st = make_host_query(&rq[i], hr[i], err);
    if (st != GEM_OK) return st;
  }
  st = relaxed_wave(ctx, hq, hr, threshold, mode, res);
  if (st != GEM_ERR_OOM) return st;
  return gem_batch_run(ctx, rq.data(), (uint32_t)rq.size(), mode, res);
}
