// Serving: continuous batching with memory-based admission.
//
// No counterpart in the reference (one query per process).  gem_submit
// admits a query when its estimated device bytes (its upper bound scaled by
// what the waves so far took of theirs) fit the admission budget.
// Worker threads, one per serving lane, each turn everything admitted and
// not yet taken into a wave, up to the lane's row limit, into one wave
// (shared filter/table launches and one persistent join launch) on their
// lane.  An in-core context serves on two lanes: the
// context itself and a lane context that borrows its resident graph (its own
// stream, arena, control block and task queue).  While one lane's wave is on
// the GPU the other lane takes the requests that arrived meanwhile, so their
// work overlaps on the device; each lane's join grid takes half of the SMs'
// blocks so that two joins fit side by side.  Out of core, each lane has
// its own partition staging buffers and copy stream, so one lane's
// partition copies run beside the other lane's join.  Results are
// identical to gem_query_run's: every query of a wave has its own plan,
// tables and counters.  While the server runs, only gem_submit and gem_poll
// may be used on the context (other calls return GEM_ERR_STATE).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "ctx.h"

using namespace gem;

struct Server {
  std::mutex mu;
  std::condition_variable cv;
  std::vector<std::thread> th;
  std::vector<gem_ctx *> lanes;  // lanes[0] is the context itself
  uint64_t saved_budget = 0;     // the context's device budget before serving split it
  bool stop = false;
  struct Req {
    uint64_t ticket;
    HostQuery q;
    int mode;
    uint64_t est;     // bytes charged to the admission budget
    uint64_t bound;   // the estimate (an upper bound of the query's bytes)
  };
  // Admission charges a query its upper bound times `scale`, learnt from the
  // waves that ran: 1.5 times the largest recent ratio of a wave's bytes to
  // its queries' bounds (at most 1).  The bound is loose (label statistics
  // only), so charging it whole would admit a fraction of what fits; a wave
  // that is admitted but does not fit is retried smaller.
  double scale = 1.0;
  std::deque<Req> pending;
  std::map<uint64_t, gem_result> done;
  uint64_t next_ticket = 1;
  uint64_t in_flight = 0, budget = 0, per_wave = 0;
  uint64_t waves = 0;
};

// Upper bound of the device scratch one query adds to a wave, from the
// graph's label statistics alone (the plan is not known at admission): per
// query vertex its rank-bitmap row with the row scan, its candidate list
// (at most the label's vertices), its bits in the wave's source and target
// membership columns and, as an edge-table source, its keys' tile counts and
// scan and an index; per query edge the larger direction's table: per-tile
// masks and positions, offsets per key, values and key positions (at most
// the arcs between the two labels); per query the join's descriptors.
// *per_wave: what every wave takes once whatever its queries (the vertex
// tiles and the write pass's units, their scans and maps, the columns'
// rounding word per vertex).
static uint64_t estimate_bytes(const gem_ctx *ctx, const HostQuery &q, uint64_t *per_wave) {
  const uint64_t nv = ctx->g.nv, nwords = (nv + 31) / 32;
  const size_t L = ctx->label_freq.size();
  auto freq = [&](uint32_t l) -> uint64_t { return l < L ? ctx->label_freq[l] : 0; };
  auto tiles = [&](uint32_t l) -> uint64_t { return l < L ? ctx->label_freq[l] + ctx->label_arcs[l] / 32 + 1 : 1; };
  auto pair_arcs = [&](uint32_t s, uint32_t t) -> uint64_t {
    if (s >= L || t >= L) return 0;
    return ctx->label_pair_arcs.empty() ? ctx->label_arcs[s] : ctx->label_pair_arcs[(size_t)s * L + t];
  };
  auto al = [](uint64_t b) -> uint64_t { return (b + 255) & ~(uint64_t)255; };
  uint64_t b = 0;
  for (uint32_t u = 0; u < q.nv; ++u) {
    const uint64_t f = freq(q.lab[u]);
    b += al(8 * nwords) + al(8 * (nwords + 1)) + al(8 * (nwords / 2048 + 2)) + al(4 * f + 4);  // row, scan, list
    b += al(4 * nwords) + 2 * al(4 * nwords);                                  // bit row, both columns
    b += al(4 * f) + al(8 * (f + 1)) + al(8 * (f / 2048 + 2));                 // source: key tiles and scan
    b += al(16 * f + 1024);                                                    // index
  }
  for (uint32_t e = 0; e < q.ne; ++e) {
    uint64_t most = 0;
    for (int dir = 0; dir < 2; ++dir) {
      const uint32_t s = q.lab[q.edges[2 * e + dir]], t = q.lab[q.edges[2 * e + 1 - dir]];
      const uint64_t ts = tiles(s), f = freq(s), v = pair_arcs(s, t);
      most = std::max<uint64_t>(most, al(4 * ts) + al(8 * (ts + 1)) + al(8 * (ts / 2048 + 2)) + al(8 * (f + 1)) +
                                2 * al(4 * v + 4));
    }
    b += most;
  }
  const uint64_t parts = ctx->part_v.empty() ? 0 : ctx->part_v.size();
  *per_wave = 2 * al(4 * nv) + 2 * (al(4 * nv + 4) + al(8 * (nv + 1)) + al(4 * (nv + ctx->g.narcs / 32 + 1))) +
              al(8 * (nv / 2048 + 2)) + al(16 * parts + 16) + (1ull << 20);
  return b + (64ull << 10) * (q.nv + 1) + (1ull << 20);
}

extern "C" gem_status gem_estimate_bytes(const gem_ctx *ctx, const gem_query *q, uint64_t *bytes) {
  if (!ctx || !q || !bytes) return GEM_ERR_ARG;
  if (!ctx->loaded) return GEM_ERR_STATE;
  HostQuery hq;
  std::string err;
  const gem_status st = make_host_query(q, hq, err);
  if (st != GEM_OK) return st;
  uint64_t per_wave = 0;
  *bytes = estimate_bytes(ctx, hq, &per_wave) + per_wave;
  return GEM_OK;
}

// One lane's worker: takes the longest run of pending requests of one mode
// that fits a wave, runs it on the lane, publishes the results.
static void server_loop(gem_ctx *root, gem_ctx *lane) {
  Server &S = *root->server;
  for (;;) {
    std::vector<Server::Req> batch;
    uint64_t wave_no = 0;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      S.cv.wait(lk, [&] { return S.stop || !S.pending.empty(); });
      if (S.stop && S.pending.empty()) return;
      uint32_t rows = 0, cap = lane->wave_max_rows;
      if (lane->wave_rows_cap) cap = std::min(cap, lane->wave_rows_cap);
      const int mode = S.pending.front().mode;
      while (!S.pending.empty() && S.pending.front().mode == mode &&
             (batch.empty() || rows + S.pending.front().q.nv <= cap)) {
        rows += S.pending.front().q.nv;
        batch.push_back(std::move(S.pending.front()));
        S.pending.pop_front();
      }
      wave_no = S.waves++;
    }
    Wave w;
    for (auto &r : batch) w.q.push_back(r.q);
    lane->arena.reset();
    gem_status st = run_wave(lane, w, 0, batch[0].mode, nullptr, 0);
    if (st != GEM_OK) {
      cudaStreamSynchronize(lane->s);
      cudaGetLastError();
    }
    if (st == GEM_ERR_OOM && batch.size() > 1) {
      // the wave's tables do not fit the lane's budget: its requests go back
      // to the front of the queue, and the lane's waves are limited to the
      // rows that would have fit (the wave's rows scaled by the bytes the
      // budget left it over the bytes it asked for, a tenth kept back; half
      // when that is not known)
      const Arena &a = lane->arena;
      double f = a.oom_need ? 0.9 * (double)a.oom_room / (double)a.oom_need : 0.5;
      f = std::min(0.9, std::max(0.25, f));
      uint64_t rows = 0;
      for (const auto &r : batch) rows += r.q.nv;
      lane->wave_rows_cap = (uint32_t)std::max<uint64_t>(1, (uint64_t)(f * (double)rows));
      if (!lane->arena.reserved) lane->arena.release(lane);
      std::lock_guard<std::mutex> lk(S.mu);
      for (size_t i = batch.size(); i-- > 0;) S.pending.push_front(std::move(batch[i]));
      S.cv.notify_all();
      continue;
    }
    std::lock_guard<std::mutex> lk(S.mu);
    if (st == GEM_OK) {
      uint64_t bound = 0;
      for (const auto &r : batch) bound += r.bound;
      if (bound) {
        const double target = std::min(1.0, 1.5 * (double)w.arena_bytes / (double)bound);
        S.scale = target > S.scale ? target : 0.8 * S.scale + 0.2 * target;
      }
    }
    for (size_t i = 0; i < batch.size(); ++i) {
      gem_result r;
      if (st == GEM_OK) {
        wave_result(lane, w, i, &r);
        r.wave = (uint32_t)wave_no;
      } else {
        std::memset(&r, 0, sizeof r);
        r.status = st;
      }
      S.done[batch[i].ticket] = r;
      S.in_flight -= batch[i].est;
    }
  }
}

void server_shutdown(gem_ctx *ctx) {
  if (!ctx->server) return;
  Server *S = ctx->server;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  for (auto &t : S->th)
    if (t.joinable()) t.join();
  for (size_t i = 1; i < S->lanes.size(); ++i) {
    merge_ooc_stats(ctx, S->lanes[i]);
    gem_ctx_destroy(S->lanes[i]);
  }
  ctx->join_grid_div = 1;
  if (S->saved_budget) ctx->budget = S->saved_budget;
  if (ctx->arena.reserved) ctx->arena.release(ctx);  // it held the lane-split budget
  delete S;
  ctx->server = nullptr;
}

// Starts the server: a second lane for in-core contexts (the remaining
// device budget split between the two), one worker thread per lane.
static gem_status server_start(gem_ctx *ctx) {
  drop_batch_lane(ctx);  // serving splits the budget between lanes of its own
  Server *S = new Server();
  ctx->server = S;
  const uint64_t cap = ctx->opts.admit_gb ? (uint64_t)ctx->opts.admit_gb << 30 : 120ull << 30;
  const uint64_t room = ctx->budget > ctx->device_bytes ? ctx->budget - ctx->device_bytes : 0;
  S->budget = cap < room ? cap : room;
  S->lanes.push_back(ctx);
  {
    gem_ctx *lane = nullptr;
    if (lane_create(ctx, room / 2, &lane) == GEM_OK) {
      S->saved_budget = ctx->budget;
      ctx->budget = ctx->device_bytes + room / 2;
      ctx->join_grid_div = 2;
      lane->join_grid_div = 2;
      S->lanes.push_back(lane);
    } else {
      cudaGetLastError();
    }
  }
  // each lane's arena: one chunk of its whole budget (no cudaMalloc or
  // cudaFree between waves), less room for the join's graph
  for (gem_ctx *l : S->lanes)
    if (l->budget > l->device_bytes + (1ull << 30)) l->arena.reserve(l, l->budget - l->device_bytes - (512ull << 20));
  for (gem_ctx *lane : S->lanes) S->th.emplace_back(server_loop, ctx, lane);
  return GEM_OK;
}

extern "C" gem_status gem_submit(gem_ctx *ctx, const gem_query *q, int mode, uint64_t *ticket) {
  if (!ctx || !q || !ticket) return GEM_ERR_ARG;
  if (mode != GEM_MODE_COUNT && mode != GEM_MODE_HASH) return GEM_ERR_ARG;
  if (!ctx->loaded) return GEM_ERR_STATE;
  HostQuery hq;
  std::string err;
  gem_status st = make_host_query(q, hq, err);
  if (st != GEM_OK) return st;
  if (!ctx->server) {
    const gem_status ss = server_start(ctx);
    if (ss != GEM_OK) return ss;
  }
  Server &S = *ctx->server;
  uint64_t per_wave = 0;
  const uint64_t bound = estimate_bytes(ctx, hq, &per_wave);
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.per_wave) {  // every lane's wave takes this once, beside its queries'
    S.per_wave = per_wave;
    const uint64_t fixed = per_wave * S.lanes.size();
    S.budget = S.budget > fixed ? S.budget - fixed : 0;
  }
  const uint64_t est = std::max<uint64_t>(1, (uint64_t)(S.scale * (double)bound));
  if (S.in_flight + est > S.budget && S.in_flight > 0) return GEM_ERR_OOM;  // busy: retry later
  S.in_flight += est;
  *ticket = S.next_ticket++;
  S.pending.push_back({*ticket, std::move(hq), mode, est, bound});
  S.cv.notify_one();
  return GEM_OK;
}

extern "C" gem_status gem_poll(gem_ctx *ctx, uint64_t ticket, gem_result *res, int *done) {
  if (!ctx || !res || !done) return GEM_ERR_ARG;
  *done = 0;
  if (!ctx->server) return GEM_ERR_STATE;
  Server &S = *ctx->server;
  std::lock_guard<std::mutex> lk(S.mu);
  auto it = S.done.find(ticket);
  if (it == S.done.end()) {
    if (ticket == 0 || ticket >= S.next_ticket) return GEM_ERR_STATE;
    return GEM_OK;
  }
  *res = it->second;
  S.done.erase(it);
  *done = 1;
  return GEM_OK;
}
