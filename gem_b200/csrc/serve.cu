// Serving: continuous batching with memory-based admission.
//
// No counterpart in the reference (one query per process).  gem_submit
// admits a query when its estimated device bytes fit the admission budget,
// and a server thread owned by the context turns everything admitted so far
// into one wave (shared filter/table launches and one persistent join launch).
// Requests that arrive while a wave is on the GPU are admitted as budget
// frees and run in the next wave, together with everything else waiting.
// Results are identical to gem_query_run's: every query of a wave has its own
// plan, tables and counters.  While the server runs, only gem_submit and
// gem_poll may be used on the context (other calls return GEM_ERR_STATE).
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
  std::thread th;
  bool stop = false;
  struct Req {
    uint64_t ticket;
    HostQuery q;
    int mode;
    uint64_t est;
  };
  std::deque<Req> pending;
  std::map<uint64_t, gem_result> done;
  uint64_t next_ticket = 1;
  uint64_t in_flight = 0, budget = 0;
  uint64_t waves = 0;
};

// Device bytes a query is expected to need: one rank-bitmap row per query
// vertex, its candidate list (bounded by the label's frequency) and, per
// query edge, the label-restricted arcs of the source candidates.
static uint64_t estimate_bytes(const gem_ctx *ctx, const HostQuery &q) {
  const uint64_t nwords = (ctx->g.nv + 31) / 32;
  uint64_t b = 0;
  for (uint32_t u = 0; u < q.nv; ++u) {
    const uint64_t f = q.lab[u] < ctx->label_freq.size() ? ctx->label_freq[q.lab[u]] : 0;
    b += nwords * 8 * 3 + f * 4;
  }
  const double nv = ctx->g.nv ? (double)ctx->g.nv : 1.0;
  for (uint32_t e = 0; e < q.ne; ++e) {
    const uint32_t a = q.edges[2 * e], c = q.edges[2 * e + 1];
    for (int dir = 0; dir < 2; ++dir) {
      const uint32_t s = dir ? c : a, t = dir ? a : c;
      const double arcs = q.lab[s] < ctx->label_arcs.size() ? (double)ctx->label_arcs[q.lab[s]] : 0.0;
      const double pt = q.lab[t] < ctx->label_freq.size() ? (double)ctx->label_freq[q.lab[t]] / nv : 0.0;
      b += (uint64_t)(arcs * (4.0 / 32 + 8.0 / 32 + pt * 4.0)) + 16;
    }
  }
  return b + (1u << 20);
}

static void server_loop(gem_ctx *ctx) {
  Server &S = *ctx->server;
  for (;;) {
    std::vector<Server::Req> batch;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      S.cv.wait(lk, [&] { return S.stop || !S.pending.empty(); });
      if (S.stop && S.pending.empty()) return;
      uint32_t rows = 0;
      const int mode = S.pending.front().mode;
      while (!S.pending.empty() && S.pending.front().mode == mode &&
             (batch.empty() || rows + S.pending.front().q.nv <= ctx->wave_max_rows)) {
        rows += S.pending.front().q.nv;
        batch.push_back(std::move(S.pending.front()));
        S.pending.pop_front();
      }
    }
    Wave w;
    for (auto &r : batch) w.q.push_back(r.q);
    ctx->arena.reset();
    gem_status st = run_wave(ctx, w, 0, batch[0].mode, nullptr, 0);
    std::lock_guard<std::mutex> lk(S.mu);
    for (size_t i = 0; i < batch.size(); ++i) {
      gem_result r;
      if (st == GEM_OK) {
        wave_result(ctx, w, i, &r);
        r.wave = (uint32_t)S.waves;
      } else {
        std::memset(&r, 0, sizeof r);
        r.status = st;
      }
      S.done[batch[i].ticket] = r;
      S.in_flight -= batch[i].est;
    }
    ++S.waves;
  }
}

void server_shutdown(gem_ctx *ctx) {
  if (!ctx->server) return;
  {
    std::lock_guard<std::mutex> lk(ctx->server->mu);
    ctx->server->stop = true;
  }
  ctx->server->cv.notify_all();
  if (ctx->server->th.joinable()) ctx->server->th.join();
  delete ctx->server;
  ctx->server = nullptr;
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
    ctx->server = new Server();
    const uint64_t cap = ctx->opts.admit_gb ? (uint64_t)ctx->opts.admit_gb << 30 : 120ull << 30;
    const uint64_t room = ctx->budget > ctx->device_bytes ? ctx->budget - ctx->device_bytes : 0;
    ctx->server->budget = cap < room ? cap : room;
    ctx->server->th = std::thread(server_loop, ctx);
  }
  Server &S = *ctx->server;
  const uint64_t est = estimate_bytes(ctx, hq);
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.in_flight + est > S.budget && S.in_flight > 0) return GEM_ERR_OOM;  // busy: retry later
  S.in_flight += est;
  *ticket = S.next_ticket++;
  S.pending.push_back({*ticket, std::move(hq), mode, est});
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
