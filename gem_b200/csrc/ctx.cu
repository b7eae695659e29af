// libgem host orchestration: the device context, the resident data graph, a
// chunked device arena, the matching-order planner, and the wave pipeline
//   filter -> compaction -> plan -> edge tables -> index -> join
// that serves gem_query_run (a wave of one query) and gem_batch_run (waves of
// many queries in one persistent join launch).
//
// Reference counterparts: main()'s phase chain (in-core/src/main.cu:140-236),
// the process globals of in-core/lib/utils/src/globals.cu, the per-phase
// allocate/scan/sync sequences of in-core/lib/structure/src/unifiedTrie.cu and
// in-core/lib/join/src/join_trie.cu.  Everything here hangs off a gem_ctx; no
// call exits the process.
#include <algorithm>
#include <chrono>
#include <functional>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "ctx.h"
#include "kernels.h"

using namespace gem;

// ---------------------------------------------------------------------------
// Error helpers
// ---------------------------------------------------------------------------
#define CU(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return e_ == cudaErrorMemoryAllocation ? GEM_ERR_OOM : GEM_ERR_CUDA;           \
    }                                                                                \
  } while (0)
#define ST(call)                      \
  do {                                \
    gem_status s_ = (call);           \
    if (s_ != GEM_OK) return s_;      \
  } while (0)

extern "C" const char *gem_strerror(gem_status s) {
  switch (s) {
    case GEM_OK: return "ok";
    case GEM_ERR_ARG: return "invalid argument";
    case GEM_ERR_OOM: return "out of device or pinned memory budget";
    case GEM_ERR_LIMIT: return "outside the supported envelope";
    case GEM_ERR_TIMEOUT: return "time cap or bounded wait expired";
    case GEM_ERR_CUDA: return "CUDA runtime error";
    case GEM_ERR_IO: return "file missing or malformed";
    case GEM_ERR_STATE: return "call out of order";
    case GEM_ERR_OVERFLOW: return "result exceeds buffer or counter";
    case GEM_ERR_INTERNAL: return "internal consistency check failed";
  }
  return "unknown status";
}

// ---------------------------------------------------------------------------
// Arena: chunks from cudaMalloc, bump allocation, reset per wave.
// ---------------------------------------------------------------------------
gem_status Arena::alloc(gem_ctx *ctx, uint64_t bytes, void **out) {
  bytes = (bytes + 255) & ~255ull;
  if (bytes == 0) bytes = 256;
  for (; cur < chunks.size(); ++cur) {
    Chunk &c = chunks[cur];
    if (c.used + bytes <= c.size) {
      *out = c.base + c.used;
      c.used += bytes;
      in_use += bytes;
      peak = std::max(peak, in_use);
      return GEM_OK;
    }
  }
  uint64_t sz = std::max<uint64_t>(bytes, 512ull << 20);
  if (ctx->device_bytes + sz > ctx->budget) {
    // chunks this wave has not used (too small for what it asked) go back
    // to the budget before the new one is taken
    size_t k = 0;
    for (size_t i = 0; i < chunks.size(); ++i) {
      if (chunks[i].used == 0) {
        cudaFree(chunks[i].base);
        ctx->device_bytes -= chunks[i].size;
        reserved = false;
      } else {
        chunks[k++] = chunks[i];
      }
    }
    chunks.resize(k);
    cur = chunks.size();
    sz = std::max<uint64_t>(bytes, 512ull << 20);
    if (ctx->device_bytes + sz > ctx->budget) sz = bytes;
    if (ctx->device_bytes + sz > ctx->budget) {
      ctx->err = "device budget exceeded: need " + std::to_string(bytes) + " more bytes";
      uint64_t held = 0;
      for (const Chunk &c : chunks) held += c.size;
      oom_need = in_use + bytes;
      oom_room = ctx->budget > ctx->device_bytes - held ? ctx->budget - (ctx->device_bytes - held) : 0;
      return GEM_ERR_OOM;
    }
  }
  char *p = nullptr;
  cudaError_t e = cudaMalloc(&p, sz);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    oom_need = oom_room = 0;
    return GEM_ERR_OOM;
  }
  ctx->device_bytes += sz;
  chunks.push_back({p, sz, bytes});
  cur = chunks.size() - 1;
  *out = p;
  in_use += bytes;
  peak = std::max(peak, in_use);
  return GEM_OK;
}
void Arena::reserve(gem_ctx *ctx, uint64_t bytes) {
  release(ctx);
  bytes &= ~((2ull << 20) - 1);
  if (bytes == 0 || ctx->device_bytes + bytes > ctx->budget) return;
  char *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  ctx->device_bytes += bytes;
  chunks.push_back({p, bytes, 0});
  reserved = true;
}
void Arena::reset() {
  for (auto &c : chunks) c.used = 0;
  cur = 0;
  in_use = 0;
}
void Arena::release(gem_ctx *ctx) {
  for (auto &c : chunks) {
    cudaFree(c.base);
    ctx->device_bytes -= c.size;
  }
  chunks.clear();
  reserved = false;
  cur = 0;
  in_use = 0;
}

template <class T>
static gem_status aalloc(gem_ctx *ctx, uint64_t n, T **out) {
  void *p = nullptr;
  gem_status s = ctx->arena.alloc(ctx, n * sizeof(T), &p);
  *out = (T *)p;
  return s;
}

// ---------------------------------------------------------------------------
// Context and graph
// ---------------------------------------------------------------------------
// A context's own execution resources: stream, events, the join's control
// block and task queue, the error words and the pinned staging buffer.
static gem_status exec_init(gem_ctx *ctx) {
  CU(cudaStreamCreateWithFlags(&ctx->s, cudaStreamNonBlocking));
  for (auto &ev : ctx->ev) CU(cudaEventCreate(&ev));
  CU(cudaMalloc(&ctx->d_ctl, sizeof(JControl)));
  CU(cudaMalloc(&ctx->d_queue, sizeof(JTask) * TASK_CAP));
  CU(cudaMalloc(&ctx->d_qends, sizeof(JQueueEnds) * QUEUE_SUBQ));
  CU(cudaMalloc(&ctx->d_err, sizeof(uint32_t) * 4));
  CU(cudaHostAlloc(&ctx->h_small, H_SMALL_BYTES, cudaHostAllocDefault));
  ctx->device_bytes += sizeof(JControl) + sizeof(JTask) * TASK_CAP + sizeof(JQueueEnds) * QUEUE_SUBQ + 16;
  return GEM_OK;
}

extern "C" gem_status gem_ctx_create(const gem_opts *opts, gem_ctx **out) {
  if (!out) return GEM_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<gem_ctx> c(new gem_ctx());
  if (opts) c->opts = *opts;
  gem_ctx *ctx = c.get();
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return GEM_ERR_CUDA;
  }
  if (ctx->opts.device < 0 || ctx->opts.device >= ndev) return GEM_ERR_ARG;
  CU(cudaSetDevice(ctx->opts.device));
  size_t fr = 0, tot = 0;
  CU(cudaMemGetInfo(&fr, &tot));
  ctx->budget = ctx->opts.device_budget_bytes ? ctx->opts.device_budget_bytes : (uint64_t)(fr * 0.9);
  if (ctx->budget > fr) ctx->budget = fr;
  CU(cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->opts.device));
  for (uint32_t m = 0; m < 3; ++m) ctx->join_bps[m] = join_blocks_per_sm(m);
  CU(cudaEventCreate(&ctx->ev_ref));
  ST(exec_init(ctx));
  *out = c.release();
  return GEM_OK;
}

// A lane's own out-of-core staging: two buffers of the root's largest
// partition, a copy stream and its events (the partition bounds on the
// device are the root's).
static gem_status lane_staging(gem_ctx *ctx, const gem_ctx *root) {
  const uint64_t b_st = (root->ooc.max_part_bytes + 255) & ~255ull;
  char *p = nullptr;
  if (ctx->device_bytes + 2 * b_st > ctx->budget || cudaMalloc(&p, 2 * b_st) != cudaSuccess) {
    cudaGetLastError();
    ctx->err = "out-of-core staging buffers of a lane do not fit the device budget";
    return GEM_ERR_OOM;
  }
  ctx->part_mem = p;
  ctx->part_bytes = 2 * b_st;
  ctx->device_bytes += 2 * b_st;
  ctx->d_part_v = root->d_part_v;
  ctx->d_stage[0] = (uint32_t *)p;
  ctx->d_stage[1] = (uint32_t *)(p + b_st);
  CU(cudaStreamCreateWithFlags(&ctx->s_copy, cudaStreamNonBlocking));
  for (int b = 0; b < 2; ++b) {
    CU(cudaEventCreateWithFlags(&ctx->ev_ready[b], cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&ctx->ev_free[b], cudaEventDisableTiming));
  }
  ctx->ooc.partitions = root->ooc.partitions;
  ctx->ooc.max_part_bytes = root->ooc.max_part_bytes;
  return GEM_OK;
}

// Serving lane over root's resident graph: everything a wave runs on of its
// own (stream, events, arena, control block, task queue, pinned staging),
// the graph and its derived indexes borrowed, the tuned schedules copied.
gem_status lane_create(gem_ctx *root, uint64_t budget, gem_ctx **out) {
  *out = nullptr;
  if (!root->loaded) return GEM_ERR_STATE;
  std::unique_ptr<gem_ctx> c(new gem_ctx());
  gem_ctx *ctx = c.get();
  ctx->opts = root->opts;
  ctx->sms = root->sms;
  for (uint32_t m = 0; m < 3; ++m) ctx->join_bps[m] = root->join_bps[m];
  ctx->budget = budget;
  ctx->loaded = true;
  ctx->borrowed_graph = true;
  ctx->g = root->g;
  ctx->vnh_off = root->vnh_off;
  ctx->vnh_slots = root->vnh_slots;
  ctx->label_freq = root->label_freq;
  ctx->label_arcs = root->label_arcs;
  ctx->label_pair_arcs = root->label_pair_arcs;
  for (int b = 0; b < 6; ++b) ctx->tune[b] = root->tune[b];
  ctx->donate_max_level = root->donate_max_level;
  ctx->closed_form_suffix = root->closed_form_suffix;
  ctx->wave_max_rows = root->wave_max_rows;
  ctx->ev_ref = root->ev_ref;
  ctx->ev_ref_recorded = root->ev_ref_recorded;
  // out of core: the pinned adjacency and the partition bounds are the
  // root's; the two staging buffers and the copy stream are the lane's own
  ctx->pinned_nbr = nullptr;
  ctx->host_nbr = root->host_nbr;
  ctx->part_v = root->part_v;
  ctx->part_a = root->part_a;
  c.release();
  gem_status st = cudaSetDevice(ctx->opts.device) == cudaSuccess ? exec_init(ctx) : GEM_ERR_CUDA;
  if (st == GEM_OK && root->opts.ooc && !root->part_v.empty()) st = lane_staging(ctx, root);
  if (st != GEM_OK) {
    cudaGetLastError();
    gem_ctx_destroy(ctx);  // its own resources only: the graph is borrowed
    return st;
  }
  ctx->budget += ctx->device_bytes;
  *out = ctx;
  return GEM_OK;
}

static void free_graph(gem_ctx *ctx) {
  if (ctx->pinned_nbr) {
    cudaFreeHost(ctx->pinned_nbr);
    ctx->pinned_nbr = nullptr;
  }
  ctx->host_nbr = nullptr;
  if (ctx->part_mem) {
    cudaFree(ctx->part_mem);
    ctx->device_bytes -= ctx->part_bytes;
  }
  ctx->part_mem = nullptr;
  ctx->part_bytes = 0;
  ctx->d_part_v = nullptr;
  ctx->d_stage[0] = ctx->d_stage[1] = nullptr;
  ctx->part_v.clear();
  ctx->part_a.clear();
  ctx->ooc = gem_ooc_stats{};
  if (ctx->graph_mem) {
    cudaFree(ctx->graph_mem);
    ctx->device_bytes -= ctx->graph_bytes;
  }
  if (ctx->vnh_mem) {
    cudaFree(ctx->vnh_mem);
    ctx->device_bytes -= ctx->vnh_bytes;
  }
  ctx->vnh_mem = nullptr;
  ctx->vnh_bytes = 0;
  ctx->vnh_off = nullptr;
  ctx->vnh_slots = nullptr;
  ctx->graph_mem = nullptr;
  ctx->graph_bytes = 0;
  ctx->g = DevGraph();
  ctx->loaded = false;
}

// The batch lane (a second context over this context's graph) and the
// budget it took; dropped before the graph changes or the context goes.
// Adds a lane's out-of-core counters to its root's and clears them.
void merge_ooc_stats(gem_ctx *root, gem_ctx *lane) {
  root->ooc.waves_streamed += lane->ooc.waves_streamed;
  root->ooc.waves_in_place += lane->ooc.waves_in_place;
  root->ooc.parts_streamed += lane->ooc.parts_streamed;
  root->ooc.bytes_streamed += lane->ooc.bytes_streamed;
  root->ooc.waves_spilled += lane->ooc.waves_spilled;
  root->ooc.bytes_spilled += lane->ooc.bytes_spilled;
  lane->ooc.waves_streamed = lane->ooc.waves_in_place = lane->ooc.parts_streamed = 0;
  lane->ooc.bytes_streamed = lane->ooc.waves_spilled = lane->ooc.bytes_spilled = 0;
}

void drop_batch_lane(gem_ctx *ctx) {
  if (!ctx->batch_lane) return;
  gem_ctx_destroy(ctx->batch_lane);
  ctx->batch_lane = nullptr;
  if (ctx->arena.reserved) ctx->arena.release(ctx);  // it held the lane-split budget
  if (ctx->batch_saved_budget) ctx->budget = ctx->batch_saved_budget;
  ctx->batch_saved_budget = 0;
}

extern "C" void gem_ctx_destroy(gem_ctx *ctx) {
  if (!ctx) return;
  server_shutdown(ctx);
  drop_batch_lane(ctx);
  cudaSetDevice(ctx->opts.device);
  cudaStreamSynchronize(ctx->s);
  ctx->arena.release(ctx);
  if (!ctx->borrowed_graph) free_graph(ctx);
  else if (ctx->part_mem) cudaFree(ctx->part_mem);  // a lane's own staging buffers
  if (ctx->ev_ref && !ctx->borrowed_graph) cudaEventDestroy(ctx->ev_ref);
  destroy_join_graph(ctx->jgraph);
  if (ctx->d_ctl) cudaFree(ctx->d_ctl);
  if (ctx->d_queue) cudaFree(ctx->d_queue);
  if (ctx->d_qends) cudaFree(ctx->d_qends);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->h_small) cudaFreeHost(ctx->h_small);
  for (auto &ev : ctx->ev)
    if (ev) cudaEventDestroy(ev);
  for (int b = 0; b < 2; ++b) {
    if (ctx->ev_ready[b]) cudaEventDestroy(ctx->ev_ready[b]);
    if (ctx->ev_free[b]) cudaEventDestroy(ctx->ev_free[b]);
  }
  if (ctx->s_copy) cudaStreamDestroy(ctx->s_copy);
  if (ctx->spill_host) cudaFreeHost(ctx->spill_host);
  if (ctx->s) cudaStreamDestroy(ctx->s);
  delete ctx;
}

extern "C" const char *gem_last_error(const gem_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

// Out-of-core: splits the adjacency into vertex ranges of at most
// ooc_part_kib KiB (a vertex whose list alone is longer gets a range of its
// own) and allocates the partition bounds and two staging buffers of the
// largest partition's size, plus the side stream and events of the copies.
// Partition bounds of a CSR: vertex ranges of at most cap_bytes of arcs (a
// vertex whose list alone is longer gets a range of its own), each as long
// as the bound allows.  pv gets the vertex bounds, pa their arc offsets.
static uint64_t partition_bounds(const gem_hgraph *hg, uint64_t cap_bytes, std::vector<uint32_t> &pv,
                                 std::vector<uint64_t> &pa) {
  const uint32_t nv = hg->nv;
  const uint64_t cap = cap_bytes / 4 ? cap_bytes / 4 : 1;  // arcs per partition
  pv.assign(1, 0);
  pa.assign(1, 0);
  uint64_t max_arcs = 0;
  for (uint32_t v = 0; v < nv;) {
    const uint64_t a0 = hg->off[v];
    uint32_t u = v + 1;
    if (hg->off[u] - a0 <= cap) {
      // the last u in (v, nv] with off[u] - a0 <= cap
      uint32_t lo = u, hi = nv + 1;
      while (hi - lo > 1) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (hg->off[mid] - a0 <= cap) lo = mid; else hi = mid;
      }
      u = lo;
    }
    pv.push_back(u);
    pa.push_back(hg->off[u]);
    max_arcs = std::max<uint64_t>(max_arcs, hg->off[u] - a0);
    v = u;
  }
  return max_arcs;
}

extern "C" gem_status gem_hgraph_partitions(const gem_hgraph *g, uint32_t part_kib, uint32_t *part_v, uint32_t cap,
                                            uint32_t *n_out) {
  if (!g || !n_out || (cap && !part_v)) return GEM_ERR_ARG;
  std::vector<uint32_t> pv;
  std::vector<uint64_t> pa;
  partition_bounds(g, (uint64_t)(part_kib ? part_kib : 16384u) << 10, pv, pa);
  *n_out = (uint32_t)pv.size() - 1;
  if (pv.size() > cap) return GEM_ERR_LIMIT;
  std::memcpy(part_v, pv.data(), 4 * pv.size());
  return GEM_OK;
}

static gem_status ooc_partitions(gem_ctx *ctx, const gem_hgraph *hg) {
  const uint64_t cap_bytes = (uint64_t)(ctx->opts.ooc_part_kib ? ctx->opts.ooc_part_kib : 16384u) << 10;
  const uint64_t max_arcs = partition_bounds(hg, cap_bytes, ctx->part_v, ctx->part_a);
  const uint32_t P = (uint32_t)ctx->part_v.size() - 1;
  auto al = [](uint64_t b) { return (b + 255) & ~255ull; };
  const uint64_t b_pv = al(4ull * (P + 1)), b_st = al(4ull * (max_arcs ? max_arcs : 1));
  const uint64_t total = b_pv + 2 * b_st;
  if (ctx->device_bytes + total > ctx->budget) {
    ctx->err = "out-of-core staging buffers do not fit the device budget";
    return GEM_ERR_OOM;
  }
  char *p = nullptr;
  if (cudaMalloc(&p, total) != cudaSuccess) {
    cudaGetLastError();
    ctx->err = "cudaMalloc out-of-core staging buffers";
    return GEM_ERR_OOM;
  }
  ctx->part_mem = p;
  ctx->part_bytes = total;
  ctx->device_bytes += total;
  ctx->d_part_v = (uint32_t *)p;
  ctx->d_stage[0] = (uint32_t *)(p + b_pv);
  ctx->d_stage[1] = (uint32_t *)(p + b_pv + b_st);
  CU(cudaMemcpyAsync(ctx->d_part_v, ctx->part_v.data(), 4ull * (P + 1), cudaMemcpyHostToDevice, ctx->s));
  if (!ctx->s_copy) CU(cudaStreamCreateWithFlags(&ctx->s_copy, cudaStreamNonBlocking));
  for (int b = 0; b < 2; ++b) {
    if (!ctx->ev_ready[b]) CU(cudaEventCreateWithFlags(&ctx->ev_ready[b], cudaEventDisableTiming));
    if (!ctx->ev_free[b]) CU(cudaEventCreateWithFlags(&ctx->ev_free[b], cudaEventDisableTiming));
  }
  ctx->ooc = gem_ooc_stats{};
  ctx->ooc.partitions = P;
  ctx->ooc.max_part_bytes = 4 * max_arcs;
  return GEM_OK;
}

extern "C" gem_status gem_ctx_ooc_stats(const gem_ctx *ctx, gem_ooc_stats *out) {
  if (!ctx || !out) return GEM_ERR_ARG;
  if (ctx->server) return GEM_ERR_STATE;  // the serving thread updates the counters
  *out = ctx->ooc;
  uint64_t arena = 0;
  for (const auto &c : ctx->arena.chunks) arena += c.size;
  out->resident_bytes = ctx->device_bytes - arena;
  return GEM_OK;
}

extern "C" gem_status gem_ctx_load_graph(gem_ctx *ctx, const gem_hgraph *hg) {
  if (!ctx || !hg) return GEM_ERR_ARG;
  if (ctx->server) return GEM_ERR_STATE;
  drop_batch_lane(ctx);
  CU(cudaSetDevice(ctx->opts.device));
  CU(cudaStreamSynchronize(ctx->s));
  ctx->arena.reset();
  free_graph(ctx);
  const uint32_t nv = hg->nv;
  const uint64_t na = hg->n_arcs();
  const uint32_t L = hg->max_label_plus1;
  const uint32_t stride = (L > 0 && L <= NLC_MAX_LABELS) ? ((L + 15) / 16) * 16 : 0;
  auto al = [](uint64_t b) { return (b + 255) & ~255ull; };
  const bool ooc = ctx->opts.ooc != 0;
  const uint64_t b_off = al(8ull * (nv + 1)), b_nbr = ooc ? 0 : al(4ull * na), b_lab = al(4ull * nv),
                 b_deg = al(4ull * nv), b_nlc = al((uint64_t)stride * nv);
  const uint64_t total = b_off + b_nbr + b_lab + b_deg + b_nlc;
  if (ctx->device_bytes + total > ctx->budget) {
    ctx->err = "graph does not fit the device budget";
    return GEM_ERR_OOM;
  }
  char *p = nullptr;
  cudaError_t e = cudaMalloc(&p, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->err = std::string("cudaMalloc graph: ") + cudaGetErrorString(e);
    return GEM_ERR_OOM;
  }
  ctx->graph_mem = p;
  ctx->graph_bytes = total;
  ctx->device_bytes += total;
  uint64_t *d_off = (uint64_t *)p;
  uint32_t *d_nbr = (uint32_t *)(p + b_off);
  uint32_t *d_lab = (uint32_t *)(p + b_off + b_nbr);
  uint32_t *d_deg = (uint32_t *)(p + b_off + b_nbr + b_lab);
  uint8_t *d_nlc = stride ? (uint8_t *)(p + b_off + b_nbr + b_lab + b_deg) : nullptr;
  CU(cudaMemcpyAsync(d_off, hg->off.data(), 8ull * (nv + 1), cudaMemcpyHostToDevice, ctx->s));
  if (ooc) {
    // Out-of-core: the adjacency array stays in pinned host memory mapped
    // into the device address space; kernels read it over the host link.
    if (ctx->opts.pinned_budget_bytes && 4ull * na > ctx->opts.pinned_budget_bytes) {
      ctx->err = "adjacency does not fit the pinned budget";
      return GEM_ERR_OOM;
    }
    void *h = nullptr;
    CU(cudaHostAlloc(&h, na ? 4ull * na : 4, cudaHostAllocMapped | cudaHostAllocPortable));
    ctx->pinned_nbr = h;
    ctx->host_nbr = h;
    if (na) std::memcpy(h, hg->nbr.data(), 4ull * na);
    CU(cudaHostGetDevicePointer((void **)&d_nbr, h, 0));
    const gem_status pst = ooc_partitions(ctx, hg);
    if (pst != GEM_OK) return pst;
  } else if (na) {
    CU(cudaMemcpyAsync(d_nbr, hg->nbr.data(), 4ull * na, cudaMemcpyHostToDevice, ctx->s));
  }
  if (nv) CU(cudaMemcpyAsync(d_lab, hg->lab.data(), 4ull * nv, cudaMemcpyHostToDevice, ctx->s));
  DevGraph g;
  g.nv = nv;
  g.narcs = na;
  g.nlabels = L;
  g.nlc_stride = stride;
  g.off = d_off;
  g.nbr = d_nbr;
  g.lab = d_lab;
  g.deg = d_deg;
  g.nlc = d_nlc;
  launch_degrees(g, d_deg, ctx->s);
  if (stride) launch_nlc(g, d_nlc, stride, ctx->s);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(ctx->s));
  // Neighbourhood hash for arc tests in the join, when it fits the device
  // budget with a quarter of the remaining budget left for the waves;
  // otherwise the join searches the sorted table lists instead.  Out of core
  // it is built from the mapped adjacency (one read over the host link) and
  // lives on the device like the tables the join reads.
  if (na) {
    std::vector<uint64_t> hoff(nv + 1);
    uint64_t n_slots = 0;
    for (uint32_t v = 0; v < nv; ++v) {
      hoff[v] = n_slots;
      const uint64_t d = hg->off[v + 1] - hg->off[v];
      if (d) {
        uint64_t size = 2;
        while (size < 2 * d) size <<= 1;
        n_slots += size;
      }
    }
    hoff[nv] = n_slots;
    const uint64_t b_hoff = al(8ull * (nv + 1)), b_slots = al(4ull * n_slots);
    const uint64_t left = ctx->budget > ctx->device_bytes ? ctx->budget - ctx->device_bytes : 0;
    char *hp = nullptr;
    if (b_hoff + b_slots <= left - left / 4 && cudaMalloc(&hp, b_hoff + b_slots) == cudaSuccess) {
      ctx->vnh_mem = hp;
      ctx->vnh_bytes = b_hoff + b_slots;
      ctx->device_bytes += ctx->vnh_bytes;
      ctx->vnh_off = (const uint64_t *)hp;
      ctx->vnh_slots = (const uint32_t *)(hp + b_hoff);
      CU(cudaMemcpyAsync(hp, hoff.data(), 8ull * (nv + 1), cudaMemcpyHostToDevice, ctx->s));
      launch_vnh_build(g, (const uint64_t *)hp, (uint32_t *)(hp + b_hoff), n_slots, ctx->s);
      CU(cudaGetLastError());
      CU(cudaStreamSynchronize(ctx->s));
    } else {
      cudaGetLastError();
    }
  }
  ctx->g = g;
  ctx->loaded = true;
  CU(cudaEventRecord(ctx->ev_ref, ctx->s));
  ctx->ev_ref_recorded = true;
  ctx->label_freq.assign(L, 0);
  ctx->label_arcs.assign(L, 0);
  for (uint32_t v = 0; v < nv; ++v) {
    ctx->label_freq[hg->lab[v]]++;
    ctx->label_arcs[hg->lab[v]] += hg->off[v + 1] - hg->off[v];
  }
  // arcs per (source label, target label): the largest any edge table between
  // vertices of those labels can be (bounds the serving admission estimate)
  ctx->label_pair_arcs.clear();
  if (L && L <= NLC_MAX_LABELS) {
    std::vector<uint64_t> pa((size_t)L * L, 0);
#pragma omp parallel
    {
      std::vector<uint64_t> mine((size_t)L * L, 0);
#pragma omp for schedule(dynamic, 4096) nowait
      for (int64_t v = 0; v < (int64_t)nv; ++v) {
        uint64_t *row = mine.data() + (size_t)hg->lab[v] * L;
        for (uint64_t i = hg->off[v]; i < hg->off[v + 1]; ++i) row[hg->lab[hg->nbr[i]]]++;
      }
#pragma omp critical
      for (size_t i = 0; i < pa.size(); ++i) pa[i] += mine[i];
    }
    ctx->label_pair_arcs.swap(pa);
  }
  return GEM_OK;
}

// ---------------------------------------------------------------------------
// Planner: matching order for the DFS join.
//
// Replaces the lattice + greedy edge choice of the reference
// (in-core/lib/structure/src/lattice.cpp:41-185, unifiedTrie.cu:939-1018),
// which at threshold 0 only decides the order of single-edge extensions.
// Here: root = fewest candidates per incident edge; then repeatedly the
// vertex with most already-placed neighbours (non-leaves first, then fewest
// candidates).  In count mode an independent set S of the query graph whose
// removal leaves the rest connected is moved to the end: no two suffix
// vertices are adjacent, so once the prefix is matched the suffix
// completions are counted by inclusion-exclusion over same-label groups
// (different labels have disjoint candidates) instead of being enumerated.
// ---------------------------------------------------------------------------
static bool connected_without(const HostQuery &q, uint32_t removed) {
  const uint32_t all = (q.nv == 32 ? 0xFFFFFFFFu : ((1u << q.nv) - 1)) & ~removed;
  if (!all) return false;
  uint32_t seen = all & (~all + 1), frontier = seen;
  while (frontier) {
    uint32_t nxt = 0;
    for (uint32_t u = 0; u < q.nv; ++u)
      if (frontier & (1u << u)) nxt |= q.adj[u];
    nxt &= all & ~seen;
    seen |= nxt;
    frontier = nxt;
  }
  return seen == all;
}

// All set partitions of {0..g-1}: term = coefficient prod_B (-1)^{|B|-1} (|B|-1)!
// with the blocks packed as 4-bit masks.
static void partition_terms(uint32_t g, std::vector<uint64_t> &out) {
  std::vector<uint32_t> blk(g, 0);
  std::function<void(uint32_t, uint32_t)> rec = [&](uint32_t i, uint32_t nb) {
    if (i == g) {
      uint32_t masks[MAX_GROUP] = {0, 0, 0, 0};
      for (uint32_t k = 0; k < g; ++k) masks[blk[k]] |= 1u << k;
      int32_t coef = 1;
      uint32_t packed = 0;
      for (uint32_t b = 0; b < nb; ++b) {
        const int sz = __builtin_popcount(masks[b]);
        int32_t f = 1;
        for (int t = 2; t < sz; ++t) f *= t;
        coef *= ((sz - 1) & 1) ? -f : f;
        packed |= masks[b] << (4 * b);
      }
      out.push_back(make_term(coef, packed));
      return;
    }
    for (uint32_t b = 0; b <= nb; ++b) {
      blk[i] = b;
      rec(i + 1, b == nb ? nb + 1 : nb);
    }
  };
  rec(0, 0);
}

void make_plan(const HostQuery &q, const uint32_t *cnt, bool count_suffix, Plan &p) {
  const uint32_t n = q.nv;
  p.n = n;
  // ---- closed-form suffix (independent set, prefix stays connected)
  uint32_t S = 0;
  if (count_suffix && n >= 2) {
    std::vector<uint32_t> cand(n);
    for (uint32_t u = 0; u < n; ++u) cand[u] = u;
    std::sort(cand.begin(), cand.end(), [&](uint32_t a, uint32_t b) {
      if (q.deg(a) != q.deg(b)) return q.deg(a) < q.deg(b);
      if (cnt[a] != cnt[b]) return cnt[a] > cnt[b];
      return a < b;
    });
    for (uint32_t u : cand) {
      if (q.adj[u] & S) continue;
      const uint32_t S2 = S | (1u << u);
      if (!connected_without(q, S2)) continue;
      uint32_t same = 0, nback = q.deg(u), groups = 0;
      for (uint32_t w = 0; w < n; ++w)
        if (S2 & (1u << w)) {
          if (q.lab[w] == q.lab[u]) {
            ++same;
            if (w != u) nback += q.deg(w);
          }
        }
      if (same > MAX_GROUP || nback > 32) continue;
      uint32_t seen_labels[QV], nl = 0;
      for (uint32_t w = 0; w < n; ++w)
        if (S2 & (1u << w)) {
          bool f = false;
          for (uint32_t t = 0; t < nl; ++t) f |= seen_labels[t] == q.lab[w];
          if (!f) seen_labels[nl++] = q.lab[w];
        }
      groups = nl;
      if (groups > MAX_GROUPS) continue;
      S = S2;
    }
  }
  const uint32_t nenum = n - (uint32_t)__builtin_popcount(S);
  p.n_enum = nenum;
  // ---- prefix order
  uint32_t used = 0;
  for (uint32_t k = 0; k < nenum; ++k) {
    int best = -1;
    uint64_t bkey[5] = {0, 0, 0, 0, 0};
    for (uint32_t u = 0; u < n; ++u) {
      if ((used | S) & (1u << u)) continue;
      const uint32_t back = __builtin_popcount(q.adj[u] & used);
      if (k > 0 && back == 0) continue;
      const uint32_t d = q.deg(u);
      uint64_t key[5];
      if (k == 0) {
        key[0] = (uint64_t)((double)cnt[u] / (double)(d + 1) * 1024.0);
        key[1] = ~(uint64_t)d;
        key[2] = u;
        key[3] = key[4] = 0;
      } else {
        key[0] = ~(uint64_t)back;
        key[1] = d <= 1 ? 1 : 0;
        key[2] = cnt[u];
        key[3] = ~(uint64_t)d;
        key[4] = u;
      }
      if (best < 0 || std::lexicographical_compare(key, key + 5, bkey, bkey + 5)) {
        best = (int)u;
        std::memcpy(bkey, key, sizeof key);
      }
    }
    const uint32_t u = (uint32_t)best;
    p.order[k] = u;
    p.level_of[u] = k;
    used |= 1u << u;
  }
  // ---- suffix levels grouped by label
  std::vector<uint32_t> suf;
  for (uint32_t u = 0; u < n; ++u)
    if (S & (1u << u)) suf.push_back(u);
  std::stable_sort(suf.begin(), suf.end(), [&](uint32_t a, uint32_t b) { return q.lab[a] < q.lab[b]; });
  for (size_t i = 0; i < suf.size(); ++i) {
    p.order[nenum + i] = suf[i];
    p.level_of[suf[i]] = nenum + (uint32_t)i;
  }
  p.groups.clear();
  for (size_t i = 0; i < suf.size();) {
    size_t j = i;
    while (j < suf.size() && q.lab[suf[j]] == q.lab[suf[i]]) ++j;
    Plan::Group gr;
    gr.first = nenum + (uint32_t)i;
    gr.size = (uint32_t)(j - i);
    partition_terms(gr.size, gr.terms);
    p.groups.push_back(gr);
    i = j;
  }
  // ---- backward neighbours, injectivity masks, index needs
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t u = p.order[k];
    p.back[k].clear();
    p.dup_mask[k] = 0;
    const uint32_t lim = k < nenum ? k : nenum;  // suffix levels see the prefix only
    for (uint32_t j = 0; j < k; ++j)
      if (q.adj[u] & (1u << p.order[j])) p.back[k].push_back(j);
    for (uint32_t j = 0; j < lim; ++j)
      if (q.lab[p.order[j]] == q.lab[u]) p.dup_mask[k] |= 1u << j;
    p.need_idx[k] = 0;
  }
  for (uint32_t k = 0; k < n; ++k)
    for (uint32_t j : p.back[k]) p.need_idx[j] = 1;
}

// Structural checks of a plan (host side, before anything reaches the device).
static bool validate_plan(const HostQuery &q, const Plan &p, std::string &why) {
  if (p.n != q.nv || p.n_enum < 1 || p.n_enum > p.n) return why = "level counts", false;
  uint32_t seen = 0;
  for (uint32_t k = 0; k < p.n; ++k) {
    if (p.order[k] >= q.nv || (seen & (1u << p.order[k]))) return why = "order is not a permutation", false;
    seen |= 1u << p.order[k];
    if (k > 0 && p.back[k].empty()) return why = "level without backward neighbour", false;
    for (uint32_t j : p.back[k]) {
      if (j >= k) return why = "backward neighbour after its level", false;
      if (k >= p.n_enum && j >= p.n_enum) return why = "suffix level keyed by a suffix level", false;
      if (!p.need_idx[j]) return why = "key level without index", false;
    }
    if (p.dup_mask[k] >> (k < p.n_enum ? k : p.n_enum)) return why = "injectivity mask beyond the prefix", false;
  }
  uint32_t covered = 0;
  for (const auto &g : p.groups) {
    if (g.size == 0 || g.size > MAX_GROUP || g.first < p.n_enum || g.first + g.size > p.n)
      return why = "suffix group bounds", false;
    uint32_t nb = 0;
    for (uint32_t k = g.first; k < g.first + g.size; ++k) nb += (uint32_t)p.back[k].size();
    if (nb > 32) return why = "suffix group lists", false;
    covered += g.size;
  }
  if (p.groups.size() > MAX_GROUPS || covered != p.n - p.n_enum) return why = "suffix groups", false;
  return true;
}

extern "C" gem_status gem_plan_query(const gem_query *q, const uint32_t *cand_counts, int closed_form,
                                     uint32_t *n_enum, uint32_t *order_out) {
  if (!q || !cand_counts || !n_enum || !order_out) return GEM_ERR_ARG;
  HostQuery hq;
  std::string err;
  const gem_status st = make_host_query(q, hq, err);
  if (st != GEM_OK) return st;
  Plan p;
  make_plan(hq, cand_counts, closed_form != 0, p);
  if (!validate_plan(hq, p, err)) return GEM_ERR_INTERNAL;
  *n_enum = p.n_enum;
  for (uint32_t k = 0; k < p.n; ++k) order_out[k] = p.order[k];
  return GEM_OK;
}

// ---------------------------------------------------------------------------
// Wave pipeline
// ---------------------------------------------------------------------------
struct EvPair {
  cudaEvent_t a, b;
};

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return ms;
}

// Runs the filter for every query of the wave; fills w.rows / counts / lists.
// Balanced lane-level counting code of a plan (JQuery::flat): the subset
// values per prefix match (at most FLAT_MAX_VALUES, each an intersection of
// at most three lists) and those needing a scan, or 0 when not eligible.
static uint32_t flat_code(const Plan &p, int mode) {
  if (mode != GEM_MODE_COUNT || p.groups.empty()) return 0;
  uint32_t nval = 0, nscan = 0;
  for (const Plan::Group &g : p.groups)
    for (uint32_t S = 1; S < (1u << g.size); ++S) {
      uint32_t nl = 0;
      for (uint32_t b = 0; b < g.size; ++b)
        if (S & (1u << b)) nl += (uint32_t)p.back[g.first + b].size();
      if (nl < 1 || nl > 3) return 0;
      ++nval;
      nscan += nl >= 2;
    }
  return nval <= FLAT_MAX_VALUES ? nval | (nscan << 8) : 0;
}

// Queries counted through the (root, first level) pair pool: count mode, an
// enumerated prefix of a root and one neighbour level, a closed-form suffix
// eligible for balanced counting, and the neighbourhood hash.
static bool pair_pool(const gem_ctx *ctx, const Plan &p, int mode) {
  return ctx->vnh_off && mode == GEM_MODE_COUNT && p.n_enum == 2 && p.n >= 3 && flat_code(p, mode) != 0;
}

// A slice of the pinned staging buffer for one copy of the current wave, or
// null when it is used up (the copy then goes through pageable memory).
static void *stage(gem_ctx *ctx, size_t bytes) {
  const size_t at = (ctx->h_used + 255) & ~(size_t)255;
  if (!ctx->h_small || at + bytes > H_SMALL_BYTES) return nullptr;
  ctx->h_used = at + bytes;
  return static_cast<char *>(ctx->h_small) + at;
}

// Host-to-device copy on the context's stream through pinned staging: the
// source may be reused as soon as this returns.
static cudaError_t h2d(gem_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (!bytes) return cudaSuccess;
  void *st = stage(ctx, bytes);
  if (!st) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->s);
  std::memcpy(st, src, bytes);
  return cudaMemcpyAsync(dst, st, bytes, cudaMemcpyHostToDevice, ctx->s);
}

// Device-to-host copy that completes with a stream synchronisation.
static cudaError_t d2h_sync(gem_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (!bytes) return cudaSuccess;
  void *st = stage(ctx, bytes);
  cudaError_t e = cudaMemcpyAsync(st ? st : dst, src, bytes, cudaMemcpyDeviceToHost, ctx->s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->s);
  if (e == cudaSuccess && st) std::memcpy(dst, st, bytes);
  return e;
}

static gem_status wave_filter(gem_ctx *ctx, Wave &w, uint32_t threshold) {
  const uint32_t nwords = (ctx->g.nv + 31) / 32;
  w.nwords = nwords;
  // Rows.  The filter predicate of a query vertex depends only on its label,
  // its degree and its neighbours' labels, so vertices that agree on the
  // three (in one query or in several) share one row: its candidate list,
  // rank bitmap and the tables it keys.
  std::map<std::vector<uint32_t>, uint32_t> row_by_sig;
  std::vector<std::vector<uint32_t>> row_sig;
  w.row_of.assign(w.q.size(), std::vector<uint32_t>());
  for (size_t i = 0; i < w.q.size(); ++i) {
    const HostQuery &q = w.sig_query ? *w.sig_query : w.q[i];
    w.row_of[i].resize(q.nv);
    for (uint32_t u = 0; u < q.nv; ++u) {
      std::vector<uint32_t> sig{q.lab[u], q.deg(u)};
      for (uint32_t v = 0; v < q.nv; ++v)
        if (q.adj[u] & (1u << v)) sig.push_back(q.lab[v]);
      std::sort(sig.begin() + 2, sig.end());
      if (w.share_rows) {
        const auto it = row_by_sig.find(sig);
        if (it != row_by_sig.end()) {
          w.row_of[i][u] = it->second;
          continue;
        }
        row_by_sig.emplace(sig, (uint32_t)row_sig.size());
      }
      w.row_of[i][u] = (uint32_t)row_sig.size();
      row_sig.push_back(std::move(sig));
    }
  }
  const uint32_t rows = (uint32_t)row_sig.size();
  // descriptors: runs of up to QV rows whose neighbour labels number at most QV
  std::vector<FilterDesc> fd;
  for (uint32_t r = 0; r < rows;) {
    FilterDesc d;
    std::memset(&d, 0, sizeof d);
    d.threshold = threshold;
    d.row_base = r;
    while (r < rows && d.nq < QV) {
      const std::vector<uint32_t> &sg = row_sig[r];
      uint32_t extra = 0;
      for (size_t i = 2; i < sg.size(); ++i) {
        bool seen = false;
        for (uint32_t k = 0; k < d.nql && !seen; ++k) seen = d.ql[k] == sg[i];
        for (size_t j = 2; j < i && !seen; ++j) seen = sg[j] == sg[i];
        extra += seen ? 0u : 1u;
      }
      if (d.nq && d.nql + extra > QV) break;
      d.lab[d.nq] = sg[0];
      d.deg[d.nq] = sg[1];
      for (size_t i = 2; i < sg.size(); ++i) {
        uint32_t k = 0;
        while (k < d.nql && d.ql[k] != sg[i]) ++k;
        if (k == d.nql) d.ql[d.nql++] = sg[i];
        d.nlc[d.nq][k]++;
      }
      ++d.nq;
      ++r;
    }
    fd.push_back(d);
  }
  w.nrows = rows;
  FilterDesc *d_fd;
  ST(aalloc(ctx, fd.size(), &d_fd));
  CU(h2d(ctx, d_fd, fd.data(), fd.size() * sizeof(FilterDesc)));
  const uint64_t nbits = (uint64_t)rows * nwords;
  ST(aalloc(ctx, nbits, &w.d_rb));
  uint64_t *d_ex, *d_tmp, *d_rows;
  ST(aalloc(ctx, nbits + 1, &d_ex));
  ST(aalloc(ctx, scan_tmp_words(nbits), &d_tmp));
  ST(aalloc(ctx, rows + 1, &d_rows));
  launch_filter(ctx->g, d_fd, (uint32_t)fd.size(), w.d_rb, nwords, ctx->s);
  launch_scan(w.d_rb, SCAN_POPC_U64LO, nbits, d_ex, d_tmp, ctx->s);
  launch_gather_strided(d_ex, nwords, rows + 1, d_rows, ctx->s);
  std::vector<uint64_t> rs(rows + 1);
  CU(d2h_sync(ctx, rs.data(), d_rows, 8ull * (rows + 1)));
  CU(cudaGetLastError());
  w.cnt.resize(rows);
  w.c_base.resize(rows + 1);
  for (uint32_t r = 0; r < rows; ++r) w.cnt[r] = (uint32_t)(rs[r + 1] - rs[r]);
  for (uint32_t r = 0; r <= rows; ++r) w.c_base[r] = rs[r] - rs[0];
  const uint64_t total = w.c_base[rows];
  uint64_t *d_cbase;
  ST(aalloc(ctx, rows + 1, &d_cbase));
  CU(h2d(ctx, d_cbase, w.c_base.data(), 8ull * (rows + 1)));
  ST(aalloc(ctx, total ? total : 1, &w.d_cand));
  ST(aalloc(ctx, nbits, &w.d_bits));
  launch_compact(w.d_rb, d_ex, rows, nwords, d_cbase, w.d_cand, ctx->s, w.d_bits);
  CU(cudaGetLastError());
  w.cand_total = total;
  // algorithmic bytes, per descriptor: labels + degrees of every vertex, the
  // label-count rows of vertices whose label occurs in its rows' neighbour
  // labels, its bit rows (write, scan, rank rewrite); then the candidate lists.
  uint64_t b = 0;
  for (const FilterDesc &d : fd) {
    uint64_t lb = 8ull * ctx->g.nv;
    for (uint32_t k = 0; k < d.nql; ++k)
      if (d.ql[k] < ctx->label_freq.size()) lb += (uint64_t)ctx->g.nlc_stride * ctx->label_freq[d.ql[k]];
    lb += 8ull * nwords * d.nq * 4;
    b += lb;
  }
  w.bytes_filter = b + 4 * total;
  return GEM_OK;
}

// Mapped pinned host memory of at least `bytes` for spilled table values
// (kept between waves, grown when needed, within the pinned budget).
static gem_status spill_buffer(gem_ctx *ctx, uint64_t bytes) {
  if (ctx->spill_bytes >= bytes) return GEM_OK;
  const uint64_t pinned_nbr = ctx->pinned_nbr ? 4ull * ctx->g.narcs : 0;
  if (ctx->opts.pinned_budget_bytes && pinned_nbr + bytes > ctx->opts.pinned_budget_bytes) {
    ctx->err = "edge tables exceed both the device and the pinned budget";
    return GEM_ERR_OOM;
  }
  if (ctx->spill_host) {
    CU(cudaStreamSynchronize(ctx->s));
    cudaFreeHost(ctx->spill_host);
    ctx->spill_host = ctx->spill_dev = nullptr;
    ctx->spill_bytes = 0;
  }
  const uint64_t sz = std::max<uint64_t>(bytes, 1ull << 30);
  if (cudaHostAlloc(&ctx->spill_host, sz, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    ctx->spill_host = nullptr;
    ctx->err = "pinned host memory for spilled edge tables unavailable";
    return GEM_ERR_OOM;
  }
  CU(cudaHostGetDevicePointer(&ctx->spill_dev, ctx->spill_host, 0));
  ctx->spill_bytes = sz;
  return GEM_OK;
}

static gem_status wave_tables(gem_ctx *ctx, Wave &w) {
  // sources and edges of every active query
  std::vector<TabSource> src;
  std::vector<TabEdge> edge;
  std::vector<uint32_t> src_row;
  std::vector<int> row_src(w.nrows, -1);
  uint64_t nkeys = 0;
  for (size_t qi = 0; qi < w.q.size(); ++qi) {
    if (!w.active[qi]) continue;
    const Plan &p = w.plan[qi];
    for (uint32_t k = 1; k < p.n; ++k)
      for (uint32_t j : p.back[k]) {
        const uint32_t r = w.row_of[qi][p.order[j]];
        if (row_src[r] < 0) {
          row_src[r] = (int)src.size();
          TabSource s;
          s.keys = w.d_cand + w.c_base[r];
          s.nkeys = w.cnt[r];
          s.pad = 0;
          s.key_base = nkeys;
          nkeys += w.cnt[r];
          src.push_back(s);
          src_row.push_back(r);
        }
      }
  }
  w.nsrc = (uint32_t)src.size();
  if (src.empty()) return GEM_OK;
  TabSource *d_src;
  ST(aalloc(ctx, src.size(), &d_src));
  CU(h2d(ctx, d_src, src.data(), src.size() * sizeof(TabSource)));
  uint32_t *d_tiles;
  uint64_t *d_tp, *d_tmp, *d_stb;
  ST(aalloc(ctx, nkeys ? nkeys : 1, &d_tiles));
  ST(aalloc(ctx, nkeys + 1, &d_tp));
  ST(aalloc(ctx, scan_tmp_words(nkeys), &d_tmp));
  ST(aalloc(ctx, src.size() + 3, &d_stb));
  launch_key_tiles(ctx->g, d_src, (uint32_t)src.size(), nkeys, d_tiles, ctx->s);
  launch_scan(d_tiles, SCAN_U32, nkeys, d_tp, d_tmp, ctx->s);
  launch_source_tile_bases(d_src, (uint32_t)src.size(), nkeys, d_tp, d_stb, ctx->s);
  // Vertex tiles: which sources hold each vertex (the source membership
  // columns, WS words per vertex) and the 32-arc tiles of every vertex that
  // some source holds; the table passes walk those tiles once for all sources.
  const uint32_t nv = ctx->g.nv;
  const uint32_t WS = (uint32_t)((src.size() + 31) / 32);
  uint32_t *d_srow, *d_S, *d_vtiles;
  uint64_t *d_vtp, *d_tmp3;
  ST(aalloc(ctx, src.size(), &d_srow));
  CU(h2d(ctx, d_srow, src_row.data(), 4 * src_row.size()));
  ST(aalloc(ctx, (uint64_t)nv * WS, &d_S));
  ST(aalloc(ctx, nv ? nv : 1, &d_vtiles));
  ST(aalloc(ctx, (uint64_t)nv + 1, &d_vtp));
  ST(aalloc(ctx, scan_tmp_words(nv), &d_tmp3));
  launch_row_columns(w.d_bits, w.nwords, d_srow, (uint32_t)src.size(), WS, nv, d_S, d_vtiles, ctx->g.deg, ctx->s);
  launch_scan(d_vtiles, SCAN_U32, nv, d_vtp, d_tmp3, ctx->s);
  // the write pass's units: up to TAB_WGROUP consecutive tiles of one vertex
  uint32_t *d_vunits;
  uint64_t *d_vgp;
  ST(aalloc(ctx, nv ? nv : 1, &d_vunits));
  ST(aalloc(ctx, (uint64_t)nv + 1, &d_vgp));
  launch_unit_counts(d_vtiles, nv, d_vunits, ctx->s);
  launch_scan(d_vunits, SCAN_U32, nv, d_vgp, d_tmp3, ctx->s);
  CU(cudaMemcpyAsync(d_stb + src.size() + 1, d_vtp + nv, 8, cudaMemcpyDeviceToDevice, ctx->s));
  CU(cudaMemcpyAsync(d_stb + src.size() + 2, d_vgp + nv, 8, cudaMemcpyDeviceToDevice, ctx->s));
  std::vector<uint64_t> stb(src.size() + 3);
  CU(d2h_sync(ctx, stb.data(), d_stb, 8 * stb.size()));
  CU(cudaGetLastError());
  const uint64_t vtiles = stb[src.size() + 1], vunits = stb[src.size() + 2];
  // edges, grouped by source: a source's tables are one range of the edges
  struct EdgeReq {
    uint32_t s, qi, j, k;
  };
  std::vector<EdgeReq> reqs;
  w.edge_of.assign(w.q.size(), {});
  for (size_t qi = 0; qi < w.q.size(); ++qi) {
    if (!w.active[qi]) continue;
    const Plan &p = w.plan[qi];
    w.edge_of[qi].assign((size_t)p.n * QV, UINT32_MAX);
    for (uint32_t k = 1; k < p.n; ++k)
      for (uint32_t j : p.back[k])
        reqs.push_back({(uint32_t)row_src[w.row_of[qi][p.order[j]]], (uint32_t)qi, j, k});
  }
  std::stable_sort(reqs.begin(), reqs.end(), [](const EdgeReq &x, const EdgeReq &y) { return x.s < y.s; });
  std::vector<uint32_t> sedge(2 * src.size(), 0);
  uint64_t tiles = 0, offs = 0;
  bool key_map = false;
  // a table is keyed by its source row and filtered by its target row: queries
  // (or twin query vertices) that need the same pair share one table
  std::map<std::pair<uint32_t, uint32_t>, uint32_t> edge_by_rows;
  std::vector<uint32_t> tgt_row;  // the target rows, one membership column bit each
  std::vector<int> row_tcol(w.nrows, -1);
  for (const EdgeReq &rq : reqs) {
    const Plan &p = w.plan[rq.qi];
    const uint32_t tgt = w.row_of[rq.qi][p.order[rq.k]];
    const uint32_t flags = (rq.qi < w.pair.size() && w.pair[rq.qi] && rq.j == 0 && rq.k == 1) ? TAB_KEY_MAP : 0u;
    key_map |= flags != 0;
    const auto found = edge_by_rows.find({rq.s, tgt});
    if (found != edge_by_rows.end()) {
      edge[found->second].flags |= flags;
      w.edge_of[rq.qi][rq.j * QV + rq.k] = found->second;
      continue;
    }
    edge_by_rows.emplace(std::make_pair(rq.s, tgt), (uint32_t)edge.size());
    TabEdge e;
    e.src = rq.s;
    e.flags = flags;
    if (row_tcol[tgt] < 0) {
      row_tcol[tgt] = (int)tgt_row.size();
      tgt_row.push_back(tgt);
    }
    e.tcol = (uint32_t)row_tcol[tgt];
    e.pad = 0;
    e.tile_base = tiles;
    e.ntiles = stb[rq.s + 1] - stb[rq.s];
    e.off_base = offs;
    e.offsets = nullptr;
    tiles += e.ntiles;
    offs += (uint64_t)src[rq.s].nkeys + 1;
    if (sedge[2 * rq.s + 1] == 0) sedge[2 * rq.s] = (uint32_t)edge.size();
    sedge[2 * rq.s + 1]++;
    w.edge_of[rq.qi][rq.j * QV + rq.k] = (uint32_t)edge.size();
    edge.push_back(e);
  }
  const uint64_t src_tiles = stb[src.size()];
  uint64_t *d_offs;
  ST(aalloc(ctx, offs, &d_offs));
  for (auto &e : edge) e.offsets = d_offs + e.off_base;
  TabEdge *d_edge;
  ST(aalloc(ctx, edge.size(), &d_edge));
  CU(h2d(ctx, d_edge, edge.data(), edge.size() * sizeof(TabEdge)));
  uint32_t *d_mask;
  uint64_t *d_vp, *d_tmp2;
  ST(aalloc(ctx, tiles ? tiles : 1, &d_mask));
  ST(aalloc(ctx, tiles + 1, &d_vp));
  ST(aalloc(ctx, scan_tmp_words(tiles), &d_tmp2));
  // the target membership columns, the tile -> vertex map, and the sources
  // and tables as the passes read them
  // target columns: whole 16-byte chunks per vertex (the count pass stages
  // them with 16-byte asynchronous copies)
  const uint32_t WT = (uint32_t)((tgt_row.size() + 127) / 128 * 4);
  if (!table_vtx_fits(WT)) {
    ctx->err = "too many edge-table target rows in one wave";
    return GEM_ERR_LIMIT;
  }
  uint32_t *d_trow, *d_B, *d_vt;
  ST(aalloc(ctx, tgt_row.size(), &d_trow));
  CU(h2d(ctx, d_trow, tgt_row.data(), 4 * tgt_row.size()));
  ST(aalloc(ctx, (uint64_t)nv * WT, &d_B));
  launch_row_columns(w.d_bits, w.nwords, d_trow, (uint32_t)tgt_row.size(), WT, nv, d_B, nullptr, nullptr, ctx->s);
  uint32_t *d_vg;
  ST(aalloc(ctx, vtiles ? vtiles : 1, &d_vt));
  launch_vertex_tile_map(d_vtp, nv, d_vt, ctx->s);
  ST(aalloc(ctx, vunits ? vunits : 1, &d_vg));
  launch_vertex_tile_map(d_vgp, nv, d_vg, ctx->s);
  std::vector<VSrc> vs(src.size());
  for (size_t i = 0; i < src.size(); ++i)
    vs[i] = VSrc{w.d_rb + (uint64_t)src_row[i] * w.nwords, src[i].key_base, stb[i], sedge[2 * i], sedge[2 * i + 1]};
  std::vector<VEdge> ve(edge.size());
  for (size_t i = 0; i < edge.size(); ++i) ve[i] = VEdge{edge[i].tile_base, edge[i].tcol, edge[i].flags};
  VSrc *d_vs;
  VEdge *d_ve;
  ST(aalloc(ctx, vs.size(), &d_vs));
  CU(h2d(ctx, d_vs, vs.data(), vs.size() * sizeof(VSrc)));
  ST(aalloc(ctx, ve.size(), &d_ve));
  CU(h2d(ctx, d_ve, ve.data(), ve.size() * sizeof(VEdge)));
  // Out-of-core: the vertex tiles of a partition (a vertex range) are one
  // range of the tile order.  Stream the partitions that hold tiles when
  // they are filled enough (their bytes at most twice what the tiles would
  // read from the mapped adjacency), else read in place.
  const uint32_t nparts = ctx->part_v.empty() ? 0u : (uint32_t)ctx->part_v.size() - 1;
  std::vector<uint64_t> pstart, pstart_w;  // each partition's first tile and first write unit
  bool streamed = false;
  if (ctx->opts.ooc && nparts && ctx->opts.ooc_stream != 2 && vtiles) {
    uint64_t *d_pb;
    ST(aalloc(ctx, 2ull * (nparts + 1), &d_pb));
    launch_gather_u64(d_vtp, ctx->d_part_v, nparts + 1, d_pb, ctx->s);
    launch_gather_u64(d_vgp, ctx->d_part_v, nparts + 1, d_pb + nparts + 1, ctx->s);
    std::vector<uint64_t> pb(2ull * (nparts + 1));
    CU(d2h_sync(ctx, pb.data(), d_pb, 16ull * (nparts + 1)));
    pstart.assign(pb.begin(), pb.begin() + nparts + 1);
    pstart_w.assign(pb.begin() + nparts + 1, pb.end());
    uint64_t need = 0;
    for (uint32_t p = 0; p < nparts; ++p)
      if (pstart[p + 1] > pstart[p]) need += 4 * (ctx->part_a[p + 1] - ctx->part_a[p]);
    streamed = ctx->opts.ooc_stream == 1 || need <= 2 * 128 * vtiles;
  }
  if (ctx->opts.ooc) ++(streamed ? ctx->ooc.waves_streamed : ctx->ooc.waves_in_place);
  // One table pass (count or write) over every vertex tile: in place, or
  // partition by partition with the copy of the next partition (side
  // stream, the other staging buffer) overlapping the kernel of the current one.
  unsigned long long *d_next;
  ST(aalloc(ctx, 1, &d_next));
  auto table_pass = [&](bool write) -> gem_status {
    VPass P;
    std::memset(&P, 0, sizeof P);
    P.next = d_next;
    P.off = ctx->g.off;
    P.nbr = ctx->g.nbr;
    P.arc_shift = 0;
    P.t0 = 0;
    P.t1 = write ? vunits : vtiles;
    P.vt = d_vt;
    P.vtp = d_vtp;
    P.vg = d_vg;
    P.vgp = d_vgp;
    P.S = d_S;
    P.WS = WS;
    P.WT = WT;
    P.B = d_B;
    P.vsrc = d_vs;
    P.vedge = d_ve;
    P.tp = d_tp;
    P.mask = d_mask;
    P.vp = d_vp;
    P.values = w.d_values;
    P.vkey = w.d_vkey;
    if (!streamed) {
      launch_table_vtx(P, write, ctx->s);
      return GEM_OK;
    }
    // a staging buffer is free once the main stream has passed what used it
    CU(cudaEventRecord(ctx->ev_free[0], ctx->s));
    CU(cudaEventRecord(ctx->ev_free[1], ctx->s));
    uint32_t k = 0;
    for (uint32_t p = 0; p < nparts; ++p) {
      if (pstart[p + 1] == pstart[p]) continue;
      const int b = (int)(k++ & 1u);
      const uint64_t a0 = ctx->part_a[p], bytes = 4 * (ctx->part_a[p + 1] - a0);
      CU(cudaStreamWaitEvent(ctx->s_copy, ctx->ev_free[b], 0));
      CU(cudaMemcpyAsync(ctx->d_stage[b], static_cast<const uint32_t *>(ctx->host_nbr) + a0, bytes,
                         cudaMemcpyHostToDevice, ctx->s_copy));
      CU(cudaEventRecord(ctx->ev_ready[b], ctx->s_copy));
      CU(cudaStreamWaitEvent(ctx->s, ctx->ev_ready[b], 0));
      P.nbr = ctx->d_stage[b];
      P.arc_shift = a0;
      P.t0 = write ? pstart_w[p] : pstart[p];
      P.t1 = write ? pstart_w[p + 1] : pstart[p + 1];
      launch_table_vtx(P, write, ctx->s);
      CU(cudaEventRecord(ctx->ev_free[b], ctx->s));
      ctx->ooc.parts_streamed += 1;
      ctx->ooc.bytes_streamed += bytes;
    }
    return GEM_OK;
  };
  CU(cudaEventRecord(ctx->ev[8], ctx->s));
  ST(table_pass(false));
  CU(cudaEventRecord(ctx->ev[9], ctx->s));
  launch_scan(d_mask, SCAN_POPC_U32, tiles, d_vp, d_tmp2, ctx->s);
  // every table's first value position and the total (table sizes order the
  // wave's queries by estimated join work)
  uint64_t *d_ebase;
  ST(aalloc(ctx, edge.size() + 1, &d_ebase));
  launch_edge_value_bases(d_edge, (uint32_t)edge.size(), d_vp, tiles, d_ebase, ctx->s);
  std::vector<uint64_t> ebase(edge.size() + 1);
  CU(d2h_sync(ctx, ebase.data(), d_ebase, 8 * ebase.size()));
  CU(cudaGetLastError());
  const uint64_t nvals = ebase[edge.size()];
  w.edge_vals.resize(edge.size());
  for (size_t e = 0; e < edge.size(); ++e) w.edge_vals[e] = ebase[e + 1] - ebase[e];
  // The values (and key positions) of the wave's tables.  Out of core, a
  // single query whose tables do not fit the device budget keeps them in
  // mapped pinned host memory, which the write pass and the join reach over
  // the host link; a batch wave that does not fit is split instead.
  w.d_vkey = nullptr;
  const uint64_t nv_alloc = nvals ? nvals : 1;
  gem_status vst = aalloc(ctx, nv_alloc, &w.d_values);
  if (vst == GEM_OK && key_map) vst = aalloc(ctx, nv_alloc, &w.d_vkey);
  if (vst == GEM_ERR_OOM && ctx->opts.ooc && w.q.size() == 1) {
    const uint64_t need = 4 * nv_alloc * (key_map ? 2 : 1);
    ST(spill_buffer(ctx, need));
    w.d_values = static_cast<uint32_t *>(ctx->spill_dev);
    w.d_vkey = key_map ? w.d_values + nv_alloc : nullptr;
    ctx->err.clear();
    ctx->ooc.waves_spilled += 1;
    ctx->ooc.bytes_spilled += need;
  } else if (vst != GEM_OK) {
    return vst;
  }
  launch_table_offsets(d_src, d_edge, (uint32_t)edge.size(), d_tp, d_vp, offs, ctx->s);
  CU(cudaEventRecord(ctx->ev[10], ctx->s));
  ST(table_pass(true));
  CU(cudaEventRecord(ctx->ev[11], ctx->s));
  w.table_passes = true;
  CU(cudaGetLastError());
  w.edges = edge;
  w.table_values = nvals;
  w.table_tiles = tiles;
  // algorithmic bytes of the two passes: per vertex tile (each pass) its
  // offsets, 32 neighbour ids and source column, and (count) the 32 target
  // columns; per tile of a source (each pass) the rank word and tile base;
  // per table tile the mask written and read and the value position; per
  // value its id (and key position); the offsets; per key its tile count
  // and scan.
  w.bytes_tables = 2 * vtiles * (16 + 32ull * 4 + 4ull * WS) + vtiles * 32ull * 4 * WT + 2 * src_tiles * 16 +
                   tiles * (4 + 4 + 8) + nvals * (key_map ? 8 : 4) + offs * 8 + nkeys * (4 + 8 + 4);
  return GEM_OK;
}

static gem_status wave_index(gem_ctx *ctx, Wave &w) {
  std::vector<CuckooTable> tabs;
  std::vector<std::pair<uint32_t, uint32_t>> who;  // (query, level)
  uint64_t slots = 0, kb = 0;
  for (size_t qi = 0; qi < w.q.size(); ++qi) {
    if (!w.active[qi]) continue;
    const Plan &p = w.plan[qi];
    for (uint32_t k = 0; k < p.n; ++k) {
      w.idx_kind[qi][k] = IDX_NONE;
      if (k == 0 || !p.need_idx[k]) continue;
      const uint32_t r = w.row_of[qi][p.order[k]];
      uint32_t kind = ctx->opts.index_kind;
      if (kind == 0) kind = IDX_RANK;
      w.idx_kind[qi][k] = kind;
      if (kind != IDX_CUCKOO) continue;
      CuckooTable t;
      std::memset(&t, 0, sizeof t);
      t.keys = w.d_cand + w.c_base[r];
      t.nkeys = w.cnt[r];
      t.key_base = kb;
      kb += t.nkeys;
      uint64_t ns = cuckoo_slots_for(t.nkeys, &t.nb0, &t.nb1);
      t.pad = (uint32_t)(slots >> 32);  // unused
      uint64_t seed = mix64(0x43554B4Full ^ ((uint64_t)qi << 32) ^ k ^ ((uint64_t)w.cuckoo_round << 48));
      t.a0 = mix64(seed) | 1ull;
      t.c0 = mix64(seed + 1);
      t.a1 = mix64(seed + 2) | 1ull;
      t.c1 = mix64(seed + 3);
      slots += ns;
      tabs.push_back(t);
      who.push_back({(uint32_t)qi, k});
    }
  }
  w.ck_tabs = nullptr;
  if (tabs.empty()) return GEM_OK;
  uint64_t *d_slots;
  uint32_t *d_sn;
  ST(aalloc(ctx, slots, &d_slots));
  ST(aalloc(ctx, tabs.size(), &d_sn));
  CU(cudaMemsetAsync(d_slots, 0xFF, slots * 8, ctx->s));
  CU(cudaMemsetAsync(d_sn, 0, tabs.size() * 4, ctx->s));
  uint64_t at = 0;
  for (size_t i = 0; i < tabs.size(); ++i) {
    CuckooTable &t = tabs[i];
    t.t0 = d_slots + at;
    t.t1 = t.t0 + (uint64_t)t.nb0 * CK_SLOTS;
    t.stash = t.t1 + (uint64_t)t.nb1 * CK_SLOTS;
    t.stash_n = d_sn + i;
    at += (uint64_t)(t.nb0 + t.nb1) * CK_SLOTS + CK_STASH;
  }
  // descriptors followed by room for the build's table lists
  void *dv;
  ST(ctx->arena.alloc(ctx, tabs.size() * sizeof(CuckooTable) + tabs.size() * 4 + 16, &dv));
  CuckooTable *d_tabs = (CuckooTable *)dv;
  CU(h2d(ctx, d_tabs, tabs.data(), tabs.size() * sizeof(CuckooTable)));
  CU(cudaMemsetAsync(ctx->d_err, 0, 4, ctx->s));
  launch_cuckoo_build(d_tabs, tabs.data(), (uint32_t)tabs.size(), ctx->d_err, ctx->s);
  CU(cudaGetLastError());
  uint32_t herr = 0;
  CU(d2h_sync(ctx, &herr, ctx->d_err, 4));
  if (herr) {
    ctx->err = "cuckoo stash overflow";
    return GEM_ERR_OVERFLOW;
  }
  for (size_t i = 0; i < tabs.size(); ++i) w.ck_of[who[i].first][who[i].second] = d_tabs + i;
  w.ck_tabs = d_tabs;
  w.bytes_index = kb * (4 + 8 + 8) + slots * 8 / 4;
  return GEM_OK;
}

// Join-work rank of query qi: enumerated levels first (the enumeration's
// exponent), then query vertices, then the values of the tables it reads.
// An estimate that multiplies per-level selectivities as if the levels were
// independent ranks dense queries on skewed graphs as cheap, which they are
// not; the prefix length is the robust part of the cost.
static double join_cost(const Wave &w, size_t qi) {
  const Plan &p = w.plan[qi];
  double vals = 0;
  for (uint32_t k = 1; k < p.n; ++k)
    for (uint32_t j : p.back[k]) {
      const uint32_t ei = w.edge_of[qi][j * QV + k];
      if (ei < w.edge_vals.size()) vals += (double)w.edge_vals[ei];
    }
  return ((double)p.n_enum * 64.0 + (double)p.n) * 1e15 + std::min(vals, 1e15 - 1);
}

static gem_status wave_join(gem_ctx *ctx, Wave &w, int mode, uint32_t *emb_dev, uint64_t emb_cap) {
  std::vector<JQuery> jq;
  std::vector<JBack> jb;
  std::vector<uint64_t> rp, terms, lpp;
  std::vector<uint32_t> lpq, lp2q;
  uint64_t lp_roots = 0;
  w.jq_index.assign(w.q.size(), UINT32_MAX);
  uint64_t roots = 0;
  // Queries take the grid's warps in order of estimated work, cheapest
  // first: under a time cap the queries that can finish do so before the
  // expensive ones take the warps, and a wave's result for a query does not
  // depend on the order.
  std::vector<size_t> order;
  std::vector<double> cost(w.q.size(), 0.0);
  for (size_t qi = 0; qi < w.q.size(); ++qi)
    if (w.active[qi]) {
      order.push_back(qi);
      cost[qi] = join_cost(w, qi);
    }
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return cost[x] < cost[y]; });
  for (const size_t qi : order) {
    const Plan &p = w.plan[qi];
    JQuery J;
    std::memset(&J, 0, sizeof J);
    J.n = p.n;
    J.n_enum = p.n_enum;
    J.n_groups = (uint32_t)p.groups.size();
    for (uint32_t gi = 0; gi < J.n_groups; ++gi) {
      J.grp_first[gi] = p.groups[gi].first;
      J.grp_size[gi] = p.groups[gi].size;
      J.term_base[gi] = (uint32_t)terms.size();
      J.term_count[gi] = (uint32_t)p.groups[gi].terms.size();
      terms.insert(terms.end(), p.groups[gi].terms.begin(), p.groups[gi].terms.end());
    }
    J.flat = flat_code(p, mode);
    J.root_u = p.order[0];
    const uint32_t r0 = w.row_of[qi][p.order[0]];
    J.root_cand = w.d_cand + w.c_base[r0];
    J.n_root = w.cnt[r0];
    J.root_base = roots;
    for (uint32_t k = 0; k < p.n; ++k) {
      JLevel &L = J.lv[k];
      L.u = p.order[k];
      L.nback = (uint32_t)p.back[k].size();
      L.back_base = (uint32_t)jb.size();
      L.dup_mask = p.dup_mask[k];
      L.idx_kind = k == 0 ? IDX_NONE : w.idx_kind[qi][k];
      L.rb = w.d_rb + (uint64_t)w.row_of[qi][p.order[k]] * w.nwords;
      L.ck = w.ck_of[qi][k];
      for (uint32_t j : p.back[k]) {
        const uint32_t ei = w.edge_of[qi][j * QV + k];
        if (ei >= w.edges.size()) {
          ctx->err = "internal: missing edge table for a backward neighbour";
          return GEM_ERR_INTERNAL;
        }
        JBack b;
        b.lvl = j;
        b.nkeys = w.cnt[w.row_of[qi][p.order[j]]];
        b.off = w.edges[ei].offsets;
        jb.push_back(b);
      }
    }
    w.jq_index[qi] = (uint32_t)jq.size();
    if (J.n == 1 || (mode == GEM_MODE_COUNT && J.n_enum == 1)) {
      // lane-parallel pool; an empty range in the ordinary pool
      lpq.push_back((uint32_t)jq.size());
      lpp.push_back(lp_roots);
      lp_roots += J.n_root;
      J.root_base = roots;
      rp.push_back(roots);
    } else if (w.pair[qi] && w.d_vkey) {
      // (root, first level) pair pool; an empty range in the ordinary pool
      lp2q.push_back((uint32_t)jq.size());
      J.root_base = roots;
      rp.push_back(roots);
    } else {
      rp.push_back(roots);
      roots += J.n_root;
    }
    jq.push_back(J);
  }
  rp.push_back(roots);
  lpp.push_back(lp_roots);
  w.out.assign(w.q.size(), JOut());
  uint32_t *d_lp2q = nullptr;
  uint64_t *d_lp2p = nullptr;
  if (jq.empty()) return GEM_OK;
  JQuery *d_jq;
  JBack *d_jb;
  uint64_t *d_rp, *d_terms;
  JOut *d_out;
  ST(aalloc(ctx, terms.size() ? terms.size() : 1, &d_terms));
  uint32_t *d_lpq;
  uint64_t *d_lpp;
  ST(aalloc(ctx, lpq.size() ? lpq.size() : 1, &d_lpq));
  ST(aalloc(ctx, lpp.size(), &d_lpp));
  if (!lpq.empty()) CU(h2d(ctx, d_lpq, lpq.data(), lpq.size() * 4));
  if (!lp2q.empty()) {
    ST(aalloc(ctx, lp2q.size(), &d_lp2q));
    ST(aalloc(ctx, lp2q.size() + 1, &d_lp2p));  // filled by the prepare kernel
    CU(h2d(ctx, d_lp2q, lp2q.data(), lp2q.size() * 4));
  }
  CU(h2d(ctx, d_lpp, lpp.data(), lpp.size() * 8));
  if (!terms.empty())
    CU(h2d(ctx, d_terms, terms.data(), terms.size() * 8));
  ST(aalloc(ctx, jq.size(), &d_jq));
  ST(aalloc(ctx, jb.size() ? jb.size() : 1, &d_jb));
  ST(aalloc(ctx, rp.size(), &d_rp));
  ST(aalloc(ctx, jq.size(), &d_out));
  CU(h2d(ctx, d_jq, jq.data(), jq.size() * sizeof(JQuery)));
  if (!jb.empty()) CU(h2d(ctx, d_jb, jb.data(), jb.size() * sizeof(JBack)));
  CU(h2d(ctx, d_rp, rp.data(), rp.size() * 8));
  const uint64_t cap_ms = ctx->opts.time_cap_ms ? ctx->opts.time_cap_ms : 600000u;
  JoinArgs a;
  std::memset(&a, 0, sizeof a);
  a.queries = d_jq;
  a.nquery = (uint32_t)jq.size();
  a.mode = (uint32_t)mode;
  a.backs = d_jb;
  a.values = w.d_values;
  a.root_prefix = d_rp;
  a.terms = d_terms;
  a.n_roots = roots;
  a.lp_query = d_lpq;
  a.lp_prefix = d_lpp;
  a.lp_nq = (uint32_t)lpq.size();
  a.lp_roots = lp_roots;
  a.lp2_query = d_lp2q;
  a.lp2_nq = (uint32_t)lp2q.size();
  a.lp2_prefix = d_lp2p;
  a.vkey = w.d_vkey;
  a.out = d_out;
  a.ctl = ctx->d_ctl;
  a.queue = ctx->d_queue;
  a.qends = ctx->d_qends;
  a.emb = emb_dev;
  a.emb_cap = emb_cap;
  // schedule: tuned per query-size bucket (largest query of the wave)
  uint32_t maxnv = 0;
  for (auto &J : jq) maxnv = std::max(maxnv, J.n);
  const Tune &tu = ctx->tune[size_bucket(maxnv)];
  a.donate_max_level = tu.donate_max_level ? tu.donate_max_level : ctx->donate_max_level;
  a.donate_min_lane = tu.donate_min_lane ? tu.donate_min_lane : 32;
  a.donate_min_desc = tu.donate_min_desc ? tu.donate_min_desc : 1;
  a.root_batch_max = tu.root_batch_max ? tu.root_batch_max : 1;
  a.lane_scan_max = tu.lane_scan_max ? tu.lane_scan_max : 48;
  a.flat_donate_blocks = tu.split_blocks ? tu.split_blocks : 32;
  a.nv = ctx->g.nv;
  a.vnh_off = ctx->vnh_off;
  a.vnh_slots = ctx->vnh_slots;
  a.n_values = w.table_values;
  a.n_backs = (uint32_t)jb.size();
  a.n_terms = (uint32_t)terms.size();
  int bps = ctx->join_bps[mode];
  if (tu.blocks_per_sm && (int)tu.blocks_per_sm < bps) bps = (int)tu.blocks_per_sm;
  bps = std::max(1, bps / (int)std::max(1u, ctx->join_grid_div));
  CU(cudaEventRecord(ctx->ev[6], ctx->s));
  CU(launch_join_graph(ctx->jgraph, a, cap_ms * 1000000ull, (uint32_t)(ctx->sms * bps), ctx->s));
  CU(cudaEventRecord(ctx->ev[7], ctx->s));
  CU(cudaGetLastError());
  std::vector<JOut> out(jq.size());
  JControl hc;
  JOut *s_out = static_cast<JOut *>(stage(ctx, out.size() * sizeof(JOut)));
  JControl *s_ctl = static_cast<JControl *>(stage(ctx, sizeof(JControl)));
  CU(cudaMemcpyAsync(s_out ? s_out : out.data(), d_out, out.size() * sizeof(JOut), cudaMemcpyDeviceToHost, ctx->s));
  CU(cudaMemcpyAsync(s_ctl ? s_ctl : &hc, ctx->d_ctl, sizeof hc, cudaMemcpyDeviceToHost, ctx->s));
  CU(cudaStreamSynchronize(ctx->s));
  if (s_out) std::memcpy(out.data(), s_out, out.size() * sizeof(JOut));
  if (s_ctl) std::memcpy(&hc, s_ctl, sizeof hc);
  w.join_ms = ev_ms(ctx->ev[6], ctx->ev[7]);
  // Donated tasks still queued when the grid stopped (deadline) were never
  // run: their queries are incomplete.
  if (hc.pending) {
    // one copy of the queue ends and one of the cells, then the host walks them
    std::vector<JQueueEnds> ends(QUEUE_SUBQ);
    std::vector<JTask> cells((size_t)QUEUE_SUBQ * QUEUE_SUBQ_CAP);
    CU(cudaMemcpy(ends.data(), ctx->d_qends, sizeof(JQueueEnds) * QUEUE_SUBQ, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(cells.data(), ctx->d_queue, sizeof(JTask) * cells.size(), cudaMemcpyDeviceToHost));
    for (uint32_t sq = 0; sq < QUEUE_SUBQ; ++sq)
      for (unsigned long long t = ends[sq].head; t < ends[sq].tail && t < ends[sq].head + QUEUE_SUBQ_CAP; ++t) {
        const uint32_t qq = cells[(size_t)sq * QUEUE_SUBQ_CAP + (t & (QUEUE_SUBQ_CAP - 1))].q;
        if (qq < out.size()) out[qq].pad[0] = 1;
      }
  }
  for (size_t qi = 0; qi < w.q.size(); ++qi)
    if (w.jq_index[qi] != UINT32_MAX) w.out[qi] = out[w.jq_index[qi]];
  w.join_nodes = out[0].nodes;
  w.join_scanned = out[0].scanned;
  w.join_probes = out[0].probes;
  w.emb_written = hc.emb_next;
  w.join_err = hc.err;
  if (hc.err == 4u /* bounds check failed (device_common.cuh DERR_BOUNDS) */) {
    static const char *sites[] = {"?", "back entry", "table key", "table range", "vertex id", "task query",
                                  "level", "root position", "suffix term", "key level"};
    ctx->err = std::string("join bounds check failed: ") + sites[hc.bad_site < 10 ? hc.bad_site : 0] +
               " index " + std::to_string(hc.bad_value) + " >= limit " + std::to_string(hc.bad_limit);
    return GEM_ERR_INTERNAL;
  }
  // algorithmic bytes: per extended partial embedding its index word and the
  // offsets pair of each table it keys; per evaluated candidate its id; per
  // binary search a 16-byte sector beyond the cached upper levels.
  uint64_t back_total = 0;
  for (auto &J : jq) back_total += 0;  // per-level entries are counted through nodes
  w.bytes_join = w.join_nodes * (8 + 16) + w.join_scanned * 4 + w.join_probes * 16 + back_total;
  return GEM_OK;
}

gem_status run_wave(gem_ctx *ctx, Wave &w, uint32_t threshold, int mode, uint32_t *emb_dev, uint64_t emb_cap) {
  ctx->h_used = 0;  // the previous wave's copies have completed (it ended with a synchronising readback)
  if (!ctx->loaded) {
    ctx->err = "no data graph loaded";
    return GEM_ERR_STATE;
  }
  CU(cudaSetDevice(ctx->opts.device));
  const uint64_t launches0 = g_launches.load();
  const size_t nq = w.q.size();
  w.row_of.assign(nq, {});
  w.active.assign(nq, 1);
  w.plan.assign(nq, Plan());
  w.idx_kind.assign(nq, std::vector<uint32_t>(QV, 0));
  w.ck_of.assign(nq, std::vector<const CuckooTable *>(QV, nullptr));
  // GEM_DEBUG_SYNC=1: synchronise after every phase so a device fault is
  // attributed to the phase that caused it.
  static const bool dbg = getenv("GEM_DEBUG_SYNC") && getenv("GEM_DEBUG_SYNC")[0] == '1';
  auto phase_sync = [&](const char *name) -> gem_status {
    if (!dbg) return GEM_OK;
    cudaError_t e = cudaStreamSynchronize(ctx->s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
      ctx->err = std::string("device error after ") + name + ": " + cudaGetErrorString(e);
      return GEM_ERR_CUDA;
    }
    return GEM_OK;
  };
  CU(cudaEventRecord(ctx->ev[0], ctx->s));
  ST(wave_filter(ctx, w, threshold));
  ST(phase_sync("filter"));
  CU(cudaEventRecord(ctx->ev[1], ctx->s));
  auto h0 = std::chrono::steady_clock::now();
  for (size_t qi = 0; qi < nq; ++qi) {
    const HostQuery &q = w.q[qi];
    bool empty = false;
    uint32_t qcnt[QV];
    for (uint32_t u = 0; u < q.nv; ++u) {
      qcnt[u] = w.cnt[w.row_of[qi][u]];
      if (qcnt[u] == 0) empty = true;
    }
    if (empty) {
      w.active[qi] = 0;
      continue;
    }
    make_plan(q, qcnt, mode == GEM_MODE_COUNT && ctx->closed_form_suffix, w.plan[qi]);
    std::string why;
    if (!validate_plan(q, w.plan[qi], why)) {
      ctx->err = "internal: invalid plan (" + why + ")";
      return GEM_ERR_INTERNAL;
    }
  }
  w.pair.assign(nq, 0);
  for (size_t qi = 0; qi < nq; ++qi) w.pair[qi] = w.active[qi] && pair_pool(ctx, w.plan[qi], mode);
  w.plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
  ST(wave_tables(ctx, w));
  ST(phase_sync("edge tables"));
  CU(cudaEventRecord(ctx->ev[2], ctx->s));
  ST(wave_index(ctx, w));
  ST(phase_sync("index"));
  CU(cudaEventRecord(ctx->ev[3], ctx->s));
  ST(wave_join(ctx, w, mode, emb_dev, emb_cap));
  ST(phase_sync("join"));
  CU(cudaEventRecord(ctx->ev[4], ctx->s));
  CU(cudaStreamSynchronize(ctx->s));
  w.filter_ms = ev_ms(ctx->ev[0], ctx->ev[1]);
  w.tables_ms = ev_ms(ctx->ev[1], ctx->ev[2]);
  w.index_ms = ev_ms(ctx->ev[2], ctx->ev[3]);
  w.total_ms = ev_ms(ctx->ev[0], ctx->ev[4]);
  if (w.table_passes) {
    w.table_pass_ms[0] = ev_ms(ctx->ev[8], ctx->ev[9]);
    w.table_pass_ms[1] = ev_ms(ctx->ev[10], ctx->ev[11]);
  }
  if (ctx->ev_ref_recorded) {
    w.t_begin_ms = ev_ms(ctx->ev_ref, ctx->ev[0]);
    w.t_end_ms = ev_ms(ctx->ev_ref, ctx->ev[4]);
  }
  w.arena_bytes = ctx->arena.in_use;
  w.launches = (uint32_t)(g_launches.load() - launches0);
  return GEM_OK;
}

void wave_result(const gem_ctx *ctx, const Wave &w, size_t qi, gem_result *r) {
  std::memset(r, 0, sizeof *r);
  r->status = GEM_OK;
  const JOut &o = w.out[qi];
  r->count = o.count;
  r->emb_hash = o.hash;
  if (o.pad[0]) r->status = w.join_err == 1 || w.join_err == 0 ? GEM_ERR_TIMEOUT : GEM_ERR_INTERNAL;
  else if (w.join_err > 1) r->status = GEM_ERR_INTERNAL;
  uint64_t ct = 0;
  for (uint32_t u = 0; u < w.q[qi].nv; ++u) ct += w.cnt[w.row_of[qi][u]];
  r->cand_total = ct;
  r->n_tables = w.active[qi] ? 0 : 0;
  if (w.active[qi]) {
    const Plan &p = w.plan[qi];
    for (uint32_t k = 1; k < p.n; ++k) r->n_tables += (uint32_t)p.back[k].size();
  }
  r->table_total = w.table_values;
  r->nodes = w.join_nodes;
  r->bytes_alg[0] = w.bytes_filter;
  r->bytes_alg[1] = w.bytes_index;
  r->bytes_alg[2] = w.bytes_tables;
  r->bytes_alg[3] = w.bytes_join;
  r->ms[GEM_PH_FILTER] = w.filter_ms;
  r->ms[GEM_PH_INDEX] = w.index_ms;
  r->ms[GEM_PH_TABLES] = w.tables_ms;
  r->ms[GEM_PH_JOIN] = w.join_ms;
  r->ms[GEM_PH_TOTAL] = w.total_ms;
  r->ms[GEM_PH_HOST] = (float)w.plan_ms;
  r->launches = w.launches;
  r->table_pass_ms[0] = w.table_pass_ms[0];
  r->table_pass_ms[1] = w.table_pass_ms[1];
  r->t_begin_ms = w.t_begin_ms;
  r->t_end_ms = w.t_end_ms;
  r->arena_bytes = w.arena_bytes;
  (void)ctx;
}

// ---------------------------------------------------------------------------
// C-ABI: queries
// ---------------------------------------------------------------------------
extern "C" gem_status gem_query_run(gem_ctx *ctx, const gem_query *q, uint32_t threshold, int mode,
                                    uint32_t *emb_out, uint64_t emb_cap, gem_result *res) {
  if (!ctx || !q || !res) return GEM_ERR_ARG;
  if (ctx->server) return GEM_ERR_STATE;
  if (mode < GEM_MODE_COUNT || mode > GEM_MODE_ENUMERATE) return GEM_ERR_ARG;
  if (mode == GEM_MODE_ENUMERATE && emb_cap && !emb_out) return GEM_ERR_ARG;
  std::memset(res, 0, sizeof *res);
  ctx->err.clear();
  if (threshold != 0) {
    ctx->err = "relaxed matching (threshold > 0) is not supported";
    res->status = GEM_ERR_LIMIT;
    return GEM_ERR_LIMIT;
  }
  Wave w;
  w.q.resize(1);
  ST(make_host_query(q, w.q[0], ctx->err));
  auto t0 = std::chrono::steady_clock::now();
  ctx->arena.reset();
  uint32_t *d_emb = nullptr;
  if (mode == GEM_MODE_ENUMERATE && emb_cap) ST(aalloc(ctx, emb_cap * q->nv, &d_emb));
  {
    const gem_status st = run_wave(ctx, w, 0, mode, d_emb, emb_cap);
    if (st != GEM_OK) {
      res->status = st;
      return st;
    }
  }
  wave_result(ctx, w, 0, res);
  if (res->status == GEM_ERR_TIMEOUT) ctx->err = "device time cap reached before the count completed";
  if (mode == GEM_MODE_ENUMERATE) {
    uint64_t nw = std::min<uint64_t>(w.emb_written, emb_cap);
    res->n_written = nw;
    if (nw) CU(cudaMemcpy(emb_out, d_emb, nw * q->nv * 4, cudaMemcpyDeviceToHost));
    if (w.emb_written > emb_cap && res->status == GEM_OK) res->status = GEM_ERR_OVERFLOW;
  }
  res->ms[GEM_PH_HOST] = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return (gem_status)res->status;
}

// Relaxed queries of `orig` at `threshold` in one wave whose filter rows are
// orig's own at that threshold (the reference's filter with slack T: a
// relaxed query's vertex loses at most T neighbours, so orig's slack
// candidates hold every relaxed query's).  All relaxed queries then share
// orig's candidate lists and the tables of the edges they keep; each is
// planned and counted exactly on its own.  GEM_ERR_OOM when the wave does
// not fit (the caller then counts them as a plain batch).
gem_status gem::relaxed_wave(gem_ctx *ctx, const HostQuery &orig, const std::vector<HostQuery> &rq,
                             uint32_t threshold, int mode, gem_result *res) {
  if (ctx->server) return GEM_ERR_STATE;
  if (mode != GEM_MODE_COUNT && mode != GEM_MODE_HASH) return GEM_ERR_ARG;
  if (rq.empty()) return GEM_OK;
  Wave w;
  w.q = rq;
  w.sig_query = &orig;
  ctx->arena.reset();
  const gem_status st = run_wave(ctx, w, threshold, mode, nullptr, 0);
  if (st != GEM_OK) {
    cudaStreamSynchronize(ctx->s);
    cudaGetLastError();
    return st;
  }
  for (size_t i = 0; i < rq.size(); ++i) {
    wave_result(ctx, w, i, &res[i]);
    res[i].wave = 0;
  }
  return GEM_OK;
}

extern "C" gem_status gem_batch_run(gem_ctx *ctx, const gem_query *qs, uint32_t n, int mode, gem_result *res) {
  if (!ctx || (n && (!qs || !res))) return GEM_ERR_ARG;
  if (ctx->server) return GEM_ERR_STATE;
  if (mode != GEM_MODE_COUNT && mode != GEM_MODE_HASH) return GEM_ERR_ARG;
  std::vector<HostQuery> all(n);
  std::vector<gem_status> vs(n, GEM_OK);
  for (uint32_t i = 0; i < n; ++i) {
    std::memset(&res[i], 0, sizeof res[i]);
    std::string e;
    vs[i] = make_host_query(&qs[i], all[i], e);
    res[i].status = vs[i];
  }
  // Waves are packed as the batch runs: as many pending queries as the
  // lane's row limit allows.  A wave that does not fit the lane's device
  // budget is retried with a released arena in smaller waves (down to single
  // queries), and the lane's limit drops to the rows that would have fit:
  // the failed wave's rows scaled by the bytes the budget left it over the
  // bytes it asked for, with a tenth kept back (half when that is not
  // known).  So later waves (and later batches) are packed to a size that
  // fits; the limit does not grow back, since a retried wave costs its
  // filter and table build.
  //
  // An in-core batch of more rows than one wave takes runs on two lanes: the
  // context and a lane context borrowing its graph (created once, kept), one
  // host thread each, the device budget left after the graph split between
  // them and each join grid on half of the blocks per SM.  One wave's join
  // then runs beside the next wave's filter and table kernels.
  std::mutex mu;
  std::deque<std::vector<uint32_t>> retry;
  uint32_t next = 0, wave_no = 0;
  gem_status first_err = GEM_OK;
  std::string lane_err;
  auto rows_of = [&](const std::vector<uint32_t> &ids) {
    uint64_t r = 0;
    for (uint32_t id : ids) r += all[id].nv;
    return r;
  };
  uint64_t total_rows = 0;
  for (uint32_t i = 0; i < n; ++i)
    if (vs[i] == GEM_OK) total_rows += all[i].nv;
  auto worker = [&](gem_ctx *lane) {
    for (;;) {
      std::vector<uint32_t> ids;
      {
        std::lock_guard<std::mutex> lk(mu);
        if (!retry.empty()) {
          ids = std::move(retry.front());
          retry.pop_front();
        } else {
          uint64_t cap = lane->wave_max_rows;
          if (lane->wave_rows_cap) cap = std::min<uint64_t>(cap, lane->wave_rows_cap);
          uint64_t rows = 0;
          while (next < n && (ids.empty() || rows + all[next].nv <= cap)) {
            if (vs[next] == GEM_OK) {
              ids.push_back(next);
              rows += all[next].nv;
            }
            ++next;
          }
        }
      }
      if (ids.empty()) {
        std::lock_guard<std::mutex> lk(mu);
        if (retry.empty() && next >= n) return;
        continue;
      }
      Wave w;
      for (uint32_t id : ids) w.q.push_back(all[id]);
      lane->arena.reset();
      const gem_status st = run_wave(lane, w, 0, mode, nullptr, 0);
      if (st != GEM_OK) {
        cudaStreamSynchronize(lane->s);  // the failed wave's copies and kernels are done before reuse
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(mu);
        if (st == GEM_ERR_OOM && ids.size() > 1) {
          // the rows that would have fit, by what the wave asked for against
          // what the budget leaves it (a tenth kept back), else half
          const Arena &a = lane->arena;
          double f = a.oom_need ? 0.9 * (double)a.oom_room / (double)a.oom_need : 0.5;
          f = std::min(0.9, std::max(0.25, f));
          const uint64_t cap = std::max<uint64_t>(1, (uint64_t)(f * (double)rows_of(ids)));
          lane->wave_rows_cap = (uint32_t)cap;
          if (!lane->arena.reserved) lane->arena.release(lane);  // a fresh arena: chunks sized for the smaller waves
          // the queries again in waves of at most cap rows (at least one query each)
          std::vector<std::vector<uint32_t>> parts(1);
          uint64_t rows = 0;
          for (uint32_t id : ids) {
            if (!parts.back().empty() && rows + all[id].nv > cap) {
              parts.emplace_back();
              rows = 0;
            }
            parts.back().push_back(id);
            rows += all[id].nv;
          }
          if (parts.size() == 1) {  // one query over the cap: halve by count
            const size_t h = ids.size() / 2;
            parts.assign({std::vector<uint32_t>(ids.begin(), ids.begin() + h),
                          std::vector<uint32_t>(ids.begin() + h, ids.end())});
          }
          for (size_t i = parts.size(); i-- > 0;) retry.push_front(std::move(parts[i]));
          continue;
        }
        for (uint32_t id : ids) res[id].status = st;
        if (first_err == GEM_OK) first_err = st;
        if (lane != ctx && lane_err.empty()) lane_err = lane->err;
        continue;
      }
      uint32_t my_wave;
      {
        std::lock_guard<std::mutex> lk(mu);
        my_wave = wave_no++;
      }
      for (size_t k = 0; k < ids.size(); ++k) {
        wave_result(lane, w, k, &res[ids[k]]);
        res[ids[k]].wave = my_wave;
      }
    }
  };
  gem_ctx *second = nullptr;
  if (ctx->opts.batch_lanes != 1 && total_rows > ctx->wave_max_rows) {
    if (!ctx->batch_lane) {
      // the graph's remaining budget, split evenly: the context's arena is
      // released so each lane grows its own within its half
      ctx->arena.release(ctx);
      const uint64_t room = ctx->budget > ctx->device_bytes ? ctx->budget - ctx->device_bytes : 0;
      if (lane_create(ctx, room / 2, &ctx->batch_lane) == GEM_OK) {
        ctx->batch_saved_budget = ctx->budget;
        ctx->budget = ctx->device_bytes + room / 2;
      } else {
        ctx->batch_lane = nullptr;
        cudaGetLastError();
      }
    }
    second = ctx->batch_lane;
  }
  if (second) {
    // each lane's arena: one chunk of its whole budget, less room for the
    // join's graph and other small allocations outside the arena
    for (gem_ctx *l : {ctx, second})
      if (!l->arena.reserved && l->budget > l->device_bytes + (1ull << 30))
        l->arena.reserve(l, l->budget - l->device_bytes - (512ull << 20));
    for (int b = 0; b < 6; ++b) second->tune[b] = ctx->tune[b];
    ctx->join_grid_div = second->join_grid_div = 2;
    std::thread t(worker, second);
    worker(ctx);
    t.join();
    ctx->join_grid_div = 1;
    merge_ooc_stats(ctx, second);
    if (!lane_err.empty() && ctx->err.empty()) ctx->err = lane_err;
  } else {
    worker(ctx);
  }
  for (uint32_t k = 0; k < n; ++k)
    if (res[k].status != GEM_OK && first_err == GEM_OK) first_err = (gem_status)res[k].status;
  return first_err;
}

// ---------------------------------------------------------------------------
// C-ABI: phase entry points
// ---------------------------------------------------------------------------
extern "C" gem_status gem_filter(gem_ctx *ctx, const gem_query *q, uint32_t threshold, uint32_t *counts,
                                 uint32_t *cand_out, uint64_t cand_cap) {
  if (!ctx || !q || !counts) return GEM_ERR_ARG;
  if (ctx->server) return GEM_ERR_STATE;
  if (!ctx->loaded) return GEM_ERR_STATE;
  Wave w;
  w.q.resize(1);
  ST(make_host_query(q, w.q[0], ctx->err));
  ctx->arena.reset();
  w.share_rows = false;  // rows in query-vertex order, one each
  ST(wave_filter(ctx, w, threshold));
  CU(cudaStreamSynchronize(ctx->s));
  for (uint32_t u = 0; u < q->nv; ++u) counts[u] = w.cnt[u];
  if (w.cand_total > cand_cap) return GEM_ERR_OVERFLOW;
  if (w.cand_total && cand_out)
    CU(cudaMemcpy(cand_out, w.d_cand, w.cand_total * 4, cudaMemcpyDeviceToHost));
  return GEM_OK;
}

extern "C" gem_status gem_edge_table(gem_ctx *ctx, const gem_query *q, uint32_t u, uint32_t wv,
                                     uint64_t *offsets_out, uint64_t offsets_cap, uint32_t *values_out,
                                     uint64_t values_cap, uint64_t *n_keys, uint64_t *n_values) {
  if (!ctx || !q || !n_keys || !n_values) return GEM_ERR_ARG;
  if (!ctx->loaded || ctx->server) return GEM_ERR_STATE;
  Wave w;
  w.q.resize(1);
  ST(make_host_query(q, w.q[0], ctx->err));
  const HostQuery &hq = w.q[0];
  if (u >= hq.nv || wv >= hq.nv || !(hq.adj[u] & (1u << wv))) return GEM_ERR_ARG;
  ctx->arena.reset();
  w.share_rows = false;  // rows in query-vertex order, one each
  w.active.assign(1, 1);
  ST(wave_filter(ctx, w, 0));
  // a two-level plan: u then w
  Plan p;
  p.n = 2;
  p.n_enum = 2;
  p.order[0] = u;
  p.order[1] = wv;
  p.back[1] = {0};
  w.plan.assign(1, p);
  ST(wave_tables(ctx, w));
  CU(cudaStreamSynchronize(ctx->s));
  const TabEdge &e = w.edges[0];
  const uint64_t nk = w.cnt[u];
  *n_keys = nk;
  std::vector<uint64_t> off(nk + 1);
  CU(cudaMemcpy(off.data(), e.offsets, 8 * (nk + 1), cudaMemcpyDeviceToHost));
  const uint64_t base = off[0];
  *n_values = off[nk] - base;
  if (offsets_cap < nk + 1 || values_cap < off[nk] - base) return GEM_ERR_OVERFLOW;
  for (uint64_t i = 0; i <= nk; ++i) offsets_out[i] = off[i] - base;
  if (off[nk] > base) CU(cudaMemcpy(values_out, w.d_values + base, 4 * (off[nk] - base), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

extern "C" gem_status gem_index_probe(gem_ctx *ctx, const gem_query *q, uint32_t u, uint32_t index_kind,
                                      const uint32_t *keys, uint32_t n_keys, uint32_t *pos_out) {
  if (!ctx || !q || (n_keys && (!keys || !pos_out))) return GEM_ERR_ARG;
  if (index_kind != IDX_RANK && index_kind != IDX_CUCKOO) return GEM_ERR_ARG;
  if (!ctx->loaded || ctx->server) return GEM_ERR_STATE;
  Wave w;
  w.q.resize(1);
  ST(make_host_query(q, w.q[0], ctx->err));
  if (u >= w.q[0].nv) return GEM_ERR_ARG;
  ctx->arena.reset();
  w.share_rows = false;  // rows in query-vertex order, one each
  w.active.assign(1, 1);
  w.idx_kind.assign(1, std::vector<uint32_t>(QV, 0));
  w.ck_of.assign(1, std::vector<const CuckooTable *>(QV, nullptr));
  ST(wave_filter(ctx, w, 0));
  uint32_t *d_keys, *d_out;
  ST(aalloc(ctx, n_keys ? n_keys : 1, &d_keys));
  ST(aalloc(ctx, n_keys ? n_keys : 1, &d_out));
  if (n_keys) CU(cudaMemcpyAsync(d_keys, keys, 4ull * n_keys, cudaMemcpyHostToDevice, ctx->s));
  if (index_kind == IDX_RANK) {
    launch_rank_probe(w.d_rb + (uint64_t)u * w.nwords, d_keys, n_keys, d_out, ctx->s);
  } else {
    Plan p;
    p.n = 2;
    p.n_enum = 2;
    p.order[0] = u == 0 ? 1 % w.q[0].nv : 0;
    p.order[1] = u;
    p.need_idx[1] = 1;
    w.plan.assign(1, p);
    const uint32_t saved = ctx->opts.index_kind;
    ctx->opts.index_kind = IDX_CUCKOO;
    gem_status s = wave_index(ctx, w);
    ctx->opts.index_kind = saved;
    if (s != GEM_OK) return s;
    launch_cuckoo_probe(w.ck_of[0][1], d_keys, n_keys, d_out, ctx->s);
  }
  CU(cudaGetLastError());
  if (n_keys) CU(cudaMemcpyAsync(pos_out, d_out, 4ull * n_keys, cudaMemcpyDeviceToHost, ctx->s));
  CU(cudaStreamSynchronize(ctx->s));
  return GEM_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: per query-size bucket, the join schedule (blocks per SM of the
// persistent grid, deepest level that donates work) with the lowest join
// time on a sample of the caller's queries.
// ---------------------------------------------------------------------------
extern "C" gem_status gem_set_schedule(gem_ctx *ctx, uint32_t query_vertices, const gem_schedule *sched) {
  if (!ctx || !sched || query_vertices == 0 || query_vertices > QV) return GEM_ERR_ARG;
  if (ctx->server) return GEM_ERR_STATE;
  Tune &t = ctx->tune[size_bucket(query_vertices)];
  t = Tune();
  t.blocks_per_sm = sched->blocks_per_sm;
  t.donate_max_level = sched->donate_max_level;
  t.donate_min_lane = sched->donate_min_lane;
  t.donate_min_desc = sched->donate_min_desc;
  t.root_batch_max = sched->root_batch_max;
  t.lane_scan_max = sched->lane_scan_max;
  t.split_blocks = sched->split_blocks;
  return GEM_OK;
}

extern "C" gem_status gem_get_schedule(gem_ctx *ctx, uint32_t query_vertices, gem_schedule *sched) {
  if (!ctx || !sched || query_vertices == 0 || query_vertices > QV) return GEM_ERR_ARG;
  const Tune &t = ctx->tune[size_bucket(query_vertices)];
  *sched = gem_schedule{};
  sched->blocks_per_sm = t.blocks_per_sm;
  sched->donate_max_level = t.donate_max_level;
  sched->donate_min_lane = t.donate_min_lane;
  sched->donate_min_desc = t.donate_min_desc;
  sched->root_batch_max = t.root_batch_max;
  sched->lane_scan_max = t.lane_scan_max;
  sched->split_blocks = t.split_blocks;
  return GEM_OK;
}

extern "C" gem_status gem_autotune(gem_ctx *ctx, const gem_query *qs, uint32_t n, int mode, uint32_t trial_cap_ms,
                                   uint32_t *report) {
  if (!ctx || (n && !qs)) return GEM_ERR_ARG;
  if (mode != GEM_MODE_COUNT && mode != GEM_MODE_HASH) return GEM_ERR_ARG;
  if (!ctx->loaded || ctx->server) return GEM_ERR_STATE;
  std::vector<HostQuery> byb[6];
  for (uint32_t i = 0; i < n; ++i) {
    HostQuery h;
    std::string e;
    if (make_host_query(&qs[i], h, e) != GEM_OK) continue;
    auto &v = byb[size_bucket(h.nv)];
    if (v.size() < 256) v.push_back(h);
  }
  const int occ = ctx->join_bps[mode];
  std::vector<uint32_t> bps_c = {(uint32_t)occ};
  if (occ > 1) bps_c.push_back((uint32_t)occ - 1);
  if (occ > 2) bps_c.push_back((uint32_t)(occ + 1) / 2);
  struct Sched {
    uint32_t dm, dml, rb, lsm, dmd, split;
  };
  const Sched sched_c[8] = {{30, 32, 1, 48, 1, 32}, {6, 32, 1, 48, 1, 32},  {2, 32, 1, 48, 1, 32},
                            {30, 256, 1, 48, 1, 32}, {30, 32, 4, 48, 1, 32}, {30, 32, 1, 8, 1, 32},
                            {30, 32, 1, 160, 1, 32}, {30, 32, 1, 48, 1, 64}};
  const uint32_t saved_cap = ctx->opts.time_cap_ms;
  ctx->opts.time_cap_ms = trial_cap_ms ? trial_cap_ms : 2000;
  gem_status st = GEM_OK;
  for (uint32_t b = 0; b < 6 && st == GEM_OK; ++b) {
    if (byb[b].empty()) continue;
    Tune best;
    double best_cost = 1e300;
    for (uint32_t bps : bps_c)
      for (const Sched &sc : sched_c) {
        ctx->tune[b].blocks_per_sm = bps;
        ctx->tune[b].donate_max_level = sc.dm;
        ctx->tune[b].donate_min_lane = sc.dml;
        ctx->tune[b].root_batch_max = sc.rb;
        ctx->tune[b].lane_scan_max = sc.lsm;
        ctx->tune[b].donate_min_desc = sc.dmd;
        ctx->tune[b].split_blocks = sc.split;
        // each candidate runs twice; the faster run counts (sub-millisecond joins are noisy)
        double cost = 1e300;
        for (int rep = 0; rep < 2 && st == GEM_OK; ++rep) {
          Wave w;
          w.q = byb[b];
          ctx->arena.reset();
          st = run_wave(ctx, w, 0, mode, nullptr, 0);
          if (st != GEM_OK) break;
          uint32_t timeouts = 0;
          for (size_t i = 0; i < w.q.size(); ++i) timeouts += w.out[i].pad[0] ? 1 : 0;
          const double c = w.join_ms + (double)timeouts * ctx->opts.time_cap_ms;
          cost = c < cost ? c : cost;
          if (timeouts) break;  // a capped trial is not repeated
        }
        if (st != GEM_OK) break;
        if (cost < best_cost) {
          best_cost = cost;
          best.blocks_per_sm = bps;
          best.donate_max_level = sc.dm;
          best.donate_min_lane = sc.dml;
          best.root_batch_max = sc.rb;
          best.lane_scan_max = sc.lsm;
          best.donate_min_desc = sc.dmd;
          best.split_blocks = sc.split;
          best.best_ms = (float)cost;
        }
      }
    ctx->tune[b] = best;
  }
  ctx->opts.time_cap_ms = saved_cap;
  if (report)
    for (uint32_t b = 0; b < 6; ++b) {
      report[3 * b] = ctx->tune[b].blocks_per_sm;
      report[3 * b + 1] = ctx->tune[b].donate_max_level | (ctx->tune[b].donate_min_lane << 8) |
                          (ctx->tune[b].root_batch_max << 20);
      report[3 * b + 2] = (uint32_t)(ctx->tune[b].best_ms * 1000.0f);
    }
  return st;
}
