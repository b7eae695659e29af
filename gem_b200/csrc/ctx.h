// Host-side state of a libgem context (not part of the C-ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gem_internal.h"
#include "kernels.h"

struct gem_ctx;
struct Server;
void server_shutdown(gem_ctx *ctx);

// Device memory in chunks obtained from cudaMalloc; bump-allocated, reset
// between waves so steady-state queries never call cudaMalloc.
struct Arena {
  struct Chunk {
    char *base;
    uint64_t size;
    uint64_t used;
  };
  std::vector<Chunk> chunks;
  size_t cur = 0;
  uint64_t in_use = 0, peak = 0;
  // the last failed allocation: what the wave would have held with it, and
  // what the budget leaves for the arena
  uint64_t oom_need = 0, oom_room = 0;
  bool reserved = false;  // one chunk holding the whole budget (batch lanes)
  gem_status alloc(gem_ctx *ctx, uint64_t bytes, void **out);
  // Replaces the chunks by one chunk of `bytes` (kept until release): waves
  // of any size then never call cudaMalloc or cudaFree, whose frees wait for
  // the whole device.  Falls back to growing chunks when it cannot allocate.
  void reserve(gem_ctx *ctx, uint64_t bytes);
  void reset();
  void release(gem_ctx *ctx);
};

// Matching order of one query.  In count mode the last n - n_enum levels
// (the suffix) form an independent set of the query graph whose completions
// are counted in closed form; suffix levels are grouped by label.
struct Plan {
  uint32_t n = 0;
  uint32_t n_enum = 0;              // levels enumerated depth-first
  uint32_t order[gem::QV] = {};     // level -> query vertex
  uint32_t level_of[gem::QV] = {};  // query vertex -> level
  std::vector<uint32_t> back[gem::QV];  // backward neighbour levels
  uint32_t dup_mask[gem::QV] = {};  // earlier enumerated levels with the same label
  uint32_t need_idx[gem::QV] = {};  // level's vertex keys a later table
  struct Group {
    uint32_t first = 0, size = 0;
    std::vector<uint64_t> terms;    // inclusion-exclusion terms (see gem::JTerm packing)
  };
  std::vector<Group> groups;
};
// count_suffix: choose a closed-form suffix (count mode only).
void make_plan(const gem::HostQuery &q, const uint32_t *cnt, bool count_suffix, Plan &p);

// One wave: a set of queries processed by shared launches.
struct Wave {
  std::vector<gem::HostQuery> q;
  // Filter rows: one per distinct (label, degree, neighbour labels) among the
  // wave's query vertices, which have the same candidates in every query.
  std::vector<std::vector<uint32_t>> row_of;  // per query, per query vertex: its row
  bool share_rows = true;           // false: one row per query vertex (the phase entry points)
  // Relaxed matching: when set, every query's filter rows are this query's
  // (the one the wave's queries relax), filtered at the wave's threshold, so
  // the relaxed queries share their candidate lists and the tables they key.
  const gem::HostQuery *sig_query = nullptr;
  std::vector<uint8_t> active;      // 0 = some C(u) empty (count 0)
  std::vector<Plan> plan;
  std::vector<std::vector<uint32_t>> idx_kind;  // per query, per level
  std::vector<std::vector<const gem::CuckooTable *>> ck_of;
  std::vector<std::vector<uint32_t>> edge_of;   // per query: [j*QV+k] -> edge index
  std::vector<uint8_t> pair;        // query counted through the (root, first level) pair pool
  uint32_t *d_vkey = nullptr;       // key positions of the pool queries' root-table values
  uint32_t nrows = 0, nwords = 0, nsrc = 0;
  uint64_t *d_rb = nullptr;       // rank bitmaps, nrows x nwords
  uint32_t *d_bits = nullptr;     // their membership bits alone, nrows x nwords
  uint32_t *d_cand = nullptr;     // candidate lists back to back
  std::vector<uint32_t> cnt;      // |C| per row
  std::vector<uint64_t> c_base;   // list start per row
  uint64_t cand_total = 0;
  std::vector<gem::TabEdge> edges;
  std::vector<uint64_t> edge_vals;  // values per table (edges[e])
  uint32_t *d_values = nullptr;
  uint64_t table_values = 0, table_tiles = 0;
  const gem::CuckooTable *ck_tabs = nullptr;
  uint32_t cuckoo_round = 0;
  std::vector<uint32_t> jq_index;
  std::vector<gem::JOut> out;
  uint64_t join_nodes = 0, join_scanned = 0, join_probes = 0, emb_written = 0;
  uint32_t join_err = 0;
  float filter_ms = 0, tables_ms = 0, index_ms = 0, join_ms = 0, total_ms = 0;
  float table_pass_ms[2] = {0, 0};  // the table kernels' count and write passes
  float t_begin_ms = 0, t_end_ms = 0;  // first and last event of the wave against the context's ev_ref
  uint64_t arena_bytes = 0;            // arena bytes the wave used
  bool table_passes = false;        // the passes ran (their events were recorded)
  double plan_ms = 0;
  uint64_t bytes_filter = 0, bytes_tables = 0, bytes_index = 0, bytes_join = 0;
  uint32_t launches = 0;
};

// Join schedule for one query-size bucket (0 = library default).
struct Tune {
  uint32_t blocks_per_sm = 0;
  uint32_t donate_max_level = 0;
  uint32_t donate_min_lane = 0;   // 0 = library default
  uint32_t root_batch_max = 0;    // 0 = library default
  uint32_t lane_scan_max = 0;     // 0 = library default
  uint32_t donate_min_desc = 0;   // 0 = library default
  uint32_t split_blocks = 0;      // 0 = library default
  float best_ms = 0;
};
// Buckets by query size: <=4, <=8, <=12, <=16, <=24, <=32 vertices.
inline uint32_t size_bucket(uint32_t nv) {
  return nv <= 4 ? 0 : nv <= 8 ? 1 : nv <= 12 ? 2 : nv <= 16 ? 3 : nv <= 24 ? 4 : 5;
}

constexpr size_t H_SMALL_BYTES = 4u << 20;  // pinned staging per context

struct gem_ctx {
  gem_opts opts{};
  cudaStream_t s = nullptr;
  cudaEvent_t ev[12] = {};
  int sms = 148;
  int join_bps[3] = {1, 1, 1};
  uint64_t budget = 0, device_bytes = 0;
  std::string err;
  // graph
  bool loaded = false;
  gem::DevGraph g;
  char *graph_mem = nullptr;
  char *vnh_mem = nullptr;           // neighbourhood hash (in-core graphs that fit)
  uint64_t vnh_bytes = 0;
  const uint64_t *vnh_off = nullptr;
  const uint32_t *vnh_slots = nullptr;
  void *pinned_nbr = nullptr;        // out-of-core: mapped pinned adjacency (owned)
  void *host_nbr = nullptr;          // the same, as the host-side source of partition copies (lanes borrow it)
  // out-of-core partition streaming: vertex ranges of at most ooc_part_kib
  // KiB of adjacency, two device staging buffers and a side copy stream
  std::vector<uint32_t> part_v;      // partition vertex bounds (partitions + 1)
  std::vector<uint64_t> part_a;      // their arc bounds
  char *part_mem = nullptr;          // d_part_v and both staging buffers
  uint64_t part_bytes = 0;
  uint32_t *d_part_v = nullptr;
  uint32_t *d_stage[2] = {nullptr, nullptr};
  cudaStream_t s_copy = nullptr;
  cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  gem_ooc_stats ooc{};
  void *spill_host = nullptr;        // out-of-core: mapped pinned values of tables that exceed the budget
  void *spill_dev = nullptr;
  uint64_t spill_bytes = 0;
  uint64_t graph_bytes = 0;
  std::vector<uint64_t> label_freq;  // vertices per label
  std::vector<uint64_t> label_arcs;  // sum of degrees per label
  std::vector<uint64_t> label_pair_arcs;  // [s * nlabels + t]: arcs from label-s to label-t vertices (<= 64 labels)
  Server *server = nullptr;          // serving thread (gem_submit / gem_poll)
  // scratch
  Arena arena;
  gem::JControl *d_ctl = nullptr;
  gem::JTask *d_queue = nullptr;
  gem::JQueueEnds *d_qends = nullptr;
  uint32_t *d_err = nullptr;
  void *h_small = nullptr;           // pinned staging for a wave's small copies (H_SMALL_BYTES)
  size_t h_used = 0;                 // bytes of h_small handed out in the current wave
  // join schedule: CUDA graph and per-size-bucket tuning (gem_autotune)
  gem::JoinGraph jgraph;
  Tune tune[6];
  // tunables
  uint32_t donate_max_level = 30;
  bool closed_form_suffix = true;
  uint32_t wave_max_rows = 4096;
  // batch packing learnt from earlier waves: the rows that would have fit of
  // the last wave that did not fit the device budget (0 = none yet)
  uint32_t wave_rows_cap = 0;
  uint32_t join_grid_div = 1;        // the join grid takes blocks_per_sm / this per SM (serving lanes: 2)
  // device timeline: waves report their first and last event against ev_ref
  // (recorded when the graph is loaded; serving lanes share their root's)
  cudaEvent_t ev_ref = nullptr;
  bool ev_ref_recorded = false;
  bool borrowed_graph = false;       // a serving lane: the graph belongs to another context
  gem_ctx *batch_lane = nullptr;     // second lane of multi-wave batches (kept until the graph changes)
  uint64_t batch_saved_budget = 0;   // the device budget before the batch lane took its half
};

// A serving lane: a context with its own stream, events, arena, control
// block and task queue that borrows `root`'s resident graph (in-core only),
// so that waves of two lanes run on the device at the same time.
gem_status lane_create(gem_ctx *root, uint64_t budget, gem_ctx **out);
// Destroys the context's batch lane, if any, and gives its budget back.
void drop_batch_lane(gem_ctx *ctx);
// Adds a lane's out-of-core counters to its root's and clears them.
void merge_ooc_stats(gem_ctx *root, gem_ctx *lane);

gem_status run_wave(gem_ctx *ctx, Wave &w, uint32_t threshold, int mode, uint32_t *emb_dev, uint64_t emb_cap);
void wave_result(const gem_ctx *ctx, const Wave &w, size_t qi, gem_result *r);
