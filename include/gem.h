/*
 * gem.h — C-ABI of libgem, a B200-native (sm_100a) edge-centric subgraph matcher.
 *
 * The reference (Seungsu-J/GEM) exposes no library API: its boundary is the
 * `GEM` executable (in-core/src/main.cu:23-275, out-of-core/src/main.cu:412-460),
 * the `t/v/e` text graph format (in-core/lib/io/src/io.cu:45-220) and a chain of
 * process-global C++ phase functions:
 *   filterSSM                                  in-core/lib/filter/include/filter.h:10
 *   HashTable::build                           in-core/lib/structure/include/unifiedTrie.cuh:58
 *   UnifiedTrieManager::initVertexTries        in-core/lib/structure/include/unifiedTrie.cuh:230
 *   UnifiedTrieManager::construct_edge_candidates  in-core/lib/structure/include/unifiedTrie.cuh:244
 *   join                                       in-core/lib/join/include/join_trie.cuh:31
 * Each entry point below names the reference piece it replaces.  All state hangs
 * off explicit handles (no process globals, no exit()); every call returns a
 * gem_status.  Plain pointers and sizes only: callers own every array they pass.
 *
 * Semantics of a match (identical to the reference at threshold 0): an
 * embedding of query q in data graph G is an injective map f: V(q) -> V(G) with
 * label(f(u)) == label(u) for every u and {f(u), f(w)} in E(G) for every query
 * edge {u, w}.  It is non-induced and no symmetry breaking is applied, so
 * automorphic copies count separately (in-core/lib/join/src/join_trie_kernel.cu
 * :270-1099 joins without any ordering constraint; injectivity is the same-label
 * duplicate check of in-core/lib/join/src/join_trie.cu:450-462).
 */
#ifndef GEM_H
#define GEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes.  Replaces `cuchk` -> exit(code)                             */
/* (in-core/lib/utils/include/cuda_helpers.cuh:20-36).                        */
/* ------------------------------------------------------------------------ */
typedef enum gem_status {
  GEM_OK = 0,
  GEM_ERR_ARG = 1,      /* invalid argument (null pointer, size out of range) */
  GEM_ERR_OOM = 2,      /* device/pinned budget exceeded; server: admission busy */
  GEM_ERR_LIMIT = 3,    /* outside supported envelope (query > 32 vertices, threshold > 0 ...) */
  GEM_ERR_TIMEOUT = 4,  /* a bounded device wait or the per-query time cap ran out */
  GEM_ERR_CUDA = 5,     /* CUDA runtime error (message in gem_last_error) */
  GEM_ERR_IO = 6,       /* file missing, malformed or inconsistent */
  GEM_ERR_STATE = 7,    /* call out of order (no graph loaded, unknown ticket ...) */
  GEM_ERR_OVERFLOW = 8, /* a result exceeded a caller buffer or a u64 counter */
  GEM_ERR_INTERNAL = 9  /* internal consistency check failed */
} gem_status;

const char *gem_strerror(gem_status s);

/* Limits of this build. */
#define GEM_MAX_QV 32u     /* query vertices (reference: MAX_VQ=16, defs.h:20) */
#define GEM_MAX_QE 496u    /* query edges: complete graph on 32 vertices       */

/* ------------------------------------------------------------------------ */
/* Host graphs (CSR with sorted adjacency).                                   */
/* Replaces cpuGraph + readGraphToCPUStandard (in-core/lib/io/src/io.cu:45).  */
/* ------------------------------------------------------------------------ */
typedef struct gem_hgraph gem_hgraph;

/* Copy caller arrays into a new host graph.  offsets: nv+1 entries, nbrs:
 * offsets[nv] entries, labels: nv entries.  The graph must be undirected
 * (every arc has its reverse), free of self loops and duplicates, with each
 * adjacency list sorted ascending; violations return GEM_ERR_ARG. */
gem_status gem_hgraph_create(uint32_t nv, const uint64_t *offsets,
                             const uint32_t *nbrs, const uint32_t *labels,
                             gem_hgraph **out);
/* Read the reference's text format: `t V E`, `v id label degree` per vertex,
 * `e src dst` per undirected edge (in-core/lib/io/src/io.cu:45-127).  Vertex
 * lines may come in any order; declared degrees must match the edges. */
gem_status gem_hgraph_read_text(const char *path, gem_hgraph **out);
/* Write the text format with ascending vertex lines and lexicographically
 * sorted (src < dst) edge lines — the layout the reference's reader needs to
 * build a sorted CSR. */
gem_status gem_hgraph_write_text(const gem_hgraph *g, const char *path);
/* R-MAT generator: 2^scale vertices, edge_factor * 2^scale sampled edges with
 * quadrant probabilities (a, b, c, 1-a-b-c); self loops and duplicates are
 * dropped and the result symmetrised.  Deterministic for a seed, independent
 * of thread count.  All labels start at 0. */
gem_status gem_hgraph_rmat(uint32_t scale, uint32_t edge_factor, double a,
                           double b, double c, uint64_t seed, gem_hgraph **out);
/* Assign labels 0..nlabels-1: uniform when zipf_s == 0, else Zipf(zipf_s)
 * with P(l) proportional to 1/(l+1)^s.  Deterministic for a seed. */
gem_status gem_hgraph_set_labels(gem_hgraph *g, uint32_t nlabels, double zipf_s,
                                 uint64_t seed);
gem_status gem_hgraph_info(const gem_hgraph *g, uint32_t *nv,
                           uint64_t *n_arcs, uint32_t *max_label_plus1,
                           uint32_t *max_degree);
/* Borrow read-only views of the CSR arrays (valid until destroy). */
gem_status gem_hgraph_view(const gem_hgraph *g, const uint64_t **offsets,
                           const uint32_t **nbrs, const uint32_t **labels);
void gem_hgraph_destroy(gem_hgraph *g);

/* ------------------------------------------------------------------------ */
/* Queries.                                                                   */
/* ------------------------------------------------------------------------ */
typedef struct gem_query {
  uint32_t nv;             /* vertices 0..nv-1, 1 <= nv <= GEM_MAX_QV */
  uint32_t ne;             /* undirected edges */
  const uint32_t *labels;  /* nv labels, compared by value with data labels */
  const uint32_t *edges;   /* 2*ne entries: (src, dst) per undirected edge */
} gem_query;

/* Read a query in the text format (same reader as data graphs).  Writes
 * nv labels and 2*ne edge endpoints (edges in file order). */
gem_status gem_query_read_text(const char *path, uint32_t *nv, uint32_t *ne,
                               uint32_t *labels /* >= GEM_MAX_QV */,
                               uint32_t *edges /* >= 2*GEM_MAX_QE */);
gem_status gem_query_write_text(const gem_query *q, const char *path);

/* Random-walk query extraction: walk from a uniformly drawn vertex until k
 * distinct vertices are visited, keep all induced edges, relabel vertices
 * 0..k-1 in visit order and copy their labels (so every query has >= 1
 * match).  density: 0 = any, 1 = sparse (average degree <= 3), 2 = dense
 * (average degree > 3).  Sparse requests whose induced walk stays dense
 * after `max_tries` walks keep the walk's first-visit tree plus induced edges
 * in vertex order while the average degree stays <= 3.  Outputs for query i:
 * ne_out[i], labels_out[i*k .. +k), edges_out[i*2*max_e .. +2*ne_out[i]). */
gem_status gem_gen_queries(const gem_hgraph *g, uint32_t k, int density,
                           uint32_t count, uint64_t seed, uint32_t max_e,
                           uint32_t *ne_out, uint32_t *labels_out,
                           uint32_t *edges_out);

/* ------------------------------------------------------------------------ */
/* Device context: one GPU, resident data graph, memory budget.              */
/* Replaces main()'s global setup + aggressive_warmup                        */
/* (in-core/src/main.cu:45-76, in-core/lib/utils/src/cuda_helpers.cu:24-73). */
/* ------------------------------------------------------------------------ */
typedef struct gem_ctx gem_ctx;

typedef struct gem_opts {
  int device;                   /* CUDA device ordinal */
  uint64_t device_budget_bytes; /* 0 = 90% of free memory at create time */
  uint64_t pinned_budget_bytes; /* pinned host pool (out-of-core mode) */
  int ooc;                      /* 1 = keep the data graph in pinned host memory */
  uint32_t time_cap_ms;         /* per-query/batch device time cap (0 = 600000) */
  uint32_t index_kind;          /* 0 = auto, 1 = rank bitmap, 2 = cuckoo hash */
  uint32_t admit_gb;            /* serving admission budget in GiB (0 = 120) */
  uint32_t ooc_part_kib;        /* out-of-core: adjacency partition streamed per table pass, KiB (0 = 16384) */
  uint32_t ooc_stream;          /* out-of-core table builds: 0 = stream partitions when the wave's
                                   sources fill them enough, 1 = always stream, 2 = never (read the
                                   mapped adjacency in place) */
  uint32_t batch_lanes;         /* in-core batches of more than one wave: 0 = run on two lanes (one
                                   wave's join beside the next wave's table build), 1 = one lane */
  uint32_t reserved[2];
} gem_opts;

gem_status gem_ctx_create(const gem_opts *opts, gem_ctx **out);
void gem_ctx_destroy(gem_ctx *ctx);
/* Thread-local description of the last failure on this context. */
const char *gem_last_error(const gem_ctx *ctx);

/* Out-of-core partition streaming counters of a context, cumulative since
 * its graph was loaded (no counterpart in the reference, whose out-of-core
 * mode keeps the data graph on the host and pages intermediate tries,
 * out-of-core/lib/structure/src/memory_manager.cu:196-839).  In out-of-core
 * mode the adjacency is split at load time into vertex ranges of at most
 * ooc_part_kib KiB (a vertex whose list is longer gets a partition of its
 * own); a table build either streams the partitions its sources touch into
 * two device staging buffers on a side stream, each copy overlapping the
 * table kernels of the previous partition, or reads the mapped adjacency in
 * place. */
typedef struct gem_ooc_stats {
  uint32_t partitions;          /* partitions of the loaded graph */
  uint32_t reserved0;
  uint64_t max_part_bytes;      /* largest partition (each staging buffer's size) */
  uint64_t waves_streamed;      /* table builds that streamed partitions */
  uint64_t waves_in_place;      /* table builds that read the mapped adjacency */
  uint64_t parts_streamed;      /* partition copies issued (two table passes per build) */
  uint64_t bytes_streamed;      /* bytes those copies moved */
  uint64_t waves_spilled;       /* single-query waves whose edge-table values exceeded the device
                                   budget and were kept in mapped pinned host memory */
  uint64_t bytes_spilled;       /* bytes of those values (and key positions) */
  uint64_t resident_bytes;      /* device bytes the context holds outside its wave scratch (graph,
                                   partitions, join queue), counted against its device budget */
} gem_ooc_stats;
/* GEM_ERR_STATE while the context serves (gem_submit): its waves update the counters. */
gem_status gem_ctx_ooc_stats(const gem_ctx *ctx, gem_ooc_stats *out);
/* The out-of-core partitions of g for a partition size of part_kib KiB (0 =
 * 16384), as gem_ctx_load_graph cuts them (no counterpart in the reference,
 * which does not partition the data graph): part_v[0..n] (n + 1 entries) are
 * the vertex bounds, *n_out = n.  GEM_ERR_LIMIT when cap < n + 1 (*n_out is
 * still set).  Host only. */
gem_status gem_hgraph_partitions(const gem_hgraph *g, uint32_t part_kib, uint32_t *part_v, uint32_t cap,
                                 uint32_t *n_out);

/* Upload (in-core) or pin (out-of-core) a host graph; derived per-graph
 * indexes (degrees, neighbour-label counts) are built on the device.
 * Replaces allocateMemGPU/copyGraphToGPU (in-core/lib/io/src/io.cu:348-452). */
gem_status gem_ctx_load_graph(gem_ctx *ctx, const gem_hgraph *g);

/* ------------------------------------------------------------------------ */
/* Queries on the device.                                                     */
/* ------------------------------------------------------------------------ */
enum {
  GEM_MODE_COUNT = 0,     /* u64 count only (the reference's output)        */
  GEM_MODE_HASH = 1,      /* count + order-independent embedding hash        */
  GEM_MODE_ENUMERATE = 2  /* count + hash + embeddings written to a buffer   */
};

/* Per-phase timing slots of gem_result.ms (device time from CUDA events). */
enum {
  GEM_PH_FILTER = 0, GEM_PH_INDEX = 1, GEM_PH_TABLES = 2, GEM_PH_JOIN = 3,
  GEM_PH_TOTAL = 4, GEM_PH_H2D = 5, GEM_PH_D2H = 6, GEM_PH_HOST = 7
};

typedef struct gem_result {
  uint64_t count;        /* number of embeddings (exact, u64) */
  uint64_t emb_hash;     /* sum over embeddings of gem_embedding_hash (HASH/ENUMERATE) */
  uint64_t n_written;    /* embeddings written (ENUMERATE) */
  uint32_t status;       /* gem_status of this query */
  uint32_t n_tables;     /* directed edge tables built */
  uint64_t cand_total;   /* sum over query vertices of |C(u)| */
  uint64_t table_total;  /* sum of edge-table value counts */
  uint64_t nodes;        /* partial embeddings extended by the join (all levels) */
  uint64_t bytes_alg[4]; /* algorithmic bytes: filter, index, tables, join */
  float ms[8];           /* GEM_PH_* (batch: times of the wave that ran this query) */
  uint32_t wave;         /* batch: index of the wave that ran this query */
  uint32_t launches;     /* kernels launched for this query's wave */
  float table_pass_ms[2]; /* device time of the wave's edge-table count pass and write pass */
  float t_begin_ms;      /* device timeline of the wave: its first and last event, in ms after */
  float t_end_ms;        /* an event recorded when the context loaded its graph */
  uint64_t arena_bytes;  /* device scratch bytes the wave used */
} gem_result;

/* Run one query end to end on the device (filter -> index -> edge tables ->
 * join), synchronously.  threshold must be 0 (exact matching; relaxed
 * matching is gem_relaxed_run).  In
 * ENUMERATE mode up to emb_cap embeddings are written to emb_out as nv u32
 * per embedding in query-vertex order (order of embeddings unspecified);
 * more than emb_cap embeddings return GEM_ERR_OVERFLOW with the exact count.
 * Replaces main()'s phase chain (in-core/src/main.cu:140-236). */
gem_status gem_query_run(gem_ctx *ctx, const gem_query *q, uint32_t threshold,
                         int mode, uint32_t *emb_out, uint64_t emb_cap,
                         gem_result *res);

/* Run many queries in one persistent join launch (waves sized to the device
 * budget), each query's result identical to gem_query_run's.
 * Replaces the out-of-core directory batch loop (out-of-core/src/main.cu:334-410). */
gem_status gem_batch_run(gem_ctx *ctx, const gem_query *qs, uint32_t n,
                         int mode, gem_result *res);

/* Relaxed matching (the reference's -t T; in-core/lib/plan/src/relax.cpp:84-142
 * and the per-relaxed-query counts of in-core/src/main.cu:229-236).  The
 * relaxed queries of q at `threshold` are its edge subsets that still connect
 * all its vertices with at most `threshold` of its edges removed; each keeps
 * q's vertices and labels.  gem_relaxed_sets lists them (host only): ets[i]
 * has bit j set when q's edge j (in q's order) is kept; fewest edges removed
 * first, then by mask descending.  gem_relaxed_run counts each exactly, as
 * its own query, with res[i] for ets[i]: in one wave whose candidate lists are
 * q's own filtered with slack `threshold` (as the reference filters at -t T),
 * so the relaxed queries share those lists and the edge tables of the edges
 * they keep (as one gem_batch_run when that wave does not fit the budget).  At most cap
 * relaxed queries: with more, GEM_ERR_LIMIT and *n_out = cap + 1.  Queries
 * with more than 64 edges return GEM_ERR_LIMIT.  A query with one edge or
 * none has only itself (the reference lists none). */
gem_status gem_relaxed_sets(const gem_query *q, uint32_t threshold, uint32_t cap, uint64_t *ets,
                            uint32_t *n_out);
gem_status gem_relaxed_run(gem_ctx *ctx, const gem_query *q, uint32_t threshold, int mode, uint32_t cap,
                           uint64_t *ets, gem_result *res, uint32_t *n_out);

/* Matching order of q (host only).  Replaces the order that the reference's
 * lattice gives single-edge extensions (in-core/lib/structure/src/lattice.cpp
 * :41-185, unifiedTrie.cu:939-1018).  cand_counts[u] is |C(u)| (gem_filter
 * returns it).  With closed_form = 1 (count mode) an independent set of q's
 * vertices whose removal leaves the rest connected moves to the end and is
 * counted in closed form: levels *n_enum .. nv-1.  order_out[k] (nv entries)
 * is the query vertex matched at level k. */
gem_status gem_plan_query(const gem_query *q, const uint32_t *cand_counts, int closed_form, uint32_t *n_enum,
                          uint32_t *order_out);

/* Autotuner (no counterpart in the reference): for each query-size bucket
 * (<=4, <=8, <=12, <=16, <=24, <=32 vertices) present in qs, runs the first
 * 256 of its queries as one wave under each candidate join schedule (blocks
 * per SM of the persistent grid, deepest level that donates work), twice per
 * candidate, each trial capped at trial_cap_ms, and keeps the fastest for
 * later waves of this context.  The sample should hold the workload's heavy
 * queries: a wave's join time is that of its slowest query.
 * Candidate schedules combine blocks per SM with the deepest donating level,
 * the smallest donated half at the lane-parallel level and the root batch.
 * report (optional, 18 entries): per bucket {blocks_per_sm,
 * donate_max_level | donate_min_lane << 8 | root_batch_max << 20, best join
 * time in us}; zeros for untuned buckets. */
gem_status gem_autotune(gem_ctx *ctx, const gem_query *qs, uint32_t n, int mode,
                        uint32_t trial_cap_ms, uint32_t *report);

/* Join schedule of one query-size bucket (no counterpart in the reference).
 * Every field 0 means the library default.  blocks_per_sm caps the
 * persistent grid; donate_max_level is the deepest level that hands work to
 * idle warps; donate_min_lane / donate_min_desc are the smallest halves of a
 * level's unread candidates worth handing over (last enumerated level /
 * other levels); root_batch_max caps the roots a warp takes at once;
 * lane_scan_max is the longest intersection a single lane works through
 * before the whole warp takes it over; split_blocks is the work (in blocks
 * of 8 scanned entries) above which a warp's chunk of last-level matches is
 * split with idle warps. */
typedef struct gem_schedule {
  uint32_t blocks_per_sm;
  uint32_t donate_max_level;
  uint32_t donate_min_lane;
  uint32_t donate_min_desc;
  uint32_t root_batch_max;
  uint32_t lane_scan_max;
  uint32_t split_blocks;
  uint32_t reserved;
} gem_schedule;

/* Set / read the schedule used for waves whose largest query has
 * query_vertices vertices (its bucket: <=4, <=8, <=12, <=16, <=24, <=32).
 * gem_autotune overwrites the schedules of the buckets it tunes. */
gem_status gem_set_schedule(gem_ctx *ctx, uint32_t query_vertices, const gem_schedule *sched);
gem_status gem_get_schedule(gem_ctx *ctx, uint32_t query_vertices, gem_schedule *sched);

/* Embedding hash of one embedding f (f[u] = data vertex of query vertex u):
 * h = mix(sum_u mix(f[u] | u << 32)) with mix the splitmix64 finaliser of
 * (x + 0x9E3779B97F4A7C15); GEM_MODE_HASH reports the sum of h over all
 * embeddings (mod 2^64), which does not depend on enumeration order. */
uint64_t gem_embedding_hash(const uint32_t *f, uint32_t nv);

/* ------------------------------------------------------------------------ */
/* Phase entry points (parity testing and tooling).                           */
/* ------------------------------------------------------------------------ */
/* Candidate filter: C(u) for every query vertex u, sorted ascending:
 * label(v) == label(u), deg(u) <= deg(v) + threshold and
 * sum_l max(0, nlc_u[l] - nlc_v[l]) <= threshold over the labels present in
 * the query.  counts[u] = |C(u)|; cand_out receives the lists back to back
 * (u = 0 first); needs sum counts <= cand_cap.
 * Replaces filterSSM (in-core/lib/filter/src/filter.cu:34-167). */
gem_status gem_filter(gem_ctx *ctx, const gem_query *q, uint32_t threshold,
                      uint32_t *counts, uint32_t *cand_out, uint64_t cand_cap);

/* Edge-candidate table T(u -> w) for the query edge {u, w}: for the i-th
 * candidate v of C(u), the values are N(v) ∩ C(w) in adjacency (ascending)
 * order.  offsets_out has |C(u)|+1 entries; values_out needs offsets[|C(u)|]
 * <= values_cap entries.  *n_keys and *n_values receive the sizes (also when
 * the buffers are too small, which returns GEM_ERR_OVERFLOW).
 * Replaces construct_edge_candidates for one directed edge
 * (in-core/lib/structure/src/unifiedTrie.cu:1020-1240). */
gem_status gem_edge_table(gem_ctx *ctx, const gem_query *q, uint32_t u,
                          uint32_t w, uint64_t *offsets_out, uint64_t offsets_cap,
                          uint32_t *values_out, uint64_t values_cap,
                          uint64_t *n_keys, uint64_t *n_values);

/* Index probe: position of each data vertex keys[i] in C(u) (or 0xFFFFFFFF
 * when absent) through the device index of kind index_kind (1 = rank bitmap,
 * 2 = cuckoo hash).  Replaces HashTable::build + hash_lookup
 * (in-core/lib/structure/src/unifiedTrie.cu:175-433,
 *  in-core/lib/structure/include/unifiedTrie.cuh:84-125). */
gem_status gem_index_probe(gem_ctx *ctx, const gem_query *q, uint32_t u,
                           uint32_t index_kind, const uint32_t *keys,
                           uint32_t n_keys, uint32_t *pos_out);

/* Candidate filter that allocates nothing (no counterpart in the reference).
 * For callers that cannot allocate device memory — code inside another
 * framework's allocator or memory pool, which owns every device byte of the
 * process, or a service whose memory is reserved up front and must not grow
 * while it serves.  The caller passes the
 * data graph as device arrays it owns (offsets nv+1, nbrs offsets[nv],
 * labels nv) and a device output array d_cand of cand_cap entries; the
 * C(u) lists are written back to back (u = 0 first) and counts[u] (host
 * array, nv_q entries) receives |C(u)|, exactly as gem_filter does.  Scratch
 * lives in a fixed device array of GEM_STATIC_SCRATCH_BYTES held by every
 * GPU that loads libgem until exit; graphs above GEM_STATIC_MAX_VERTICES
 * vertices return GEM_ERR_LIMIT; more candidates than cand_cap return
 * GEM_ERR_OVERFLOW with exact counts.  All calls on a device share that
 * array, so calls whose work overlaps on the GPU race: order them on one
 * stream.  Every call looks up the array's address in the caller's current
 * context.  stream is a cudaStream_t (NULL = legacy default stream); the
 * call blocks until the stream has finished its work (it reads each
 * candidate count back), so it cannot be made during stream capture.  All
 * four device pointers must be non-null; a neighbour id >= nv or offsets
 * that decrease or run past offsets[nv] are skipped on the device and
 * return GEM_ERR_ARG. */
#define GEM_STATIC_SCRATCH_BYTES (4u << 20)
#define GEM_STATIC_MAX_VERTICES 8000000u
gem_status gem_filter_static(const uint64_t *d_offsets, const uint32_t *d_nbrs,
                             const uint32_t *d_labels, uint32_t nv,
                             const gem_query *q, uint32_t threshold,
                             uint32_t *counts, uint32_t *d_cand,
                             uint64_t cand_cap, void *stream);

/* ------------------------------------------------------------------------ */
/* Serving: continuous batching with memory-based admission.                 */
/* The first gem_submit starts a server thread on the context; from then on  */
/* only gem_submit and gem_poll are accepted (others return GEM_ERR_STATE)   */
/* until gem_ctx_destroy.  Admitted requests run in waves: everything        */
/* admitted while a wave is on the GPU forms the next wave.                  */
/* ------------------------------------------------------------------------ */
/* An upper bound of the device scratch a wave of q alone takes, from the
 * resident graph's label statistics (host only, no counterpart in the
 * reference).  gem_submit charges the admission budget this bound times a
 * factor (at most 1) learnt from the bytes its waves took of their
 * queries' bounds. */
gem_status gem_estimate_bytes(const gem_ctx *ctx, const gem_query *q, uint64_t *bytes);
/* Submit a query; returns GEM_ERR_OOM when its charge does not fit the
 * admission budget right now (caller retries later). */
gem_status gem_submit(gem_ctx *ctx, const gem_query *q, int mode,
                      uint64_t *ticket);
/* Advance the server (admit queued work, launch, retire finished queries)
 * and report whether `ticket` is done; *done = 1 fills *res. */
gem_status gem_poll(gem_ctx *ctx, uint64_t ticket, gem_result *res, int *done);

#ifdef __cplusplus
}
#endif

#endif /* GEM_H */
