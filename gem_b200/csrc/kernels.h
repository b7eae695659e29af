// Launch wrappers and descriptor structs shared by the host orchestration
// (ctx.cu) and the kernel translation units.  All pointers are device
// pointers unless named h_*.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <atomic>

namespace gem {

// Number of kernels libgem has launched (all contexts); read by the C-ABI
// results so callers can report their launch counts.
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

constexpr uint32_t QV = 32;           // max query vertices
constexpr uint32_t NLC_MAX_LABELS = 64;  // per-vertex label-count table kept up to this many labels

// ---------------------------------------------------------------------------
// Graph (device-resident CSR plus derived per-vertex data)
// ---------------------------------------------------------------------------
struct DevGraph {
  uint32_t nv = 0;
  uint64_t narcs = 0;
  uint32_t nlabels = 0;     // max label + 1
  uint32_t nlc_stride = 0;  // bytes per vertex in nlc (0: no table)
  const uint64_t *off = nullptr;
  const uint32_t *nbr = nullptr;
  const uint32_t *lab = nullptr;
  const uint32_t *deg = nullptr;
  const uint8_t *nlc = nullptr;  // saturating neighbour-label counts
};

// Per-graph derived data, built once at load time.
void launch_degrees(const DevGraph &g, uint32_t *deg, cudaStream_t s);
void launch_nlc(const DevGraph &g, uint8_t *nlc, uint32_t stride, cudaStream_t s);

// Neighbourhood hash: per vertex u an open-addressed table of its neighbours
// (u32, empty = VNH_EMPTY) of a power of two >= 2 deg(u) slots, at
// [hoff[u], hoff[u+1]) of `slots`; a neighbour v starts probing at the top
// log2(size) bits of v * VNH_MULT and moves to the next slot (mod size).
// It answers "is (u, v) an arc" in about one load, where a binary search of
// a hub's sorted adjacency takes a dozen dependent loads.
constexpr uint32_t VNH_EMPTY = 0xFFFFFFFFu;
constexpr uint64_t VNH_MULT = 0x9E3779B97F4A7C15ull;
void launch_vnh_build(const DevGraph &g, const uint64_t *hoff, uint32_t *slots, uint64_t n_slots,
                      cudaStream_t s);

// ---------------------------------------------------------------------------
// Generic exclusive scan (u64 results, n + 1 entries: out[n] = total)
// ---------------------------------------------------------------------------
enum ScanInput : uint32_t {
  SCAN_POPC_U64LO = 0,  // popcount of the low 32 bits of a u64 word
  SCAN_POPC_U32 = 1,    // popcount of a u32 word
  SCAN_U32 = 2,         // plain u32 values
};
// out[i] = in[i * stride] for i < n.
void launch_gather_strided(const uint64_t *in, uint64_t stride, uint32_t n, uint64_t *out, cudaStream_t s);
// *deadline = device global timer + cap_ns.
void launch_set_deadline(unsigned long long *deadline, uint64_t cap_ns, cudaStream_t s);
// tmp needs scan_tmp_words(n) u64 words.
uint64_t scan_tmp_words(uint64_t n);
void launch_scan(const void *in, ScanInput kind, uint64_t n, uint64_t *out, uint64_t *tmp,
                 cudaStream_t s);

// ---------------------------------------------------------------------------
// Filter
// ---------------------------------------------------------------------------
struct FilterDesc {          // one query of a wave
  uint32_t nq;               // query vertices
  uint32_t nql;              // distinct labels in the query
  uint32_t threshold;
  uint32_t row_base;         // first rank-bitmap row of this query
  uint32_t ql[QV];           // distinct labels
  uint32_t lab[QV];          // label of each query vertex
  uint32_t deg[QV];          // query degree of each vertex
  uint8_t nlc[QV][QV];       // nlc[u][k]: neighbours of u with label ql[k]
};

// Writes the candidate bit of every (query vertex, data vertex) pair into the
// low halves of rb (rows of nwords u64, row = row_base + u).
void launch_filter(const DevGraph &g, const FilterDesc *d_desc, uint32_t nquery, uint64_t *rb,
                   uint32_t nwords, cudaStream_t s);
// Given ex = exclusive scan of popcounts over all rows, writes the per-word
// ranks into the high halves of rb and the sorted candidate lists
// cand[c_base[row] ...].
// bit_rows (optional, nrows x nwords u32): the membership bits alone, half
// the bytes of rb for tests that need no rank.
void launch_compact(uint64_t *rb, const uint64_t *ex, uint32_t nrows, uint32_t nwords,
                    const uint64_t *c_base, uint32_t *cand, cudaStream_t s, uint32_t *bit_rows = nullptr);

// ---------------------------------------------------------------------------
// Edge-candidate tables
// ---------------------------------------------------------------------------
struct TabSource {           // a (query, query vertex) whose candidates are table keys
  const uint32_t *keys;      // C(u), sorted
  uint32_t nkeys;
  uint32_t pad;
  uint64_t key_base;         // first index of this source in the flattened key space
};
struct TabEdge {             // a directed table T(u -> w)
  uint32_t src;              // index into TabSource
  uint32_t flags;            // TAB_KEY_MAP: the write pass also records each value's key position
  uint32_t tcol;             // the target row's bit in the target membership columns
  uint32_t pad;
  uint64_t tile_base;        // first tile of this edge in the flattened edge-tile space
  uint64_t ntiles;
  uint64_t off_base;         // first entry of this edge in the flattened offsets space
  uint64_t *offsets;         // nkeys + 1 absolute positions into the values array
};
// tiles[k] = ceil(deg(key k) / 32) over the flattened key space.
void launch_key_tiles(const DevGraph &g, const TabSource *d_src, uint32_t nsrc, uint64_t nkeys,
                      uint32_t *tiles, cudaStream_t s);
// Membership columns of a list of rows: out[v * W + c] bit b = v is in row
// rows[32c + b] (bits: membership bit rows, nwords u32 words per row).  With
// vtiles, vtiles[v] = ceil(deg(v) / 32) for a vertex in any of the rows, else 0.
void launch_row_columns(const uint32_t *bits, uint32_t nwords, const uint32_t *rows, uint32_t nrows, uint32_t W,
                        uint32_t nv, uint32_t *out, uint32_t *vtiles, const uint32_t *deg, cudaStream_t s);
// vt[t] = v for every vertex tile t in [vtp[v], vtp[v + 1]).
void launch_vertex_tile_map(const uint64_t *vtp, uint32_t nv, uint32_t *vt, cudaStream_t s);
// Write-pass units: out[v] = ceil(vtiles[v] / TAB_WGROUP).
constexpr uint32_t TAB_WGROUP = 4;
void launch_unit_counts(const uint32_t *vtiles, uint32_t nv, uint32_t *out, cudaStream_t s);
// out[i] = a[idx[i]].
void launch_gather_u64(const uint64_t *a, const uint32_t *idx, uint32_t n, uint64_t *out, cudaStream_t s);
struct VSrc {                // a table source as the vertex-tile passes see it
  const uint64_t *rb;        // rank bitmap row of its candidates
  uint64_t key_base;         // first key in the flattened key space
  uint64_t stb;              // tp[key_base]: its first tile
  uint32_t e0, ne;           // its tables: edges [e0, e0 + ne)
};
struct VEdge {
  uint64_t tile_base;
  uint32_t tcol;
  uint32_t flags;
};
// One table pass over units [t0, t1): the count pass's units are vertex
// tiles (vt: tile -> vertex, vtp: first tile of each vertex), the write
// pass's up to TAB_WGROUP consecutive tiles of one vertex (vg, vgp).  Arcs are read at nbr[arc - arc_shift], with off the
// device offsets of the data graph.  S: the source membership columns (WS
// words per vertex), B: the target membership columns (WT words per vertex).
// count: mask[edge.tile_base + lt] = the 32-bit membership mask of tile lt of
// the edge's source; write: the values (and key positions) at vp.
struct VPass {
  const uint64_t *off;
  const uint32_t *nbr;
  uint64_t arc_shift;
  uint64_t t0, t1;
  const uint32_t *vt;
  const uint64_t *vtp;
  const uint32_t *vg;        // write pass: unit -> vertex (units of up to 4 tiles of one vertex)
  const uint64_t *vgp;       // first unit of each vertex
  const uint32_t *S;
  uint32_t WS;
  uint32_t WT;
  uint32_t WTp;              // set by the launcher
  uint32_t pad;
  const uint32_t *B;
  const VSrc *vsrc;
  const VEdge *vedge;
  const uint64_t *tp;
  uint32_t *mask;
  const uint64_t *vp;
  uint32_t *values;
  uint32_t *vkey;
  unsigned long long *next;  // tile counter of the launch (zeroed by the launcher)
};
void launch_table_vtx(const VPass &P, bool write, cudaStream_t s);
// Whether the count pass can stage WT-word target columns (WT a multiple of
// 4, at most 128: 4,096 target rows).
bool table_vtx_fits(uint32_t WT);
// out[i] = tp[d_src[i].key_base] for i < nsrc, out[nsrc] = tp[nkeys].
void launch_source_tile_bases(const TabSource *d_src, uint32_t nsrc, uint64_t nkeys, const uint64_t *tp,
                              uint64_t *out, cudaStream_t s);
// out[e] = vp[edges[e].tile_base] for e < nedge and out[nedge] = vp[tiles]:
// the first value position of every table (and the total), so that table e
// holds out[e + 1] - out[e] values.
void launch_edge_value_bases(const TabEdge *d_edge, uint32_t nedge, const uint64_t *vp, uint64_t tiles,
                             uint64_t *out, cudaStream_t s);
void launch_table_offsets(const TabSource *d_src, const TabEdge *d_edge, uint32_t nedge,
                          const uint64_t *tp, const uint64_t *vp, uint64_t total_offsets,
                          cudaStream_t s);
constexpr uint32_t TAB_KEY_MAP = 1;

// ---------------------------------------------------------------------------
// Cuckoo hash: vertex id -> position in C(u).  Two bucketised tables of
// 128-byte buckets (16 slots of {key, pos}) plus a small stash.
// ---------------------------------------------------------------------------
constexpr uint32_t CK_SLOTS = 16;         // slots per bucket (one 128-byte line)
constexpr uint32_t CK_STASH = 64;
constexpr uint32_t CK_MAX_KICKS = 64;
constexpr uint64_t CK_EMPTY = ~0ull;
struct CuckooTable {
  uint64_t *t0;              // nb0 * 16 slots
  uint64_t *t1;              // nb1 * 16 slots
  uint64_t *stash;           // CK_STASH slots
  uint32_t *stash_n;
  uint32_t nb0, nb1;
  uint64_t a0, c0, a1, c1;   // multiply-add hash parameters
  const uint32_t *keys;      // C(u)
  uint32_t nkeys;
  uint32_t pad;
  uint64_t key_base;         // first key of this table in the flattened build space
};
uint64_t cuckoo_slots_for(uint32_t nkeys, uint32_t *nb0, uint32_t *nb1);
// Builds every table (keys inserted with pos = index); small tables are
// assembled in shared memory and written out with coalesced stores.
// Slots (t0, t1, stash) must be preset to CK_EMPTY and stash_n to 0.
void launch_cuckoo_build(const CuckooTable *d_tabs, const CuckooTable *h_tabs, uint32_t ntab,
                         uint32_t *err, cudaStream_t s);
void launch_cuckoo_probe(const CuckooTable *d_tab, const uint32_t *keys, uint32_t n, uint32_t *out,
                         cudaStream_t s);
void launch_rank_probe(const uint64_t *rb, const uint32_t *keys, uint32_t n, uint32_t *out,
                       cudaStream_t s);

// ---------------------------------------------------------------------------
// Join (warp-level DFS over the matching order)
// ---------------------------------------------------------------------------
constexpr uint32_t IDX_NONE = 0, IDX_RANK = 1, IDX_CUCKOO = 2;

struct JLevel {
  uint32_t u;          // query vertex matched at this level
  uint32_t nback;      // backward neighbours (tables keyed by earlier levels)
  uint32_t back_base;  // first entry in the JBack array
  uint32_t dup_mask;   // earlier levels with the same label (injectivity)
  uint32_t idx_kind;   // how this level's vertex finds its position in C(u)
  uint32_t pad;
  const uint64_t *rb;          // IDX_RANK
  const CuckooTable *ck;       // IDX_CUCKOO
};
struct JBack {
  uint32_t lvl;              // level of the key vertex
  uint32_t nkeys;            // keys of the table (offsets has nkeys + 1 entries)
  const uint64_t *off;       // table offsets (absolute into the values array)
};
// Join: per-warp shared-memory cache of suffix lists (slots x entries).
constexpr uint32_t LIST_CACHE_SLOTS = 2;
// 512 entries per slot: with 72 KiB of dynamic shared memory per block (two
// blocks per SM) the rest of the SM's 228 KiB of shared memory / L1 serves as
// L1 for the join's table and hash loads; 1,024-entry slots measured 10%
// slower on the headline batch.
constexpr uint32_t LIST_CACHE_CAP = 512;
constexpr uint32_t JOIN_WARPS_PER_BLOCK = 8;
// Balanced lane-level counting: per warp, up to FLAT_MAX_JOBS intersections
// (one per subset of a prefix match) shared out in blocks of 8 entries.
constexpr uint32_t FLAT_MAX_VALUES = 4;  // subset values per prefix match
constexpr uint32_t FLAT_MAX_JOBS = 96;
constexpr uint32_t FLAT_JOB_BYTES = 40;
constexpr uint32_t FLAT_WARP_BYTES = FLAT_MAX_JOBS * (FLAT_JOB_BYTES + 8) + 16;
// Ranges of the suffix lists keyed by prefix levels, per warp: 32 {lo, hi}
// pairs and a header (the first suffix back entry).
constexpr uint32_t SUFFIX_RANGE_BYTES = 32 * 16 + 16;
constexpr uint32_t JOIN_WARP_SMEM = LIST_CACHE_SLOTS * LIST_CACHE_CAP * 4 + FLAT_WARP_BYTES + SUFFIX_RANGE_BYTES;
constexpr uint32_t JOIN_DYN_SMEM = JOIN_WARPS_PER_BLOCK * JOIN_WARP_SMEM;
constexpr uint32_t MAX_GROUPS = 16;   // label groups of a closed-form suffix
constexpr uint32_t MAX_GROUP = 4;     // members of one group (15 subsets, 15 partitions)
// Inclusion-exclusion term: coefficient in the high 32 bits (two's
// complement), then up to four 4-bit block masks over the group's members
// (block b in bits 4b..4b+3; a zero mask ends the list).
inline uint64_t make_term(int32_t coef, uint32_t packed_blocks) {
  return ((uint64_t)(uint32_t)coef << 32) | packed_blocks;
}
struct JQuery {
  uint32_t n;                // query vertices (levels)
  uint32_t root_u;
  const uint32_t *root_cand; // C(root)
  uint32_t n_root;
  uint32_t n_enum;           // levels enumerated; levels n_enum..n-1 are counted in closed form
  uint64_t root_base;        // first global root index of this query
  uint32_t n_groups;         // label groups of the suffix
  uint32_t flat;             // balanced lane-level counting: subset values per prefix match
                             // (bits 0-7; 0 = not eligible) and those needing a scan (bits 8-15)
  uint32_t grp_first[MAX_GROUPS];
  uint32_t grp_size[MAX_GROUPS];
  uint32_t term_base[MAX_GROUPS];
  uint32_t term_count[MAX_GROUPS];
  JLevel lv[QV];             // lv[0] describes the root's index only
};
struct JOut {                // per query, accumulated with atomics
  unsigned long long count;
  unsigned long long hash;
  unsigned long long written;
  unsigned long long nodes;      // extended partial embeddings
  unsigned long long scanned;    // source-list elements evaluated
  unsigned long long probes;     // binary-search and index probes
  unsigned long long pad[2];     // pad[0] != 0: some work of this query was abandoned
};
// Donation queue: QUEUE_SUBQ sub-queues of QUEUE_SUBQ_CAP cells each, so
// that thousands of polling warps spread their atomics over many lines.
constexpr uint32_t QUEUE_SUBQ = 128;
constexpr uint32_t QUEUE_SUBQ_CAP = 256;                    // power of two
constexpr uint32_t TASK_CAP = QUEUE_SUBQ * QUEUE_SUBQ_CAP;  // donation queue cells
// A push skips a sub-queue holding this many tasks; the other half of the
// cells is room for the warps that passed the check at the same time.
constexpr uint32_t QUEUE_SUBQ_FILL = QUEUE_SUBQ_CAP / 2;
struct JQueueEnds {  // one sub-queue; head and tail on lines of their own
  alignas(128) unsigned long long head;  // next position to take
  alignas(128) unsigned long long tail;  // next position to reserve
};
struct JTask {
  unsigned long long seq;
  uint32_t q, lvl, src;      // query, level whose candidates are donated, source back entry
  uint32_t pad;
  uint64_t begin, end;       // range in the values array
  uint64_t hs;               // hash prefix of levels < lvl
  uint32_t f[QV];
  uint32_t idx[QV];
};
// Zeroed before every launch (except the queue cells' sequence numbers).
// Every counter that many warps update or poll sits on a 128-byte line of
// its own, so the atomics on one do not queue behind traffic to the others.
struct JControl {
  alignas(128) unsigned long long lp_next;    // next root of the lane-parallel pool
  alignas(128) unsigned long long lp2_next;   // next chunk of the (root, first level) pair pool
  alignas(128) unsigned long long root_next;  // next root of the ordinary pool
  alignas(128) unsigned long long pending;    // tasks published and not yet taken
  alignas(128) unsigned int busy;             // warps holding work
  alignas(128) unsigned int idle;             // warps waiting for donated work
  alignas(128) unsigned long long emb_next;   // enumerate cursor
  alignas(128) unsigned int err;              // read-mostly: error word, then cold fields
  unsigned int pad;
  unsigned long long deadline_ns;
  unsigned long long bad_site;   // first failed bounds check: site id
  unsigned long long bad_value;  // ... the offending index
  unsigned long long bad_limit;  // ... and its limit
};

enum : uint32_t { MODE_COUNT = 0, MODE_HASH = 1, MODE_ENUM = 2 };
struct JoinArgs {
  const JQuery *queries;
  uint32_t nquery;
  uint32_t mode;
  const JBack *backs;
  JQueueEnds *qends;          // QUEUE_SUBQ sub-queue ends (cells in `queue`)
  const uint32_t *values;     // edge-table values of the whole wave
  const uint64_t *root_prefix; // nquery + 1 global root offsets
  // Lane-parallel root pool: queries whose only enumerated level is the root
  // (count mode with n_enum == 1, or single-vertex queries); 32 roots per warp.
  const uint32_t *lp_query;    // query index of each pool segment
  const uint64_t *lp_prefix;   // lp_nq + 1 root offsets
  uint32_t lp_nq;
  uint32_t pad_lp;
  uint64_t lp_roots;
  const uint64_t *terms;      // inclusion-exclusion terms of every query's suffix groups
  uint64_t n_roots;
  JOut *out;
  JControl *ctl;
  JTask *queue;
  uint32_t *emb;             // ENUM: output buffer
  uint64_t emb_cap;          // embeddings that fit
  uint32_t donate_max_level; // donate candidates of levels <= this
  uint32_t donate_min_lane;  // smallest donated half at the lane-parallel level
  uint32_t donate_min_desc;  // smallest donated half at other levels
  uint32_t root_batch_max;   // largest root batch a warp takes at once
  uint32_t lane_scan_max;    // longest intersection one lane does alone
  uint32_t nv;               // data vertices (bounds of rank-bitmap probes)
  uint32_t flat_donate_blocks; // balanced counting: chunks above this many blocks are split with idle warps
  const uint32_t *lp2_query; // queries whose prefix is (root, first level): their pair pool
  uint32_t lp2_nq;
  const uint64_t *lp2_prefix; // lp2_nq + 1 chunk-padded pair offsets (written by the prepare kernel)
  const uint32_t *vkey;       // per value of the pool queries' root tables: its key's position
  const uint64_t *vnh_off;   // neighbourhood hash offsets (nv + 1), or null: binary search
  const uint32_t *vnh_slots;
  uint64_t n_values;         // entries of `values`
  uint32_t n_backs;          // entries of `backs`
  uint32_t n_terms;          // entries of `terms`
};
// The join of a wave as a CUDA graph: a prepare kernel (zero the control
// block and the per-query outputs, reset the task queue, set the device
// deadline) followed by the persistent join.  One executable graph is built
// per (mode, grid) and reused; each wave only updates the two kernel nodes'
// parameters before cudaGraphLaunch.
struct JoinGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t prep = nullptr, join = nullptr;
  uint32_t mode = 0, grid = 0;
};
cudaError_t launch_join_graph(JoinGraph &jg, const JoinArgs &a, uint64_t cap_ns, uint32_t grid, cudaStream_t s);
void destroy_join_graph(JoinGraph &jg);
int join_blocks_per_sm(uint32_t mode);

}  // namespace gem
