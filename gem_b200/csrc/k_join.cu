// Edge join: depth-first extension of partial embeddings, one warp per task.
//
// Replaces the reference's level-at-a-time join (in-core/lib/join/src/
// join_trie.cu:1087-1277: direct_join 397-718, refer_join 720-1023,
// host_select 116-395 and the kernels of join_trie_kernel.cu:85-1099), which
// materialises every intermediate level as {vertex, parent} columns, runs a
// count kernel, a CUB scan, a host sync and an allocation per step, and only
// skips materialising the last level.  Same result (the number of injective,
// label-preserving, edge-preserving maps), different execution:
//
//  * the matching order is a chain of levels; level k's candidates are the
//    edge-table lists T(u_j -> u_k)[pos of f(u_j) in C(u_j)] of all its
//    backward neighbours u_j (tree edge and non-tree edges alike): the
//    shortest list is scanned 32 candidates at a time (one per lane) and the
//    others are probed by binary search, which covers the reference's
//    "select" step for non-tree edges;
//  * injectivity compares a candidate with the earlier levels of the same
//    label only (the reference's dup_check_type, join_trie.cu:450-462);
//  * the state of level L lives in lane L's registers (levels <= 32), so a
//    warp's whole DFS stack costs a few registers per lane and no memory;
//  * count mode: the planner's closed-form suffix (an independent set of
//    query vertices, e.g. the leaves of a tree) is counted by
//    inclusion-exclusion instead of being enumerated, one candidate of the
//    last enumerated level per lane (32 prefix matches in flight per warp);
//  * one persistent grid serves every query of a wave: warps take root
//    candidates from a global counter and, once roots run out, receive work
//    donated by busy warps (half of the unread candidates of a shallow
//    level) through a bounded lock-free queue.  Every wait is bounded by the
//    device deadline; an expired deadline sets a TIMEOUT status;
//  * every indexed access is bounds-checked against the wave's sizes; a
//    failed check records (site, value, limit) in the control block, skips
//    the access and stops the grid.
#include "device_common.cuh"
#include "index_device.cuh"
#include "kernels.h"

namespace gem {

using namespace dev;

struct LaneState {   // lane L holds the state of level L
  uint32_t f;        // matched data vertex
  uint32_t idx;      // position of f in C(u_L)
  uint64_t hs;       // hash prefix over levels 0..L
  uint64_t pos;      // next unread position of the level's source range
  uint64_t end;      // end of the level's source range
  uint64_t cbase;    // first position of the current chunk
  uint32_t mask;     // candidates of the current chunk not yet descended
  uint32_t src;      // back entry scanned at this level
};

struct Stats {
  uint64_t nodes = 0, scanned = 0, probes = 0;
};

// Bounds-check sites (reported through JControl::bad_site).
enum : uint32_t {
  SITE_BACK = 1,     // back-entry index
  SITE_KEY = 2,      // table key (position of the key vertex)
  SITE_RANGE = 3,    // table range outside the values array
  SITE_VERTEX = 4,   // data vertex id of an index probe
  SITE_QUERY = 5,    // query index of a task
  SITE_LEVEL = 6,    // level of a task or of a descent
  SITE_ROOT = 7,     // root position
  SITE_TERM = 8,     // inclusion-exclusion term index
  SITE_KEYLVL = 9    // key level after the probing level
};

__device__ __forceinline__ unsigned long long ld_vol(const unsigned long long *p) {
  return *reinterpret_cast<const volatile unsigned long long *>(p);
}
__device__ __forceinline__ unsigned int ld_vol(const unsigned int *p) {
  return *reinterpret_cast<const volatile unsigned int *>(p);
}

// True when idx < lim; otherwise records the first violation and stops the grid.
__device__ __forceinline__ bool inb(const JoinArgs &a, uint32_t site, uint64_t idx, uint64_t lim) {
  if (idx < lim) return true;
  if (atomicCAS(&a.ctl->err, DERR_NONE, DERR_BOUNDS) == DERR_NONE) {
    a.ctl->bad_site = site;
    a.ctl->bad_value = idx;
    a.ctl->bad_limit = lim;
  }
  return false;
}

// Warp-uniform: true once the error word is set or the time cap has passed
// (the cap then sets the error word, so every warp stops at its next look).
__device__ __forceinline__ bool stop_now(const JoinArgs &a, uint64_t deadline) {
  int stop = 0;
  if (lane_id() == 0) {
    if (ld_vol(&a.ctl->err) != DERR_NONE) {
      stop = 1;
    } else if (globaltimer_ns() > deadline) {
      set_error(&a.ctl->err, DERR_TIMEOUT);
      stop = 1;
    }
  }
  return __shfl_sync(FULL, stop, 0) != 0;
}

// Warp-uniform: the error word is set (a count cut short by the cap may
// have been added since the last look).
__device__ __forceinline__ bool err_set(const JoinArgs &a) {
  return __shfl_sync(FULL, lane_id() == 0 ? (int)(ld_vol(&a.ctl->err) != DERR_NONE) : 0, 0) != 0;
}

// Range [lo, hi) of table entry b at key position kidx (checked).
__device__ __forceinline__ void table_range(const JoinArgs &a, const JBack *b, uint32_t kidx, uint64_t &lo,
                                            uint64_t &hi) {
  lo = hi = 0;
  if (!inb(a, SITE_KEY, kidx, b->nkeys)) return;
  const uint64_t l = __ldg(b->off + kidx), h = __ldg(b->off + kidx + 1);
  if (!inb(a, SITE_RANGE, h, a.n_values + 1) || !inb(a, SITE_RANGE, l, h + 1)) return;
  lo = l;
  hi = h;
}

// Per back entry i (lane i < nback): the list T(u_j -> u_L)[idx_j] as the
// absolute range [lo, hi) of the values array.
__device__ __forceinline__ void level_ranges(const JoinArgs &a, const JLevel *__restrict__ L, const LaneState &c,
                                             uint32_t &nback, uint64_t &my_lo, uint64_t &my_hi,
                                             uint32_t *my_kv = nullptr) {
  const uint32_t lane = lane_id();
  nback = L->nback;
  uint32_t klvl = 0;
  const JBack *b = nullptr;
  if (lane < nback && inb(a, SITE_BACK, (uint64_t)L->back_base + lane, a.n_backs)) {
    b = a.backs + L->back_base + lane;
    klvl = b->lvl & 31u;
  }
  const uint32_t kidx = __shfl_sync(FULL, c.idx, klvl);
  const uint32_t kv = __shfl_sync(FULL, c.f, klvl);  // the list's key vertex f(u_j)
  if (my_kv) *my_kv = kv;
  my_lo = my_hi = 0;
  if (b) table_range(a, b, kidx, my_lo, my_hi);
}

// level_ranges plus the shortest entry (lowest index on ties) and its range,
// identical in every lane.
__device__ __forceinline__ void level_lists(const JoinArgs &a, const JLevel *__restrict__ L, const LaneState &c,
                                            uint32_t &nback, uint64_t &my_lo, uint64_t &my_hi, uint32_t &src,
                                            uint64_t &s_lo, uint64_t &s_hi) {
  const uint32_t lane = lane_id();
  level_ranges(a, L, c, nback, my_lo, my_hi);
  uint64_t best = lane < nback ? my_hi - my_lo : ~0ull;
  uint32_t bl = lane;
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    const uint64_t ob = __shfl_xor_sync(FULL, best, d);
    const uint32_t ol = __shfl_xor_sync(FULL, bl, d);
    if (ob < best || (ob == best && ol < bl)) {
      best = ob;
      bl = ol;
    }
  }
  src = bl;
  s_lo = __shfl_sync(FULL, my_lo, src);
  s_hi = __shfl_sync(FULL, my_hi, src);
}

// Evaluates the chunk [cpos, min(cpos + 32, end)) of the source list: a lane's
// candidate survives if every other backward list contains it and no earlier
// same-label level holds it.  Returns the ballot; *w receives the lane's value.
// ---------------------------------------------------------------------------
// Arc tests through the neighbourhood hash.  A list T(u_j -> u_s)[f_j] is
// N(f_j) restricted to C(u_s), so a value already known to be in C(u_s) is
// in the list exactly when (f_j, value) is an arc.
// ---------------------------------------------------------------------------
struct VnhRow {
  uint64_t b, mask;  // first slot and size - 1 of the vertex's table (mask ~0: no neighbours)
  uint32_t shift;    // 64 - log2(size)
};

__device__ __forceinline__ VnhRow vnh_row(const JoinArgs &a, uint32_t u) {
  VnhRow r;
  r.b = __ldg(a.vnh_off + u);
  const uint64_t size = __ldg(a.vnh_off + u + 1) - r.b;
  r.mask = size ? size - 1 : ~0ull;
  r.shift = size ? 1 + __clzll(size) : 0;
  return r;
}

__device__ __forceinline__ bool vnh_has(const JoinArgs &a, const VnhRow &r, uint32_t v) {
  if (r.mask == ~0ull) return false;
  uint64_t pos = (v * VNH_MULT) >> r.shift;
  for (uint64_t k = 0; k <= r.mask; ++k) {
    const uint32_t x = __ldg(a.vnh_slots + r.b + pos);
    if (x == v) return true;
    if (x == VNH_EMPTY) return false;
    pos = (pos + 1) & r.mask;
  }
  return false;
}

// Arc tests of up to 8 keys (the bits of `want`) against one vertex's
// table; the probes of all keys are issued together.  Returns the keys found.
__device__ __forceinline__ uint32_t vnh_has8(const JoinArgs &a, const VnhRow &r, const uint32_t (&v)[8],
                                             uint32_t want) {
  if (r.mask == ~0ull) return 0;
  uint64_t pos[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) pos[k] = (v[k] * VNH_MULT) >> r.shift;
  uint32_t found = 0, open = want;
  for (uint64_t step = 0; open && step <= r.mask; ++step) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if ((open >> k) & 1u) {
        const uint32_t x = __ldg(a.vnh_slots + r.b + pos[k]);
        if (x == v[k]) {
          found |= 1u << k;
          open &= ~(1u << k);
        } else if (x == VNH_EMPTY) {
          open &= ~(1u << k);
        } else {
          pos[k] = (pos[k] + 1) & r.mask;
        }
      }
    }
  }
  return found;
}

// The source list and the probed lists all lie in C(u_L), so with the
// neighbourhood hash a probe of list T(u_j -> u_L)[f_j] is the arc test
// (f_j, w); without it, a binary search of the list.
__device__ __forceinline__ uint32_t eval_chunk(const JoinArgs &a, uint64_t cpos, uint64_t end, uint32_t nback,
                                               uint32_t src, uint64_t my_lo, uint64_t my_hi, uint32_t my_kv,
                                               uint32_t dup_mask, const LaneState &c, uint32_t *w_out, Stats &st) {
  const uint32_t lane = lane_id();
  const uint64_t e = cpos + lane;
  bool ok = e < end;
  uint32_t w = ok ? __ldg(a.values + e) : 0u;
  for (uint32_t i = 0; i < nback; ++i) {
    const uint64_t lo = __shfl_sync(FULL, my_lo, i), hi = __shfl_sync(FULL, my_hi, i);
    const uint32_t kv = __shfl_sync(FULL, my_kv, i);
    if (i == src) continue;
    if (ok) ok = a.vnh_off ? vnh_has(a, vnh_row(a, kv), w) : contains_u32(a.values, lo, hi, w);
  }
  for (uint32_t dm = dup_mask; dm; dm &= dm - 1) {
    const uint32_t j = __ffs(dm) - 1;
    const uint32_t fj = __shfl_sync(FULL, c.f, j);
    if (w == fj) ok = false;
  }
  if (lane == 0) {
    const uint64_t k = (end - cpos) < 32 ? (end - cpos) : 32;
    st.scanned += k;
    st.probes += (uint64_t)(nback - 1) * k;
  }
  *w_out = w;
  return __ballot_sync(FULL, ok);
}

__device__ __forceinline__ uint32_t index_of(const JoinArgs &a, const JLevel *__restrict__ L, uint32_t w) {
  const uint32_t kind = L->idx_kind;
  if (kind == IDX_NONE) return 0u;
  if (!inb(a, SITE_VERTEX, w, a.nv)) return 0xFFFFFFFFu;
  if (kind == IDX_RANK) return rank_lookup(L->rb, w);
  return ck_lookup(L->ck, w);
}

// ---------------------------------------------------------------------------
// Per-warp list cache in shared memory.  A suffix list keyed by an earlier
// level than the last enumerated one is the same for all 32 lanes of a chunk
// and usually for every chunk of the same prefix, so the warp copies the two
// longest of them (up to LIST_CACHE_CAP entries each) into shared memory and
// membership tests against them become shared-memory binary searches instead
// of chains of dependent L2 loads.  A slot is tagged by the list's absolute
// range in the values array, which identifies the list for the whole launch.
// ---------------------------------------------------------------------------
struct ListCache {
  uint32_t *buf;            // LIST_CACHE_SLOTS * LIST_CACHE_CAP entries
  unsigned long long *tag;  // {lo, hi} per slot
  unsigned long long *rng;  // {lo, hi} of suffix back entries b0 + i (lo ~0: not keyed by the prefix); rng[64] = b0
};

__device__ __forceinline__ int cache_slot(const ListCache &lc, uint64_t lo, uint64_t hi) {
  if (hi <= lo) return -1;
#pragma unroll
  for (int k = 0; k < (int)LIST_CACHE_SLOTS; ++k)
    if (lc.tag[2 * k] == lo && lc.tag[2 * k + 1] == hi) return k;
  return -1;
}

__device__ __forceinline__ bool smem_contains(const uint32_t *b, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (b[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < n && b[lo] == x;
}

// Membership of up to 8 keys (the bits of `want`) in the sorted shared-memory
// list b[0, n): the eight binary searches advance together.
__device__ __forceinline__ uint32_t smem_member8(const uint32_t *b, uint32_t n, const uint32_t (&v)[8],
                                                 uint32_t want) {
  uint32_t l[8], h[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    l[k] = 0;
    h[k] = ((want >> k) & 1u) ? n : 0;
  }
  for (uint32_t span = n; span; span >>= 1) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (l[k] < h[k]) {
        const uint32_t mid = (l[k] + h[k]) >> 1;
        if (b[mid] < v[k]) l[k] = mid + 1; else h[k] = mid;
      }
    }
  }
  uint32_t found = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (((want >> k) & 1u) && l[k] < n && b[l[k]] == v[k]) found |= 1u << k;
  return found;
}

// x in list [lo, hi): from the cache slot when there is one, else by binary
// search of the values array from *cur (lists are probed in ascending x, so
// the search start only moves forward).
__device__ __forceinline__ bool list_member(const JoinArgs &a, const ListCache &lc, int slot, uint64_t lo,
                                            uint64_t hi, uint64_t &cur, uint32_t x) {
  if (slot >= 0) return smem_contains(lc.buf + slot * LIST_CACHE_CAP, (uint32_t)(hi - lo), x);
  const uint64_t p = lower_bound_u32(a.values, cur, hi, x);
  cur = p;
  return p < hi && __ldg(a.values + p) == x;
}

// Membership of up to 8 ascending keys in the sorted list [lo, hi) of the
// values array: eight binary searches advance together, so every step issues
// eight independent loads instead of one.  Returns a bit per key found
// (bit k for key k, among the `n` valid keys); *cur moves to the lower bound
// of the last key, where the next block of larger keys starts.
__device__ __forceinline__ uint32_t list_member8(const JoinArgs &a, uint64_t &cur, uint64_t hi, const uint32_t (&v)[8],
                                                 uint32_t n) {
  const uint32_t *__restrict__ base = a.values + cur;
  const uint32_t len = (uint32_t)(hi - cur);
  uint32_t l[8], h[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    l[k] = 0;
    h[k] = (uint32_t)k < n ? len : 0;
  }
  for (uint32_t span = len; span; span >>= 1) {  // ceil(log2(len + 1)) rounds
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (l[k] < h[k]) {
        const uint32_t mid = (l[k] + h[k]) >> 1;
        if (__ldg(base + mid) < v[k]) l[k] = mid + 1; else h[k] = mid;
      }
    }
  }
  uint32_t found = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if ((uint32_t)k < n && l[k] < len && __ldg(base + l[k]) == v[k]) found |= 1u << k;
  if (n) cur += l[n - 1 < 8 ? n - 1 : 7];
  return found;
}

// Warp-collective: caches the longest suffix lists keyed by levels below L
// (the prefix is sf/sidx).  Lists already cached stay in their slots.
__device__ void cache_suffix_lists(const JoinArgs &a, const JQuery *__restrict__ Q, uint32_t L,
                                   const uint32_t *sidx, const ListCache &lc, bool copy = true) {
  const uint32_t lane = lane_id();
  const uint32_t n = Q->n, ne = Q->n_enum;
  if (ne >= n || n > QV) {
    lc.rng[2 * lane] = ~0ull;
    __syncwarp();
    return;
  }
  const uint32_t b0 = Q->lv[ne].back_base, b1 = Q->lv[n - 1].back_base + Q->lv[n - 1].nback;
  uint64_t my_lo = 0, my_hi = 0, my_len = 0;
  if (b1 > b0 && lane < b1 - b0 && inb(a, SITE_BACK, (uint64_t)b0 + lane, a.n_backs)) {
    const JBack *b = a.backs + b0 + lane;
    const uint32_t kl = b->lvl;
    if (kl < L) {
      table_range(a, b, sidx[kl], my_lo, my_hi);
      const uint64_t len = my_hi - my_lo;
      if (len >= 4 && len <= LIST_CACHE_CAP) my_len = len;
      lc.rng[2 * lane] = my_lo;
      lc.rng[2 * lane + 1] = my_hi;
    } else {
      lc.rng[2 * lane] = ~0ull;
    }
  } else {
    lc.rng[2 * lane] = ~0ull;
  }
  if (lane == 0) lc.rng[64] = b0;
  __syncwarp();  // every lane reads the range table
  if (!copy) return;
  uint64_t pick_lo[LIST_CACHE_SLOTS], pick_hi[LIST_CACHE_SLOTS];
#pragma unroll
  for (int k = 0; k < (int)LIST_CACHE_SLOTS; ++k) {
    uint64_t best = my_len;
    uint32_t bl = lane;
#pragma unroll
    for (int d = 16; d; d >>= 1) {
      const uint64_t ob = __shfl_xor_sync(FULL, best, d);
      const uint32_t ol = __shfl_xor_sync(FULL, bl, d);
      if (ob > best || (ob == best && ol < bl)) {
        best = ob;
        bl = ol;
      }
    }
    pick_lo[k] = __shfl_sync(FULL, my_lo, bl);
    pick_hi[k] = best ? __shfl_sync(FULL, my_hi, bl) : pick_lo[k];
    if (lane == bl) my_len = 0;  // the next round picks another list
  }
  // keep what is cached already; fill the other picks into the free slots
  uint32_t used = 0;
#pragma unroll
  for (int k = 0; k < (int)LIST_CACHE_SLOTS; ++k) {
    const int s = cache_slot(lc, pick_lo[k], pick_hi[k]);
    if (s >= 0) used |= 1u << s;
  }
#pragma unroll
  for (int k = 0; k < (int)LIST_CACHE_SLOTS; ++k) {
    if (pick_hi[k] <= pick_lo[k] || cache_slot(lc, pick_lo[k], pick_hi[k]) >= 0) continue;
    const uint32_t free_slots = ~used & ((1u << LIST_CACHE_SLOTS) - 1u);
    if (!free_slots) break;
    const uint32_t s = __ffs(free_slots) - 1;
    used |= 1u << s;
    uint32_t *dst = lc.buf + s * LIST_CACHE_CAP;
    const uint32_t len = (uint32_t)(pick_hi[k] - pick_lo[k]);
    for (uint32_t j = lane; j < len; j += 32) dst[j] = __ldg(a.values + pick_lo[k] + j);
    __syncwarp();
    if (lane == 0) {
      lc.tag[2 * s] = pick_lo[k];
      lc.tag[2 * s + 1] = pick_hi[k];
    }
    __syncwarp();
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Count mode, closed-form suffix.  The suffix levels form an independent set
// of the query graph, so once the prefix is matched each suffix level's
// candidates are fixed: A_i = intersection of its backward lists minus the
// prefix vertices of its label.  Levels of different labels have disjoint
// candidates; within a label group the number of injective assignments is
// sum over set partitions pi of the group of
//   prod_{B in pi} (-1)^{|B|-1} (|B|-1)! * |intersection_{i in B} A_i|
// (inclusion-exclusion over coincidences).  All arithmetic wraps mod 2^64,
// which is exact whenever the count itself fits in 64 bits.
//
// Every lane owns one candidate w of the last enumerated level L (position
// widx in C(u_L)); the earlier levels' vertices and positions come from the
// warp's shared copy (sf, sidx).  Lists are addressed by index through the
// members' backward entries, so no per-lane arrays are needed.
// ---------------------------------------------------------------------------
struct LaneCtx {
  const JQuery *Q;
  uint32_t L, w, widx;
  const uint32_t *sf, *sidx;
  ListCache lc;
  uint64_t deadline;  // device time cap (%globaltimer ns)
  // prefix level ownp (if < QV) is this lane's own, not the warp's shared prefix
  uint32_t ownp = 0xFFu, wp = 0, widxp = 0;
};

// Vertex and candidate position of prefix level j for this lane.
__device__ __forceinline__ uint32_t lvl_vertex(const LaneCtx &x, uint32_t j) {
  return j == x.L ? x.w : j == x.ownp ? x.wp : x.sf[j];
}
__device__ __forceinline__ uint32_t lvl_index(const LaneCtx &x, uint32_t j) {
  return j == x.L ? x.widx : j == x.ownp ? x.widxp : x.sidx[j];
}

// List li of the subset `members` of a suffix group: its range, its key
// vertex (f of the key level) and the level of the member it belongs to.
__device__ __forceinline__ void lane_list(const JoinArgs &a, const LaneCtx &x, uint32_t first, uint32_t members,
                                          uint32_t li, uint64_t &lo, uint64_t &hi, uint32_t &kv, uint32_t &mlvl) {
  lo = hi = 0;
  kv = 0;
  mlvl = first;
  for (uint32_t m = members; m; m &= m - 1) {
    mlvl = (first + __ffs(m) - 1) & 31u;
    const JLevel *M = &x.Q->lv[mlvl];
    const uint32_t nb = M->nback;
    if (li < nb) {
      if (!inb(a, SITE_BACK, (uint64_t)M->back_base + li, a.n_backs)) return;
      const JBack *b = a.backs + M->back_base + li;
      const uint32_t kl = b->lvl;
      if (!inb(a, SITE_KEYLVL, kl, (uint64_t)x.L + 1)) return;
      kv = lvl_vertex(x, kl);
      if (kl < x.L && kl != x.ownp) {  // keyed by the shared prefix: the warp's range table has it
        const uint32_t ti = M->back_base + li - (uint32_t)x.lc.rng[64];
        if (ti < 32 && x.lc.rng[2 * ti] != ~0ull) {
          lo = x.lc.rng[2 * ti];
          hi = x.lc.rng[2 * ti + 1];
          return;
        }
      }
      const uint32_t kidx = lvl_index(x, kl);
      table_range(a, b, kidx, lo, hi);
      return;
    }
    li -= nb;
  }
}

// v in list (range [lo, hi), key vertex kv, member level ml) when v is known
// to be in C(u of level vl): an arc test, plus a candidate test when the
// list belongs to another member.
__device__ __forceinline__ bool vnh_list_has(const JoinArgs &a, const JQuery *Q, uint32_t kv, uint32_t ml,
                                             uint32_t vl, uint32_t v) {
  if (!vnh_has(a, vnh_row(a, kv), v)) return false;
  return ml == vl || (v < a.nv && rank_member(Q->lv[ml].rb, v));
}


// Lists of one subset, at most three: ranges computed once, cached lists read
// from shared memory, the others probed through the neighbourhood hash (or
// searched from a moving start without it).
__device__ uint64_t lane_subset_count3(const JoinArgs &a, const LaneCtx &x, uint32_t first, uint32_t members,
                                       uint32_t nl, uint32_t dup_mask, Stats &st, bool &heavy) {
  uint64_t lo0 = 0, hi0 = 0, lo1 = 0, hi1 = 0, lo2 = 0, hi2 = 0;
  uint32_t kv0 = 0, kv1 = 0, kv2 = 0, ml0 = 0, ml1 = 0, ml2 = 0;
  lane_list(a, x, first, members, 0, lo0, hi0, kv0, ml0);
  if (nl > 1) lane_list(a, x, first, members, 1, lo1, hi1, kv1, ml1);
  if (nl > 2) lane_list(a, x, first, members, 2, lo2, hi2, kv2, ml2);
  // the shortest list (s) is scanned; the other two (a, b) are probed
  uint64_t slo = lo0, shi = hi0, alo = lo1, ahi = hi1, blo = lo2, bhi = hi2;
  uint32_t skv = kv0, sml = ml0, akv = kv1, aml = ml1, bkv = kv2, bml = ml2;
  if (nl > 1 && hi1 - lo1 < shi - slo) {
    slo = lo1; shi = hi1; skv = kv1; sml = ml1;
    alo = lo0; ahi = hi0; akv = kv0; aml = ml0;
  }
  if (nl > 2 && hi2 - lo2 < shi - slo) {
    blo = slo; bhi = shi; bkv = skv; bml = sml;
    slo = lo2; shi = hi2; skv = kv2; sml = ml2;
  }
  const uint64_t len = shi - slo;
  const int ss = cache_slot(x.lc, slo, shi);
  const bool hash = a.vnh_off != nullptr;
  // Lists with one range are one list (members that share a filter row and
  // key levels share their tables): the intersection is the list itself.
  if (nl == 1 || (alo == slo && ahi == shi && (nl < 3 || (blo == slo && bhi == shi)))) {
    uint64_t c = len, cur = slo;
    for (uint32_t dm = dup_mask; dm; dm &= dm - 1) {
      const uint32_t j = __ffs(dm) - 1;
      const uint32_t v = lvl_vertex(x, j);  // a prefix vertex: not known to be in C(u_s)
      cur = slo;
      const bool in = ss >= 0 || !hash ? list_member(a, x.lc, ss, slo, shi, cur, v)
                                       : vnh_list_has(a, x.Q, skv, sml, ~0u, v);
      if (in) --c;
    }
    st.probes += __popc(dup_mask);
    return c;
  }
  const int sa = cache_slot(x.lc, alo, ahi), sb = nl > 2 ? cache_slot(x.lc, blo, bhi) : 0;
  // A lane intersects at most lane_scan_max entries by itself (2x that with
  // the neighbourhood hash, 8x when the scanned and the probed lists are all
  // in shared memory); longer intersections are deferred to the whole warp
  // (warp_suffix_count).
  const bool all_shared = ss >= 0 && sa >= 0 && sb >= 0;
  const uint64_t lim = all_shared ? 8ull * a.lane_scan_max : hash ? 2ull * a.lane_scan_max : a.lane_scan_max;
  if (len > lim) {
    heavy = true;
    return 0;
  }
  VnhRow ra = {}, rb = {};
  if (hash && sa < 0) ra = vnh_row(a, akv);
  if (hash && nl > 2 && sb < 0) rb = vnh_row(a, bkv);
  const uint64_t *rba = x.Q->lv[aml & 31u].rb, *rbb = x.Q->lv[bml & 31u].rb;
  uint64_t c = 0, ca = alo, cb = blo;
  const uint32_t *sbuf = ss >= 0 ? x.lc.buf + ss * LIST_CACHE_CAP : nullptr;
  for (uint64_t e0 = 0; e0 < len; e0 += 8) {
    // eight entries of the scanned list per step; their loads, and their
    // probes of the other lists, overlap
    const uint32_t n = len - e0 < 8 ? (uint32_t)(len - e0) : 8u;
    uint32_t vv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      vv[k] = (uint32_t)k >= n ? 0xFFFFFFFFu : sbuf ? sbuf[e0 + k] : __ldg(a.values + slo + e0 + k);
    uint32_t okm = (1u << n) - 1u;
    for (uint32_t dm = dup_mask; dm; dm &= dm - 1) {
      const uint32_t j = __ffs(dm) - 1;
      const uint32_t d = lvl_vertex(x, j);
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (vv[k] == d) okm &= ~(1u << k);
    }
    if (okm) {
      if (sa >= 0) {
        okm &= smem_member8(x.lc.buf + sa * LIST_CACHE_CAP, (uint32_t)(ahi - alo), vv, okm);
      } else if (hash) {
        okm &= vnh_has8(a, ra, vv, okm);
        if (aml != sml) {
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (((okm >> k) & 1u) && !(vv[k] < a.nv && rank_member(rba, vv[k]))) okm &= ~(1u << k);
        }
      } else {
        okm &= list_member8(a, ca, ahi, vv, n);
      }
    }
    if (okm && nl > 2) {
      if (sb >= 0) {
        okm &= smem_member8(x.lc.buf + sb * LIST_CACHE_CAP, (uint32_t)(bhi - blo), vv, okm);
      } else if (hash) {
        okm &= vnh_has8(a, rb, vv, okm);
        if (bml != sml) {
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (((okm >> k) & 1u) && !(vv[k] < a.nv && rank_member(rbb, vv[k]))) okm &= ~(1u << k);
        }
      } else {
        okm &= list_member8(a, cb, bhi, vv, n);
      }
    }
    c += __popc(okm);
  }
  st.scanned += len;
  st.probes += len * (nl - 1);
  return c;
}

__device__ uint64_t lane_subset_count(const JoinArgs &a, const LaneCtx &x, uint32_t first, uint32_t members,
                                      uint32_t dup_mask, Stats &st, bool &heavy) {
  uint32_t nl = 0;
  for (uint32_t m = members; m; m &= m - 1) nl += x.Q->lv[(first + __ffs(m) - 1) & 31u].nback;
  if (nl <= 3) return lane_subset_count3(a, x, first, members, nl, dup_mask, st, heavy);
  uint32_t s = 0, s_ml = 0;
  uint64_t s_lo = 0, s_hi = 0;
  for (uint32_t i = 0; i < nl; ++i) {
    uint64_t lo, hi;
    uint32_t kv, ml;
    lane_list(a, x, first, members, i, lo, hi, kv, ml);
    if (i == 0 || hi - lo < s_hi - s_lo) {
      s = i;
      s_lo = lo;
      s_hi = hi;
      s_ml = ml;
    }
  }
  // A lane intersects at most a.lane_scan_max source entries by itself;
  // longer intersections are deferred to the whole warp (warp_suffix_count).
  if (s_hi - s_lo > a.lane_scan_max) {
    heavy = true;
    return 0;
  }
  uint64_t c = 0;
  for (uint64_t e = s_lo; e < s_hi; ++e) {
    const uint32_t v = __ldg(a.values + e);
    bool ok = true;
    for (uint32_t dm = dup_mask; dm && ok; dm &= dm - 1) {
      const uint32_t j = __ffs(dm) - 1;
      ok = v != lvl_vertex(x, j);
    }
    for (uint32_t i = 0; i < nl && ok; ++i) {
      if (i == s) continue;
      uint64_t lo, hi;
      uint32_t kv, ml;
      lane_list(a, x, first, members, i, lo, hi, kv, ml);
      const int slot = cache_slot(x.lc, lo, hi);
      uint64_t cur = lo;
      ok = slot >= 0 || !a.vnh_off ? list_member(a, x.lc, slot, lo, hi, cur, v)
                                   : vnh_list_has(a, x.Q, kv, ml, s_ml, v);
    }
    c += ok;
  }
  st.scanned += s_hi - s_lo;
  st.probes += (s_hi - s_lo) * (nl - 1);
  return c;
}

// ---------------------------------------------------------------------------
// Balanced lane-level counting.  The per-lane form above makes a chunk last as
// long as its longest intersection; here every intersection of the chunk
// (one per prefix match and subset with two or more lists) becomes a job in
// the warp's shared memory, the jobs' blocks of 8 scanned entries are dealt
// round-robin to all 32 lanes, and each lane then assembles its own prefix
// match's inclusion-exclusion from the job results.  Used when the
// neighbourhood hash exists and the query's suffix has at most
// FLAT_MAX_VALUES subset values of at most three lists each.
// ---------------------------------------------------------------------------
struct FJob {
  uint64_t s;     // scanned list: start in the values array, or offset in its cache slot
  uint64_t ra;    // probe a: cached list length, or hash row start | log2(size) << 58 (63: no neighbours)
  uint64_t rb;    // probe b (three-list subsets)
  uint32_t len;   // scanned entries
  uint32_t w;     // the prefix match's vertex at level L (a duplicate candidate)
  uint32_t dup;   // earlier same-label levels
  uint32_t meta;  // bit 0: three lists; bits 1-2 / 3-4 / 5-6: cache slot + 1 (0: none) of the
                  // scanned list and of probes a, b; bits 7-11 / 12-16 / 17-21: their member levels
};
static_assert(sizeof(FJob) == FLAT_JOB_BYTES, "job record size");

__device__ __forceinline__ uint64_t flat_probe_word(const JoinArgs &a, int slot, uint64_t lo, uint64_t hi,
                                                    uint32_t kv) {
  if (slot >= 0) return hi - lo;
  const uint64_t b = __ldg(a.vnh_off + kv), size = __ldg(a.vnh_off + kv + 1) - b;
  const uint64_t lg = size ? 63 - __clzll(size) : 63;
  return b | (lg << 58);
}

// Keys among `want` that are in the probed list (word from flat_probe_word,
// slot1 = cache slot + 1 or 0); keys come from a list of member level sml.
__device__ __forceinline__ uint32_t flat_probe8(const JoinArgs &a, const JQuery *Q, const ListCache &lc,
                                                uint32_t slot1, uint64_t word, uint32_t ml, uint32_t sml,
                                                const uint32_t (&vv)[8], uint32_t want) {
  if (!want) return 0;
  if (slot1) return smem_member8(lc.buf + (slot1 - 1) * LIST_CACHE_CAP, (uint32_t)word, vv, want);
  const uint64_t lg = word >> 58;
  if (lg == 63) return 0;
  VnhRow r;
  r.b = word & ((1ull << 58) - 1);
  r.mask = (1ull << lg) - 1;
  r.shift = 64 - (uint32_t)lg;
  uint32_t f = vnh_has8(a, r, vv, want);
  if (ml != sml) {
    const uint64_t *rbm = Q->lv[ml & 31u].rb;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (((f >> k) & 1u) && !(vv[k] < a.nv && rank_member(rbm, vv[k]))) f &= ~(1u << k);
  }
  return f;
}

__device__ bool queue_push(const JoinArgs &a, uint32_t q, uint32_t lvl, uint32_t src, uint64_t begin, uint64_t end,
                           uint64_t hs, const LaneState &c);

// Where the chunk came from, for handing part of it to idle warps.
struct FlatOrigin {
  uint32_t q, src;
  uint64_t pos, end;  // the chunk's positions [pos, end) in the source list
};

// v (any vertex) in a list: its cache slot, the neighbourhood hash with a
// candidate test, or a binary search.
__device__ __forceinline__ bool list_has_vertex(const JoinArgs &a, const LaneCtx &x, int slot, uint64_t lo,
                                                uint64_t hi, uint32_t kv, uint32_t ml, uint32_t v) {
  if (slot >= 0) return smem_contains(x.lc.buf + slot * LIST_CACHE_CAP, (uint32_t)(hi - lo), v);
  if (a.vnh_off) return vnh_list_has(a, x.Q, kv, ml, ~0u, v);
  uint64_t cur = lo;
  return list_member(a, x.lc, -1, lo, hi, cur, v);
}

// Counts the suffix completions of the chunk's prefix matches (lanes in m);
// *my_cnt receives this lane's.  While the chunk holds more than
// a.flat_donate_blocks blocks and other warps are idle, the positions of the
// upper half of its work go to the queue (the recipient evaluates them
// again) and their lanes count nothing here.  Returns false, having done
// nothing, when the chunk's jobs do not fit the job table.
__device__ __forceinline__ bool flat_lane_chunk(const JoinArgs &a, const LaneCtx &x, uint32_t m, char *fbase,
                                                const FlatOrigin &org, const LaneState &c, bool &pushed,
                                                Stats &st, uint64_t &my_cnt) {
  const uint32_t lane = lane_id();
  const JQuery *Q = x.Q;
  const uint32_t nscan = (Q->flat >> 8) & 0xFFu;
  const uint32_t nact = __popc(m);
  if (nact * nscan > FLAT_MAX_JOBS) return false;
  FJob *jobs = reinterpret_cast<FJob *>(fbase);
  uint32_t *res = reinterpret_cast<uint32_t *>(fbase + FLAT_MAX_JOBS * FLAT_JOB_BYTES);
  uint32_t *start = res + FLAT_MAX_JOBS;
  bool act = (m >> lane) & 1u;
  const uint32_t jbase = __popc(m & ((1u << lane) - 1u)) * nscan;
  const uint32_t ng = Q->n_groups < MAX_GROUPS ? Q->n_groups : MAX_GROUPS;
  uint64_t val[FLAT_MAX_VALUES] = {0, 0, 0, 0};  // one-list values, or the duplicate corrections of jobs
  uint32_t my_blocks = 0;
  // ---- stage 1: this lane's subsets: one-list values directly, the others as jobs
  if (act) {
    uint32_t k = 0, jn = 0;
    for (uint32_t g = 0; g < ng; ++g) {
      const uint32_t first = Q->grp_first[g], gs = Q->grp_size[g] < MAX_GROUP ? Q->grp_size[g] : MAX_GROUP;
      const uint32_t dup = Q->lv[first & 31u].dup_mask;
      for (uint32_t S = 1; S < (1u << gs) && k < FLAT_MAX_VALUES; ++S, ++k) {
        uint32_t nl = 0;
        for (uint32_t mm = S; mm; mm &= mm - 1) nl += Q->lv[(first + __ffs(mm) - 1) & 31u].nback;
        uint64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        uint32_t kv[3] = {0, 0, 0}, ml[3] = {0, 0, 0};
#pragma unroll
        for (uint32_t i = 0; i < 3; ++i)
          if (i < nl) lane_list(a, x, first, S, i, lo[i], hi[i], kv[i], ml[i]);
        uint32_t s = 0;
        uint64_t best = hi[0] - lo[0];
        if (nl > 1 && hi[1] - lo[1] < best) {
          s = 1;
          best = hi[1] - lo[1];
        }
        if (nl > 2 && hi[2] - lo[2] < best) s = 2;
        const uint64_t slo = s == 0 ? lo[0] : s == 1 ? lo[1] : lo[2];
        const uint64_t shi = s == 0 ? hi[0] : s == 1 ? hi[1] : hi[2];
        const uint32_t skv = s == 0 ? kv[0] : s == 1 ? kv[1] : kv[2];
        const uint32_t sml = s == 0 ? ml[0] : s == 1 ? ml[1] : ml[2];
        const int ss = cache_slot(x.lc, slo, shi);
        if (nl == 1) {
          uint64_t cnt = shi - slo, cur = slo;
          for (uint32_t dm = dup; dm; dm &= dm - 1) {
            const uint32_t j = __ffs(dm) - 1;
            const uint32_t v = lvl_vertex(x, j);
            cur = slo;
            const bool in = ss >= 0 ? list_member(a, x.lc, ss, slo, shi, cur, v)
                                    : vnh_list_has(a, Q, skv, sml, ~0u, v);
            if (in) --cnt;
          }
          val[k] = cnt;
          continue;
        }
        // the probed lists: the two (or one) other than s
        const uint32_t ia = s == 0 ? 1 : 0, ib = s == 2 ? 1 : 2;
        const uint64_t alo = ia == 0 ? lo[0] : lo[1], ahi = ia == 0 ? hi[0] : hi[1];
        const uint64_t blo = ib == 1 ? lo[1] : lo[2], bhi = ib == 1 ? hi[1] : hi[2];
        const uint32_t akv = ia == 0 ? kv[0] : kv[1], bkv = ib == 1 ? kv[1] : kv[2];
        const uint32_t aml = ia == 0 ? ml[0] : ml[1], bml = ib == 1 ? ml[1] : ml[2];
        const int sa = cache_slot(x.lc, alo, ahi), sb = nl > 2 ? cache_slot(x.lc, blo, bhi) : -1;
        // With a shared prefix the blocks skip the earlier same-label
        // vertices themselves; with a per-lane level the job counts the whole
        // intersection and those vertices (distinct) found in it are
        // subtracted afterwards.
        uint64_t corr = 0;
        for (uint32_t dm = x.ownp < QV ? dup : 0u; dm; dm &= dm - 1) {
          const uint32_t d = lvl_vertex(x, __ffs(dm) - 1);
          if (list_has_vertex(a, x, ss, slo, shi, skv, sml, d) && list_has_vertex(a, x, sa, alo, ahi, akv, aml, d) &&
              (nl < 3 || list_has_vertex(a, x, sb, blo, bhi, bkv, bml, d)))
            ++corr;
        }
        val[k] = corr;
        FJob jb;
        jb.s = ss >= 0 ? 0 : slo;
        jb.len = (uint32_t)(shi - slo);
        jb.ra = flat_probe_word(a, sa, alo, ahi, akv);
        jb.rb = nl > 2 ? flat_probe_word(a, sb, blo, bhi, bkv) : 0;
        jb.w = x.w;
        jb.dup = x.ownp < QV ? 0u : dup;
        jb.meta = (nl > 2 ? 1u : 0u) | ((uint32_t)(ss + 1) << 1) | ((uint32_t)(sa + 1) << 3) |
                  ((uint32_t)(sb + 1) << 5) | ((sml & 31u) << 7) | ((aml & 31u) << 12) | ((bml & 31u) << 17);
        jobs[jbase + jn] = jb;
        res[jbase + jn] = 0;
        my_blocks += (jb.len + 7) >> 3;
        st.scanned += jb.len;
        st.probes += (uint64_t)jb.len * (nl - 1);
        ++jn;
      }
    }
  }
  // ---- job starts (in blocks of 8 entries): lanes in order, jobs in order
  uint32_t incl = my_blocks;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL, incl, d);
    if (lane >= (uint32_t)d) incl += o;
  }
  uint32_t total = __shfl_sync(FULL, incl, 31);
  // hand the upper half of the work to idle warps while the chunk is large
  uint32_t keep = m;  // lanes whose prefix matches stay here
  uint64_t give_end = org.end;
  while (org.q != ~0u && total > a.flat_donate_blocks) {
    const int idle_now = __shfl_sync(FULL, lane == 0 ? (int)(ld_vol(&a.ctl->idle) > 0) : 0, 0);
    if (!idle_now) break;
    // first lane whose work starts at or after half of the remaining blocks
    const uint32_t cut = __ballot_sync(FULL, ((keep >> lane) & 1u) && incl - my_blocks >= total / 2);
    if (!cut) break;
    const uint32_t s0 = __ffs(cut) - 1;
    if (!queue_push(a, org.q, x.L, org.src, org.pos + s0, give_end, 0ull, c)) break;
    pushed = true;
    give_end = org.pos + s0;
    keep &= (1u << s0) - 1u;
    total = __shfl_sync(FULL, incl - my_blocks, s0);
  }
  act = act && ((keep >> lane) & 1u);
  if (act) {
    uint32_t b = incl - my_blocks;
    for (uint32_t i = 0; i < nscan; ++i) {
      start[jbase + i] = b;
      b += (jobs[jbase + i].len + 7) >> 3;
    }
  }
  const uint32_t njobs = __popc(keep) * nscan;
  if (lane == 0) start[njobs] = total;
  __syncwarp();
  // ---- stage 2: blocks dealt round-robin; partial counts summed per job
  uint32_t cur_j = 0, cur_c = 0;
  for (uint32_t base = 0; base < total; base += 32) {
    if (((base >> 5) & 15u) == 15u && stop_now(a, x.deadline)) break;
    const uint32_t bid = base + lane;
    if (bid < total) {
      uint32_t lo = cur_j, hi = njobs;  // last job whose start <= bid (jobs only move forward)
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (start[mid] <= bid) lo = mid; else hi = mid;
      }
      if (lo != cur_j && cur_c) {
        atomicAdd(res + cur_j, cur_c);
        cur_c = 0;
      }
      cur_j = lo;
      const FJob jb = jobs[lo];
      const uint32_t off = (bid - start[lo]) << 3;
      const uint32_t n = jb.len - off < 8 ? jb.len - off : 8u;
      const uint32_t ss1 = (jb.meta >> 1) & 3u, sa1 = (jb.meta >> 3) & 3u, sb1 = (jb.meta >> 5) & 3u;
      const uint32_t sml = (jb.meta >> 7) & 31u, aml = (jb.meta >> 12) & 31u, bml = (jb.meta >> 17) & 31u;
      uint32_t vv[8];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        vv[k] = (uint32_t)k >= n ? 0xFFFFFFFFu
                : ss1 ? x.lc.buf[(ss1 - 1) * LIST_CACHE_CAP + off + k]
                      : __ldg(a.values + jb.s + off + k);
      uint32_t okm = (1u << n) - 1u;
      for (uint32_t dm = jb.dup; dm; dm &= dm - 1) {  // shared prefix: jb.w is level L, the rest shared
        const uint32_t j = __ffs(dm) - 1;
        const uint32_t d = j == x.L ? jb.w : x.sf[j];
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (vv[k] == d) okm &= ~(1u << k);
      }
      okm &= flat_probe8(a, Q, x.lc, sa1, jb.ra, aml, sml, vv, okm);
      if (jb.meta & 1u) okm &= flat_probe8(a, Q, x.lc, sb1, jb.rb, bml, sml, vv, okm);
      cur_c += __popc(okm);
    }
  }
  if (cur_c) atomicAdd(res + cur_j, cur_c);
  __syncwarp();
  // ---- stage 3: this lane's inclusion-exclusion
  my_cnt = 0;
  if (act) {
    uint64_t total_c = 1;
    uint32_t k = 0, jn = 0;
    for (uint32_t g = 0; g < ng && k < FLAT_MAX_VALUES; ++g) {
      const uint32_t first = Q->grp_first[g], gs = Q->grp_size[g] < MAX_GROUP ? Q->grp_size[g] : MAX_GROUP;
      uint64_t sv[4] = {0, 0, 0, 0};
      for (uint32_t S = 1; S < (1u << gs) && k < FLAT_MAX_VALUES; ++S, ++k) {
        uint32_t nl = 0;
        for (uint32_t mm = S; mm; mm &= mm - 1) nl += Q->lv[(first + __ffs(mm) - 1) & 31u].nback;
        const uint64_t v = nl == 1 ? val[k] : (uint64_t)res[jbase + jn++] - val[k];
        if (S < 4) sv[S] = v;
      }
      if (gs == 1) {
        total_c *= sv[1];
        continue;
      }
      uint64_t G = 0;
      const uint32_t tb = Q->term_base[g], tc = Q->term_count[g];
      for (uint32_t t = 0; t < tc; ++t) {
        if (!inb(a, SITE_TERM, (uint64_t)tb + t, a.n_terms)) break;
        const uint64_t term = __ldg(a.terms + tb + t);
        uint64_t prod = (uint64_t)(int64_t)(int32_t)(uint32_t)(term >> 32);
        const uint32_t blocks = (uint32_t)term;
        for (uint32_t b = 0; b < MAX_GROUP; ++b) {
          const uint32_t mk = (blocks >> (4 * b)) & 15u;
          if (!mk) break;
          prod *= mk < 4 ? sv[mk] : 0ull;
        }
        G += prod;
      }
      total_c *= G;
    }
    my_cnt = total_c;
  }
  return true;
}

// Suffix completions of one lane's prefix match; sets `heavy` (and returns
// 0) when an intersection is too long for one lane.
__device__ uint64_t lane_suffix_count(const JoinArgs &a, const LaneCtx &x, Stats &st, bool &heavy) {
  const JQuery *Q = x.Q;
  uint64_t total = 1;
  const uint32_t ng = Q->n_groups < MAX_GROUPS ? Q->n_groups : MAX_GROUPS;
  for (uint32_t g = 0; g < ng && total; ++g) {
    const uint32_t first = Q->grp_first[g];
    const uint32_t gs = Q->grp_size[g] < MAX_GROUP ? Q->grp_size[g] : MAX_GROUP;
    const uint32_t dup_mask = Q->lv[first & 31u].dup_mask;
    if (gs == 1) {
      total *= lane_subset_count(a, x, first, 1u, dup_mask, st, heavy);
      if (heavy) return 0;
      continue;
    }
    uint64_t sv[1u << MAX_GROUP];
    for (uint32_t S = 0; S < (1u << MAX_GROUP); ++S) sv[S] = 0;
    for (uint32_t S = 1; S < (1u << gs); ++S) {
      sv[S] = lane_subset_count(a, x, first, S, dup_mask, st, heavy);
      if (heavy) return 0;
      if (sv[S] == 0 && __popc(S) == 1) return 0;
    }
    uint64_t G = 0;
    const uint32_t tb = Q->term_base[g], tc = Q->term_count[g];
    for (uint32_t t = 0; t < tc; ++t) {
      if (!inb(a, SITE_TERM, (uint64_t)tb + t, a.n_terms)) return 0;
      const uint64_t term = __ldg(a.terms + tb + t);
      uint64_t prod = (uint64_t)(int64_t)(int32_t)(uint32_t)(term >> 32);
      const uint32_t blocks = (uint32_t)term;
      for (uint32_t b = 0; b < MAX_GROUP; ++b) {
        const uint32_t mk = (blocks >> (4 * b)) & 15u;
        if (!mk) break;
        prod *= sv[mk];
      }
      G += prod;
    }
    total *= G;
  }
  return total;
}

// Warp-cooperative form for one deferred (heavy) prefix match: every lane
// receives the same context; lists are spread one per lane and the shortest
// is scanned 32 entries at a time.
__device__ uint64_t warp_subset_count(const JoinArgs &a, const LaneCtx &x, uint32_t first, uint32_t members,
                                      uint32_t dup_mask, Stats &st) {
  const uint32_t lane = lane_id();
  uint32_t nl = 0;
  for (uint32_t m = members; m; m &= m - 1) nl += x.Q->lv[(first + __ffs(m) - 1) & 31u].nback;
  nl = nl < 32 ? nl : 32;
  uint64_t my_lo = 0, my_hi = 0;
  uint32_t my_kv = 0, my_ml = 0;
  if (lane < nl) lane_list(a, x, first, members, lane, my_lo, my_hi, my_kv, my_ml);
  uint64_t best = lane < nl ? my_hi - my_lo : ~0ull;
  uint32_t bl = lane;
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    const uint64_t ob = __shfl_xor_sync(FULL, best, d);
    const uint32_t ol = __shfl_xor_sync(FULL, bl, d);
    if (ob < best || (ob == best && ol < bl)) {
      best = ob;
      bl = ol;
    }
  }
  const uint32_t src = bl;
  const uint64_t s_lo = __shfl_sync(FULL, my_lo, src), s_hi = __shfl_sync(FULL, my_hi, src);
  const uint32_t s_kv = __shfl_sync(FULL, my_kv, src), s_ml = __shfl_sync(FULL, my_ml, src);
  const bool hash = a.vnh_off != nullptr;
  if (nl == 1) {
    bool hit = false;
    uint64_t cur = s_lo;
    if ((dup_mask >> lane) & 1u) {
      const uint32_t v = lvl_vertex(x, lane);  // a prefix vertex: not known to be in C(u_s)
      const int slot = cache_slot(x.lc, s_lo, s_hi);
      hit = slot >= 0 || !hash ? list_member(a, x.lc, slot, s_lo, s_hi, cur, v)
                               : vnh_list_has(a, x.Q, s_kv, s_ml, ~0u, v);
    }
    return (s_hi - s_lo) - (uint64_t)__popc(__ballot_sync(FULL, hit));
  }
  // cached lists: the scanned one is read from, the probed ones searched in, shared memory
  const int my_slot = lane < nl ? cache_slot(x.lc, my_lo, my_hi) : -1;
  const int s_slot = __shfl_sync(FULL, my_slot, src);
  // Merge intersection: 32 entries of the shortest list per step (one per
  // lane) against coalesced 32-entry windows of every other list; list i's
  // read cursor lives in lane i.  A window that ends below the step's first
  // entry is skipped with one binary search (galloping for skewed lengths).
  uint64_t cur = my_lo;
  uint64_t cnt = 0;
  uint32_t step = 0;
  for (uint64_t cp = s_lo; cp < s_hi; cp += 32) {
    // merges look at the time cap and the error word first and every 16
    // steps; past the cap the partial count is dropped with the query (the
    // error word marks it incomplete wherever the count is retired)
    if ((step++ & 15u) == 0 && stop_now(a, x.deadline)) break;
    const uint64_t e = cp + lane;
    bool ok = e < s_hi;
    const uint32_t v = !ok ? 0xFFFFFFFFu
                           : s_slot >= 0 ? x.lc.buf[s_slot * LIST_CACHE_CAP + (uint32_t)(e - s_lo)]
                                         : __ldg(a.values + e);
    const uint32_t last = (uint32_t)((s_hi - cp) < 32 ? (s_hi - cp - 1) : 31);
    const uint32_t vmin = __shfl_sync(FULL, v, 0), vmax = __shfl_sync(FULL, v, last);
    for (uint32_t i = 0; i < nl; ++i) {
      if (i == src) continue;
      const int sl = __shfl_sync(FULL, my_slot, i);
      if (sl >= 0) {
        const uint32_t ln = (uint32_t)(__shfl_sync(FULL, my_hi, i) - __shfl_sync(FULL, my_lo, i));
        ok = ok && smem_contains(x.lc.buf + sl * LIST_CACHE_CAP, ln, v);
        continue;
      }
      if (hash) {  // v is in C(u of the scanned list's member)
        const uint32_t kv = __shfl_sync(FULL, my_kv, i), ml = __shfl_sync(FULL, my_ml, i);
        ok = ok && vnh_list_has(a, x.Q, kv, ml, s_ml, v);
        continue;
      }
      uint64_t bp = __shfl_sync(FULL, cur, i);
      const uint64_t be = __shfl_sync(FULL, my_hi, i);
      bool found = false;
      if (bp < be) {
        const uint64_t probe = bp + 31 < be ? bp + 31 : be - 1;
        if (__ldg(a.values + probe) < vmin) bp = lower_bound_u32(a.values, probe + 1, be, vmin);
      }
      while (bp < be) {
        const uint64_t j = bp + lane;
        const uint32_t b = j < be ? __ldg(a.values + j) : 0xFFFFFFFFu;
        const uint32_t bl = (uint32_t)((be - bp) < 32 ? (be - bp - 1) : 31);
        const uint32_t bmax = __shfl_sync(FULL, b, bl);
        // lane-register binary search of v among the window's 32 values
        uint32_t lo = 0, hi = bl + 1;
#pragma unroll
        for (int step = 0; step < 6; ++step) {
          const uint32_t mid = (lo + hi) >> 1;
          const uint32_t bm = __shfl_sync(FULL, b, mid & 31u);
          if (lo < hi) {
            if (bm < v) lo = mid + 1; else hi = mid;
          }
        }
        const uint32_t bf = __shfl_sync(FULL, b, lo & 31u);
        found |= lo <= bl && bf == v;
        if (bmax >= vmax) break;  // entries > vmax may serve the next step
        bp += 32;
      }
      ok = ok && found;
      if (lane == i) cur = bp;
    }
    for (uint32_t dm = dup_mask; dm && ok; dm &= dm - 1) {
      const uint32_t j = __ffs(dm) - 1;
      ok = v != lvl_vertex(x, j);
    }
    cnt += __popc(__ballot_sync(FULL, ok));
  }
  if (lane == 0) {
    st.scanned += s_hi - s_lo;
    st.probes += (s_hi - s_lo) * (nl - 1);
  }
  return cnt;
}

__device__ uint64_t warp_suffix_count(const JoinArgs &a, const LaneCtx &x, Stats &st) {
  const JQuery *Q = x.Q;
  uint64_t total = 1;
  const uint32_t ng = Q->n_groups < MAX_GROUPS ? Q->n_groups : MAX_GROUPS;
  for (uint32_t g = 0; g < ng && total; ++g) {
    const uint32_t first = Q->grp_first[g];
    const uint32_t gs = Q->grp_size[g] < MAX_GROUP ? Q->grp_size[g] : MAX_GROUP;
    const uint32_t dup_mask = Q->lv[first & 31u].dup_mask;
    uint64_t sv[1u << MAX_GROUP];
    for (uint32_t S = 0; S < (1u << MAX_GROUP); ++S) sv[S] = 0;
    bool empty = false;
    for (uint32_t S = 1; S < (1u << gs); ++S) {
      sv[S] = warp_subset_count(a, x, first, S, dup_mask, st);
      if (sv[S] == 0 && __popc(S) == 1) {
        empty = true;
        break;
      }
    }
    if (empty) return 0;
    if (gs == 1) {
      total *= sv[1];
      continue;
    }
    uint64_t G = 0;
    const uint32_t tb = Q->term_base[g], tc = Q->term_count[g];
    for (uint32_t t = 0; t < tc; ++t) {
      if (!inb(a, SITE_TERM, (uint64_t)tb + t, a.n_terms)) return 0;
      const uint64_t term = __ldg(a.terms + tb + t);
      uint64_t prod = (uint64_t)(int64_t)(int32_t)(uint32_t)(term >> 32);
      const uint32_t blocks = (uint32_t)term;
      for (uint32_t b = 0; b < MAX_GROUP; ++b) {
        const uint32_t mk = (blocks >> (4 * b)) & 15u;
        if (!mk) break;
        prod *= sv[mk];
      }
      G += prod;
    }
    total *= G;
  }
  return total;
}

// ---------------------------------------------------------------------------
// Donation queue: QUEUE_SUBQ bounded MPMC sub-queues of sequence-numbered
// cells.  A push reserves a position with an atomic add on one sub-queue's
// tail (a reservation cannot lose a race), writes the cell and publishes it;
// a pop scans the sub-queues with all 32 lanes and takes a published cell
// with a CAS on that sub-queue's head.  `pending` counts published tasks not
// yet taken.  Called by a whole warp; lane 0 does the atomics.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_global_id() {
  return blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
}

__device__ __forceinline__ JTask *queue_cell(const JoinArgs &a, uint32_t sq, unsigned long long pos) {
  return a.queue + sq * QUEUE_SUBQ_CAP + (pos & (QUEUE_SUBQ_CAP - 1));
}

__device__ bool queue_push(const JoinArgs &a, uint32_t q, uint32_t lvl, uint32_t src, uint64_t begin, uint64_t end,
                           uint64_t hs, const LaneState &c) {
  const uint32_t lane = lane_id();
  JControl *ctl = a.ctl;
  unsigned long long slot = 0;
  uint32_t sq = 0;
  int ok = 0;
  if (lane == 0) {
    const uint32_t q0 = warp_global_id() % QUEUE_SUBQ;
    for (uint32_t k = 0; k < 4; ++k) {
      sq = (q0 + 37u * k) % QUEUE_SUBQ;
      // head first: the tail read after it is never smaller
      const unsigned long long h = ld_vol(&a.qends[sq].head), t = ld_vol(&a.qends[sq].tail);
      if (t - h >= QUEUE_SUBQ_FILL) continue;
      // A reserved position is never given back.  Its cell is free once the
      // pop of the previous lap released it, which has happened unless more
      // than QUEUE_SUBQ_CAP - QUEUE_SUBQ_FILL warps passed the check together;
      // a wait that runs out stops the grid with an overflow error.
      slot = atomicAdd(&a.qends[sq].tail, 1ull);
      const JTask *cell = queue_cell(a, sq, slot);
      ok = 1;
      for (uint32_t spin = 0; ld_vol(&cell->seq) != slot; ++spin) {
        if (spin >= 4096) {
          set_error(&ctl->err, DERR_OVERFLOW);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
      break;
    }
  }
  ok = __shfl_sync(FULL, ok, 0);
  if (!ok) return false;
  slot = __shfl_sync(FULL, slot, 0);
  sq = __shfl_sync(FULL, sq, 0);
  JTask *cell = queue_cell(a, sq, slot);
  if (lane < lvl) {
    cell->f[lane] = c.f;
    cell->idx[lane] = c.idx;
  }
  if (lane == 0) {
    cell->q = q;
    cell->lvl = lvl;
    cell->src = src;
    cell->begin = begin;
    cell->end = end;
    cell->hs = hs;
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    *reinterpret_cast<volatile unsigned long long *>(&cell->seq) = slot + 1;
    atomicAdd(&ctl->pending, 1ull);  // after publishing, before this warp's busy release
  }
  return true;
}

struct PoppedTask {
  uint32_t q, lvl, src;
  uint64_t begin, end, hs;
};

// Takes one published task.  The caller raises `busy` and then lowers
// `pending`, so that a task is always counted by one of the two.
__device__ bool queue_pop(const JoinArgs &a, PoppedTask &t, LaneState &c) {
  const uint32_t lane = lane_id();
  JControl *ctl = a.ctl;
  const unsigned long long pend = __shfl_sync(FULL, lane == 0 ? ld_vol(&ctl->pending) : 0ull, 0);
  if (!pend) return false;
  // one bit per sub-queue that holds tasks, rotated to start at this warp's own
  const uint32_t q0 = warp_global_id() % QUEUE_SUBQ;
  uint32_t nonempty[QUEUE_SUBQ / 32];
#pragma unroll
  for (uint32_t r = 0; r < QUEUE_SUBQ / 32; ++r) {
    const uint32_t sq = (q0 + 32 * r + lane) % QUEUE_SUBQ;
    const unsigned long long h = ld_vol(&a.qends[sq].head), tl = ld_vol(&a.qends[sq].tail);
    nonempty[r] = __ballot_sync(FULL, h < tl);
  }
  unsigned long long slot = 0;
  uint32_t sq_got = 0;
  int ok = 0;
  if (lane == 0) {
    uint32_t attempts = 0;
    for (uint32_t r = 0; r < QUEUE_SUBQ / 32 && !ok && attempts < 8; ++r)
      for (uint32_t bits = nonempty[r]; bits && !ok && attempts < 8; bits &= bits - 1, ++attempts) {
        const uint32_t sq = (q0 + 32 * r + __ffs(bits) - 1) % QUEUE_SUBQ;
        unsigned long long pos = ld_vol(&a.qends[sq].head);
        for (int tries = 0; tries < 4; ++tries) {
          const unsigned long long seq = ld_vol(&queue_cell(a, sq, pos)->seq);
          const long long dif = (long long)seq - (long long)(pos + 1);
          if (dif == 0) {
            const unsigned long long prev = atomicCAS(&a.qends[sq].head, pos, pos + 1);
            if (prev == pos) {
              ok = 1;
              slot = pos;
              sq_got = sq;
              break;
            }
            pos = prev;  // another warp took it: try the position after
          } else if (dif < 0) {
            break;  // empty, or the task at the head is not published yet
          } else {
            pos = ld_vol(&a.qends[sq].head);
          }
        }
      }
  }
  ok = __shfl_sync(FULL, ok, 0);
  if (!ok) return false;
  slot = __shfl_sync(FULL, slot, 0);
  sq_got = __shfl_sync(FULL, sq_got, 0);
  __threadfence();
  JTask *cell = queue_cell(a, sq_got, slot);
  t.q = __ldcg(&cell->q);
  t.lvl = __ldcg(&cell->lvl);
  t.src = __ldcg(&cell->src);
  t.begin = __ldcg(reinterpret_cast<const unsigned long long *>(&cell->begin));
  t.end = __ldcg(reinterpret_cast<const unsigned long long *>(&cell->end));
  t.hs = __ldcg(reinterpret_cast<const unsigned long long *>(&cell->hs));
  if (lane < t.lvl && lane < QV) {
    c.f = __ldcg(&cell->f[lane]);
    c.idx = __ldcg(&cell->idx[lane]);
  }
  __syncwarp();
  __threadfence();
  if (lane == 0) *reinterpret_cast<volatile unsigned long long *>(&cell->seq) = slot + QUEUE_SUBQ_CAP;
  return true;
}

__device__ __forceinline__ uint32_t find_query(const uint64_t *__restrict__ rp, uint32_t nq, uint64_t r) {
  uint32_t lo = 0, hi = nq;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(rp + mid) <= r) lo = mid; else hi = mid;
  }
  return lo;
}

// Marks query q incomplete and, once, withdraws every unclaimed root so the
// grid drains quickly; the queries owning withdrawn roots are marked too.
__device__ void abandon(const JoinArgs &a, uint32_t q) {
  if (q < a.nquery) atomicOr(&a.out[q].pad[0], 1ull);
  const unsigned long long r0 = atomicExch(&a.ctl->root_next, (unsigned long long)a.n_roots);
  if (r0 < a.n_roots)
    for (uint32_t k = find_query(a.root_prefix, a.nquery, r0); k < a.nquery; ++k) atomicOr(&a.out[k].pad[0], 1ull);
}

template <uint32_t MODE>
__device__ __forceinline__ void emit_last(const JoinArgs &a, const JQuery *__restrict__ Q, uint32_t lvl, uint32_t m,
                                          uint32_t w, const LaneState &c, uint64_t &lane_cnt, uint64_t &lane_hash) {
  const uint32_t lane = lane_id();
  const bool ok = (m >> lane) & 1u;
  const uint64_t hsp = __shfl_sync(FULL, c.hs, lvl - 1);
  if (ok) {
    lane_cnt += 1;
    lane_hash += mix64(hsp + emb_term(Q->lv[lvl].u, w));
  }
  if (MODE == MODE_ENUM) {
    unsigned long long base = 0;
    if (lane == 0 && m) base = atomicAdd(&a.ctl->emb_next, (unsigned long long)__popc(m));
    base = __shfl_sync(FULL, base, 0);
    const uint64_t slot = base + __popc(m & ((1u << lane) - 1u));
    const bool wr = ok && slot < a.emb_cap;
    const uint32_t n = Q->n;
    for (uint32_t j = 0; j < lvl; ++j) {
      const uint32_t fj = __shfl_sync(FULL, c.f, j);
      if (wr) a.emb[slot * n + Q->lv[j].u] = fj;
    }
    if (wr) a.emb[slot * n + Q->lv[lvl].u] = w;
  }
}

template <uint32_t MODE>
__global__ void __launch_bounds__(256, 2) join_kernel(JoinArgs a) {
  const uint32_t lane = lane_id();
  JControl *ctl = a.ctl;
  const uint64_t deadline = ctl->deadline_ns;
  __shared__ uint32_t s_pref[JOIN_WARPS_PER_BLOCK][2][QV];  // per warp: f and idx of the enumerated prefix
  __shared__ unsigned long long s_ctag[JOIN_WARPS_PER_BLOCK][2 * LIST_CACHE_SLOTS];
  extern __shared__ uint32_t s_lcache[];  // JOIN_DYN_SMEM bytes: per warp LIST_CACHE_SLOTS lists
  uint32_t *sf = s_pref[threadIdx.x >> 5][0], *sidx = s_pref[threadIdx.x >> 5][1];
  ListCache lc;
  // per warp: the list cache, then the balanced-counting job table
  lc.buf = s_lcache + (threadIdx.x >> 5) * (JOIN_WARP_SMEM / 4);
  char *fbuf = reinterpret_cast<char *>(lc.buf + LIST_CACHE_SLOTS * LIST_CACHE_CAP);
  lc.rng = reinterpret_cast<unsigned long long *>(fbuf + FLAT_WARP_BYTES);
  lc.rng[2 * lane] = ~0ull;
  if (lane == 0) lc.rng[64] = 0;
  lc.tag = s_ctag[threadIdx.x >> 5];
  if (lane < 2 * LIST_CACHE_SLOTS) lc.tag[lane] = 0ull;  // empty: no list has lo == hi == 0 and hi > lo
  __syncwarp();
  LaneState c;
  c.f = 0; c.idx = 0; c.hs = 0; c.pos = 0; c.end = 0; c.cbase = 0; c.mask = 0; c.src = 0;
  Stats st;
  bool idle_registered = false;
  // Root batch held by this warp ([rb_cur, rb_end) of the ordinary pool); the
  // warp counts as busy from the batch grab until its last root retires.
  uint64_t rb_cur = 0, rb_end = 0;
  const uint64_t total_warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  bool pushed = false;  // donated work since the last busy decrement
  // The prefix changes only with a new task or a descent: the suffix lists
  // keyed by it are looked up once per prefix (epoch), not once per chunk.
  uint32_t epoch = 0, filled_epoch = 0xFFFFFFFFu;

  // ---------------------------------------------------------------- lane-parallel roots
  // Queries whose only enumerated level is the root: one root per lane.
  if (a.lp_roots) {
    uint32_t it = 0;
    for (;;) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&ctl->lp_next, 32ull);
      base = __shfl_sync(FULL, base, 0);
      if (base >= a.lp_roots) break;
      if ((++it & 15u) == 0) {
        int stop = 0;
        if (lane == 0) {
          if (ld_vol(&ctl->err) != DERR_NONE) stop = 1;
          else if (globaltimer_ns() > deadline) {
            set_error(&ctl->err, DERR_TIMEOUT);
            stop = 1;
          }
          if (stop) {
            // this block and every unclaimed root of the pool are abandoned
            const unsigned long long r0 = atomicExch(&ctl->lp_next, (unsigned long long)a.lp_roots);
            const unsigned long long from = base < r0 ? base : r0;
            for (uint32_t k = find_query(a.lp_prefix, a.lp_nq, from); k < a.lp_nq; ++k)
              atomicOr(&a.out[a.lp_query[k]].pad[0], 1ull);
          }
        }
        if (__shfl_sync(FULL, stop, 0)) break;
      }
      const uint64_t r = base + lane;
      bool heavy = false;
      uint32_t hq = 0, hw = 0, hidx = 0;
      if (r < a.lp_roots) {
        const uint32_t k = find_query(a.lp_prefix, a.lp_nq, r);
        const uint32_t q = a.lp_query[k];
        if (inb(a, SITE_QUERY, q, a.nquery)) {
          const JQuery *Q = a.queries + q;
          const uint64_t rl = r - __ldg(a.lp_prefix + k);
          if (inb(a, SITE_ROOT, rl, Q->n_root)) {
            const uint32_t w0 = __ldg(Q->root_cand + rl);
            uint64_t cnt = 0, h = 0;
            if (Q->n == 1) {
              cnt = 1;
              if (MODE != MODE_COUNT) h = mix64(emb_term(Q->root_u, w0));
              if (MODE == MODE_ENUM) {
                const unsigned long long s = atomicAdd(&ctl->emb_next, 1ull);
                if (s < a.emb_cap) a.emb[s] = w0;
              }
            } else {
              LaneCtx x;
              x.Q = Q;
              x.L = 0;
              x.w = w0;
              x.widx = (uint32_t)rl;
              x.sf = sf;
              x.sidx = sidx;
              x.lc = lc;
              x.deadline = deadline;
              cnt = lane_suffix_count(a, x, st, heavy);
              hq = q;
              hw = w0;
              hidx = (uint32_t)rl;
            }
            if (cnt) atomicAdd(&a.out[q].count, (unsigned long long)cnt);
            if (h) atomicAdd(&a.out[q].hash, (unsigned long long)h);
          }
        }
      }
      // roots whose intersections are long: the whole warp, one at a time
      for (uint32_t hm = __ballot_sync(FULL, heavy); hm; hm &= hm - 1) {
        const uint32_t hl = __ffs(hm) - 1;
        const uint32_t qh = __shfl_sync(FULL, hq, hl);
        LaneCtx x;
        x.Q = a.queries + qh;
        x.L = 0;
        x.w = __shfl_sync(FULL, hw, hl);
        x.widx = __shfl_sync(FULL, hidx, hl);
        x.sf = sf;
        x.sidx = sidx;
        x.lc = lc;
        x.deadline = deadline;
        const uint64_t k = warp_suffix_count(a, x, st);
        if (lane == 0 && k) atomicAdd(&a.out[qh].count, (unsigned long long)k);
      }
      if (lane == 0) st.nodes += (a.lp_roots - base) < 32 ? (a.lp_roots - base) : 32;
      if (err_set(a)) {
        // a count of this chunk may have been cut short: its queries and every
        // unclaimed root of the pool are incomplete
        if (lane == 0) {
          const unsigned long long r0 = atomicExch(&ctl->lp_next, (unsigned long long)a.lp_roots);
          const unsigned long long from = base < r0 ? base : r0;
          for (uint32_t k = find_query(a.lp_prefix, a.lp_nq, from); k < a.lp_nq; ++k)
            atomicOr(&a.out[a.lp_query[k]].pad[0], 1ull);
        }
        break;
      }
    }
  }

  // ---------------------------------------------------------------- (root, first level) pairs
  // Queries whose enumerated prefix is a root and one neighbour level: their
  // prefix matches are the entries of the root's edge table, taken 32 at a
  // time (each query's range padded to whole chunks), one match per lane with
  // its own root, so short neighbour lists still fill the warp.
  if (a.lp2_nq) {
    const uint64_t total = a.lp2_prefix[a.lp2_nq];
    uint32_t it = 0;
    for (;;) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&ctl->lp2_next, 32ull);
      base = __shfl_sync(FULL, base, 0);
      if (base >= total) break;
      if ((++it & 15u) == 0) {
        int stop = 0;
        if (lane == 0) {
          if (ld_vol(&ctl->err) != DERR_NONE) stop = 1;
          else if (globaltimer_ns() > deadline) {
            set_error(&ctl->err, DERR_TIMEOUT);
            stop = 1;
          }
          if (stop) {
            // this chunk and every unclaimed one are abandoned
            const unsigned long long r0 = atomicExch(&ctl->lp2_next, (unsigned long long)total);
            const unsigned long long from = base < r0 ? base : r0;
            for (uint32_t k = find_query(a.lp2_prefix, a.lp2_nq, from); k < a.lp2_nq; ++k)
              atomicOr(&a.out[a.lp2_query[k]].pad[0], 1ull);
          }
        }
        if (__shfl_sync(FULL, stop, 0)) break;
      }
      const uint32_t qk = find_query(a.lp2_prefix, a.lp2_nq, base);
      const uint32_t q = a.lp2_query[qk];
      if (!inb(a, SITE_QUERY, q, a.nquery)) break;
      const JQuery *Q = a.queries + q;
      const JLevel *L1 = &Q->lv[1];
      if (!inb(a, SITE_BACK, L1->back_base, a.n_backs)) break;
      const JBack *b = a.backs + L1->back_base;
      const uint64_t e0 = __ldg(b->off), e1 = __ldg(b->off + b->nkeys);
      const uint64_t p = e0 + (base - __ldg(a.lp2_prefix + qk)) + lane;
      bool valid = p < e1 && inb(a, SITE_RANGE, p, a.n_values);
      uint32_t f0 = 0, k0 = 0, f1 = 0, i1 = 0;
      if (valid) {
        k0 = __ldg(a.vkey + p);
        valid = inb(a, SITE_ROOT, k0, Q->n_root);
        if (valid) {
          f0 = __ldg(Q->root_cand + k0);
          f1 = __ldg(a.values + p);
          i1 = index_of(a, L1, f1);
        }
      }
      const uint32_t m = __ballot_sync(FULL, valid);
      LaneCtx x;
      x.Q = Q;
      x.L = 1;
      x.w = f1;
      x.widx = i1;
      x.sf = sf;
      x.sidx = sidx;
      x.lc = lc;
      x.deadline = deadline;
      x.ownp = 0;
      x.wp = f0;
      x.widxp = k0;
      FlatOrigin org;
      org.q = ~0u;  // lanes hold different roots: no task can carry the chunk
      org.src = 0;
      org.pos = org.end = 0;
      uint64_t cnt = 0;
      if (!flat_lane_chunk(a, x, m, fbuf, org, c, pushed, st, cnt)) {
        bool heavy = false;
        cnt = valid ? lane_suffix_count(a, x, st, heavy) : 0;
        for (uint32_t hm = __ballot_sync(FULL, heavy); hm; hm &= hm - 1) {
          const uint32_t hl = __ffs(hm) - 1;
          LaneCtx y = x;
          y.w = __shfl_sync(FULL, f1, hl);
          y.widx = __shfl_sync(FULL, i1, hl);
          y.wp = __shfl_sync(FULL, f0, hl);
          y.widxp = __shfl_sync(FULL, k0, hl);
          const uint64_t k = warp_suffix_count(a, y, st);
          if (lane == hl) cnt += k;
        }
      }
#pragma unroll
      for (int d = 16; d; d >>= 1) cnt += __shfl_xor_sync(FULL, cnt, d);
      if (lane == 0) {
        if (cnt) atomicAdd(&a.out[q].count, (unsigned long long)cnt);
        st.nodes += __popc(m);
      }
      if (err_set(a)) {
        // this chunk's count may have been cut short: its query and every
        // unclaimed chunk's are incomplete
        if (lane == 0) {
          const unsigned long long r0 = atomicExch(&ctl->lp2_next, (unsigned long long)total);
          const unsigned long long from = base < r0 ? base : r0;
          for (uint32_t k = find_query(a.lp2_prefix, a.lp2_nq, from); k < a.lp2_nq; ++k)
            atomicOr(&a.out[a.lp2_query[k]].pad[0], 1ull);
        }
        break;
      }
    }
  }

  for (;;) {
    // ------------------------------------------------------------ acquire
    uint32_t q = 0, base_lvl = 0, lvl = 0;
    bool have = false, from_root = false;
    uint64_t r = 0;
    if (!idle_registered) {
      if (rb_cur >= rb_end) {
        // guided batches: a quarter of the remaining roots per warp, 1..16
        unsigned long long rr = 0, cnt = 1;
        if (lane == 0) {
          const unsigned long long seen = ld_vol(&ctl->root_next);
          const unsigned long long left = seen < a.n_roots ? a.n_roots - seen : 0;
          cnt = left / (4ull * total_warps);
          cnt = cnt < 1 ? 1 : (cnt > a.root_batch_max ? a.root_batch_max : cnt);
          atomicAdd(&ctl->busy, 1u);
          __threadfence();
          rr = atomicAdd(&ctl->root_next, cnt);
          if (rr >= a.n_roots) atomicSub(&ctl->busy, 1u);
        }
        rb_cur = __shfl_sync(FULL, rr, 0);
        cnt = __shfl_sync(FULL, cnt, 0);
        rb_end = rb_cur < a.n_roots ? (rb_cur + cnt < a.n_roots ? rb_cur + cnt : a.n_roots) : rb_cur;
      }
      r = rb_cur < rb_end ? rb_cur++ : a.n_roots;
      // warp-uniform: lane 0 reads the error word for the whole warp
      const int err_set = __shfl_sync(FULL, lane == 0 ? (int)(ld_vol(&ctl->err) != DERR_NONE) : 0, 0);
      if (r < a.n_roots && err_set) {
        // past the deadline: this root and the rest of the batch are not processed
        if (lane == 0) {
          const uint32_t q0 = find_query(a.root_prefix, a.nquery, r);
          const uint32_t q1 = find_query(a.root_prefix, a.nquery, rb_end - 1);
          for (uint32_t k = q0; k <= q1; ++k) atomicOr(&a.out[k].pad[0], 1ull);
          abandon(a, q0);
          if (pushed) __threadfence();
          atomicSub(&ctl->busy, 1u);
        }
        pushed = false;
        rb_cur = rb_end;
        r = a.n_roots;
      }
      if (r < a.n_roots) {
        have = true;
        from_root = true;
      } else {
        idle_registered = true;
        if (lane == 0) atomicAdd(&ctl->idle, 1u);
      }
    }
    if (!have) {
      uint32_t backoff = 64;
      for (;;) {
        // Only a warp that holds work counts as busy: pollers must not keep
        // `busy` above zero, or no poller could ever observe quiescence.
        PoppedTask t;
        if (queue_pop(a, t, c)) {
          if (lane == 0) {
            atomicAdd(&ctl->busy, 1u);
            atomicSub(&ctl->idle, 1u);
            __threadfence();  // busy is raised before pending drops
            atomicAdd(&ctl->pending, ~0ull);
          }
          idle_registered = false;  // a finished donated task re-registers as idle below
          q = t.q;
          lvl = base_lvl = t.lvl;
          have = true;
          if (!inb(a, SITE_QUERY, q, a.nquery) || !inb(a, SITE_LEVEL, lvl, a.queries[q].n) || lvl == 0 ||
              !inb(a, SITE_RANGE, t.end, a.n_values + 1) || !inb(a, SITE_RANGE, t.begin, t.end + 1)) {
            lvl = 0;  // unusable task: nothing to run (a failed check stops the grid)
            base_lvl = 1;
            q = 0;
          } else {
            if (lane == lvl - 1) c.hs = t.hs;
            if (lane == lvl) {
              c.src = t.src;
              c.pos = t.begin;
              c.end = t.end;
              c.mask = 0;
            }
          }
          break;
        }
        int leave = 0, pending = 0;
        if (lane == 0) {
          const unsigned int b = ld_vol(&ctl->busy);
          __threadfence();  // `pending` is read after `busy`
          const bool empty = ld_vol(&ctl->pending) == 0;
          pending = !empty;
          if (b == 0 && empty) leave = 1;
          if (ld_vol(&ctl->err) != DERR_NONE) leave = 1;
          if (globaltimer_ns() > deadline) {
            set_error(&ctl->err, DERR_TIMEOUT);
            leave = 1;
          }
        }
        if (__shfl_sync(FULL, leave, 0)) break;
        // tasks are published but other warps won them: retry soon
        if (__shfl_sync(FULL, pending, 0)) backoff = 256;
        __nanosleep(backoff);
        backoff = backoff < 16384 ? backoff * 2 : 16384;
      }
      if (!have) {
        if (lane == 0) atomicSub(&ctl->idle, 1u);
        break;
      }
    }

    // ------------------------------------------------------------ set up
    ++epoch;
    uint64_t lane_cnt = 0, lane_hash = 0;
    const JQuery *__restrict__ Q = a.queries + q;
    if (from_root) {
      q = find_query(a.root_prefix, a.nquery, r);
      Q = a.queries + q;
      const uint64_t rl = r - Q->root_base;
      lvl = 0;
      base_lvl = 1;
      if (inb(a, SITE_ROOT, rl, Q->n_root)) {
        const uint32_t w0 = __ldg(Q->root_cand + rl);
        const uint64_t h0 = MODE == MODE_COUNT ? 0ull : emb_term(Q->root_u, w0);
        if (lane == 0) {
          c.f = w0;
          c.idx = (uint32_t)rl;
          c.hs = h0;
        }
        st.nodes += lane == 0;
        if (Q->n >= 2) {
          uint32_t nb, src;
          uint64_t lo, hi, s_lo, s_hi;
          level_lists(a, &Q->lv[1], c, nb, lo, hi, src, s_lo, s_hi);
          if (lane == 1) {
            c.src = src;
            c.pos = s_lo;
            c.end = s_hi;
            c.mask = 0;
          }
          lvl = base_lvl = 1;
        }
      }
    }

    // ------------------------------------------------------------ DFS
    const uint32_t n = Q->n;
    uint32_t iter = 0;
    bool abort = false;
    while (lvl >= base_lvl && lvl != 0) {
      const JLevel *__restrict__ L = &Q->lv[lvl & 31u];
      const uint32_t mask = __shfl_sync(FULL, c.mask, lvl);
      if (mask == 0) {
        const uint64_t pos = __shfl_sync(FULL, c.pos, lvl), end = __shfl_sync(FULL, c.end, lvl);
        if (pos >= end) {
          --lvl;
          continue;
        }
        if ((++iter & 3u) == 0) {
          int stop = 0;
          if (lane == 0) {
            if (ld_vol(&ctl->err) != DERR_NONE) stop = 1;
            else if (globaltimer_ns() > deadline) {
              set_error(&ctl->err, DERR_TIMEOUT);
              stop = 1;
            }
          }
          if (__shfl_sync(FULL, stop, 0)) {
            abort = true;
            break;
          }
        }
        uint32_t nb, kv;
        uint64_t lo, hi;
        level_ranges(a, L, c, nb, lo, hi, &kv);
        const uint32_t src = __shfl_sync(FULL, c.src, lvl);
        uint32_t w;
        const uint32_t m = eval_chunk(a, pos, end, nb, src, lo, hi, kv, L->dup_mask, c, &w, st);
        if (MODE != MODE_COUNT && lvl == n - 1) {
          emit_last<MODE>(a, Q, lvl, m, w, c, lane_cnt, lane_hash);
          if (lane == lvl) c.pos = pos + 32;
          continue;
        }
        uint64_t new_end = end;
        // Donate the unread half of this level when another warp is idle and
        // the half is at least the tuned minimum (separate minimums for the
        // lane-parallel level, cheap per candidate, and for levels whose
        // candidates open subtrees).
        const bool lane_level = MODE == MODE_COUNT && lvl + 1 >= Q->n_enum;
        const uint64_t min_half = lane_level ? a.donate_min_lane : a.donate_min_desc;
        if (lvl <= a.donate_max_level && end >= pos + 32 + 2 * min_half) {
          // warp-uniform: lane 0 reads the idle count for the whole warp
          const int idle_now = __shfl_sync(FULL, lane == 0 ? (int)(ld_vol(&ctl->idle) > 0) : 0, 0);
          if (idle_now) {
            const uint64_t rem = pos + 32;
            const uint64_t mid = rem + ((((end - rem) >> 1) + 31) & ~31ull);
            if (mid < end) {
              const uint64_t hsp = MODE == MODE_COUNT ? 0ull : __shfl_sync(FULL, c.hs, lvl - 1);
              if (queue_push(a, q, lvl, src, mid, end, hsp, c)) {
                new_end = mid;
                pushed = true;
              }
            }
          }
        }
        if (lane_level) {
          // last enumerated level: each lane counts its own candidate's
          // suffix completions (32 prefix matches in flight per warp)
          if (lane < lvl) {
            sf[lane] = c.f;
            sidx[lane] = c.idx;
          }
          __syncwarp();
          if (lvl > 0 && filled_epoch != epoch) {
            // copying lists into shared memory pays only when the prefix has
            // more than this chunk at its last level
            cache_suffix_lists(a, Q, lvl, sidx, lc, end > pos + 32);
            filled_epoch = epoch;
          }
          bool flat_done = false;
          if (Q->flat && a.vnh_off) {
            LaneCtx x;
            x.Q = Q;
            x.L = lvl;
            x.w = w;
            x.widx = ((m >> lane) & 1u) ? index_of(a, L, w) : 0u;
            x.sf = sf;
            x.sidx = sidx;
            x.lc = lc;
            x.deadline = deadline;
            FlatOrigin org;
            org.q = q;
            org.src = src;
            org.pos = pos;
            org.end = end < pos + 32 ? end : pos + 32;
            uint64_t fc = 0;
            flat_done = flat_lane_chunk(a, x, m, fbuf, org, c, pushed, st, fc);
            if (flat_done) lane_cnt += fc;
          }
          bool heavy = false;
          uint32_t widx = 0;
          uint64_t my_cnt = 0;
          if (!flat_done && ((m >> lane) & 1u)) {
            LaneCtx x;
            x.Q = Q;
            x.L = lvl;
            x.w = w;
            x.widx = widx = index_of(a, L, w);
            x.sf = sf;
            x.sidx = sidx;
            x.lc = lc;
            x.deadline = deadline;
            my_cnt = lane_suffix_count(a, x, st, heavy);
          }
          // Candidates whose intersections are long are counted by the whole
          // warp, one at a time.  When another warp is idle, the chunk's
          // positions from the first of the upper half of them on go to the
          // queue as one task; the recipient evaluates them all again, so
          // their counts here are dropped.
          uint32_t hm = __ballot_sync(FULL, heavy);
          uint64_t give_end = end < pos + 32 ? end : pos + 32;  // chunk positions not yet given away
          while (hm & (hm - 1)) {
            const int idle_now = __shfl_sync(FULL, lane == 0 ? (int)(ld_vol(&ctl->idle) > 0) : 0, 0);
            if (!idle_now) break;
            uint32_t upper = hm;
            for (uint32_t k = __popc(hm) >> 1; k; --k) upper &= upper - 1;
            const uint32_t s0 = __ffs(upper) - 1;
            if (!queue_push(a, q, lvl, src, pos + s0, give_end, 0ull, c)) break;
            hm &= (1u << s0) - 1u;
            if (lane >= s0 && pos + lane < give_end) my_cnt = 0;
            give_end = pos + s0;
            pushed = true;
          }
          lane_cnt += my_cnt;
          for (; hm; hm &= hm - 1) {
            const uint32_t hl = __ffs(hm) - 1;
            LaneCtx x;
            x.Q = Q;
            x.L = lvl;
            x.w = __shfl_sync(FULL, w, hl);
            x.widx = __shfl_sync(FULL, widx, hl);
            x.sf = sf;
            x.sidx = sidx;
            x.lc = lc;
            x.deadline = deadline;
            const uint64_t k = warp_suffix_count(a, x, st);
            if (lane == 0) lane_cnt += k;
          }
          __syncwarp();
          if (lane == 0) st.nodes += __popc(m);
          if (lane == lvl) {
            c.pos = pos + 32;
            c.end = new_end;
          }
        } else if (lane == lvl) {
          c.cbase = pos;
          c.pos = pos + 32;
          c.mask = m;
          c.end = new_end;
        }
        continue;
      }
      // descend into the lowest remaining candidate
      const uint32_t b = __ffs(mask) - 1;
      const uint64_t cb = __shfl_sync(FULL, c.cbase, lvl);
      uint32_t rest = mask & (mask - 1);
      // Each survivor of the chunk opens a subtree of its own: when another
      // warp is idle, the upper half of the remaining survivors goes to the
      // queue as the source range that holds them (the recipient evaluates
      // that range again and finds the same survivors).
      if (rest && lvl <= a.donate_max_level) {
        const int idle_now = __shfl_sync(FULL, lane == 0 ? (int)(ld_vol(&ctl->idle) > 0) : 0, 0);
        if (idle_now) {
          uint32_t upper = rest;
          for (uint32_t k = __popc(rest) >> 1; k; --k) upper &= upper - 1;  // drop the lower half
          const uint32_t s = __ffs(upper) - 1, hb = 31 - __clz(rest);
          const uint32_t src = __shfl_sync(FULL, c.src, lvl);
          const uint64_t hsp = MODE == MODE_COUNT ? 0ull : __shfl_sync(FULL, c.hs, lvl - 1);
          if (queue_push(a, q, lvl, src, cb + s, cb + hb + 1, hsp, c)) {
            rest &= (1u << s) - 1u;
            pushed = true;
          }
        }
      }
      if (lane == lvl) c.mask = rest;
      const uint32_t w = __ldg(a.values + cb + b);
      const uint32_t widx = index_of(a, L, w);
      const uint64_t hsp = MODE == MODE_COUNT ? 0ull : __shfl_sync(FULL, c.hs, lvl - 1);
      if (lane == lvl) {
        c.f = w;
        c.idx = widx;
        if (MODE != MODE_COUNT) c.hs = hsp + emb_term(L->u, w);
      }
      if (lane == 0) {
        st.nodes += 1;
        st.probes += L->idx_kind != IDX_NONE;
      }
      const uint32_t nxt = lvl + 1;
      ++epoch;
      if (!inb(a, SITE_LEVEL, nxt, n)) {
        abort = true;
        break;
      }
      uint32_t nb, src;
      uint64_t lo, hi, s_lo, s_hi;
      level_lists(a, &Q->lv[nxt], c, nb, lo, hi, src, s_lo, s_hi);
      if (lane == nxt) {
        c.src = src;
        c.pos = s_lo;
        c.end = s_hi;
        c.mask = 0;
      }
      lvl = nxt;
    }

    // ------------------------------------------------------------ retire
    uint64_t tc = lane_cnt, th = lane_hash;
#pragma unroll
    for (int d = 16; d; d >>= 1) {
      tc += __shfl_xor_sync(FULL, tc, d);
      th += __shfl_xor_sync(FULL, th, d);
    }
    const bool release = abort || !from_root || rb_cur >= rb_end;
    // a count of this task may have been cut short by the cap since the last
    // look: with the error word set, its query is incomplete
    const bool cut = !abort && err_set(a);
    if (lane == 0) {
      if (cut) atomicOr(&a.out[q].pad[0], 1ull);
      if (abort) {
        abandon(a, q);
        if (from_root && rb_cur < rb_end) {
          const uint32_t q1 = find_query(a.root_prefix, a.nquery, rb_end - 1);
          for (uint32_t k = q; k <= q1; ++k) atomicOr(&a.out[k].pad[0], 1ull);
        }
      }
      if (tc) atomicAdd(&a.out[q].count, (unsigned long long)tc);
      if (MODE != MODE_COUNT && th) atomicAdd(&a.out[q].hash, (unsigned long long)th);
      if (release) {
        if (pushed) __threadfence();  // donated tasks are visible before quiescence can be observed
        atomicSub(&ctl->busy, 1u);
      }
    }
    if (release) pushed = false;
    if (abort) break;
    if (!from_root && !idle_registered) {
      idle_registered = true;
      if (lane == 0) atomicAdd(&ctl->idle, 1u);
    }
  }
  if (lane == 0 && (st.nodes | st.scanned | st.probes)) {
    atomicAdd(&a.out[0].nodes, (unsigned long long)st.nodes);
    atomicAdd(&a.out[0].scanned, (unsigned long long)st.scanned);
    atomicAdd(&a.out[0].probes, (unsigned long long)st.probes);
  }
}

// Zeroes the control block and the per-query outputs, resets the task queue
// and sets the deadline; runs right before the join in the same graph.
__global__ void join_prepare_kernel(JControl *ctl, JOut *out, uint32_t nquery, JTask *cells, JQueueEnds *qends,
                                    uint64_t cap_ns, const JQuery *queries, const JBack *backs,
                                    const uint32_t *lp2q, uint32_t lp2_nq, uint64_t *lp2_prefix) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  // pair pool: each query's (root, first level) pairs are the entries of its
  // root table, padded to whole chunks of 32 so no chunk spans two queries;
  // block 0 scans the padded sizes, one query per thread
  if (blockIdx.x == 0 && lp2_nq) {
    __shared__ uint64_t wsum[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint64_t carry = 0;
    for (uint32_t b0 = 0; b0 < lp2_nq; b0 += blockDim.x) {
      const uint32_t i = b0 + threadIdx.x;
      uint64_t n = 0;
      if (i < lp2_nq) {
        const JQuery *Q = queries + lp2q[i];
        const JBack *b = backs + Q->lv[1].back_base;
        n = ((b->off[b->nkeys] - b->off[0]) + 31) & ~31ull;
      }
      uint64_t incl = n;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(FULL, incl, d);
        if (lane >= (uint32_t)d) incl += o;
      }
      if (lane == 31) wsum[warp] = incl;
      __syncthreads();
      uint64_t before = carry, tile = 0;
      for (uint32_t w = 0; w < nw; ++w) {
        if (w < warp) before += wsum[w];
        tile += wsum[w];
      }
      if (i < lp2_nq) lp2_prefix[i] = before + incl - n;
      carry += tile;
      __syncthreads();  // wsum is rewritten by the next step
    }
    if (threadIdx.x == 0) lp2_prefix[lp2_nq] = carry;
  }
  for (uint32_t i = t; i < TASK_CAP; i += nt) cells[i].seq = i & (QUEUE_SUBQ_CAP - 1);
  for (uint32_t i = t; i < QUEUE_SUBQ; i += nt) {
    qends[i].head = 0;
    qends[i].tail = 0;
  }
  unsigned long long *o = reinterpret_cast<unsigned long long *>(out);
  const uint32_t words = nquery * (uint32_t)(sizeof(JOut) / 8);
  for (uint32_t i = t; i < words; i += nt) o[i] = 0ull;
  if (t == 0) {
    JControl z;
    memset(&z, 0, sizeof z);
    z.deadline_ns = globaltimer_ns() + cap_ns;
    *ctl = z;
  }
}

static void *join_fn(uint32_t mode) {
  if (mode == MODE_COUNT) return (void *)join_kernel<MODE_COUNT>;
  if (mode == MODE_HASH) return (void *)join_kernel<MODE_HASH>;
  return (void *)join_kernel<MODE_ENUM>;
}

// The list cache takes JOIN_DYN_SMEM of dynamic shared memory per block,
// above the default 48 KiB limit: every join instance opts in once.
static cudaError_t join_smem_optin() {
  static cudaError_t done = [] {
    for (uint32_t m : {MODE_COUNT, MODE_HASH, MODE_ENUM}) {
      const cudaError_t e =
          cudaFuncSetAttribute(join_fn(m), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JOIN_DYN_SMEM);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }();
  return done;
}

int join_blocks_per_sm(uint32_t mode) {
  int n = 0;
  if (join_smem_optin() != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, join_fn(mode), JOIN_WARPS_PER_BLOCK * 32, JOIN_DYN_SMEM) !=
          cudaSuccess ||
      n <= 0) {
    cudaGetLastError();
    n = 1;
  }
  return n;
}

void destroy_join_graph(JoinGraph &jg) {
  if (jg.exec) cudaGraphExecDestroy(jg.exec);
  if (jg.graph) cudaGraphDestroy(jg.graph);
  jg = JoinGraph();
}

cudaError_t launch_join_graph(JoinGraph &jg, const JoinArgs &a, uint64_t cap_ns, uint32_t grid, cudaStream_t s) {
  JoinArgs args = a;
  JControl *ctl = a.ctl;
  JOut *out = a.out;
  uint32_t nq = a.nquery;
  JTask *cells = a.queue;
  JQueueEnds *qends = a.qends;
  uint64_t cap = cap_ns;
  const JQuery *queries = a.queries;
  const JBack *backs = a.backs;
  const uint32_t *lp2q = a.lp2_query;
  uint32_t lp2_nq = a.lp2_nq;
  uint64_t *lp2_prefix = const_cast<uint64_t *>(a.lp2_prefix);
  void *prep_params[] = {&ctl, &out, &nq, &cells, &qends, &cap, &queries, &backs, &lp2q, &lp2_nq, &lp2_prefix};
  void *join_params[] = {&args};
  cudaKernelNodeParams pp = {};
  pp.func = (void *)join_prepare_kernel;
  pp.gridDim = dim3(32);
  pp.blockDim = dim3(256);
  pp.kernelParams = prep_params;
  cudaKernelNodeParams jp = {};
  jp.func = join_fn(a.mode);
  jp.gridDim = dim3(grid);
  jp.blockDim = dim3(JOIN_WARPS_PER_BLOCK * 32);
  jp.sharedMemBytes = JOIN_DYN_SMEM;
  jp.kernelParams = join_params;
  cudaError_t e;
  if ((e = join_smem_optin()) != cudaSuccess) return e;
  if (!jg.exec || jg.mode != a.mode || jg.grid != grid) {
    destroy_join_graph(jg);
    if ((e = cudaGraphCreate(&jg.graph, 0)) != cudaSuccess) return e;
    if ((e = cudaGraphAddKernelNode(&jg.prep, jg.graph, nullptr, 0, &pp)) != cudaSuccess) return e;
    if ((e = cudaGraphAddKernelNode(&jg.join, jg.graph, &jg.prep, 1, &jp)) != cudaSuccess) return e;
    if ((e = cudaGraphInstantiate(&jg.exec, jg.graph, 0)) != cudaSuccess) return e;
    jg.mode = a.mode;
    jg.grid = grid;
  } else {
    if ((e = cudaGraphExecKernelNodeSetParams(jg.exec, jg.prep, &pp)) != cudaSuccess) return e;
    if ((e = cudaGraphExecKernelNodeSetParams(jg.exec, jg.join, &jp)) != cudaSuccess) return e;
  }
  count_launch(2);
  return cudaGraphLaunch(jg.exec, s);
}

}  // namespace gem
