/*
 * oracle.c — CPU oracle for the subgraph-matching path.  TEST INFRASTRUCTURE:
 * only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark load this; the product (libgem) never links or calls it.
 *
 * It restates, in plain C, the reference's semantics for the three artefacts
 * the GPU path produces:
 *   1. candidate sets C(u)     — in-core/lib/filter/src/filter_kernel.cu:122-283
 *                                (LDfilterSSM_kernel), out-of-core/lib/filter/
 *                                src/filter.cu:61-240 (CPU filterSSM);
 *   2. edge-candidate tables   — in-core/lib/structure/src/construct_kernel.cu
 *                                :1183-1300 (count/write_bitmap_task1),
 *                                out-of-core/lib/structure/src/unifiedTrie.cu
 *                                :1224-1427 (construct_edge_candidates_cpu);
 *   3. the embedding count     — the join chain of in-core/lib/join/src/
 *                                join_trie.cu:1087-1277 at threshold 0: injective
 *                                (same-label duplicate check, join_trie.cu:450-462),
 *                                label-preserving, non-induced, no symmetry
 *                                breaking.
 * The count here is computed by straightforward backtracking from the raw
 * definition (no candidate filter), so it also checks the GPU filter's
 * soundness.  oracle_brute enumerates every injective map on tiny graphs and
 * checks the backtracker itself.  Parity pins: the reference has no tests,
 * golden vectors or fixtures; the committed fixtures under tests/golden/
 * hold hand-derived answers and counts printed by the reference binary.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAX_QV 32

static uint64_t or_mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

/* Same definition as gem_embedding_hash in include/gem.h. */
uint64_t oracle_emb_hash(const uint32_t *f, uint32_t n) {
  uint64_t s = 0;
  for (uint32_t u = 0; u < n; ++u) s += or_mix64((uint64_t)f[u] | ((uint64_t)u << 32));
  return or_mix64(s);
}

static int has_arc(const uint64_t *off, const uint32_t *nbr, uint32_t a, uint32_t b) {
  uint64_t lo = off[a], hi = off[a + 1];
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (nbr[mid] < b) lo = mid + 1; else hi = mid;
  }
  return lo < off[a + 1] && nbr[lo] == b;
}

static void build_qadj(uint32_t qn, uint32_t qm, const uint32_t *qedges, uint32_t *qadj) {
  for (uint32_t u = 0; u < qn; ++u) qadj[u] = 0;
  for (uint32_t e = 0; e < qm; ++e) {
    qadj[qedges[2 * e]] |= 1u << qedges[2 * e + 1];
    qadj[qedges[2 * e + 1]] |= 1u << qedges[2 * e];
  }
}

/*
 * Filter: writes |C(u)| to counts[u] and the sorted lists back to back into
 * cand (capacity cand_cap).  Returns 0, or -1 when cand_cap is too small.
 * Predicate (in-core filter_kernel.cu:196-257; out-of-core filter.cu:93-240):
 * label(v) == label(u), deg_q(u) <= deg(v) + T, and the neighbour-label-count
 * deficit sum_l max(0, nlc_u[l] - nlc_v[l]) <= T, where nlc counts only the
 * labels that occur in the query (the reference maps every other data label
 * to one sentinel at or above NUM_VLQ and skips it).
 */
int oracle_filter(uint32_t nv, const uint64_t *off, const uint32_t *nbr, const uint32_t *lab,
                  uint32_t qn, const uint32_t *qlab, uint32_t qm, const uint32_t *qedges,
                  uint32_t T, uint32_t *counts, uint32_t *cand, uint64_t cand_cap) {
  uint32_t qadj[OR_MAX_QV];
  build_qadj(qn, qm, qedges, qadj);
  /* distinct query labels -> local ids */
  uint32_t ql[OR_MAX_QV], nql = 0;
  for (uint32_t u = 0; u < qn; ++u) {
    uint32_t k = 0;
    while (k < nql && ql[k] != qlab[u]) ++k;
    if (k == nql) ql[nql++] = qlab[u];
  }
  uint32_t qnlc[OR_MAX_QV][OR_MAX_QV];
  memset(qnlc, 0, sizeof qnlc);
  for (uint32_t u = 0; u < qn; ++u)
    for (uint32_t w = 0; w < qn; ++w)
      if (qadj[u] & (1u << w)) {
        uint32_t k = 0;
        while (ql[k] != qlab[w]) ++k;
        qnlc[u][k]++;
      }
  uint64_t pos = 0;
  for (uint32_t u = 0; u < qn; ++u) {
    uint32_t du = (uint32_t)__builtin_popcount(qadj[u]);
    uint32_t c = 0;
    for (uint32_t v = 0; v < nv; ++v) {
      if (lab[v] != qlab[u]) continue;
      uint32_t dv = (uint32_t)(off[v + 1] - off[v]);
      if (!(du <= dv + T)) continue;
      uint32_t dnlc[OR_MAX_QV];
      memset(dnlc, 0, sizeof dnlc);
      for (uint64_t i = off[v]; i < off[v + 1]; ++i) {
        uint32_t l = lab[nbr[i]];
        for (uint32_t k = 0; k < nql; ++k)
          if (ql[k] == l) { dnlc[k]++; break; }
      }
      uint32_t diff = 0;
      for (uint32_t k = 0; k < nql; ++k)
        if (qnlc[u][k] > dnlc[k]) diff += qnlc[u][k] - dnlc[k];
      if (diff > T) continue;
      if (pos >= cand_cap) return -1;
      cand[pos++] = v;
      ++c;
    }
    counts[u] = c;
  }
  return 0;
}

/*
 * Edge-candidate table T(u -> w) from candidate lists: for i in [0, nu),
 * values = [x in N(cu[i]) : x in C(w)] in adjacency order; offsets CSR with
 * nu + 1 entries (in-core construct_kernel.cu:1205-1229 and the scan that
 * feeds getMax, unifiedTrie.cu:1138-1161).  Returns total values, or -1 when
 * values_cap is too small (offsets still complete).
 */
int64_t oracle_edge_table(uint32_t nv, const uint64_t *off, const uint32_t *nbr,
                          const uint32_t *cu, uint32_t nu, const uint32_t *cw, uint32_t nw,
                          uint64_t *offsets, uint32_t *values, uint64_t values_cap) {
  uint8_t *inw = (uint8_t *)calloc(nv ? nv : 1, 1);
  if (!inw) return -2;
  for (uint32_t i = 0; i < nw; ++i) inw[cw[i]] = 1;
  uint64_t p = 0;
  int overflow = 0;
  offsets[0] = 0;
  for (uint32_t i = 0; i < nu; ++i) {
    uint32_t v = cu[i];
    for (uint64_t j = off[v]; j < off[v + 1]; ++j)
      if (inw[nbr[j]]) {
        if (p < values_cap) values[p] = nbr[j]; else overflow = 1;
        ++p;
      }
    offsets[i + 1] = p;
  }
  free(inw);
  return overflow ? -1 : (int64_t)p;
}

/*
 * The same filter on threads (nt <= 0: min(16, omp_get_max_threads()), the
 * worker count of the reference's out-of-core filterSSM, out-of-core/lib/
 * filter/src/filter.cu:47-58): data vertices in parallel, each vertex's
 * neighbour-label counts computed once and tested against every query vertex,
 * then the lists compacted in vertex order.  Same output as oracle_filter.
 */
int oracle_filter_mt(uint32_t nv, const uint64_t *off, const uint32_t *nbr, const uint32_t *lab,
                     uint32_t qn, const uint32_t *qlab, uint32_t qm, const uint32_t *qedges,
                     uint32_t T, uint32_t *counts, uint32_t *cand, uint64_t cand_cap, int nt) {
  if (nt <= 0) {
    nt = omp_get_max_threads();
    if (nt > 16) nt = 16;
  }
  uint32_t qadj[OR_MAX_QV];
  build_qadj(qn, qm, qedges, qadj);
  uint32_t ql[OR_MAX_QV], nql = 0;
  for (uint32_t u = 0; u < qn; ++u) {
    uint32_t k = 0;
    while (k < nql && ql[k] != qlab[u]) ++k;
    if (k == nql) ql[nql++] = qlab[u];
  }
  uint32_t qnlc[OR_MAX_QV][OR_MAX_QV], qdeg[OR_MAX_QV];
  memset(qnlc, 0, sizeof qnlc);
  for (uint32_t u = 0; u < qn; ++u) {
    qdeg[u] = (uint32_t)__builtin_popcount(qadj[u]);
    for (uint32_t w = 0; w < qn; ++w)
      if (qadj[u] & (1u << w)) {
        uint32_t k = 0;
        while (ql[k] != qlab[w]) ++k;
        qnlc[u][k]++;
      }
  }
  uint32_t *mask = (uint32_t *)malloc((nv ? nv : 1) * sizeof(uint32_t));
  if (!mask) return -2;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (int64_t vi = 0; vi < (int64_t)nv; ++vi) {
    const uint32_t v = (uint32_t)vi;
    uint32_t m = 0;
    for (uint32_t u = 0; u < qn; ++u)
      if (lab[v] == qlab[u] && qdeg[u] <= (uint32_t)(off[v + 1] - off[v]) + T) m |= 1u << u;
    if (m) {
      uint32_t dnlc[OR_MAX_QV];
      memset(dnlc, 0, sizeof dnlc);
      for (uint64_t i = off[v]; i < off[v + 1]; ++i) {
        const uint32_t l = lab[nbr[i]];
        for (uint32_t k = 0; k < nql; ++k)
          if (ql[k] == l) { dnlc[k]++; break; }
      }
      for (uint32_t mm = m; mm; mm &= mm - 1) {
        const uint32_t u = (uint32_t)__builtin_ctz(mm);
        uint32_t diff = 0;
        for (uint32_t k = 0; k < nql; ++k)
          if (qnlc[u][k] > dnlc[k]) diff += qnlc[u][k] - dnlc[k];
        if (diff > T) m &= ~(1u << u);
      }
    }
    mask[v] = m;
  }
  uint64_t pos = 0;
  int overflow = 0;
  for (uint32_t u = 0; u < qn; ++u) {
    uint32_t c = 0;
    for (uint32_t v = 0; v < nv; ++v)
      if ((mask[v] >> u) & 1u) {
        if (pos < cand_cap) cand[pos] = v; else overflow = 1;
        ++pos;
        ++c;
      }
    counts[u] = c;
  }
  free(mask);
  return overflow ? -1 : 0;
}

/*
 * The same edge-candidate table on threads (nt <= 0: min(4,
 * omp_get_max_threads()), the worker count of the reference's out-of-core
 * construct_edge_candidates_cpu, out-of-core/lib/structure/src/unifiedTrie.cu
 * :26-37): a parallel count pass over the keys, a prefix sum, a parallel write
 * pass.  Same output as oracle_edge_table.
 */
int64_t oracle_edge_table_mt(uint32_t nv, const uint64_t *off, const uint32_t *nbr,
                             const uint32_t *cu, uint32_t nu, const uint32_t *cw, uint32_t nw,
                             uint64_t *offsets, uint32_t *values, uint64_t values_cap, int nt) {
  if (nt <= 0) {
    nt = omp_get_max_threads();
    if (nt > 4) nt = 4;
  }
  uint8_t *inw = (uint8_t *)calloc(nv ? nv : 1, 1);
  if (!inw) return -2;
  for (uint32_t i = 0; i < nw; ++i) inw[cw[i]] = 1;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
  for (int64_t ii = 0; ii < (int64_t)nu; ++ii) {
    const uint32_t v = cu[ii];
    uint64_t c = 0;
    for (uint64_t j = off[v]; j < off[v + 1]; ++j) c += inw[nbr[j]];
    offsets[ii + 1] = c;
  }
  offsets[0] = 0;
  for (uint32_t i = 0; i < nu; ++i) offsets[i + 1] += offsets[i];
  const uint64_t total = offsets[nu];
  if (total > values_cap) {
    free(inw);
    return -1;
  }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
  for (int64_t ii = 0; ii < (int64_t)nu; ++ii) {
    const uint32_t v = cu[ii];
    uint64_t p = offsets[ii];
    for (uint64_t j = off[v]; j < off[v + 1]; ++j)
      if (inw[nbr[j]]) values[p++] = nbr[j];
  }
  free(inw);
  return (int64_t)total;
}

/* ---------------------------------------------------------------------- */
/* Backtracking counter                                                    */
/* ---------------------------------------------------------------------- */
typedef struct {
  uint32_t n;
  uint32_t order[OR_MAX_QV];      /* matching order */
  uint32_t parent[OR_MAX_QV];     /* level of the neighbour whose adjacency is scanned */
  uint32_t nback[OR_MAX_QV];      /* other backward neighbours (levels) */
  uint32_t back[OR_MAX_QV][OR_MAX_QV];
  uint32_t label[OR_MAX_QV];      /* label by level */
  uint32_t qdeg[OR_MAX_QV];       /* query degree by level */
} or_plan;

static void make_plan(uint32_t qn, const uint32_t *qlab, const uint32_t *qadj, or_plan *p) {
  p->n = qn;
  uint32_t used = 0, pos_of[OR_MAX_QV];
  for (uint32_t k = 0; k < qn; ++k) {
    int best = -1;
    int bb = -1, bd = -1;
    for (uint32_t u = 0; u < qn; ++u) {
      if (used & (1u << u)) continue;
      int b = __builtin_popcount(qadj[u] & used);
      int d = __builtin_popcount(qadj[u]);
      if (k > 0 && b == 0) continue;
      if (b > bb || (b == bb && d > bd)) { best = (int)u; bb = b; bd = d; }
    }
    uint32_t u = (uint32_t)best;
    p->order[k] = u;
    pos_of[u] = k;
    used |= 1u << u;
    p->label[k] = qlab[u];
    p->qdeg[k] = (uint32_t)__builtin_popcount(qadj[u]);
    p->nback[k] = 0;
    p->parent[k] = 0;
    int first = 1;
    for (uint32_t j = 0; j < k; ++j) {
      if (qadj[u] & (1u << p->order[j])) {
        if (first) { p->parent[k] = j; first = 0; }
        else p->back[k][p->nback[k]++] = j;
      }
    }
  }
  (void)pos_of;
}

typedef struct {
  const uint64_t *off;
  const uint32_t *nbr;
  const uint32_t *lab;
  const or_plan *p;
  uint64_t count, hash, nodes, work;
  int want_hash;
  uint64_t node_cap;
  volatile int *abort_flag;
  uint32_t f[OR_MAX_QV];          /* by level */
  uint64_t hsum[OR_MAX_QV + 1];   /* prefix sums of per-vertex hash terms */
} or_walker;

static void walk(or_walker *w, uint32_t k) {
  const or_plan *p = w->p;
  const uint32_t u = p->order[k];
  const uint32_t par = w->f[p->parent[k]];
  const uint32_t last = (k + 1 == p->n);
  w->work += w->off[par + 1] - w->off[par];
  if (w->node_cap && w->work > w->node_cap) { *w->abort_flag = 1; return; }
  if (*w->abort_flag) return;
  for (uint64_t i = w->off[par]; i < w->off[par + 1]; ++i) {
    uint32_t x = w->nbr[i];
    if (w->lab[x] != p->label[k]) continue;
    if ((uint32_t)(w->off[x + 1] - w->off[x]) < p->qdeg[k]) continue;
    int ok = 1;
    for (uint32_t j = 0; j < k && ok; ++j) if (w->f[j] == x) ok = 0;
    for (uint32_t b = 0; b < p->nback[k] && ok; ++b)
      if (!has_arc(w->off, w->nbr, w->f[p->back[k][b]], x)) ok = 0;
    if (!ok) continue;
    uint64_t term = w->want_hash ? or_mix64((uint64_t)x | ((uint64_t)u << 32)) : 0;
    if (last) {
      w->count++;
      if (w->want_hash) w->hash += or_mix64(w->hsum[k] + term);
    } else {
      w->nodes++;
      w->f[k] = x;
      w->hsum[k + 1] = w->hsum[k] + term;
      walk(w, k + 1);
    }
  }
}

/*
 * Count embeddings.  threads <= 0 uses all OpenMP threads.  work_cap > 0
 * aborts after about that many scanned adjacency entries and returns 1
 * (count incomplete).  Returns 0 when complete; nodes_out receives the number
 * of partial embeddings extended (every level but the last).
 */
int oracle_count(uint32_t nv, const uint64_t *off, const uint32_t *nbr, const uint32_t *lab,
                 uint32_t qn, const uint32_t *qlab, uint32_t qm, const uint32_t *qedges,
                 int threads, int want_hash, uint64_t node_cap,
                 uint64_t *count_out, uint64_t *hash_out, uint64_t *nodes_out) {
  uint32_t qadj[OR_MAX_QV];
  if (qn == 0 || qn > OR_MAX_QV) return -1;
  build_qadj(qn, qm, qedges, qadj);
  or_plan p;
  make_plan(qn, qlab, qadj, &p);
  uint64_t count = 0, hash = 0, nodes = 0, shared_work = 0;
  volatile int abort_flag = 0;
  const uint32_t u0 = p.order[0];
  int nt = threads;
#ifdef _OPENMP
  if (nt <= 0) nt = omp_get_max_threads();
#else
  nt = 1;
#endif
#pragma omp parallel num_threads(nt) reduction(+ : count, hash, nodes)
  {
    or_walker w;
    w.off = off; w.nbr = nbr; w.lab = lab; w.p = &p;
    w.count = 0; w.hash = 0; w.nodes = 0; w.work = 0; w.want_hash = want_hash;
    w.node_cap = node_cap; w.abort_flag = &abort_flag;
    w.hsum[0] = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t v = 0; v < (int64_t)nv; ++v) {
      if (abort_flag) continue;
      if (lab[v] != qlab[u0]) continue;
      if ((uint32_t)(off[v + 1] - off[v]) < p.qdeg[0]) continue;
      uint64_t term = want_hash ? or_mix64((uint64_t)(uint32_t)v | ((uint64_t)u0 << 32)) : 0;
      if (qn == 1) {
        w.count++;
        if (want_hash) w.hash += or_mix64(term);
        continue;
      }
      w.f[0] = (uint32_t)v;
      w.hsum[1] = term;
      w.nodes++;
      uint64_t before = w.work;
      walk(&w, 1);
      if (node_cap) {
        uint64_t d = w.work - before + 1, tot;
#pragma omp atomic capture
        { shared_work += d; tot = shared_work; }
        if (tot > node_cap) abort_flag = 1;
        w.work = 0;
      }
    }
    count += w.count;
    hash += w.hash;
    nodes += w.nodes;
  }
  *count_out = count;
  if (hash_out) *hash_out = hash;
  if (nodes_out) *nodes_out = nodes;
  return abort_flag ? 1 : 0;
}

/*
 * Brute force over all injective maps (tiny graphs only): returns the count
 * and the hash.  Used to check oracle_count itself.
 */
static void brute_rec(uint32_t k, uint32_t qn, uint32_t nv, const uint64_t *off, const uint32_t *nbr,
                      const uint32_t *lab, const uint32_t *qlab, const uint32_t *qadj,
                      uint32_t *f, uint64_t *count, uint64_t *hash) {
  if (k == qn) {
    for (uint32_t a = 0; a < qn; ++a)
      for (uint32_t b = a + 1; b < qn; ++b)
        if ((qadj[a] & (1u << b)) && !has_arc(off, nbr, f[a], f[b])) return;
    (*count)++;
    *hash += oracle_emb_hash(f, qn);
    return;
  }
  for (uint32_t v = 0; v < nv; ++v) {
    if (lab[v] != qlab[k]) continue;
    int used = 0;
    for (uint32_t j = 0; j < k; ++j) if (f[j] == v) used = 1;
    if (used) continue;
    f[k] = v;
    brute_rec(k + 1, qn, nv, off, nbr, lab, qlab, qadj, f, count, hash);
  }
}

int oracle_brute(uint32_t nv, const uint64_t *off, const uint32_t *nbr, const uint32_t *lab,
                 uint32_t qn, const uint32_t *qlab, uint32_t qm, const uint32_t *qedges,
                 uint64_t *count_out, uint64_t *hash_out) {
  uint32_t qadj[OR_MAX_QV], f[OR_MAX_QV];
  if (qn == 0 || qn > 8 || nv > 64) return -1;
  build_qadj(qn, qm, qedges, qadj);
  uint64_t c = 0, h = 0;
  brute_rec(0, qn, nv, off, nbr, lab, qlab, qadj, f, &c, &h);
  *count_out = c;
  *hash_out = h;
  return 0;
}
