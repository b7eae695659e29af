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
#include <math.h>
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
  const uint32_t *lastc;          /* count mode, a last level keyed by one neighbour only: per data vertex
                                     its neighbours with that level's label and least degree (else null) */
  uint32_t f[OR_MAX_QV];          /* by level */
  uint64_t hsum[OR_MAX_QV + 1];   /* prefix sums of per-vertex hash terms */
} or_walker;

static void walk(or_walker *w, uint32_t k) {
  const or_plan *p = w->p;
  const uint32_t u = p->order[k];
  const uint32_t par = w->f[p->parent[k]];
  const uint32_t last = (k + 1 == p->n);
  if (last && w->lastc) {
    /* The last level counted without listing it, as the reference's last
       join step does (only the count of each row's extensions, in-core/lib/
       join/src/join_trie.cu:1204): the parent's neighbours with the label
       and degree, minus the earlier matches among them (injectivity). */
    uint64_t c = w->lastc[par];
    for (uint32_t j = 0; j < k; ++j) {
      const uint32_t y = w->f[j];
      if (w->lab[y] == p->label[k] && (uint32_t)(w->off[y + 1] - w->off[y]) >= p->qdeg[k] &&
          has_arc(w->off, w->nbr, par, y))
        --c;
    }
    w->count += c;
    w->work += 1 + k;
    return;
  }
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
  /* count mode: a last level whose only backward neighbour is its parent is
     counted from per-vertex neighbour counts instead of being listed */
  uint32_t *lastc = NULL;
  if (!want_hash && qn >= 2 && p.nback[qn - 1] == 0) {
    lastc = (uint32_t *)malloc((size_t)nv * sizeof(uint32_t));
    if (lastc) {
      const uint32_t L = p.label[qn - 1], D = p.qdeg[qn - 1];
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
      for (int64_t v = 0; v < (int64_t)nv; ++v) {
        uint32_t c = 0;
        for (uint64_t i = off[v]; i < off[v + 1]; ++i) {
          const uint32_t x = nbr[i];
          c += lab[x] == L && (uint32_t)(off[x + 1] - off[x]) >= D;
        }
        lastc[v] = c;
      }
    }
  }
#pragma omp parallel num_threads(nt) reduction(+ : count, hash, nodes)
  {
    or_walker w;
    w.off = off; w.nbr = nbr; w.lab = lab; w.p = &p;
    w.count = 0; w.hash = 0; w.nodes = 0; w.work = 0; w.want_hash = want_hash;
    w.node_cap = node_cap; w.abort_flag = &abort_flag;
    w.lastc = lastc;
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
  free(lastc);
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

/* ------------------------------------------------------------------------
 * Seeded workload generators, restated so that the benchmark's reference arm
 * builds its inputs without loading libgem.  They produce the same graphs and
 * queries as gem_hgraph_rmat, gem_hgraph_set_labels and gem_gen_queries (a
 * CPU test checks equality): counter-based splitmix64 draws, R-MAT quadrant
 * descent, Zipf labels by inverse CDF, random-walk queries with induced
 * edges.  The CSR of a simple undirected graph with sorted adjacency is
 * unique, so any correct construction gives the same arrays.
 * ------------------------------------------------------------------------ */
static uint64_t or_rng_at(uint64_t s, uint64_t i) { return or_mix64(or_mix64(s) ^ (i * 0xD1B54A32D192ED03ull)); }
static double or_u01(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

/* LSD radix sort of n keys of `bits` bits (11-bit digits). */
static int or_radix_sort(uint64_t *k, uint64_t n, uint32_t bits) {
  uint64_t *tmp = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
  uint64_t *cnt = (uint64_t *)malloc(2048 * sizeof(uint64_t));
  if (!tmp || !cnt) { free(tmp); free(cnt); return -1; }
  for (uint32_t sh = 0; sh < bits; sh += 11) {
    memset(cnt, 0, 2048 * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) cnt[(k[i] >> sh) & 2047]++;
    uint64_t s = 0;
    for (uint32_t d = 0; d < 2048; ++d) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
    for (uint64_t i = 0; i < n; ++i) tmp[cnt[(k[i] >> sh) & 2047]++] = k[i];
    memcpy(k, tmp, n * sizeof(uint64_t));
  }
  free(tmp);
  free(cnt);
  return 0;
}

/*
 * R-MAT: 2^scale vertices, edge_factor * 2^scale sampled edges; edge i draws
 * one splitmix64 stream from (seed, i) and descends `scale` levels, taking
 * quadrant (0,0), (0,1), (1,0) or (1,1) with probabilities a, b, c, 1-a-b-c
 * compared on the draw's top 53 bits.  Self loops and duplicates are dropped,
 * the rest symmetrised.  off gets nv+1 entries; *nbr_out is malloc'd (the
 * caller frees it with oracle_free).  Returns 0, or -1 on bad arguments or
 * memory.
 */
int oracle_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, uint64_t *off,
                uint32_t **nbr_out, uint64_t *n_arcs) {
  if (scale == 0 || scale > 31 || edge_factor == 0 || !off || !nbr_out || !n_arcs) return -1;
  const uint32_t nv = 1u << scale;
  const uint64_t m = (uint64_t)edge_factor << scale;
  const uint64_t ta = (uint64_t)(a * 9007199254740992.0), tb = (uint64_t)((a + b) * 9007199254740992.0),
                 tc = (uint64_t)((a + b + c) * 9007199254740992.0);
  uint64_t *keys = (uint64_t *)malloc(m * sizeof(uint64_t));
  if (!keys) return -1;
  const uint64_t drop = ~0ull;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i) {
    uint64_t s = or_rng_at(seed, (uint64_t)i);
    uint32_t src = 0, dst = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      s = or_mix64(s);
      const uint64_t r = s >> 11;
      const uint32_t bs = r >= tb, bd = (r >= ta && r < tb) || r >= tc;
      src = (src << 1) | bs;
      dst = (dst << 1) | bd;
    }
    keys[i] = src == dst ? drop : ((uint64_t)(src < dst ? src : dst) << scale) | (src < dst ? dst : src);
  }
  /* drop markers: move them out before sorting the 2*scale-bit keys */
  uint64_t n = 0;
  for (uint64_t i = 0; i < m; ++i)
    if (keys[i] != drop) keys[n++] = keys[i];
  if (or_radix_sort(keys, n, 2 * scale) != 0) { free(keys); return -1; }
  uint64_t u = 0;
  for (uint64_t i = 0; i < n; ++i)
    if (u == 0 || keys[u - 1] != keys[i]) keys[u++] = keys[i];
  const uint64_t mask = ((uint64_t)1 << scale) - 1;
  uint64_t *lower = (uint64_t *)calloc((size_t)nv + 1, sizeof(uint64_t));
  uint64_t *pos = (uint64_t *)malloc(((size_t)nv + 1) * sizeof(uint64_t));
  uint64_t *lpos = (uint64_t *)malloc(((size_t)nv + 1) * sizeof(uint64_t));
  uint32_t *nbr = (uint32_t *)malloc((2 * u ? 2 * u : 1) * sizeof(uint32_t));
  if (!lower || !pos || !lpos || !nbr) { free(keys); free(lower); free(pos); free(lpos); free(nbr); return -1; }
  for (uint32_t v = 0; v <= nv; ++v) off[v] = 0;
  for (uint64_t i = 0; i < u; ++i) {
    off[(keys[i] >> scale) + 1]++;  /* upper neighbour of lo */
    off[(keys[i] & mask) + 1]++;    /* lower neighbour of hi */
    lower[keys[i] & mask]++;
  }
  for (uint32_t v = 0; v < nv; ++v) off[v + 1] += off[v];
  /* each list: its lower neighbours (< v) then its upper ones (> v); keys in
     (lo, hi) order fill both parts in ascending order */
  for (uint32_t v = 0; v < nv; ++v) { lpos[v] = off[v]; pos[v] = off[v] + lower[v]; }
  for (uint64_t i = 0; i < u; ++i) {
    const uint32_t lo = (uint32_t)(keys[i] >> scale), hi = (uint32_t)(keys[i] & mask);
    nbr[pos[lo]++] = hi;
    nbr[lpos[hi]++] = lo;
  }
  free(keys);
  free(lower);
  free(pos);
  free(lpos);
  *nbr_out = nbr;
  *n_arcs = 2 * u;
  return 0;
}

void oracle_free(void *p) { free(p); }

/* Labels 0..nlabels-1 (uniform when zipf_s == 0, else P(l) ~ 1/(l+1)^s): vertex
 * v draws u = u01(stream seed, draw v) and takes the first l with cdf[l] > u. */
int oracle_set_labels(uint32_t nv, uint32_t nlabels, double zipf_s, uint64_t seed, uint32_t *lab) {
  if (nlabels == 0 || zipf_s < 0 || !lab) return -1;
  double *cdf = (double *)malloc(nlabels * sizeof(double));
  if (!cdf) return -1;
  double tot = 0;
  for (uint32_t l = 0; l < nlabels; ++l) {
    tot += zipf_s == 0 ? 1.0 : pow((double)(l + 1), -zipf_s);
    cdf[l] = tot;
  }
  for (uint32_t l = 0; l < nlabels; ++l) cdf[l] /= tot;
  cdf[nlabels - 1] = 1.0;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)nv; ++v) {
    const double x = or_u01(or_rng_at(seed, (uint64_t)v));
    uint32_t lo = 0, hi = nlabels;  /* first l with cdf[l] > x */
    while (lo < hi) {
      const uint32_t mid = (lo + hi) / 2;
      if (cdf[mid] > x) hi = mid; else lo = mid + 1;
    }
    lab[v] = lo < nlabels ? lo : nlabels - 1;
  }
  free(cdf);
  return 0;
}

/*
 * Random-walk queries (density 0 any, 1 sparse = average degree <= 3, 2 dense
 * = above 3).  Query qi draws from stream mix64(seed) ^ mix64(qi + 0x51).  Up
 * to 4096 walks: a start vertex with neighbours, then uniform neighbour steps
 * (at most 64k + 256) until k distinct vertices, numbered in visit order; the
 * query keeps all induced edges.  The first walk that reaches k vertices is
 * kept unless a later one meets the density.  An unsatisfied sparse request
 * keeps the first-visit tree edges plus induced (i, j) edges in order while
 * the average degree stays <= 3, sorted.  Outputs as gem_gen_queries:
 * ne_out[qi], labels_out[qi*k ..), edges_out[qi*2*max_e ..).  Returns 0, -1
 * (arguments), -2 (no walk reached k vertices) or -3 (more than max_e edges).
 */
int oracle_gen_queries(uint32_t nv, const uint64_t *off, const uint32_t *nbr, const uint32_t *lab, uint32_t k,
                       int density, uint32_t count, uint64_t seed, uint32_t max_e, uint32_t *ne_out,
                       uint32_t *labels_out, uint32_t *edges_out) {
  if (k == 0 || k > OR_MAX_QV || k > nv || density < 0 || density > 2 || off[nv] == 0) return -1;
  int fail = 0;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t qi = 0; qi < (int64_t)count; ++qi) {
    const uint64_t stream = or_mix64(seed) ^ or_mix64((uint64_t)qi + 0x51ull);
    uint64_t draw = 0;
    uint32_t vis[OR_MAX_QV], best[OR_MAX_QV], tree[OR_MAX_QV][2], btree[OR_MAX_QV][2];
    uint32_t nbest = 0, ntree = 0, nbtree = 0;
    int done = 0;
    for (uint32_t attempt = 0; attempt < 4096 && !done; ++attempt) {
      uint32_t s;
      do { s = (uint32_t)(or_rng_at(stream, draw++) % nv); } while (off[s + 1] == off[s]);
      uint32_t nvis = 1, cur = s, cur_local = 0;
      vis[0] = s;
      ntree = 0;
      for (uint64_t steps = 0, cap = 64ull * k + 256; nvis < k && steps < cap; ++steps) {
        const uint64_t d = off[cur + 1] - off[cur];
        const uint32_t nx = nbr[off[cur] + or_rng_at(stream, draw++) % d];
        uint32_t j = 0;
        while (j < nvis && vis[j] != nx) ++j;
        if (j == nvis) {
          vis[nvis++] = nx;
          tree[ntree][0] = cur_local;
          tree[ntree][1] = j;
          ++ntree;
        }
        cur = nx;
        cur_local = j;
      }
      if (nvis < k) continue;
      uint32_t m = 0;
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = i + 1; j < k; ++j) m += (uint32_t)has_arc(off, nbr, vis[i], vis[j]);
      const int dense = 2.0 * m / k > 3.0;
      const int ok = density == 0 || (density == 1 && !dense) || (density == 2 && dense);
      if (nbest == 0 || ok) {
        memcpy(best, vis, k * sizeof(uint32_t));
        memcpy(btree, tree, ntree * sizeof(tree[0]));
        nbest = k;
        nbtree = ntree;
      }
      if (ok) done = 1;
    }
    if (nbest == 0) {
#pragma omp atomic write
      fail = -2;
      continue;
    }
    uint32_t ne = 0;
    uint32_t *eo = edges_out + (size_t)qi * 2 * max_e;
    if (done || density != 1) {
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = i + 1; j < k; ++j)
          if (has_arc(off, nbr, best[i], best[j])) {
            if (ne < max_e) { eo[2 * ne] = i; eo[2 * ne + 1] = j; }
            ++ne;
          }
    } else {
      uint32_t has[OR_MAX_QV] = {0};  /* has[i] bit j: tree edge (i, j), i < j */
      uint32_t e[OR_MAX_QV * OR_MAX_QV][2];
      for (uint32_t t = 0; t < nbtree; ++t) {
        const uint32_t i = btree[t][0] < btree[t][1] ? btree[t][0] : btree[t][1];
        const uint32_t j = btree[t][0] < btree[t][1] ? btree[t][1] : btree[t][0];
        has[i] |= 1u << j;
        e[ne][0] = i;
        e[ne][1] = j;
        ++ne;
      }
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = i + 1; j < k; ++j) {
          if (has[i] >> j & 1u) continue;
          if (2.0 * (ne + 1) / k > 3.0) { i = k; break; }
          if (has_arc(off, nbr, best[i], best[j])) { e[ne][0] = i; e[ne][1] = j; ++ne; }
        }
      /* sort (i, j) pairs */
      for (uint32_t x = 1; x < ne; ++x)
        for (uint32_t y = x; y > 0 && (e[y - 1][0] > e[y][0] || (e[y - 1][0] == e[y][0] && e[y - 1][1] > e[y][1])); --y) {
          uint32_t t0 = e[y][0], t1 = e[y][1];
          e[y][0] = e[y - 1][0]; e[y][1] = e[y - 1][1];
          e[y - 1][0] = t0; e[y - 1][1] = t1;
        }
      for (uint32_t t = 0; t < ne && t < max_e; ++t) { eo[2 * t] = e[t][0]; eo[2 * t + 1] = e[t][1]; }
    }
    if (ne > max_e) {
#pragma omp atomic write
      fail = -3;
      continue;
    }
    ne_out[qi] = ne;
    for (uint32_t i = 0; i < k; ++i) labels_out[(size_t)qi * k + i] = lab[best[i]];
  }
  return fail;
}
