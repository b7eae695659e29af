// Candidate filter and compaction.
//
// Same predicate as the reference's LDfilterSSM_kernel
// (in-core/lib/filter/src/filter_kernel.cu:122-283) and the CPU filterSSM
// (out-of-core/lib/filter/src/filter.cu:160-240): label equality, query degree
// <= data degree + T, and a neighbour-label-count deficit <= T over the labels
// that occur in the query.  Layout differences: one warp covers 32
// consecutive data vertices (one per lane, coalesced label/degree loads), the
// per-vertex label counts come from the table built at graph load, every
// query of a wave is evaluated against a tile while it is in registers, and
// each (query vertex, tile) result is one ballot word.  The compaction turns
// the bit rows into sorted candidate lists and leaves a per-word rank in the
// high half of each word, so the same row answers "is v in C(u)" and "where
// is v in C(u)" with one 8-byte load.
#include "device_common.cuh"
#include "kernels.h"

namespace gem {

__global__ void __launch_bounds__(256) filter_kernel(DevGraph g, const FilterDesc *__restrict__ descs,
                                                     uint32_t nquery, uint64_t *__restrict__ rb,
                                                     uint32_t nwords) {
  const uint32_t lane = dev::lane_id();
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t t = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); t < nwords; t += nwarps) {
    const uint64_t v = t * 32 + lane;
    const bool valid = v < g.nv;
    const uint32_t l = valid ? __ldg(g.lab + v) : 0u;
    const uint32_t d = valid ? __ldg(g.deg + v) : 0u;
    const uint8_t *row = (g.nlc_stride && valid) ? g.nlc + v * g.nlc_stride : nullptr;
    // this block's group of queries (blockIdx.y): small graphs have too few
    // tiles to fill the GPU with whole waves of queries per warp
    const uint32_t qper = (nquery + gridDim.y - 1) / gridDim.y;
    const uint32_t q0 = blockIdx.y * qper, q1 = q0 + qper < nquery ? q0 + qper : nquery;
    for (uint32_t qi = q0; qi < q1; ++qi) {
      const FilterDesc *q = descs + qi;
      const uint32_t nq = q->nq, T = q->threshold, nql = q->nql;
      uint32_t pmask = 0;
      if (valid)
        for (uint32_t u = 0; u < nq; ++u)
          if (l == q->lab[u] && q->deg[u] <= d + T) pmask |= 1u << u;
      if (__ballot_sync(dev::FULL, pmask != 0)) {
        if (pmask) {
          uint32_t cnt[QV];
          if (row) {
            for (uint32_t k = 0; k < nql; ++k) {
              uint32_t lk = q->ql[k];
              cnt[k] = lk < g.nlabels ? (uint32_t)__ldg(row + lk) : 0u;
            }
          } else {
            for (uint32_t k = 0; k < nql; ++k) cnt[k] = 0;
            for (uint64_t i = g.off[v], e = g.off[v + 1]; i < e; ++i) {
              uint32_t ln = __ldg(g.lab + __ldg(g.nbr + i));
              for (uint32_t k = 0; k < nql; ++k)
                if (q->ql[k] == ln) { cnt[k]++; break; }
            }
          }
          uint32_t m = pmask;
          while (m) {
            uint32_t u = __ffs(m) - 1;
            m &= m - 1;
            uint32_t diff = 0;
            for (uint32_t k = 0; k < nql; ++k) {
              uint32_t qc = q->nlc[u][k];
              if (qc > cnt[k]) diff += qc - cnt[k];
            }
            if (diff > T) pmask &= ~(1u << u);
          }
        }
      }
      uint32_t word = 0;
      for (uint32_t u = 0; u < nq; ++u) {
        uint32_t b = __ballot_sync(dev::FULL, (pmask >> u) & 1u);
        if (lane == u) word = b;
      }
      if (lane < nq) rb[(uint64_t)(q->row_base + lane) * nwords + t] = (uint64_t)word;
    }
  }
}

void launch_filter(const DevGraph &g, const FilterDesc *d_desc, uint32_t nquery, uint64_t *rb, uint32_t nwords,
                   cudaStream_t s) {
  if (nwords == 0 || nquery == 0) return;
  uint64_t blocks = (nwords + 7) / 8;
  if (blocks > 148ull * 16) blocks = 148ull * 16;
  // split the wave's queries over grid.y until about 148 x 48 warps run
  uint64_t groups = (148ull * 48 + nwords - 1) / nwords;
  if (groups > nquery) groups = nquery;
  if (groups > 65535) groups = 65535;
  if (groups == 0) groups = 1;
  count_launch();
  filter_kernel<<<dim3((uint32_t)blocks, (uint32_t)groups), 256, 0, s>>>(g, d_desc, nquery, rb, nwords);
}

__global__ void compact_kernel(uint64_t *__restrict__ rb, const uint64_t *__restrict__ ex, uint32_t nrows,
                               uint32_t nwords, const uint64_t *__restrict__ c_base, uint32_t *__restrict__ cand,
                               uint32_t *__restrict__ bit_rows) {
  const uint64_t n = (uint64_t)nrows * nwords;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(i / nwords), w = (uint32_t)(i % nwords);
    const uint32_t bits = (uint32_t)rb[i];
    const uint64_t rank = ex[i] - ex[(uint64_t)r * nwords];
    rb[i] = (rank << 32) | bits;
    if (bit_rows) bit_rows[i] = bits;
    uint32_t m = bits, j = 0;
    uint32_t *dst = cand + c_base[r] + rank;
    while (m) {
      uint32_t b = __ffs(m) - 1;
      m &= m - 1;
      dst[j++] = w * 32u + b;
    }
  }
}

void launch_compact(uint64_t *rb, const uint64_t *ex, uint32_t nrows, uint32_t nwords, const uint64_t *c_base,
                    uint32_t *cand, cudaStream_t s, uint32_t *bit_rows) {
  uint64_t n = (uint64_t)nrows * nwords;
  if (n == 0) return;
  uint64_t blocks = (n + 255) / 256;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  count_launch();
  compact_kernel<<<(uint32_t)blocks, 256, 0, s>>>(rb, ex, nrows, nwords, c_base, cand, bit_rows);
}

}  // namespace gem
