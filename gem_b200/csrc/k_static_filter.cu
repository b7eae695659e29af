// Candidate filter that allocates nothing: gem_filter_static.
//
// For callers that must not allocate device memory themselves or through the
// library — code running inside another framework's memory pool or allocator,
// which owns every device byte of the process, or a service whose memory is
// reserved up front and must not grow while it serves.  The caller passes the data graph and the
// output buffer as device pointers it already owns; the scratch the filter
// needs (one bit row with per-word ranks, its scan and the scan's partial
// sums) lives in a fixed, file-scope device array.
//
// Limits and sharing:
//  * the scratch array holds GEM_STATIC_SCRATCH_BYTES (4 MiB) on every GPU
//    that loads libgem, until the process exits; graphs with more than
//    GEM_STATIC_MAX_VERTICES vertices are rejected with GEM_ERR_LIMIT;
//  * every call on a device uses the same array, which keeps the last call's
//    contents: two calls whose work overlaps on that GPU (different streams,
//    threads or processes sharing a context) race and corrupt each other —
//    order them on one stream;
//  * every call looks up the array's device address (cudaGetSymbolAddress,
//    with the caller's device current) instead of caching it: after
//    cudaDeviceReset, or under another context of the same device, the
//    array lives at another address, and a cached one would be stale;
//  * a call blocks on its stream (it reads each row's candidate count back
//    before writing the list), so it cannot be made during stream capture;
//  * the graph arrays are checked on the device: a neighbour id >= nv or an
//    offset that decreases or runs past offsets[nv] is skipped, recorded in
//    the array's last word, and returns GEM_ERR_ARG.
// The predicate is the one of gem_filter (in-core/lib/filter/src/
// filter_kernel.cu:122-283): label, degree and neighbour-label counts, here
// computed from the adjacency of each label-and-degree survivor because no
// per-graph label-count table exists.
#include <cstring>
#include <string>

#include "../../include/gem.h"
#include "gem_internal.h"
#include "device_common.cuh"
#include "kernels.h"

namespace gem {

constexpr uint64_t STATIC_SCRATCH_WORDS = GEM_STATIC_SCRATCH_BYTES / 8;

// The scratch array: [0, nwords) bit row (low half bits, high half rank),
// [nwords, 2 nwords + 1) exclusive scan, then the scan's partials; its last
// word is the malformed-graph flag.
static __device__ __align__(256) uint64_t g_static_scratch[STATIC_SCRATCH_WORDS];

// One query vertex u against 32 consecutive data vertices per warp; degrees
// come from the offsets and label counts from the adjacency.
__global__ void __launch_bounds__(256) static_filter_row_kernel(const uint64_t *__restrict__ off,
                                                                const uint32_t *__restrict__ nbr,
                                                                const uint32_t *__restrict__ lab, uint32_t nv,
                                                                FilterDesc q, uint32_t u, uint64_t *__restrict__ row,
                                                                uint32_t nwords, uint32_t *bad) {
  const uint32_t lane = dev::lane_id();
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t n_arcs = __ldg(off + nv);
  for (uint64_t t = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); t < nwords; t += nwarps) {
    const uint64_t v = t * 32 + lane;
    bool pass = false;
    if (v < nv && __ldg(lab + v) == q.lab[u]) {
      const uint64_t b = __ldg(off + v), e = __ldg(off + v + 1);
      if (b > e || e > n_arcs) {
        dev::set_error(bad, dev::DERR_BOUNDS);  // offsets not a CSR: the list is not read
      } else if (q.deg[u] <= (uint32_t)(e - b) + q.threshold) {
        uint32_t cnt[QV];
        for (uint32_t k = 0; k < q.nql; ++k) cnt[k] = 0;
        for (uint64_t i = b; i < e; ++i) {
          const uint32_t nb = __ldg(nbr + i);
          if (nb >= nv) {
            dev::set_error(bad, dev::DERR_BOUNDS);  // neighbour id out of range: not looked up
            continue;
          }
          const uint32_t ln = __ldg(lab + nb);
          for (uint32_t k = 0; k < q.nql; ++k)
            if (q.ql[k] == ln) {
              cnt[k]++;
              break;
            }
        }
        uint32_t diff = 0;
        for (uint32_t k = 0; k < q.nql; ++k)
          if (q.nlc[u][k] > cnt[k]) diff += q.nlc[u][k] - cnt[k];
        pass = diff <= q.threshold;
      }
    }
    const uint32_t word = __ballot_sync(dev::FULL, pass);
    if (lane == 0) row[t] = word;
  }
}

// Device address of the scratch array in the caller's current context, looked
// up on every call (a cached address goes stale after cudaDeviceReset or in
// another context of the same device).
static gem_status static_scratch_address(uint64_t **out) {
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return GEM_ERR_CUDA;
  }
  *out = (uint64_t *)p;
  return GEM_OK;
}

}  // namespace gem

using namespace gem;

extern "C" gem_status gem_filter_static(const uint64_t *d_offsets, const uint32_t *d_nbrs, const uint32_t *d_labels,
                                        uint32_t nv, const gem_query *q, uint32_t threshold, uint32_t *counts,
                                        uint32_t *d_cand, uint64_t cand_cap, void *stream) {
  if (!d_offsets || !d_nbrs || !d_labels || !q || !counts || (cand_cap && !d_cand)) return GEM_ERR_ARG;
  HostQuery hq;
  std::string err;
  gem_status st = make_host_query(q, hq, err);
  if (st != GEM_OK) return st;
  if ((uint64_t)nv > GEM_STATIC_MAX_VERTICES) return GEM_ERR_LIMIT;
  const uint32_t nwords = (nv + 31) / 32;
  const uint64_t need = 2ull * nwords + 1 + scan_tmp_words(nwords);
  if (need + 1 > STATIC_SCRATCH_WORDS) return GEM_ERR_LIMIT;
  uint64_t *scratch = nullptr;
  st = static_scratch_address(&scratch);
  if (st != GEM_OK) return st;
  uint64_t *row = scratch, *ex = scratch + nwords, *tmp = scratch + 2ull * nwords + 1;
  uint32_t *bad = (uint32_t *)(scratch + STATIC_SCRATCH_WORDS - 1);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(bad, 0, 4, s) != cudaSuccess) {  // the previous call's flag
    cudaGetLastError();
    return GEM_ERR_CUDA;
  }
  // query description (same fields as gem_filter's)
  FilterDesc d;
  std::memset(&d, 0, sizeof d);
  d.nq = hq.nv;
  d.threshold = threshold;
  for (uint32_t u = 0; u < hq.nv; ++u) {
    d.lab[u] = hq.lab[u];
    d.deg[u] = hq.deg(u);
    uint32_t k = 0;
    while (k < d.nql && d.ql[k] != hq.lab[u]) ++k;
    if (k == d.nql) d.ql[d.nql++] = hq.lab[u];
  }
  for (uint32_t u = 0; u < hq.nv; ++u)
    for (uint32_t w = 0; w < hq.nv; ++w)
      if (hq.adj[u] & (1u << w)) {
        uint32_t k = 0;
        while (d.ql[k] != hq.lab[w]) ++k;
        d.nlc[u][k]++;
      }
  uint64_t at = 0;
  st = GEM_OK;
  for (uint32_t u = 0; u < hq.nv; ++u) {
    uint64_t blocks = (nwords + 7) / 8;
    if (blocks > 148ull * 16) blocks = 148ull * 16;
    if (blocks == 0) blocks = 1;
    count_launch();
    static_filter_row_kernel<<<(uint32_t)blocks, 256, 0, s>>>(d_offsets, d_nbrs, d_labels, nv, d, u, row, nwords,
                                                               bad);
    launch_scan(row, SCAN_POPC_U64LO, nwords, ex, tmp, s);
    uint64_t total = 0;
    uint32_t malformed = 0;
    if (cudaMemcpyAsync(&total, ex + nwords, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&malformed, bad, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      cudaGetLastError();
      return GEM_ERR_CUDA;
    }
    if (malformed) return GEM_ERR_ARG;  // not a CSR of nv vertices: nothing written for this row
    counts[u] = (uint32_t)total;
    if (at + total > cand_cap) {
      st = GEM_ERR_OVERFLOW;  // counts stay exact; lists stop here
      at += total;
      continue;
    }
    // write C(u) at d_cand + at (the row's list base is ex[0], always 0)
    launch_compact(row, ex, 1, nwords, ex, d_cand + at, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      cudaGetLastError();
      return GEM_ERR_CUDA;
    }
    at += total;
  }
  if (cudaGetLastError() != cudaSuccess) return GEM_ERR_CUDA;
  return st;
}
