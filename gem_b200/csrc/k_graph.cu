// Per-graph derived arrays (degrees, neighbour-label counts) and the
// device-wide exclusive scan used by the filter compaction and the table
// builder.
//
// The reference recomputes every data vertex's neighbour-label counts inside
// each query's filter kernel (in-core/lib/filter/src/filter_kernel.cu:196-232)
// and scans with CUB once per query vertex (in-core/lib/filter/src/filter.cu
// :81-100).  Here the counts are built once when the graph is loaded (one byte
// per (vertex, label), saturating at 255 — exact for the filter because query
// degrees are at most 31) and all rows of a wave share one flattened scan.
#include "device_common.cuh"
#include "kernels.h"

namespace gem {

std::atomic<uint64_t> g_launches{0};

__global__ void degrees_kernel(const uint64_t *__restrict__ off, uint32_t nv, uint32_t *__restrict__ deg) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = (uint32_t)(off[v + 1] - off[v]);
}

void launch_degrees(const DevGraph &g, uint32_t *deg, cudaStream_t s) {
  if (g.nv == 0) return;
  uint32_t blocks = (uint32_t)((g.nv + 255) / 256);
  if (blocks > 148u * 32u) blocks = 148u * 32u;
  count_launch();
  degrees_kernel<<<blocks, 256, 0, s>>>(g.off, g.nv, deg);
}

// One warp per vertex; a shared histogram per warp.
__global__ void __launch_bounds__(256) nlc_kernel(const uint64_t *__restrict__ off,
                                                  const uint32_t *__restrict__ nbr,
                                                  const uint32_t *__restrict__ lab, uint32_t nv,
                                                  uint32_t nlabels, uint8_t *__restrict__ nlc,
                                                  uint32_t stride) {
  __shared__ uint32_t hist[8][NLC_MAX_LABELS];
  const uint32_t lane = dev::lane_id(), w = threadIdx.x >> 5;
  const uint64_t nwarps = (uint64_t)gridDim.x * 8;
  for (uint64_t v = blockIdx.x * 8ull + w; v < nv; v += nwarps) {
    for (uint32_t l = lane; l < stride; l += 32) hist[w][l] = 0;
    __syncwarp();
    const uint64_t b = off[v], e = off[v + 1];
    for (uint64_t i = b + lane; i < e; i += 32) {
      uint32_t l = __ldg(lab + __ldg(nbr + i));
      if (l < nlabels) atomicAdd(&hist[w][l], 1u);
    }
    __syncwarp();
    for (uint32_t l = lane; l < stride; l += 32) {
      uint32_t c = hist[w][l];
      nlc[v * stride + l] = (uint8_t)(c > 255u ? 255u : c);
    }
    __syncwarp();
  }
}

void launch_nlc(const DevGraph &g, uint8_t *nlc, uint32_t stride, cudaStream_t s) {
  if (g.nv == 0) return;
  uint64_t warps = g.nv;
  uint64_t blocks = (warps + 7) / 8;
  if (blocks > 148ull * 64) blocks = 148ull * 64;
  count_launch();
  nlc_kernel<<<(uint32_t)blocks, 256, 0, s>>>(g.off, g.nbr, g.lab, g.nv, g.nlabels, nlc, stride);
}

// ---------------------------------------------------------------------------
// Exclusive scan: 2048 items per block (256 threads x 8 consecutive items).
// ---------------------------------------------------------------------------
// One warp per vertex inserts its neighbours into the vertex's table.
__global__ void __launch_bounds__(256) vnh_build_kernel(const uint64_t *__restrict__ off,
                                                        const uint32_t *__restrict__ nbr, uint32_t nv,
                                                        const uint64_t *__restrict__ hoff, uint32_t *slots) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t u = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); u < nv; u += nw) {
    const uint64_t b = hoff[u], size = hoff[u + 1] - b;
    if (!size) continue;
    const uint32_t lg = 63 - __clzll(size);
    for (uint64_t i = off[u] + lane; i < off[u + 1]; i += 32) {
      const uint32_t v = nbr[i];
      uint64_t pos = (v * VNH_MULT) >> (64 - lg);
      for (uint64_t k = 0; k < size; ++k) {  // size >= 2 deg: a free slot exists
        const uint32_t prev = atomicCAS(slots + b + pos, VNH_EMPTY, v);
        if (prev == VNH_EMPTY || prev == v) break;
        pos = (pos + 1) & (size - 1);
      }
    }
  }
}

void launch_vnh_build(const DevGraph &g, const uint64_t *hoff, uint32_t *slots, uint64_t n_slots,
                      cudaStream_t s) {
  if (!g.nv || !n_slots) return;
  cudaMemsetAsync(slots, 0xFF, n_slots * 4, s);
  uint64_t blocks = ((uint64_t)g.nv + 7) / 8;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  count_launch();
  vnh_build_kernel<<<(uint32_t)blocks, 256, 0, s>>>(g.off, g.nbr, g.nv, hoff, slots);
}

constexpr uint32_t SCAN_T = 256, SCAN_I = 8, SCAN_B = SCAN_T * SCAN_I;

template <ScanInput K>
__device__ __forceinline__ uint32_t scan_item(const void *in, uint64_t i) {
  if (K == SCAN_POPC_U64LO) return (uint32_t)__popc((uint32_t)__ldg((const uint64_t *)in + i));
  if (K == SCAN_POPC_U32) return (uint32_t)__popc(__ldg((const uint32_t *)in + i));
  return __ldg((const uint32_t *)in + i);
}

// Exclusive block scan of one u64 per thread; returns the block total in *total.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t x, uint64_t *total) {
  __shared__ uint64_t wsum[SCAN_T / 32];
  const uint32_t lane = dev::lane_id(), w = threadIdx.x >> 5;
  uint64_t inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint64_t y = __shfl_up_sync(dev::FULL, inc, d);
    if (lane >= (uint32_t)d) inc += y;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint64_t v = lane < SCAN_T / 32 ? wsum[lane] : 0, vi = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint64_t y = __shfl_up_sync(dev::FULL, vi, d);
      if (lane >= (uint32_t)d) vi += y;
    }
    if (lane < SCAN_T / 32) wsum[lane] = vi - v;
    if (lane == SCAN_T / 32 - 1) *total = vi;
  }
  __syncthreads();
  uint64_t r = wsum[w] + inc - x;
  __syncthreads();
  return r;
}

// A thread's SCAN_I consecutive items: 16-byte loads when they are whole
// and the input is 16-byte aligned, else one by one.
template <ScanInput K>
__device__ __forceinline__ void scan_items(const void *in, uint64_t n, uint64_t base, uint32_t (&v)[SCAN_I]) {
  if (base + SCAN_I <= n && ((uintptr_t)in & 15u) == 0) {
    if (K == SCAN_POPC_U64LO) {
      const uint4 *p = (const uint4 *)((const uint64_t *)in + base);
#pragma unroll
      for (uint32_t j = 0; j < SCAN_I / 2; ++j) {
        const uint4 a = __ldg(p + j);
        v[2 * j] = __popc(a.x);
        v[2 * j + 1] = __popc(a.z);
      }
    } else {
      const uint4 *p = (const uint4 *)((const uint32_t *)in + base);
#pragma unroll
      for (uint32_t j = 0; j < SCAN_I / 4; ++j) {
        const uint4 a = __ldg(p + j);
        v[4 * j] = K == SCAN_POPC_U32 ? __popc(a.x) : a.x;
        v[4 * j + 1] = K == SCAN_POPC_U32 ? __popc(a.y) : a.y;
        v[4 * j + 2] = K == SCAN_POPC_U32 ? __popc(a.z) : a.z;
        v[4 * j + 3] = K == SCAN_POPC_U32 ? __popc(a.w) : a.w;
      }
    }
    return;
  }
#pragma unroll
  for (uint32_t j = 0; j < SCAN_I; ++j) v[j] = base + j < n ? scan_item<K>(in, base + j) : 0u;
}

template <ScanInput K>
__global__ void __launch_bounds__(SCAN_T) scan_partial_kernel(const void *in, uint64_t n, uint64_t *part) {
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_B + (uint64_t)threadIdx.x * SCAN_I;
  uint32_t v[SCAN_I];
  scan_items<K>(in, n, base, v);
  uint64_t s = 0;
#pragma unroll
  for (uint32_t j = 0; j < SCAN_I; ++j) s += v[j];
  __shared__ uint64_t tot;
  (void)block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// Single block: exclusive scan of nb partials in place; part[nb] = total.
__global__ void __launch_bounds__(1024) scan_top_kernel(uint64_t *part, uint64_t nb, uint64_t *out, uint64_t n) {
  __shared__ uint64_t wsum[32];
  __shared__ uint64_t carry_s;
  const uint32_t lane = dev::lane_id(), w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (uint64_t base = 0; base < nb; base += 1024) {
    uint64_t i = base + threadIdx.x;
    uint64_t x = i < nb ? part[i] : 0, inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint64_t y = __shfl_up_sync(dev::FULL, inc, d);
      if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
      uint64_t v = wsum[lane], vi = v;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint64_t y = __shfl_up_sync(dev::FULL, vi, d);
        if (lane >= (uint32_t)d) vi += y;
      }
      wsum[lane] = vi - v;
    }
    __syncthreads();
    uint64_t carry = carry_s;
    uint64_t ex = carry + wsum[w] + inc - x;
    if (i < nb) part[i] = ex;
    __syncthreads();
    if (threadIdx.x == 1023) carry_s = ex + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[nb] = carry_s;
    out[n] = carry_s;
  }
}

template <ScanInput K>
__global__ void __launch_bounds__(SCAN_T) scan_final_kernel(const void *in, uint64_t n, const uint64_t *part,
                                                            uint64_t *out) {
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_B + (uint64_t)threadIdx.x * SCAN_I;
  uint32_t v[SCAN_I];
  scan_items<K>(in, n, base, v);
  uint64_t s = 0;
#pragma unroll
  for (uint32_t j = 0; j < SCAN_I; ++j) s += v[j];
  __shared__ uint64_t tot;
  uint64_t ex = block_exclusive_scan(s, &tot) + part[blockIdx.x];
  uint64_t o[SCAN_I];
#pragma unroll
  for (uint32_t j = 0; j < SCAN_I; ++j) {
    o[j] = ex;
    ex += v[j];
  }
  if (base + SCAN_I <= n && ((uintptr_t)(out + base) & 15u) == 0) {
    ulonglong2 *q = (ulonglong2 *)(out + base);  // 16-byte stores
#pragma unroll
    for (uint32_t j = 0; j < SCAN_I / 2; ++j) q[j] = make_ulonglong2(o[2 * j], o[2 * j + 1]);
  } else {
#pragma unroll
    for (uint32_t j = 0; j < SCAN_I; ++j)
      if (base + j < n) out[base + j] = o[j];
  }
}

__global__ void gather_strided_kernel(const uint64_t *__restrict__ in, uint64_t stride, uint32_t n,
                                      uint64_t *__restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i * stride];
}

void launch_gather_strided(const uint64_t *in, uint64_t stride, uint32_t n, uint64_t *out, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  gather_strided_kernel<<<(n + 255) / 256, 256, 0, s>>>(in, stride, n, out);
}

__global__ void set_deadline_kernel(unsigned long long *deadline, unsigned long long cap_ns) {
  *deadline = dev::globaltimer_ns() + cap_ns;
}

void launch_set_deadline(unsigned long long *deadline, uint64_t cap_ns, cudaStream_t s) {
  count_launch();
  set_deadline_kernel<<<1, 1, 0, s>>>(deadline, cap_ns);
}

uint64_t scan_tmp_words(uint64_t n) { return (n + SCAN_B - 1) / SCAN_B + 2; }

void launch_scan(const void *in, ScanInput kind, uint64_t n, uint64_t *out, uint64_t *tmp, cudaStream_t s) {
  const uint64_t nb = (n + SCAN_B - 1) / SCAN_B;
  if (n == 0) {
    cudaMemsetAsync(out, 0, sizeof(uint64_t), s);
    return;
  }
  switch (kind) {
    case SCAN_POPC_U64LO:
      count_launch();
      scan_partial_kernel<SCAN_POPC_U64LO><<<(uint32_t)nb, SCAN_T, 0, s>>>(in, n, tmp);
      count_launch();
      scan_top_kernel<<<1, 1024, 0, s>>>(tmp, nb, out, n);
      count_launch();
      scan_final_kernel<SCAN_POPC_U64LO><<<(uint32_t)nb, SCAN_T, 0, s>>>(in, n, tmp, out);
      break;
    case SCAN_POPC_U32:
      count_launch();
      scan_partial_kernel<SCAN_POPC_U32><<<(uint32_t)nb, SCAN_T, 0, s>>>(in, n, tmp);
      count_launch();
      scan_top_kernel<<<1, 1024, 0, s>>>(tmp, nb, out, n);
      count_launch();
      scan_final_kernel<SCAN_POPC_U32><<<(uint32_t)nb, SCAN_T, 0, s>>>(in, n, tmp, out);
      break;
    default:
      count_launch();
      scan_partial_kernel<SCAN_U32><<<(uint32_t)nb, SCAN_T, 0, s>>>(in, n, tmp);
      count_launch();
      scan_top_kernel<<<1, 1024, 0, s>>>(tmp, nb, out, n);
      count_launch();
      scan_final_kernel<SCAN_U32><<<(uint32_t)nb, SCAN_T, 0, s>>>(in, n, tmp, out);
      break;
  }
}

}  // namespace gem
