// Edge-candidate tables T(u -> w): for the i-th candidate v of C(u), the
// neighbours of v that are candidates of w, in adjacency order.
//
// The reference (in-core/lib/structure/src/unifiedTrie.cu:1093-1240 with the
// kernels of construct_kernel.cu:1183-1340) runs, per directed query edge, a
// count kernel over 32-neighbour tiles, a CUB scan over the tiles of the
// *whole* data graph, a max kernel and a write kernel, with host syncs in
// between.  Here all tables of a wave share each launch, and the passes walk
// the data graph's vertex tiles (32 arcs of one vertex) once: each tile
// serves every source row whose candidates hold its vertex (in a batch of
// queries a vertex is a candidate of many rows), and membership of an arc's
// target in every target row is one word of that target's membership
// column, staged in shared memory.  The tables keep the per-source layout
// (a key's values at the key's tiles of its source), so the offsets, the
// scans and the join see the same tables as a pass over each source would
// write.
#include "device_common.cuh"
#include "kernels.h"

namespace gem {

__device__ __forceinline__ uint32_t find_src(const TabSource *__restrict__ src, uint32_t nsrc, uint64_t k) {
  uint32_t lo = 0, hi = nsrc;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (src[mid].key_base <= k) lo = mid; else hi = mid;
  }
  return lo;
}


__global__ void key_tiles_kernel(DevGraph g, const TabSource *__restrict__ src, uint32_t nsrc, uint64_t nkeys,
                                 uint32_t *__restrict__ tiles) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nkeys; k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s = find_src(src, nsrc, k);
    uint32_t v = __ldg(src[s].keys + (k - src[s].key_base));
    tiles[k] = (__ldg(g.deg + v) + 31u) >> 5;
  }
}


void launch_key_tiles(const DevGraph &g, const TabSource *d_src, uint32_t nsrc, uint64_t nkeys, uint32_t *tiles,
                      cudaStream_t s) {
  if (nkeys == 0) return;
  uint64_t blocks = (nkeys + 255) / 256;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  count_launch();
  key_tiles_kernel<<<(uint32_t)blocks, 256, 0, s>>>(g, d_src, nsrc, nkeys, tiles);
}

__global__ void source_tile_bases_kernel(const TabSource *__restrict__ src, uint32_t nsrc, uint64_t nkeys,
                                         const uint64_t *__restrict__ tp, uint64_t *__restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= nsrc; i += gridDim.x * blockDim.x)
    out[i] = tp[i < nsrc ? src[i].key_base : nkeys];
}

void launch_source_tile_bases(const TabSource *d_src, uint32_t nsrc, uint64_t nkeys, const uint64_t *tp,
                              uint64_t *out, cudaStream_t s) {
  count_launch();
  source_tile_bases_kernel<<<(nsrc + 256) / 256, 256, 0, s>>>(d_src, nsrc, nkeys, tp, out);
}

// Membership columns: out[v * W + c] holds, in bit b, whether vertex v is in
// row rows[32c + b] (bits: the wave's membership bit rows, 32 vertices per
// word).  One block per 32-vertex word j: each warp transposes 32 rows x 32
// vertices with 32 ballots.  With vtiles, vtiles[v] = ceil(deg(v) / 32) for a
// vertex in at least one of the rows, else 0.
__global__ void __launch_bounds__(256) row_columns_kernel(const uint32_t *__restrict__ bits, uint32_t nwords,
                                                          const uint32_t *__restrict__ rows, uint32_t nrows,
                                                          uint32_t W, uint32_t nv, uint32_t *__restrict__ out,
                                                          uint32_t *__restrict__ vtiles,
                                                          const uint32_t *__restrict__ deg) {
  __shared__ uint32_t any[32];
  const uint32_t lane = dev::lane_id(), warp = threadIdx.x >> 5;
  for (uint32_t j = blockIdx.x; j < nwords; j += gridDim.x) {
    if (threadIdx.x < 32) any[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t v = j * 32u + lane;
    uint32_t seen = 0;
    for (uint32_t c = warp; c < W; c += blockDim.x >> 5) {
      const uint32_t r = c * 32u + lane;
      const uint32_t word = r < nrows ? __ldg(bits + (uint64_t)__ldg(rows + r) * nwords + j) : 0u;
      uint32_t col = 0;
#pragma unroll
      for (uint32_t b = 0; b < 32; ++b) {
        const uint32_t m = __ballot_sync(dev::FULL, (word >> b) & 1u);
        if (lane == b) col = m;
      }
      if (v < nv) out[(uint64_t)v * W + c] = col;
      seen |= col;
    }
    if (vtiles) {
      if (seen) atomicOr(any + lane, 1u);
      __syncthreads();
      if (warp == 0 && v < nv) vtiles[v] = any[lane] ? (__ldg(deg + v) + 31u) >> 5 : 0u;
    }
    __syncthreads();  // any[] is reset by the next word
  }
}

void launch_row_columns(const uint32_t *bits, uint32_t nwords, const uint32_t *rows, uint32_t nrows, uint32_t W,
                        uint32_t nv, uint32_t *out, uint32_t *vtiles, const uint32_t *deg, cudaStream_t s) {
  if (nwords == 0) return;
  uint32_t blocks = nwords < 148u * 16 ? nwords : 148u * 16;
  count_launch();
  row_columns_kernel<<<blocks, 256, 0, s>>>(bits, nwords, rows, nrows, W, nv, out, vtiles, deg);
}

// vt[t] = v for every tile t in [vtp[v], vtp[v + 1]).
__global__ void vertex_tile_map_kernel(const uint64_t *__restrict__ vtp, uint32_t nv, uint32_t *__restrict__ vt) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    for (uint64_t t = __ldg(vtp + v), e = __ldg(vtp + v + 1); t < e; ++t) vt[t] = v;
}

void launch_vertex_tile_map(const uint64_t *vtp, uint32_t nv, uint32_t *vt, cudaStream_t s) {
  if (nv == 0) return;
  uint32_t blocks = (nv + 255) / 256;
  if (blocks > 148u * 16) blocks = 148u * 16;
  count_launch();
  vertex_tile_map_kernel<<<blocks, 256, 0, s>>>(vtp, nv, vt);
}

__global__ void unit_counts_kernel(const uint32_t *__restrict__ vtiles, uint32_t nv, uint32_t *__restrict__ out) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    out[v] = (__ldg(vtiles + v) + TAB_WGROUP - 1) / TAB_WGROUP;
}

void launch_unit_counts(const uint32_t *vtiles, uint32_t nv, uint32_t *out, cudaStream_t s) {
  if (nv == 0) return;
  uint32_t blocks = (nv + 255) / 256;
  if (blocks > 148u * 16) blocks = 148u * 16;
  count_launch();
  unit_counts_kernel<<<blocks, 256, 0, s>>>(vtiles, nv, out);
}

__global__ void gather_u64_kernel(const uint64_t *__restrict__ a, const uint32_t *__restrict__ idx, uint32_t n,
                                  uint64_t *__restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = __ldg(a + __ldg(idx + i));
}

void launch_gather_u64(const uint64_t *a, const uint32_t *idx, uint32_t n, uint64_t *out, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  gather_u64_kernel<<<(n + 255) / 256, 256, 0, s>>>(a, idx, n, out);
}

// 16-byte asynchronous copy global -> shared (both 16-byte aligned),
// bypassing L1; cp_async_wait_all waits for this thread's copies.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Position of the (r + 1)-th set bit of m (r < popc(m)).
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t r) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t w = 16; w >= 1; w >>= 1) {
    const uint32_t low = __popc(m & ((1u << w) - 1u));
    if (r >= low) {
      r -= low;
      m >>= w;
      pos += w;
    }
  }
  return pos;
}

// The table passes over vertex tiles.  One warp per tile (32 arcs of one
// vertex v): the arcs are read once for every source whose candidates hold
// v.  Those sources are the set bits of v's source column; the warp takes
// them 32 at a time, one per lane, and each lane computes its source's key
// position of v (rank bitmap) and tile index (tp).  The tables of those
// sources are then flattened into (source, table) pairs, again one per
// lane, 32 at a time:
//   count: each lane tests its table's target column bit (tcol) for the 32
//          arcs of the tile (the warp stages the arcs' target columns in
//          shared memory, one column per arc) and writes the tile's mask;
//   write: each lane reads its pair's mask and value position into a
//          per-warp record (records of empty masks dropped); then for each
//          record the lanes, one per arc, write the arcs whose bit is set
//          (and the key position) at the value position plus their rank in
//          the mask.
// The mask and value positions are those of the source's own tile order
// (mask[tile_base + lt], lt = the tile's index among the source's tiles), so
// both passes lay out every table exactly as a pass over the sources would.
constexpr uint32_t TAB_GRAB = 1;  // units a warp takes from the counter at a time (1: the narrowest window)

struct VRec {
  uint64_t vb;  // first value position of the pair's tile
  uint32_t m;   // the tile's mask
  uint32_t kf;  // key position to record, or 0xFFFFFFFF (no key map)
};

template <bool WRITE>
__global__ void __launch_bounds__(256) table_vtx_kernel(VPass P) {
  constexpr uint32_t G = WRITE ? TAB_WGROUP : 1u;  // tiles of one vertex per unit
  extern __shared__ uint32_t stage[];  // count: 32 target columns per warp
  __shared__ VRec rec[WRITE ? 8 : 1][32 * G];  // write: the records of one round
  const uint32_t lane = dev::lane_id(), warp = threadIdx.x >> 5;
  for (;;) {
    // units are taken in order from one counter, so the units in flight
    // stay a narrow window of consecutive vertices
    unsigned long long got = 0;
    if (lane == 0) got = atomicAdd(P.next, (unsigned long long)TAB_GRAB);
    const uint64_t t0 = P.t0 + __shfl_sync(dev::FULL, got, 0);
    if (t0 >= P.t1) break;
    const uint64_t t1 = t0 + TAB_GRAB < P.t1 ? t0 + TAB_GRAB : P.t1;
    for (uint64_t t = t0; t < t1; ++t) {
    // the unit: tiles c .. c + nt - 1 of vertex v
    uint32_t v, nt = 1;
    uint64_t c;
    if (WRITE) {
      v = __ldg(P.vg + t);
      c = (t - __ldg(P.vgp + v)) * G;
      const uint64_t tv = __ldg(P.vtp + v + 1) - __ldg(P.vtp + v);
      nt = tv - c < G ? (uint32_t)(tv - c) : G;
    } else {
      v = __ldg(P.vt + t);
      c = t - __ldg(P.vtp + v);
    }
    const uint64_t a0 = __ldg(P.off + v), a1 = __ldg(P.off + v + 1);
    uint32_t xs[G];
#pragma unroll
    for (uint32_t i = 0; i < G; ++i) {
      const uint64_t arc = a0 + (c + i) * 32u + lane;
      xs[i] = i < nt && arc < a1 ? __ldg(P.nbr + (arc - P.arc_shift)) : 0u;
    }
    const bool valid = a0 + c * 32u + lane < a1;  // lane's arc of the unit's first tile
    const uint32_t nvalid = a1 - a0 - c * 32u < 32u ? (uint32_t)(a1 - a0 - c * 32u) : 32u;  // valid lanes: a prefix
    const uint32_t x = xs[0];
    if (!WRITE) {
      // stage the target columns of the tile's arcs with asynchronous 16-byte
      // copies (all in flight at once): lane = (row in group, 16-byte chunk)
      __syncwarp();  // the previous tile's reads of the stage are done
      const uint32_t ch = P.WT >> 2, rpi = 32u / ch;  // chunks per column, columns per round
      const uint32_t r = lane / ch, q = lane - r * ch;
      uint32_t *wst = stage + (uint64_t)warp * 32u * P.WTp;
      for (uint32_t g = 0; g < nvalid; g += rpi) {
        const uint32_t l = g + r;
        const uint32_t xl = __shfl_sync(dev::FULL, x, l < 32u ? l : 0u);
        if (r < rpi && l < nvalid) cp_async16(wst + l * P.WTp + q * 4u, P.B + (uint64_t)xl * P.WT + q * 4u);
      }
      cp_async_wait_all();
      __syncwarp();
    }
    const uint32_t *sv = P.S + (uint64_t)v * P.WS;
    for (uint32_t wb = 0; wb < P.WS; wb += 32) {
      const uint32_t word = wb + lane < P.WS ? __ldg(sv + wb + lane) : 0u;
      const uint32_t cnt = __popc(word);
      uint32_t incl = cnt;
#pragma unroll
      for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(dev::FULL, incl, d);
        if (lane >= d) incl += y;
      }
      const uint32_t total = __shfl_sync(dev::FULL, incl, 31);
      for (uint32_t b = 0; b < total; b += 32) {
        // lane i takes the (b + i)-th source of this word range: the first
        // lane j whose inclusive count exceeds it holds it
        const uint32_t q = b + lane;
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step >= 1; step >>= 1)
          if (__shfl_sync(dev::FULL, incl, j + step - 1) <= q) j += step;
        const uint32_t wj = __shfl_sync(dev::FULL, word, j);
        const uint32_t exj = __shfl_sync(dev::FULL, incl - cnt, j);
        uint32_t k = 0, e0 = 0, ne = 0;
        uint64_t lt = 0;
        if (q < total) {
          const VSrc &src = P.vsrc[(wb + j) * 32u + nth_set_bit(wj, q - exj)];
          const uint64_t rw = __ldg(src.rb + (v >> 5));
          k = (uint32_t)(rw >> 32) + __popc((uint32_t)rw & ((1u << (v & 31u)) - 1u));
          lt = __ldg(P.tp + src.key_base + k) - src.stb + c;
          e0 = src.e0;
          ne = src.ne;
        }
        // the (source, table) pairs of these sources, one per lane
        uint32_t pin = ne;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
          const uint32_t y = __shfl_up_sync(dev::FULL, pin, d);
          if (lane >= d) pin += y;
        }
        const uint32_t npairs = __shfl_sync(dev::FULL, pin, 31);
        for (uint32_t pb = 0; pb < npairs; pb += 32) {
          const uint32_t p = pb + lane;
          uint32_t o = 0;  // the source lane of pair p
#pragma unroll
          for (uint32_t step = 16; step >= 1; step >>= 1)
            if (__shfl_sync(dev::FULL, pin, o + step - 1) <= p) o += step;
          const uint32_t u = p - (__shfl_sync(dev::FULL, pin, o) - __shfl_sync(dev::FULL, ne, o));
          const uint32_t pe = __shfl_sync(dev::FULL, e0, o) + u;
          const uint64_t plt = __shfl_sync(dev::FULL, lt, o);
          const uint32_t pk = __shfl_sync(dev::FULL, k, o);
          const bool have = p < npairs;
          const VEdge E = have ? P.vedge[pe] : VEdge{0, 0, 0};
          const uint64_t maddr = E.tile_base + plt;
          if (!WRITE) {
            const uint32_t *col = stage + (uint64_t)warp * 32u * P.WTp + (E.tcol >> 5);
            const uint32_t sh = E.tcol & 31u, st = P.WTp;
            uint32_t m = 0, l = 0;
            for (; l + 4 <= nvalid; l += 4) {
              const uint32_t w0 = col[l * st], w1 = col[(l + 1) * st], w2 = col[(l + 2) * st], w3 = col[(l + 3) * st];
              m |= (((w0 >> sh) & 1u) | (((w1 >> sh) & 1u) << 1) | (((w2 >> sh) & 1u) << 2) | (((w3 >> sh) & 1u) << 3)) << l;
            }
            for (; l < nvalid; ++l) m |= ((col[l * st] >> sh) & 1u) << l;
            if (have) P.mask[maddr] = m;
          } else {
            // records of the pair's tiles that have values, packed to the
            // front; the tile's index in the unit rides in the top byte of
            // the value position.  A key's tiles are consecutive in its
            // source's tile order, so the unit's masks and positions are
            // consecutive words.
            const uint32_t kf = have && (E.flags & TAB_KEY_MAP) ? pk : 0xFFFFFFFFu;
            const uint32_t below = (1u << lane) - 1u;
            uint32_t m[G];
            uint64_t vb[G];
#pragma unroll
            for (uint32_t i = 0; i < G; ++i) {
              m[i] = have && i < nt ? __ldg(P.mask + maddr + i) : 0u;
              vb[i] = have && i < nt ? __ldg(P.vp + maddr + i) : 0ull;
            }
            __syncwarp();  // the previous round's records are read
            uint32_t nr = 0;
#pragma unroll
            for (uint32_t i = 0; i < G; ++i) {
              const uint32_t nz = __ballot_sync(dev::FULL, m[i] != 0u);
              if (m[i]) rec[warp][nr + __popc(nz & below)] = VRec{vb[i] | ((uint64_t)i << 56), m[i], kf};
              nr += __popc(nz);
            }
            __syncwarp();
            for (uint32_t i = 0; i < nr; ++i) {
              const VRec r0 = rec[warp][i];
              if ((r0.m >> lane) & 1u) {
                const uint32_t ti = (uint32_t)(r0.vb >> 56);
                uint32_t xi = xs[0];
#pragma unroll
                for (uint32_t j = 1; j < G; ++j) xi = ti == j ? xs[j] : xi;
                const uint64_t pos = (r0.vb & ((1ull << 56) - 1)) + __popc(r0.m & below);
                P.values[pos] = xi;
                if (r0.kf != 0xFFFFFFFFu) P.vkey[pos] = r0.kf;
              }
            }
          }
        }
      }
    }
    }
  }
}

// Warps per block of the count pass: each warp stages 32 target columns of
// WTp words; blocks stay within 96 KB of shared memory so that two fit an SM.
static uint32_t count_warps(uint32_t WTp) {
  const uint64_t per_warp = 32ull * WTp * 4;
  const uint64_t w = (96ull << 10) / per_warp;
  return w > 8 ? 8u : w < 1 ? 1u : (uint32_t)w;
}

// Target columns are staged in 16-byte chunks, at most one per lane per
// column: WT (a multiple of 4) words up to 128.
bool table_vtx_fits(uint32_t WT) { return WT % 4 == 0 && WT >= 4 && WT <= 128; }

// Persistent grid: what the SMs hold at once (blocks per SM by occupancy).
// Its warps take tiles in order from the launch's counter, so the tiles in
// flight are a window of consecutive vertices, and the rank words, tile
// bases, masks and positions they read are the same few lines per source
// and table, which stay in L2 while the window passes (a static stride lets
// the warps drift apart until they touch the whole order at once).
static uint32_t resident_blocks(const void *fn, int threads, size_t smem, uint64_t want) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  uint64_t b = (uint64_t)(sms > 0 ? sms : 148) * (uint64_t)(per_sm > 0 ? per_sm : 1);
  if (b > want) b = want;
  return (uint32_t)(b ? b : 1);
}

void launch_table_vtx(const VPass &P0, bool write, cudaStream_t s) {
  if (P0.t1 <= P0.t0) return;
  VPass P = P0;
  P.WTp = P.WT;  // the lanes of a pair round read one staged column each: no stride padding
  const uint32_t warps = write ? 8u : count_warps(P.WTp);
  const uint64_t want = (P.t1 - P.t0 + warps - 1) / warps;
  cudaMemsetAsync(P.next, 0, sizeof(unsigned long long), s);
  count_launch();
  if (write) {
    const uint32_t blocks = resident_blocks((const void *)table_vtx_kernel<true>, 256, 0, want);
    table_vtx_kernel<true><<<blocks, 256, 0, s>>>(P);
  } else {
    const size_t smem = (size_t)warps * 32 * P.WTp * 4;
    cudaFuncSetAttribute(table_vtx_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const uint32_t blocks = resident_blocks((const void *)table_vtx_kernel<false>, (int)warps * 32, smem, want);
    table_vtx_kernel<false><<<blocks, warps * 32, smem, s>>>(P);
  }
}

__global__ void edge_value_bases_kernel(const TabEdge *__restrict__ edges, uint32_t nedge,
                                       const uint64_t *__restrict__ vp, uint64_t tiles, uint64_t *__restrict__ out) {
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e <= nedge; e += gridDim.x * blockDim.x)
    out[e] = vp[e < nedge ? edges[e].tile_base : tiles];
}

void launch_edge_value_bases(const TabEdge *d_edge, uint32_t nedge, const uint64_t *vp, uint64_t tiles,
                             uint64_t *out, cudaStream_t s) {
  count_launch();
  edge_value_bases_kernel<<<(nedge + 256) / 256, 256, 0, s>>>(d_edge, nedge, vp, tiles, out);
}

__device__ __forceinline__ uint32_t find_edge_off(const TabEdge *__restrict__ e, uint32_t ne, uint64_t i) {
  uint32_t lo = 0, hi = ne;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (e[mid].off_base <= i) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void table_offsets_kernel(const TabSource *__restrict__ srcs, const TabEdge *__restrict__ edges,
                                     uint32_t nedge, const uint64_t *__restrict__ tp, const uint64_t *__restrict__ vp,
                                     uint64_t total) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e = find_edge_off(edges, nedge, i);
    const TabEdge E = edges[e];
    const TabSource S = srcs[E.src];
    const uint64_t key = i - E.off_base;  // 0..nkeys
    const uint64_t lt = tp[S.key_base + key] - tp[S.key_base];
    E.offsets[key] = vp[E.tile_base + lt];
  }
}

void launch_table_offsets(const TabSource *d_src, const TabEdge *d_edge, uint32_t nedge, const uint64_t *tp,
                          const uint64_t *vp, uint64_t total_offsets, cudaStream_t s) {
  if (total_offsets == 0) return;
  uint64_t blocks = (total_offsets + 255) / 256;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  count_launch();
  table_offsets_kernel<<<(uint32_t)blocks, 256, 0, s>>>(d_src, d_edge, nedge, tp, vp, total_offsets);
}

}  // namespace gem
