// Edge-candidate tables T(u -> w): for the i-th candidate v of C(u), the
// neighbours of v that are candidates of w, in adjacency order.
//
// The reference (in-core/lib/structure/src/unifiedTrie.cu:1093-1240 with the
// kernels of construct_kernel.cu:1183-1340) runs, per directed query edge, a
// count kernel over 32-neighbour tiles, a CUB scan over the tiles of the
// *whole* data graph, a max kernel and a write kernel, with host syncs in
// between.  Here the tile space is compacted to the arcs of C(u) only, all
// edges of a wave share each launch, every warp owns a fixed run of tiles (so
// hub vertices do not serialise on one warp), and membership in C(w) is one
// bit of w's rank bitmap.
#include "device_common.cuh"
#include "kernels.h"

namespace gem {

// Last index i in [lo, hi) with a[i] <= x (requires a[lo] <= x).
__device__ __forceinline__ uint64_t last_le(const uint64_t *__restrict__ a, uint64_t lo, uint64_t hi, uint64_t x) {
  while (hi - lo > 1) {
    uint64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= x) lo = mid; else hi = mid;
  }
  return lo;
}

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

// Tile t of the flattened source-tile space (the 32-arc tiles of every key of
// every source): the key it belongs to and its source.
__global__ void tile_keys_kernel(const TabSource *__restrict__ src, uint32_t nsrc, uint64_t nkeys,
                                 const uint64_t *__restrict__ tp, uint32_t *__restrict__ tkey,
                                 uint32_t *__restrict__ tsrc) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nkeys; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = find_src(src, nsrc, k);
    for (uint64_t t = tp[k], e = tp[k + 1]; t < e; ++t) {
      tkey[t] = (uint32_t)k;
      tsrc[t] = s;
    }
  }
}

void launch_tile_keys(const TabSource *d_src, uint32_t nsrc, uint64_t nkeys, const uint64_t *tp, uint32_t *tkey,
                      uint32_t *tsrc, cudaStream_t s) {
  if (nkeys == 0) return;
  uint64_t blocks = (nkeys + 255) / 256;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  count_launch();
  tile_keys_kernel<<<(uint32_t)blocks, 256, 0, s>>>(d_src, nsrc, nkeys, tp, tkey, tsrc);
}

// One warp per TILE_UNROLL consecutive source tiles: the tiles' key, vertex,
// offsets and neighbour loads are independent and overlap; each tile is then
// tested against (count) or copied for (write) every edge of its source, so
// a source's adjacency is read once however many tables it keys.  The warps
// cover positions [t0, t1) of the tile order `tord` (identity when null), and
// a key's arcs are read at nbr[arc - arc_shift]: the resident (or mapped)
// adjacency with shift 0, or a streamed partition that starts at arc_shift.
constexpr int TILE_UNROLL = 4;

template <bool WRITE>
__global__ void __launch_bounds__(256) table_src_kernel(TabPass P, const TabSource *__restrict__ srcs,
                                                        const uint32_t *__restrict__ sedge,
                                                        const TabEdge *__restrict__ edges,
                                                        const uint64_t *__restrict__ tp,
                                                        const uint32_t *__restrict__ tkey,
                                                        const uint32_t *__restrict__ tsrc,
                                                        uint32_t *__restrict__ mask, const uint64_t *__restrict__ vp,
                                                        uint32_t *__restrict__ values, uint32_t *__restrict__ vkey) {
  const uint32_t lane = dev::lane_id();
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t base = P.t0 + (blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5)) * TILE_UNROLL;
       base < P.t1; base += nwarps * TILE_UNROLL) {
    uint32_t x[TILE_UNROLL], sx[TILE_UNROLL], kx[TILE_UNROLL];
    uint64_t lt[TILE_UNROLL];
    bool xv[TILE_UNROLL];
#pragma unroll
    for (int i = 0; i < TILE_UNROLL; ++i) {
      const bool tv = base + i < P.t1;
      const uint64_t t = !tv ? 0ull : P.tord ? (uint64_t)__ldg(P.tord + base + i) : base + i;
      const uint32_t k = tv ? __ldg(tkey + t) : 0u, sidx = tv ? __ldg(tsrc + t) : 0u;
      const uint64_t kb = srcs[sidx].key_base;
      const uint32_t *keys = srcs[sidx].keys;
      const uint32_t v = tv ? __ldg(keys + (k - kb)) : 0u;
      const uint64_t tk = tv ? __ldg(tp + k) : 0ull, stb = tv ? __ldg(tp + kb) : 0ull;
      const uint64_t a0 = tv ? __ldg(P.off + v) : 0ull, a1 = tv ? __ldg(P.off + v + 1) : 0ull;
      const uint64_t arc = a0 + (t - tk) * 32 + lane;
      sx[i] = sidx;
      kx[i] = (uint32_t)(k - kb);  // the key's position in its source's candidate list
      lt[i] = t - stb;  // the tile's index among its source's tiles
      xv[i] = tv && arc < a1;
      x[i] = xv[i] ? __ldg(P.nbr + (arc - P.arc_shift)) : 0u;
    }
    // Common case: the warp's tiles all belong to one source (a source has
    // many tiles).  Then each table of the source is read once for all of
    // them, and its TILE_UNROLL membership probes (count) or mask / position
    // loads (write) are issued together.
    bool same = base + TILE_UNROLL <= P.t1;
#pragma unroll
    for (int i = 1; i < TILE_UNROLL; ++i) same = same && sx[i] == sx[0];
    if (same) {
      const uint32_t e0 = __ldg(sedge + 2 * sx[0]), ne = __ldg(sedge + 2 * sx[0] + 1);
      for (uint32_t e = e0; e < e0 + ne; ++e) {
        const uint64_t tb = edges[e].tile_base;
        if (!WRITE) {
          const uint32_t *bw = edges[e].bits_w;
          bool hit[TILE_UNROLL];
#pragma unroll
          for (int i = 0; i < TILE_UNROLL; ++i) hit[i] = xv[i] && ((__ldg(bw + (x[i] >> 5)) >> (x[i] & 31u)) & 1u);
#pragma unroll
          for (int i = 0; i < TILE_UNROLL; ++i) {
            const uint32_t m = __ballot_sync(dev::FULL, hit[i]);
            if (lane == 0) mask[tb + lt[i]] = m;
          }
        } else {
          uint32_t m[TILE_UNROLL];
          uint64_t vb[TILE_UNROLL];
#pragma unroll
          for (int i = 0; i < TILE_UNROLL; ++i) {
            m[i] = __ldg(mask + tb + lt[i]);
            vb[i] = __ldg(vp + tb + lt[i]);
          }
          const bool km = (edges[e].flags & TAB_KEY_MAP) != 0;
#pragma unroll
          for (int i = 0; i < TILE_UNROLL; ++i)
            if (m[i] & (1u << lane)) {
              const uint64_t pos = vb[i] + __popc(m[i] & ((1u << lane) - 1u));
              values[pos] = x[i];
              if (km) vkey[pos] = kx[i];
            }
        }
      }
      continue;
    }
#pragma unroll
    for (int i = 0; i < TILE_UNROLL; ++i) {
      if (base + i >= P.t1) break;  // the same in every lane
      const uint32_t e0 = __ldg(sedge + 2 * sx[i]), ne = __ldg(sedge + 2 * sx[i] + 1);
      for (uint32_t e = e0; e < e0 + ne; ++e) {
        const uint64_t et = edges[e].tile_base + lt[i];
        if (!WRITE) {
          const bool hit = xv[i] && ((__ldg(edges[e].bits_w + (x[i] >> 5)) >> (x[i] & 31u)) & 1u);
          const uint32_t m = __ballot_sync(dev::FULL, hit);
          if (lane == 0) mask[et] = m;
        } else {
          const uint32_t m = __ldg(mask + et);
          if (m & (1u << lane)) {
            const uint64_t pos = __ldg(vp + et) + __popc(m & ((1u << lane) - 1u));
            values[pos] = x[i];
            if (edges[e].flags & TAB_KEY_MAP) vkey[pos] = kx[i];
          }
        }
      }
    }
  }
}

static uint32_t src_tile_blocks(uint64_t ntile) {
  uint64_t warps = (ntile + TILE_UNROLL - 1) / TILE_UNROLL;
  uint64_t blocks = (warps + 7) / 8;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  if (blocks == 0) blocks = 1;
  return (uint32_t)blocks;
}

void launch_table_count(const TabPass &P, const TabSource *d_src, const uint32_t *sedge, const TabEdge *d_edge,
                        const uint64_t *tp, const uint32_t *tkey, const uint32_t *tsrc, uint32_t *mask,
                        cudaStream_t s) {
  if (P.t1 <= P.t0) return;
  count_launch();
  table_src_kernel<false><<<src_tile_blocks(P.t1 - P.t0), 256, 0, s>>>(P, d_src, sedge, d_edge, tp, tkey, tsrc, mask,
                                                                        nullptr, nullptr, nullptr);
}

void launch_table_write(const TabPass &P, const TabSource *d_src, const uint32_t *sedge, const TabEdge *d_edge,
                        const uint64_t *tp, const uint32_t *tkey, const uint32_t *tsrc, const uint32_t *mask,
                        const uint64_t *vp, uint32_t *values, uint32_t *vkey, cudaStream_t s) {
  if (P.t1 <= P.t0) return;
  count_launch();
  table_src_kernel<true><<<src_tile_blocks(P.t1 - P.t0), 256, 0, s>>>(P, d_src, sedge, d_edge, tp, tkey, tsrc,
                                                                       const_cast<uint32_t *>(mask), vp, values, vkey);
}

// Partition of every source tile (by its key vertex: the partition whose
// vertex range [part_v[p], part_v[p + 1]) holds it) and the tiles per
// partition.  Partitions are few (adjacency bytes / partition size), so the
// counts go through a shared-memory histogram when they fit one.
__global__ void tile_partition_kernel(const TabSource *__restrict__ srcs, const uint32_t *__restrict__ tkey,
                                      const uint32_t *__restrict__ tsrc, uint64_t ntile,
                                      const uint32_t *__restrict__ part_v, uint32_t nparts,
                                      uint32_t *__restrict__ tpart, uint32_t *__restrict__ hist) {
  __shared__ uint32_t sh[TILE_PART_SMEM];
  const bool local = nparts <= TILE_PART_SMEM;
  if (local)
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ntile; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t sidx = __ldg(tsrc + t);
    const uint32_t v = __ldg(srcs[sidx].keys + (__ldg(tkey + t) - srcs[sidx].key_base));
    uint32_t lo = 0, hi = nparts;  // last p with part_v[p] <= v
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(part_v + mid) <= v) lo = mid; else hi = mid;
    }
    tpart[t] = lo;
    if (local) atomicAdd(sh + lo, 1u); else atomicAdd(hist + lo, 1u);
  }
  __syncthreads();
  if (local)
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x)
      if (sh[i]) atomicAdd(hist + i, sh[i]);
}

// tord[cursor[p]++] = t for every tile t of partition p (cursor starts at the
// partition's first position); the order within a partition is immaterial.
// Partitions are few, so a per-tile global atomic would serialise on a
// handful of cursors: each block counts a chunk of SCATTER_ITEMS tiles per
// thread in shared memory (one atomic per warp and partition, lanes of the
// same partition found with __match_any_sync), reserves each partition's
// range with one global atomic, then writes.
constexpr int SCATTER_ITEMS = 8;

__global__ void __launch_bounds__(256) tile_scatter_kernel(const uint32_t *__restrict__ tpart, uint64_t ntile,
                                                           uint32_t nparts, uint32_t *__restrict__ cursor,
                                                           uint32_t *__restrict__ tord) {
  __shared__ uint32_t cnt[TILE_PART_SMEM], base[TILE_PART_SMEM];
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t chunk = (uint64_t)blockDim.x * SCATTER_ITEMS;
  for (uint64_t c0 = blockIdx.x * chunk; c0 < ntile; c0 += (uint64_t)gridDim.x * chunk) {
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    uint32_t pp[SCATTER_ITEMS], off[SCATTER_ITEMS];
#pragma unroll
    for (int it = 0; it < SCATTER_ITEMS; ++it) {
      const uint64_t t = c0 + (uint64_t)it * blockDim.x + threadIdx.x;
      const uint32_t p = t < ntile ? __ldg(tpart + t) : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(dev::FULL, p);
      const uint32_t leader = __ffs(peers) - 1;
      uint32_t o = 0;
      if (lane == leader && p != 0xFFFFFFFFu) o = atomicAdd(cnt + p, (uint32_t)__popc(peers));
      pp[it] = p;
      off[it] = __shfl_sync(dev::FULL, o, leader) + __popc(peers & ((1u << lane) - 1u));
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) base[i] = cnt[i] ? atomicAdd(cursor + i, cnt[i]) : 0u;
    __syncthreads();
#pragma unroll
    for (int it = 0; it < SCATTER_ITEMS; ++it)
      if (pp[it] != 0xFFFFFFFFu) tord[base[pp[it]] + off[it]] = (uint32_t)(c0 + (uint64_t)it * blockDim.x + threadIdx.x);
    __syncthreads();  // cnt and base are reset by the next chunk
  }
}

// Fallback for more partitions than the shared-memory tables hold.
__global__ void tile_scatter_global_kernel(const uint32_t *__restrict__ tpart, uint64_t ntile,
                                           uint32_t *__restrict__ cursor, uint32_t *__restrict__ tord) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ntile; t += (uint64_t)gridDim.x * blockDim.x)
    tord[atomicAdd(cursor + __ldg(tpart + t), 1u)] = (uint32_t)t;
}

void launch_tile_partition(const TabSource *d_src, const uint32_t *tkey, const uint32_t *tsrc, uint64_t ntile,
                           const uint32_t *part_v, uint32_t nparts, uint32_t *tpart, uint32_t *hist, cudaStream_t s) {
  if (ntile == 0) return;
  uint64_t blocks = (ntile + 255) / 256;
  if (blocks > 148ull * 8) blocks = 148ull * 8;
  count_launch();
  tile_partition_kernel<<<(uint32_t)blocks, 256, 0, s>>>(d_src, tkey, tsrc, ntile, part_v, nparts, tpart, hist);
}

void launch_tile_scatter(const uint32_t *tpart, uint64_t ntile, uint32_t nparts, uint32_t *cursor, uint32_t *tord,
                         cudaStream_t s) {
  if (ntile == 0) return;
  count_launch();
  if (nparts <= TILE_PART_SMEM) {
    uint64_t blocks = (ntile + 256 * SCATTER_ITEMS - 1) / (256 * SCATTER_ITEMS);
    if (blocks > 148ull * 8) blocks = 148ull * 8;
    tile_scatter_kernel<<<(uint32_t)blocks, 256, 0, s>>>(tpart, ntile, nparts, cursor, tord);
  } else {
    uint64_t blocks = (ntile + 255) / 256;
    if (blocks > 148ull * 32) blocks = 148ull * 32;
    tile_scatter_global_kernel<<<(uint32_t)blocks, 256, 0, s>>>(tpart, ntile, cursor, tord);
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
