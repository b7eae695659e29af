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

constexpr uint32_t TILES_PER_WARP = 16;

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

__device__ __forceinline__ uint32_t find_edge(const TabEdge *__restrict__ e, uint32_t ne, uint64_t t) {
  uint32_t lo = 0, hi = ne;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (e[mid].tile_base <= t) lo = mid; else hi = mid;
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

// Walks the tiles [t0, t1) of the flattened edge-tile space; calls
// fn(edge, arc_index_or_~0, nbr) once per lane per tile with the tile index.
template <bool WRITE>
__global__ void __launch_bounds__(256) table_tiles_kernel(DevGraph g, const TabSource *__restrict__ srcs,
                                                          const TabEdge *__restrict__ edges, uint32_t nedge,
                                                          const uint64_t *__restrict__ tp, uint64_t total_tiles,
                                                          uint32_t *__restrict__ mask, const uint64_t *__restrict__ vp,
                                                          uint32_t *__restrict__ values) {
  const uint32_t lane = dev::lane_id();
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t t0 = (blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5)) * TILES_PER_WARP;
       t0 < total_tiles; t0 += nwarps * TILES_PER_WARP) {
    const uint64_t t1 = min(t0 + TILES_PER_WARP, total_tiles);
    uint32_t e = find_edge(edges, nedge, t0);
    TabEdge E = edges[e];
    TabSource S = srcs[E.src];
    uint64_t sbase = tp[S.key_base];
    uint64_t st = sbase + (t0 - E.tile_base);
    uint64_t k = last_le(tp, S.key_base, S.key_base + S.nkeys, st);
    uint64_t k_next_tile = __ldg(tp + k + 1);
    uint32_t v = __ldg(S.keys + (k - S.key_base));
    uint64_t a0 = __ldg(g.off + v), a1 = __ldg(g.off + v + 1);
    for (uint64_t t = t0; t < t1; ++t, ++st) {
      if (t >= E.tile_base + E.ntiles) {  // next edge
        e = find_edge(edges, nedge, t);
        E = edges[e];
        S = srcs[E.src];
        sbase = tp[S.key_base];
        st = sbase + (t - E.tile_base);
        k = last_le(tp, S.key_base, S.key_base + S.nkeys, st);
        k_next_tile = __ldg(tp + k + 1);
        v = __ldg(S.keys + (k - S.key_base));
        a0 = __ldg(g.off + v);
        a1 = __ldg(g.off + v + 1);
      }
      while (st >= k_next_tile) {  // next key with at least one tile
        ++k;
        k_next_tile = __ldg(tp + k + 1);
        v = __ldg(S.keys + (k - S.key_base));
        a0 = __ldg(g.off + v);
        a1 = __ldg(g.off + v + 1);
      }
      const uint64_t arc = a0 + (st - __ldg(tp + k)) * 32 + lane;
      if (!WRITE) {
        bool hit = false;
        if (arc < a1) hit = dev::rank_member(E.rb_w, __ldg(g.nbr + arc));
        uint32_t m = __ballot_sync(dev::FULL, hit);
        if (lane == 0) mask[t] = m;
      } else {
        uint32_t m = __ldg(mask + t);
        if (m & (1u << lane)) {
          uint64_t pos = __ldg(vp + t) + __popc(m & ((1u << lane) - 1u));
          values[pos] = __ldg(g.nbr + arc);
        }
      }
    }
  }
}

static uint32_t tile_blocks(uint64_t total_tiles) {
  uint64_t warps = (total_tiles + TILES_PER_WARP - 1) / TILES_PER_WARP;
  uint64_t blocks = (warps + 7) / 8;
  if (blocks > 148ull * 16) blocks = 148ull * 16;
  if (blocks == 0) blocks = 1;
  return (uint32_t)blocks;
}

void launch_table_count(const DevGraph &g, const TabSource *d_src, const TabEdge *d_edge, uint32_t nedge,
                        const uint64_t *tp, uint64_t total_tiles, uint32_t *mask, cudaStream_t s) {
  if (total_tiles == 0) return;
  count_launch();
  table_tiles_kernel<false><<<tile_blocks(total_tiles), 256, 0, s>>>(g, d_src, d_edge, nedge, tp, total_tiles, mask,
                                                                     nullptr, nullptr);
}

void launch_table_write(const DevGraph &g, const TabSource *d_src, const TabEdge *d_edge, uint32_t nedge,
                        const uint64_t *tp, uint64_t total_tiles, const uint32_t *mask, const uint64_t *vp,
                        uint32_t *values, cudaStream_t s) {
  if (total_tiles == 0) return;
  count_launch();
  table_tiles_kernel<true><<<tile_blocks(total_tiles), 256, 0, s>>>(g, d_src, d_edge, nedge, tp, total_tiles,
                                                                    const_cast<uint32_t *>(mask), vp, values);
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
