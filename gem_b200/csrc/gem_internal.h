// Internal declarations shared by the host (C++) and device (CUDA) parts of
// libgem.  Nothing here is part of the C-ABI (include/gem.h is).
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gem.h"

struct gem_hgraph {
  uint32_t nv = 0;
  std::vector<uint64_t> off;  // nv + 1
  std::vector<uint32_t> nbr;  // off[nv], each list sorted ascending
  std::vector<uint32_t> lab;  // nv
  uint32_t max_label_plus1 = 0;
  uint32_t max_degree = 0;

  uint64_t n_arcs() const { return off.empty() ? 0 : off[nv]; }
  void refresh_stats();
};

namespace gem {

// splitmix64 (Steele, Lea, Flood 2014; constants as published by Vigna).
inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Counter-based uniform draws: stream `s`, draw `i`.
inline uint64_t rng_at(uint64_t s, uint64_t i) {
  return mix64(mix64(s) ^ (i * 0xD1B54A32D192ED03ull));
}
inline double u01(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// Parallel LSD radix sort of 64-bit keys that fit in `bits` bits.
void radix_sort_u64(std::vector<uint64_t> &keys, uint32_t bits);

// A query in plain host form after validation.
struct HostQuery {
  uint32_t nv = 0, ne = 0;
  uint32_t lab[GEM_MAX_QV];
  uint32_t adj[GEM_MAX_QV];  // bitmask of neighbours
  std::vector<uint32_t> edges;  // 2*ne (as given)
  uint32_t deg(uint32_t u) const { return (uint32_t)__builtin_popcount(adj[u]); }
};

// Validates q (sizes, ranges, no self loops or duplicate edges); connectivity
// is required for nv > 1.
gem_status make_host_query(const gem_query *q, HostQuery &out, std::string &err);
// Relaxed queries rq of orig counted in one wave that shares orig's filter
// rows at `threshold` (ctx.cu); GEM_ERR_OOM when that wave does not fit.
gem_status relaxed_wave(gem_ctx *ctx, const HostQuery &orig, const std::vector<HostQuery> &rq, uint32_t threshold,
                        int mode, gem_result *res);

}  // namespace gem
