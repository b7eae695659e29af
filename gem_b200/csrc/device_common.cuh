// Device helpers shared by the kernels of libgem (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gem {
namespace dev {

constexpr uint32_t FULL = 0xFFFFFFFFu;

// Device error word values (written with atomicCAS so the first cause wins).
enum : uint32_t {
  DERR_NONE = 0,
  DERR_TIMEOUT = 1,   // a bounded wait or the time cap ran out
  DERR_OVERFLOW = 2,  // a fixed-capacity structure (cuckoo stash, output) overflowed
  DERR_INTERNAL = 3,  // an index or invariant check failed
  DERR_BOUNDS = 4     // a bounds check failed; the kernel skipped the access
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void set_error(uint32_t *err, uint32_t code) {
  atomicCAS(err, DERR_NONE, code);
}

// splitmix64 finaliser of (x + golden gamma); identical to gem::mix64 on the host.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Hash term of (query vertex u, data vertex v) used by the embedding hash.
__device__ __forceinline__ uint64_t emb_term(uint32_t u, uint32_t v) {
  return mix64((uint64_t)v | ((uint64_t)u << 32));
}

// First index i in [lo, hi) with a[i] >= x (hi if none).
__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t *__restrict__ a, uint64_t lo,
                                                    uint64_t hi, uint32_t x) {
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains_u32(const uint32_t *__restrict__ a, uint64_t lo, uint64_t hi,
                                             uint32_t x) {
  uint64_t p = lower_bound_u32(a, lo, hi, x);
  return p < hi && __ldg(a + p) == x;
}

// Position of v in a sorted candidate list through its rank bitmap: one
// 64-bit word per 32 data vertices, bits in the low half and the number of
// members before this word in the high half.  Returns 0xFFFFFFFF if absent.
__device__ __forceinline__ uint32_t rank_lookup(const uint64_t *__restrict__ rb, uint32_t v) {
  uint64_t w = __ldg(rb + (v >> 5));
  uint32_t bits = (uint32_t)w, bit = 1u << (v & 31u);
  if (!(bits & bit)) return 0xFFFFFFFFu;
  return (uint32_t)(w >> 32) + (uint32_t)__popc(bits & (bit - 1u));
}

__device__ __forceinline__ bool rank_member(const uint64_t *__restrict__ rb, uint32_t v) {
  return (uint32_t)__ldg(rb + (v >> 5)) & (1u << (v & 31u));
}

}  // namespace dev
}  // namespace gem
