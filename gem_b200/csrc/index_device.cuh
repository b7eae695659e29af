// Device-side probes of the vertex -> position indexes (shared by the index
// and join translation units).
#pragma once

#include "device_common.cuh"
#include "kernels.h"

namespace gem {

__host__ __device__ __forceinline__ uint32_t ck_bucket(uint32_t key, uint64_t a, uint64_t c, uint32_t nb) {
  uint32_t h = (uint32_t)((a * (uint64_t)key + c) >> 32);
  return (uint32_t)(((uint64_t)h * nb) >> 32);
}

__device__ __forceinline__ uint32_t ck_probe_bucket(const uint64_t *__restrict__ b, uint32_t key, bool *stop) {
  const uint4 *p = reinterpret_cast<const uint4 *>(b);
#pragma unroll 2
  for (uint32_t i = 0; i < CK_SLOTS / 2; ++i) {
    uint4 x = __ldg(p + i);
    if (x.x == key) return x.y;
    if (x.z == key) return x.w;
    if (x.x == 0xFFFFFFFFu || x.z == 0xFFFFFFFFu) { *stop = true; return 0xFFFFFFFFu; }
  }
  return 0xFFFFFFFFu;
}

__device__ __forceinline__ uint32_t ck_lookup(const CuckooTable *__restrict__ Tp, uint32_t key) {
  const uint32_t nb0 = Tp->nb0, nb1 = Tp->nb1;
  bool stop = false;
  uint32_t r = ck_probe_bucket(Tp->t0 + (uint64_t)ck_bucket(key, Tp->a0, Tp->c0, nb0) * CK_SLOTS, key, &stop);
  if (r != 0xFFFFFFFFu) return r;
  stop = false;
  r = ck_probe_bucket(Tp->t1 + (uint64_t)ck_bucket(key, Tp->a1, Tp->c1, nb1) * CK_SLOTS, key, &stop);
  if (r != 0xFFFFFFFFu) return r;
  uint32_t ns = *Tp->stash_n;
  if (ns > CK_STASH) ns = CK_STASH;
  for (uint32_t i = 0; i < ns; ++i) {
    uint64_t x = Tp->stash[i];
    if ((uint32_t)x == key) return (uint32_t)(x >> 32);
  }
  return 0xFFFFFFFFu;
}


}  // namespace gem
