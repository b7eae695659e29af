// Vertex -> position-in-C(u) indexes.
//
// Cuckoo hash: replaces HashTable::build / buildHashKeys / hash_lookup
// (in-core/lib/structure/src/unifiedTrie.cu:175-433,
//  in-core/lib/structure/src/cuckooHash.cu:9-147,
//  in-core/lib/structure/include/unifiedTrie.cuh:77-125).  The reference keeps
// 8 keys per 32-byte bucket in two tables with a separate position array,
// rebuilds a whole table from the host whenever one insert exceeds 64 kicks,
// and uses warp ballots over partial masks.  Here a bucket is one 128-byte
// line of 16 {key, position} slots, so a hit costs one line; table 0 holds
// about 8 keys per bucket (load 0.5), table 1 takes the overflow, kicks are
// bounded and the rare leftovers go to a 64-entry stash (an overflowing stash
// sets an error status instead of looping).  Tables of up to a few thousand
// keys are assembled in shared memory by one block and copied out with
// coalesced 16-byte stores.
//
// Rank bitmap: the filter's bit rows with a per-word prefix count; the
// position of v is the prefix plus a popcount (one 8-byte load).
#include "device_common.cuh"
#include "kernels.h"
#include "index_device.cuh"

#include <vector>

namespace gem {

uint64_t cuckoo_slots_for(uint32_t nkeys, uint32_t *nb0, uint32_t *nb1) {
  uint32_t b0 = (nkeys + 7) / 8, b1 = (nkeys + 31) / 32;
  if (b0 == 0) b0 = 1;
  if (b1 == 0) b1 = 1;
  if (nb0) *nb0 = b0;
  if (nb1) *nb1 = b1;
  return (uint64_t)(b0 + b1) * CK_SLOTS + CK_STASH;
}

__device__ __forceinline__ bool ck_try_bucket(uint64_t *b, uint64_t item) {
  volatile uint64_t *vb = b;
  for (uint32_t s = 0; s < CK_SLOTS; ++s) {
    if (vb[s] == CK_EMPTY) {
      if (atomicCAS((unsigned long long *)(b + s), (unsigned long long)CK_EMPTY, (unsigned long long)item) ==
          (unsigned long long)CK_EMPTY)
        return true;
    }
  }
  return false;
}

// Inserts item = pos << 32 | key into the tables t0/t1 (either global or
// shared memory); overflow goes to the stash in global memory.
__device__ bool ck_insert(uint64_t *t0, uint64_t *t1, const CuckooTable &T, uint64_t item, uint32_t *err) {
  uint32_t tbl = 0;
  for (uint32_t kick = 0; kick < CK_MAX_KICKS; ++kick) {
    const uint32_t key = (uint32_t)item;
    uint64_t *b0 = t0 + (uint64_t)ck_bucket(key, T.a0, T.c0, T.nb0) * CK_SLOTS;
    uint64_t *b1 = t1 + (uint64_t)ck_bucket(key, T.a1, T.c1, T.nb1) * CK_SLOTS;
    uint64_t *first = tbl == 0 ? b0 : b1, *second = tbl == 0 ? b1 : b0;
    if (ck_try_bucket(first, item)) return true;
    if (ck_try_bucket(second, item)) return true;
    // Both buckets full: displace a slot of `first`; the displaced item lives
    // in its own bucket of that table, so it retries the other table first.
    uint32_t s = (uint32_t)(dev::mix64(((uint64_t)key << 8) ^ kick) & (CK_SLOTS - 1));
    item = (uint64_t)atomicExch((unsigned long long *)(first + s), (unsigned long long)item);
    if (item == CK_EMPTY) return true;
    tbl ^= 1u;
  }
  uint32_t i = atomicAdd(T.stash_n, 1u);
  if (i < CK_STASH) {
    T.stash[i] = item;
    return true;
  }
  dev::set_error(err, dev::DERR_OVERFLOW);
  return false;
}

// One block per small table, built in shared memory.
__global__ void __launch_bounds__(256) cuckoo_build_smem_kernel(const CuckooTable *__restrict__ tabs,
                                                                const uint32_t *__restrict__ which, uint32_t *err) {
  extern __shared__ uint64_t sm[];
  const CuckooTable T = tabs[which[blockIdx.x]];
  const uint32_t nslots = (T.nb0 + T.nb1) * CK_SLOTS;
  for (uint32_t i = threadIdx.x; i < nslots; i += blockDim.x) sm[i] = CK_EMPTY;
  __syncthreads();
  uint64_t *s0 = sm, *s1 = sm + (uint64_t)T.nb0 * CK_SLOTS;
  for (uint32_t i = threadIdx.x; i < T.nkeys; i += blockDim.x) {
    uint64_t item = ((uint64_t)i << 32) | __ldg(T.keys + i);
    ck_insert(s0, s1, T, item, err);
  }
  __syncthreads();
  // t0 and t1 are contiguous in global memory (t1 = t0 + nb0 * 16).
  const uint4 *src = reinterpret_cast<const uint4 *>(sm);
  uint4 *dst = reinterpret_cast<uint4 *>(T.t0);
  for (uint32_t i = threadIdx.x; i < nslots / 2; i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ uint32_t find_table(const CuckooTable *__restrict__ tabs, const uint32_t *__restrict__ which,
                                               uint32_t n, uint64_t k) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (tabs[which[mid]].key_base <= k) lo = mid; else hi = mid;
  }
  return which[lo];
}

// Large tables: one thread per key over the flattened key space of the
// selected tables (their key_base values ascend in `which` order).
__global__ void cuckoo_build_global_kernel(const CuckooTable *__restrict__ tabs, const uint32_t *__restrict__ which,
                                           uint32_t nwhich, uint64_t k0, uint64_t k1, uint32_t *err) {
  for (uint64_t k = k0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < k1; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = find_table(tabs, which, nwhich, k);
    const CuckooTable &T = tabs[t];
    const uint32_t i = (uint32_t)(k - T.key_base);
    if (i >= T.nkeys) continue;
    uint64_t item = ((uint64_t)i << 32) | __ldg(T.keys + i);
    ck_insert(T.t0, T.t1, T, item, err);
  }
}

constexpr uint32_t CK_SMEM_MAX_BYTES = 96 * 1024;

void launch_cuckoo_build(const CuckooTable *d_tabs, const CuckooTable *h_tabs, uint32_t ntab, uint32_t *err,
                         cudaStream_t s) {
  // The caller allocates d_tabs with room for ntab extra u32 after the
  // descriptors; the lists of small and large tables go there.  The H2D copy
  // from pageable memory is staged before cudaMemcpyAsync returns.
  uint32_t *d_which = reinterpret_cast<uint32_t *>(const_cast<CuckooTable *>(d_tabs) + ntab);
  static thread_local std::vector<uint32_t> small, large;
  small.clear();
  large.clear();
  uint32_t max_smem = 0;
  uint64_t k0 = ~0ull, k1 = 0;
  for (uint32_t i = 0; i < ntab; ++i) {
    const CuckooTable &T = h_tabs[i];
    if (T.nkeys == 0) continue;
    uint32_t bytes = (T.nb0 + T.nb1) * CK_SLOTS * 8u;
    if (bytes <= CK_SMEM_MAX_BYTES) {
      small.push_back(i);
      if (bytes > max_smem) max_smem = bytes;
    } else {
      large.push_back(i);
      if (T.key_base < k0) k0 = T.key_base;
      if (T.key_base + T.nkeys > k1) k1 = T.key_base + T.nkeys;
    }
  }
  std::vector<uint32_t> all(small);
  all.insert(all.end(), large.begin(), large.end());
  if (all.empty()) return;
  cudaMemcpyAsync(d_which, all.data(), all.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
  if (!small.empty()) {
    cudaFuncSetAttribute(cuckoo_build_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)CK_SMEM_MAX_BYTES);
    count_launch();
    cuckoo_build_smem_kernel<<<(uint32_t)small.size(), 256, max_smem, s>>>(d_tabs, d_which, err);
  }
  if (!large.empty()) {
    uint64_t n = k1 - k0;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > 148ull * 32) blocks = 148ull * 32;
    count_launch();
    cuckoo_build_global_kernel<<<(uint32_t)blocks, 256, 0, s>>>(d_tabs, d_which + small.size(),
                                                                (uint32_t)large.size(), k0, k1, err);
  }
}

__global__ void cuckoo_probe_kernel(const CuckooTable *T, const uint32_t *keys, uint32_t n, uint32_t *out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = ck_lookup(T, keys[i]);
}

__global__ void rank_probe_kernel(const uint64_t *rb, const uint32_t *keys, uint32_t n, uint32_t *out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = dev::rank_lookup(rb, keys[i]);
}

void launch_cuckoo_probe(const CuckooTable *d_tab, const uint32_t *keys, uint32_t n, uint32_t *out, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  cuckoo_probe_kernel<<<(n + 255) / 256 > 4096 ? 4096 : (n + 255) / 256, 256, 0, s>>>(d_tab, keys, n, out);
}

void launch_rank_probe(const uint64_t *rb, const uint32_t *keys, uint32_t n, uint32_t *out, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  rank_probe_kernel<<<(n + 255) / 256 > 4096 ? 4096 : (n + 255) / 256, 256, 0, s>>>(rb, keys, n, out);
}

}  // namespace gem
