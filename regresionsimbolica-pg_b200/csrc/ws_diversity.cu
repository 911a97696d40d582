// ws_diversity.cu -- structural hashing, deduplication and sharing penalties
// (diversity_kernels.cu of the reference), restated.
//
//   ws_population_hashes       polynomial hash (base 31, mod 2^64) of each program up to its first
//                              PAD, and the bitmask of the variables it uses
//   ws_var_presence            the variable bitmask alone
//   ws_structural_dedup        groups programs by hash through an open-addressing table; one
//                              program per group is the original, the others point to it
//   ws_count_unique            programs whose duplicate flag is 0
//   ws_replacement_positions   indices of the duplicates
//   ws_fitness_sharing_penalty per-island counts of an 8-token prefix hash; log2(count) above a
//                              threshold
//
// The reference resolves dedup groups and replacement order with atomics, so WHICH member of a
// group is the original, and the order of the replacement positions, depend on thread timing
// there.  Here the original of a group is its lowest index and positions come out ascending:
// the same groups, the same counts, deterministic.
#include <cuda_runtime.h>
#include <cstdint>

#include "ws_internal.h"

namespace ws {
namespace {

constexpr int64_t kDedupSlots = int64_t(1) << 20;  // the caller's hash_table (diversity_kernels.cu:115)
constexpr int kDedupProbes = 16;
constexpr int64_t kShareSlots = int64_t(1) << 18;   // per island (:116)

unsigned blocks_for(int64_t n, int t) {
  int64_t g = (n + t - 1) / t;
  const int64_t cap = (int64_t)device_info().sm_count * 32;
  return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

// compute_population_hashes_kernel / compute_var_presence_kernel (diversity_kernels.cu:29-72,
// 465-488); variables beyond bit 31 do not fit the int32 mask and are left out of it.
// VEC: rows are 16-byte aligned multiples of 16 bytes and are read 16 bytes at a time.
template <bool VEC>
__global__ void __launch_bounds__(256) hash_kernel(const uint8_t* __restrict__ pop, int64_t B,
                                                   int L, int pad, int x0, int nv,
                                                   int64_t* __restrict__ hashes,
                                                   int32_t* __restrict__ presence) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t* row = pop + b * L;
    uint64_t h = 0ull, p = 1ull;
    int32_t mask = 0;
    bool open = true;
    auto take = [&](int t) {
      if (!open || t == pad) {
        open = false;
        return;
      }
      h += (uint64_t)t * p;
      p *= 31ull;
      const int v = t - x0;
      if (t >= x0 && v < nv && v < 32) mask |= (int32_t)(1u << v);
    };
    if (VEC) {
      const uint4* r4 = reinterpret_cast<const uint4*>(row);
      for (int c = 0; c < (L >> 4) && open; ++c) {
        const uint4 w = r4[c];
        const uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int j = 0; j < 4; ++j) take((int)((words[q] >> (8 * j)) & 0xFFu));
      }
    } else {
      for (int i = 0; i < L && open; ++i) take(row[i]);
    }
    if (hashes) hashes[b] = (int64_t)h;
    if (presence) presence[b] = mask;
  }
}

// Dedup pass 1: a program claims an empty slot for its hash, or joins the slot that already
// holds its hash and lowers the slot's index to its own (atomicMin: the group's lowest index
// remains); other hashes move it to the next slot, at most kDedupProbes times.
__global__ void __launch_bounds__(256) dedup_insert_kernel(const int64_t* __restrict__ hashes,
                                                           int64_t B, int64_t* table) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    const int64_t h = hashes[b];
    int64_t slot = h & (kDedupSlots - 1);
    for (int a = 0; a <= kDedupProbes; ++a) {
      unsigned long long* cell = reinterpret_cast<unsigned long long*>(table + slot);
      const unsigned long long old = atomicCAS(cell, ~0ull, (unsigned long long)b);
      if (old == ~0ull) break;  // claimed
      // an index this call cannot have written (a table left over from a larger population)
      // is a foreign entry: probe on rather than read past the hashes
      if (old < (unsigned long long)B && hashes[(int64_t)old] == h) {  // this hash's slot (indices in it only ever decrease)
        atomicMin(reinterpret_cast<long long*>(cell), (long long)b);
        break;
      }
      slot = (slot + 1) & (kDedupSlots - 1);
    }
  }
}

// Dedup pass 2: the original of a program is the index its hash's slot ended with.
__global__ void __launch_bounds__(256) dedup_lookup_kernel(const int64_t* __restrict__ hashes,
                                                           int64_t B,
                                                           const int64_t* __restrict__ table,
                                                           int32_t* __restrict__ dup,
                                                           int64_t* __restrict__ orig) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    const int64_t h = hashes[b];
    int64_t slot = h & (kDedupSlots - 1);
    int64_t o = b;  // not found within the probes: unique (the reference's fallback)
    for (int a = 0; a <= kDedupProbes; ++a) {
      const int64_t c = table[slot];
      if (c < 0) break;
      if (c < B && hashes[c] == h) {
        o = c;
        break;
      }
      slot = (slot + 1) & (kDedupSlots - 1);
    }
    dup[b] = o != b ? 1 : 0;
    orig[b] = o;
  }
}

// One block walks the flags in tiles of 1024 threads x 16 flags: each thread loads its 16
// consecutive flags (four 16-byte loads when aligned: a warp reads 2 KB contiguous), keeps the
// selected ones as a bit mask, and a block scan of the per-thread counts (warp shuffles, then the
// 32 warp totals) gives every thread its first output position; positions come out ascending, the
// running total carries from tile to tile.  count_unique: count the non-duplicates instead.
constexpr int kScanPer = 16;
__global__ void __launch_bounds__(1024) dup_scan_kernel(const int32_t* __restrict__ dup,
                                                        int64_t B, int64_t* __restrict__ pos,
                                                        int64_t* __restrict__ count,
                                                        int count_unique) {
  __shared__ int64_t wsum[32];
  __shared__ int64_t s_total;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int want = count_unique ? 0 : 1;
  const bool vec = ((uintptr_t)dup & 15u) == 0;
  const bool write = !count_unique && pos != nullptr;
  int64_t base = 0;  // selected flags before this tile (the same in every thread)
  for (int64_t t0 = 0; t0 < B; t0 += 1024 * kScanPer) {
    const int64_t i0 = t0 + (int64_t)t * kScanPer;
    uint32_t bits = 0u;
    if (vec && i0 + kScanPer <= B) {
      const int4* src = reinterpret_cast<const int4*>(dup + i0);
#pragma unroll
      for (int q = 0; q < kScanPer / 4; ++q) {
        const int4 v = src[q];
        bits |= (uint32_t)(v.x == want) << (4 * q) | (uint32_t)(v.y == want) << (4 * q + 1) |
                (uint32_t)(v.z == want) << (4 * q + 2) | (uint32_t)(v.w == want) << (4 * q + 3);
      }
    } else {
      for (int k = 0; k < kScanPer; ++k)
        if (i0 + k < B && dup[i0 + k] == want) bits |= 1u << k;
    }
    const int c = __popc(bits);
    int incl = c;  // inclusive scan over the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;  // warp totals
    __syncthreads();
    if (w == 0) {  // exclusive offsets of the warps (each lane rewrites its own slot only)
      const int64_t v = wsum[lane];
      int64_t iv = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t u = __shfl_up_sync(0xFFFFFFFFu, iv, o);
        if (lane >= o) iv += u;
      }
      wsum[lane] = iv - v;
      if (lane == 31) s_total = iv;  // the tile's selected flags
    }
    __syncthreads();
    if (write && bits) {
      int64_t o = base + wsum[w] + (incl - c);
      for (uint32_t m = bits; m; m &= m - 1) pos[o++] = i0 + __ffs(m) - 1;
    }
    base += s_total;
    __syncthreads();  // wsum and s_total are rewritten by the next tile
  }
  if (t == 0) count[0] = base;
}

// fitness_sharing_hash8 / count / penalty kernels (diversity_kernels.cu:224-319): the first
// min(hash_len, L, 8) tokens weighted by powers of 31 (the eighth by 1103515245), then the
// 32-bit-constant avalanche; per-island tables of 2^18 slots with 32 linear probes.
__device__ __forceinline__ uint64_t share_hash(const uint8_t* row, int L, int hash_len) {
  const uint64_t w[8] = {1ull, 31ull, 961ull, 29791ull, 923521ull, 28629151ull, 887503681ull,
                         1103515245ull};
  uint64_t h = 0ull;
  int lim = hash_len < L ? hash_len : L;
  if (lim > 8) lim = 8;
  if (L >= 8 && ((uintptr_t)row & 7u) == 0) {  // the 8-token prefix in one load
    const uint64_t v = *reinterpret_cast<const uint64_t*>(row);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (i < lim) h += ((v >> (8 * i)) & 0xFFull) * w[i];
  } else {
    for (int i = 0; i < lim; ++i) h += (uint64_t)row[i] * w[i];
  }
  h ^= h >> 16;
  h *= 0x7feb352dull;
  h ^= h >> 15;
  h *= 0x846ca68bull;
  h ^= h >> 16;
  return h;
}

__device__ __forceinline__ int island_of(int64_t b, int n_islands, int island_size) {
  int64_t is = island_size > 0 ? b / island_size : 0;
  return (int)(is >= n_islands ? n_islands - 1 : is);
}

__global__ void __launch_bounds__(256) share_count_kernel(const uint8_t* __restrict__ pop,
                                                          int64_t B, int L, int n_islands,
                                                          int island_size, int hash_len,
                                                          int64_t* keys, int32_t* counts) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    const int isl = island_of(b, n_islands, island_size);
    const uint64_t h = share_hash(pop + b * L, L, hash_len);
    const int64_t base = (int64_t)isl * kShareSlots;
    int64_t slot = (int64_t)(h & (kShareSlots - 1));
    for (int a = 0; a < 32; ++a) {
      const unsigned long long old = atomicCAS(
          reinterpret_cast<unsigned long long*>(keys + base + slot), ~0ull, (unsigned long long)h);
      if (old == ~0ull || old == (unsigned long long)h) {
        atomicAdd(counts + base + slot, 1);
        break;
      }
      slot = (slot + 1) & (kShareSlots - 1);
    }
  }
}

__global__ void __launch_bounds__(256) share_penalty_kernel(const uint8_t* __restrict__ pop,
                                                            int64_t B, int L, int n_islands,
                                                            int island_size, int threshold,
                                                            int hash_len,
                                                            const int64_t* __restrict__ keys,
                                                            const int32_t* __restrict__ counts,
                                                            float* __restrict__ out) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    const int isl = island_of(b, n_islands, island_size);
    const uint64_t h = share_hash(pop + b * L, L, hash_len);
    const int64_t base = (int64_t)isl * kShareSlots;
    int64_t slot = (int64_t)(h & (kShareSlots - 1));
    int c = 1;
    for (int a = 0; a < 32; ++a) {
      const int64_t k = keys[base + slot];
      if (k == (int64_t)h) {
        c = counts[base + slot];
        break;
      }
      if (k == -1) break;
      slot = (slot + 1) & (kShareSlots - 1);
    }
    out[b] = c > threshold ? log2f((float)c) : 0.0f;
  }
}

ws_status after(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, what);
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

ws_status ws_population_hashes(const uint8_t* population, int64_t B, int64_t L, int64_t* hashes,
                               int32_t* var_presence, int32_t pad_id, int32_t id_x_start,
                               int32_t num_vars, void* stream) {
  clear_error();
  if (B < 0 || L < 0) return fail("negative size");
  if (B == 0) return WS_OK;
  if ((L > 0 && !population) || (!hashes && !var_presence)) return fail("null tensor pointer");
  if (L % 16 == 0 && ((uintptr_t)population & 15u) == 0)
    hash_kernel<true><<<blocks_for(B, 256), 256, 0, (cudaStream_t)stream>>>(
        population, B, (int)L, pad_id, id_x_start, num_vars, hashes, var_presence);
  else
    hash_kernel<false><<<blocks_for(B, 256), 256, 0, (cudaStream_t)stream>>>(
        population, B, (int)L, pad_id, id_x_start, num_vars, hashes, var_presence);
  return after("population hash launch");
}

ws_status ws_structural_dedup(const int64_t* hashes, int64_t B, int64_t* hash_table,
                              int32_t* duplicate_mask, int64_t* original_index, void* stream) {
  clear_error();
  if (B < 0) return fail("negative size");
  if (B == 0) return WS_OK;
  if (!hashes || !hash_table || !duplicate_mask || !original_index)
    return fail("null tensor pointer");
  const unsigned g = blocks_for(B, 256);
  dedup_insert_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(hashes, B, hash_table);
  dedup_lookup_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(hashes, B, hash_table, duplicate_mask,
                                                           original_index);
  return after("structural dedup launch");
}

ws_status ws_count_unique(const int32_t* duplicate_mask, int64_t B, int64_t* out_count,
                          void* stream) {
  clear_error();
  if (B < 0) return fail("negative size");
  if (!out_count || (B > 0 && !duplicate_mask)) return fail("null tensor pointer");
  dup_scan_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(duplicate_mask, B, nullptr, out_count, 1);
  return after("count unique launch");
}

ws_status ws_replacement_positions(const int32_t* duplicate_mask, int64_t B, int64_t* positions,
                                   int64_t* n_replacements, void* stream) {
  clear_error();
  if (B < 0) return fail("negative size");
  if (!n_replacements || (B > 0 && (!duplicate_mask || !positions)))
    return fail("null tensor pointer");
  dup_scan_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(duplicate_mask, B, positions,
                                                        n_replacements, 0);
  return after("replacement positions launch");
}

ws_status ws_fitness_sharing_penalty(const uint8_t* population, int64_t B, int64_t L,
                                     int32_t n_islands, int32_t island_size, int32_t threshold,
                                     int32_t hash_len, int64_t* keys, int32_t* counts,
                                     float* out_penalty, void* stream) {
  clear_error();
  if (B < 0 || L < 0 || n_islands < 1) return fail("invalid size");
  if (B == 0) return WS_OK;
  if (!population || !keys || !counts || !out_penalty) return fail("null tensor pointer");
  const unsigned g = blocks_for(B, 256);
  share_count_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(population, B, (int)L, n_islands,
                                                          island_size, hash_len, keys, counts);
  share_penalty_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(population, B, (int)L, n_islands,
                                                            island_size, threshold, hash_len, keys,
                                                            counts, out_penalty);
  return after("fitness sharing launch");
}

int64_t ws_dedup_table_slots(void) { return kDedupSlots; }
int64_t ws_sharing_table_slots(void) { return kShareSlots; }

}  // extern "C"
