// ws_evolve.cu -- the device steps of one evolve_generation call.
//
// Replaces the kernels that `evolve_generation` (bindings.cpp:474 -> rpn_kernels.cu:1810-2237)
// launches between its torch random draws; the host sequence (the draws, their order, the torch
// glue) lives in rpn_cuda_native.evolve_generation.  Each step reproduces the reference kernel's
// results bit for bit:
//   - subtree range of a row at a random end (select_subtree_range_indirect_kernel,
//     rpn_kernels.cu:597-640): end = floor(u * len), the start found by walking back until the
//     arity balance closes;
//   - crossover validity (validate_crossover_lengths_kernel, :642-679) ANDed with the candidate
//     mask (the reference's logical_and_);
//   - splice of parent rows into child rows, with the point mutation of the children whose draw
//     is below the cut (crossover_splicing_mutation_kernel, :1020-1105; without mutation it is
//     crossover_splicing_kernel, :927-1016);
//   - point mutation of copied rows (mutation_philox_indirect_kernel, :747-770);
//   - SBX of the parents' constants (sbx_constants_kernel, :1225-1261) and the constant transfer
//     that follows the spliced `C` tokens (crossover_constants_kernel, :1107-1223);
//   - hoist mutation (hoist_mutation_indirect_kernel, :1363-1411): a reservoir draw over the
//     row's subtrees with the 64-bit LCG x -> x * 6364136223846793005 + 1, then the subtree moved
//     to the front.
// The point mutation draws Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers:
// as easy as 1, 2, 3", SC 2011) with counter (row * L + position, generation lo, generation hi,
// row) and key (seed lo, seed hi); word 0 decides, word 1 picks the same-arity replacement.
#include <cuda_runtime.h>
#include <cstdint>

#include "ws_internal.h"

namespace ws {
namespace {

__device__ __forceinline__ int arity_of(const int32_t* ar, int vocab, int tok) {
  return tok < vocab ? ar[tok] : 0;
}

// Philox4x32 with 10 rounds: multipliers 0xD2511F53 / 0xCD9E8D57, key bumps 0x9E3779B9 /
// 0xBB67AE85 (the published constants).
__device__ __forceinline__ uint4 philox_4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t p0h = __umulhi(0xD2511F53u, c.x), p0l = 0xD2511F53u * c.x;
    const uint32_t p1h = __umulhi(0xCD9E8D57u, c.z), p1l = 0xCD9E8D57u * c.z;
    c = make_uint4(p1h ^ c.y ^ k0, p1l, p0h ^ c.w ^ k1, p0l);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ uint8_t philox_mutate(uint8_t tok, uint64_t row, int pos, int L,
                                                 const ws_point_mutation& m, int pad) {
  if ((int)tok == pad) return tok;
  const uint4 ctr = make_uint4((uint32_t)(row * (uint64_t)L + (uint64_t)pos),
                               (uint32_t)m.generation, (uint32_t)(m.generation >> 32),
                               (uint32_t)row);
  const uint4 r = philox_4x32_10(ctr, (uint32_t)m.seed, (uint32_t)(m.seed >> 32));
  const float u = ((float)r.x + 0.5f) * 2.3283064365386963e-10f;
  if (u >= m.rate) return tok;
  const int a = arity_of(m.arities, m.vocab, tok);
  if (a == 0 && m.n0 > 0) return m.ids0[r.y % (uint32_t)m.n0];
  if (a == 1 && m.n1 > 0) return m.ids1[r.y % (uint32_t)m.n1];
  if (a == 2 && m.n2 > 0) return m.ids2[r.y % (uint32_t)m.n2];
  return tok;
}

__global__ void __launch_bounds__(256) subtree_pick_kernel(const uint8_t* __restrict__ pop,
                                                           const int64_t* __restrict__ rows,
                                                           int64_t N, int L,
                                                           const int32_t* __restrict__ ar,
                                                           int vocab, const float* __restrict__ u,
                                                           int64_t* __restrict__ out_len,
                                                           int64_t* __restrict__ out_s,
                                                           int64_t* __restrict__ out_e, int pad) {
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t* row = pop + (rows ? rows[n] : n) * (int64_t)L;
    int len = 0;
    while (len < L && (int)row[len] != pad) ++len;
    if (len < 1) len = 1;
    int e = (int)(u[n] * (float)len);
    if (e < 0) e = 0;
    if (e >= len) e = len - 1;
    int s = e;
    const int a = arity_of(ar, vocab, row[e]);
    if (a > 0) {
      int need = a;
      for (int j = e - 1; j >= 0 && (int)row[j] != pad; --j) {
        need += arity_of(ar, vocab, row[j]) - 1;
        if (need == 0) {
          s = j;
          break;
        }
      }
    }
    out_len[n] = len;
    out_s[n] = s;
    out_e[n] = e;
  }
}

__global__ void __launch_bounds__(256) splice_valid_kernel(
    const int64_t* __restrict__ len1, const int64_t* __restrict__ len2,
    const int64_t* __restrict__ s1, const int64_t* __restrict__ e1,
    const int64_t* __restrict__ s2, const int64_t* __restrict__ e2,
    const uint8_t* __restrict__ candidate, uint8_t* __restrict__ valid, int64_t N, int64_t L) {
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n1 = s1[n] + (e2[n] - s2[n] + 1) + (len1[n] - (e1[n] + 1));
    const int64_t n2 = s2[n] + (e1[n] - s1[n] + 1) + (len2[n] - (e2[n] + 1));
    const bool ok = n1 <= L && n2 <= L;
    valid[n] = (ok && (!candidate || candidate[n] != 0)) ? 1 : 0;
  }
}

// One thread per (pair, position): the two children's bytes at that position.
__global__ void __launch_bounds__(256) splice_rows_kernel(
    const uint8_t* __restrict__ p1src, const uint8_t* __restrict__ p2src,
    const int64_t* __restrict__ p1_rows, const int64_t* __restrict__ p2_rows,
    const int64_t* __restrict__ c1_rows, const int64_t* __restrict__ c2_rows,
    const int64_t* __restrict__ s1v, const int64_t* __restrict__ e1v,
    const int64_t* __restrict__ s2v, const int64_t* __restrict__ e2v,
    const uint8_t* __restrict__ cx_mask, uint8_t* child1, uint8_t* child2, int64_t N, int L,
    int pad, const float* __restrict__ ind_rand, float cut, ws_point_mutation m, int mutate) {
  const int64_t total = N * (int64_t)L;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = i / L;
    const int t = (int)(i - n * L);
    const int64_t r1 = p1_rows ? p1_rows[n] : n, r2 = p2_rows ? p2_rows[n] : n;
    const int64_t o1 = c1_rows ? c1_rows[n] : n, o2 = c2_rows ? c2_rows[n] : n;
    const uint8_t* a = p1src + r1 * (int64_t)L;
    const uint8_t* b = p2src + r2 * (int64_t)L;
    uint8_t v1, v2;
    if (cx_mask && cx_mask[n] == 0) {
      v1 = a[t];
      v2 = b[t];
    } else {
      const int64_t s1 = s1v[n], e1 = e1v[n], s2 = s2v[n], e2 = e2v[n];
      const int64_t cut1 = s1 + (e2 - s2 + 1), cut2 = s2 + (e1 - s1 + 1);
      // child 1 = a[0, s1) + b[s2, e2] + a(e1, ...); child 2 the mirror image
      int64_t j1;
      const uint8_t* from1;
      if (t < s1) { j1 = t; from1 = a; }
      else if (t < cut1) { j1 = s2 + (t - s1); from1 = b; }
      else { j1 = e1 + 1 + (t - cut1); from1 = a; }
      v1 = (j1 >= 0 && j1 < L) ? from1[j1] : (uint8_t)pad;
      int64_t j2;
      const uint8_t* from2;
      if (t < s2) { j2 = t; from2 = b; }
      else if (t < cut2) { j2 = s1 + (t - s2); from2 = a; }
      else { j2 = e2 + 1 + (t - cut2); from2 = b; }
      v2 = (j2 >= 0 && j2 < L) ? from2[j2] : (uint8_t)pad;
    }
    if (mutate) {
      if (o1 != 0 && ind_rand[o1] < cut) v1 = philox_mutate(v1, (uint64_t)o1, t, L, m, pad);
      if (o2 != 0 && ind_rand[o2] < cut) v2 = philox_mutate(v2, (uint64_t)o2, t, L, m, pad);
    }
    child1[o1 * (int64_t)L + t] = v1;
    child2[o2 * (int64_t)L + t] = v2;
  }
}

__global__ void __launch_bounds__(256) mutate_rows_kernel(uint8_t* pop,
                                                          const int64_t* __restrict__ rows,
                                                          int64_t N, int L,
                                                          const float* __restrict__ ind_rand,
                                                          float cut, ws_point_mutation m,
                                                          int pad) {
  const int64_t total = N * (int64_t)L;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = i / L;
    const int t = (int)(i - n * L);
    const int64_t row = rows[n];
    if (row == 0 || ind_rand[row] >= cut) continue;
    uint8_t* p = pop + row * (int64_t)L + t;
    *p = philox_mutate(*p, (uint64_t)row, t, L, m, pad);
  }
}

__global__ void __launch_bounds__(256) sbx_kernel(const float* __restrict__ consts,
                                                  const int64_t* __restrict__ p1_rows,
                                                  const int64_t* __restrict__ p2_rows,
                                                  const float* __restrict__ u_sbx,
                                                  const float* __restrict__ mask_rand,
                                                  float* __restrict__ out1,
                                                  float* __restrict__ out2, int64_t total,
                                                  int64_t K, float eta) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pair = i / K, k = i - pair * K;
    const float c1 = consts[(p1_rows ? p1_rows[pair] : pair) * K + k];
    const float c2 = consts[(p2_rows ? p2_rows[pair] : pair) * K + k];
    if (mask_rand[i] >= 0.5f) {
      out1[i] = c1;
      out2[i] = c2;
      continue;
    }
    // simulated binary crossover with distribution index eta
    const float u = u_sbx[i];
    const float inv = 1.0f / (eta + 1.0f);
    float beta;
    if (u <= 0.5f) {
      beta = powf(2.0f * u, inv);
    } else {
      const float denom = fminf(fmaxf(1.0f - u, 1e-7f), 1.0f);
      beta = powf(1.0f / (2.0f * denom), inv);
    }
    out1[i] = 0.5f * ((1.0f + beta) * c1 + (1.0f - beta) * c2);
    out2[i] = 0.5f * ((1.0f - beta) * c1 + (1.0f + beta) * c2);
  }
}

// The constants of one child, in the order its `C` tokens appear: the head's from parent A (its
// own C numbering), the spliced subtree's from parent B (numbered from B's start), the tail's
// from A (numbering continued past A's removed subtree); unused slots take A's values slot by
// slot.
__device__ void child_constants(const uint8_t* a, const uint8_t* b, const float* ca,
                                const float* cb, int64_t sa, int64_t ea, int64_t sb, int64_t eb,
                                int L, int K, int idC, float* out) {
  int w = 0, na = 0, nb = 0;
  for (int64_t i = 0; i < sa; ++i)
    if (a[i] == idC) {
      if (w < K && na < K) out[w++] = ca[na];
      ++na;
    }
  for (int64_t i = 0; i < sb; ++i) nb += (b[i] == idC);
  for (int64_t i = sb; i <= eb; ++i)
    if (b[i] == idC) {
      if (w < K && nb < K) out[w++] = cb[nb];
      ++nb;
    }
  for (int64_t i = sa; i <= ea; ++i) na += (a[i] == idC);
  for (int64_t i = ea + 1; i < L; ++i)
    if (a[i] == idC) {
      if (w < K && na < K) out[w++] = ca[na];
      ++na;
    }
  for (; w < K; ++w) out[w] = ca[w];
}

__global__ void __launch_bounds__(256) splice_consts_kernel(
    const uint8_t* __restrict__ pop, const int64_t* __restrict__ p1_rows,
    const int64_t* __restrict__ p2_rows, const float* __restrict__ cons1,
    const float* __restrict__ cons2, const int64_t* __restrict__ s1v,
    const int64_t* __restrict__ e1v, const int64_t* __restrict__ s2v,
    const int64_t* __restrict__ e2v, const uint8_t* __restrict__ cx_mask, float* child,
    const int64_t* __restrict__ c1_rows, const int64_t* __restrict__ c2_rows, int64_t N, int L,
    int K, int idC) {
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t* a = pop + (p1_rows ? p1_rows[n] : n) * (int64_t)L;
    const uint8_t* b = pop + (p2_rows ? p2_rows[n] : n) * (int64_t)L;
    const float* ca = cons1 + n * K;
    const float* cb = cons2 + n * K;
    float* o1 = child + (c1_rows ? c1_rows[n] : n) * (int64_t)K;
    float* o2 = child + (c2_rows ? c2_rows[n] : n) * (int64_t)K;
    if (cx_mask && cx_mask[n] == 0) {
      for (int k = 0; k < K; ++k) {
        o1[k] = ca[k];
        o2[k] = cb[k];
      }
      continue;
    }
    const int64_t s1 = s1v[n], e1 = e1v[n], s2 = s2v[n], e2 = e2v[n];
    child_constants(a, b, ca, cb, s1, e1, s2, e2, L, K, idC, o1);
    child_constants(b, a, cb, ca, s2, e2, s1, e1, L, K, idC, o2);
  }
}

__global__ void __launch_bounds__(128) hoist_rows_kernel(uint8_t* pop,
                                                         const int64_t* __restrict__ rows,
                                                         int64_t N, int L,
                                                         const int32_t* __restrict__ ar,
                                                         int vocab,
                                                         const int64_t* __restrict__ rand_ints,
                                                         int pad) {
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (int64_t)gridDim.x * blockDim.x) {
    uint8_t* row = pop + rows[n] * (int64_t)L;
    uint64_t state = (uint64_t)rand_ints[n];
    int pick_s = -1, pick_e = -1, seen = 0;
    for (int e = 0; e < L && (int)row[e] != pad; ++e) {
      const int a = arity_of(ar, vocab, row[e]);
      int s = e;
      bool ok = a == 0;
      if (a > 0) {
        int need = a;
        for (int j = e - 1; j >= 0 && (int)row[j] != pad; --j) {
          need += arity_of(ar, vocab, row[j]) - 1;
          if (need == 0) {
            s = j;
            ok = true;
            break;
          }
        }
      }
      if (!ok) continue;
      ++seen;  // reservoir sampling: the k-th subtree replaces the pick with probability 1/k
      state = state * 6364136223846793005ull + 1ull;
      if (state % (uint64_t)seen == 0) {
        pick_s = s;
        pick_e = e;
      }
    }
    if (pick_e < 0) continue;
    const int len = pick_e - pick_s + 1;
    for (int i = 0; i < len; ++i) row[i] = row[pick_s + i];
    for (int i = len; i < L; ++i) row[i] = (uint8_t)pad;
  }
}

// The same hoist with one warp per row (rows of at most kHoistStagedL tokens): the row and the
// arity table sit in shared memory, each lane runs the backward subtree scan for its own end
// positions e = lane, lane + 32, ..., and the reservoir sampling then walks the valid positions
// in ascending order from a ballot mask -- the same LCG steps and the same picks as one thread
// walking e = 0, 1, 2, ... -- identically in every lane.
constexpr int kHoistStagedL = 255;
constexpr int kHoistWarps = 4;
__global__ void __launch_bounds__(32 * kHoistWarps) hoist_rows_warp_kernel(
    uint8_t* pop, const int64_t* __restrict__ rows, int64_t N, int L,
    const int32_t* __restrict__ ar, int vocab, const int64_t* __restrict__ rand_ints, int pad) {
  __shared__ int32_t s_ar[256];
  __shared__ uint8_t s_row[kHoistWarps][256];
  __shared__ uint8_t s_start[kHoistWarps][256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) s_ar[t] = t < vocab ? ar[t] : 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* srow = s_row[w];
  uint8_t* sst = s_start[w];
  for (int64_t n = (int64_t)blockIdx.x * kHoistWarps + w; n < N;
       n += (int64_t)gridDim.x * kHoistWarps) {
    uint8_t* row = pop + rows[n] * (int64_t)L;
    int len = L;  // the first PAD
    for (int c0 = 0; c0 < L; c0 += 32) {
      const int i = c0 + lane;
      const uint8_t b = i < L ? row[i] : (uint8_t)pad;
      if (i < L) srow[i] = b;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, i < L && (int)b == pad);
      if (m) {
        len = c0 + __ffs(m) - 1;
        break;
      }
    }
    __syncwarp();
    const uint64_t state0 = (uint64_t)rand_ints[n];
    uint64_t state = state0;
    int pick_s = -1, pick_e = -1, seen = 0;
    for (int c0 = 0; c0 < len; c0 += 32) {
      const int e = c0 + lane;
      bool ok = false;
      int s = e;
      if (e < len) {
        const int a = s_ar[srow[e]];
        ok = a == 0;
        if (a > 0) {
          int need = a;
          for (int j = e - 1; j >= 0; --j) {
            need += s_ar[srow[j]] - 1;
            if (need == 0) {
              s = j;
              ok = true;
              break;
            }
          }
        }
        sst[e] = (uint8_t)s;
      }
      unsigned m = __ballot_sync(0xFFFFFFFFu, ok);
      __syncwarp();
      for (; m; m &= m - 1) {  // valid subtrees in ascending end position: reservoir sampling
        const int e2 = c0 + __ffs(m) - 1;
        ++seen;
        state = state * 6364136223846793005ull + 1ull;
        if (state % (uint64_t)seen == 0) {
          pick_e = e2;
          pick_s = sst[e2];
        }
      }
    }
    if (pick_e >= 0) {
      const int cnt = pick_e - pick_s + 1;
      for (int i = lane; i < L; i += 32) row[i] = i < cnt ? srow[pick_s + i] : (uint8_t)pad;
    }
    __syncwarp();  // the row buffers are rewritten for the next row
  }
}

unsigned grid_for(int64_t n, int threads) {
  const int64_t g = (n + threads - 1) / threads;
  return (unsigned)(g < 65535 * 16 ? (g > 0 ? g : 1) : 65535 * 16);
}

ws_status launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, what);
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" ws_status ws_subtree_pick(const uint8_t* population, const int64_t* rows, int64_t N,
                                     int64_t L, const int32_t* arities, int32_t vocab,
                                     const float* u, int64_t* out_len, int64_t* out_start,
                                     int64_t* out_end, int32_t pad_id, void* stream) {
  clear_error();
  if (N < 0 || L < 1 || L > 65535) return fail("subtree_pick: bad shape");
  if (N == 0) return WS_OK;
  if (!population || !arities || !u || !out_len || !out_start || !out_end)
    return fail("null tensor pointer");
  subtree_pick_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      population, rows, N, (int)L, arities, vocab, u, out_len, out_start, out_end, pad_id);
  return launched("subtree_pick");
}

extern "C" ws_status ws_splice_valid(const int64_t* len1, const int64_t* len2, const int64_t* s1,
                                     const int64_t* e1, const int64_t* s2, const int64_t* e2,
                                     const uint8_t* candidate, uint8_t* valid, int64_t N,
                                     int64_t L, void* stream) {
  clear_error();
  if (N < 0) return fail("splice_valid: bad shape");
  if (N == 0) return WS_OK;
  if (!len1 || !len2 || !s1 || !e1 || !s2 || !e2 || !valid) return fail("null tensor pointer");
  splice_valid_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      len1, len2, s1, e1, s2, e2, candidate, valid, N, L);
  return launched("splice_valid");
}

extern "C" ws_status ws_splice_rows(const uint8_t* parent1, const uint8_t* parent2,
                                    const int64_t* p1_rows, const int64_t* p2_rows,
                                    const int64_t* c1_rows, const int64_t* c2_rows,
                                    const int64_t* s1, const int64_t* e1, const int64_t* s2,
                                    const int64_t* e2, const uint8_t* cx_mask, uint8_t* child1,
                                    uint8_t* child2, int64_t N, int64_t L, int32_t pad_id,
                                    const float* individual_rand, float cut,
                                    const ws_point_mutation* mutation, void* stream) {
  clear_error();
  if (N < 0 || L < 1 || L > 65535) return fail("splice_rows: bad shape");
  if (N == 0) return WS_OK;
  if (!parent1 || !parent2 || !s1 || !e1 || !s2 || !e2 || !child1 || !child2)
    return fail("null tensor pointer");
  if (mutation && (!individual_rand || !mutation->arities)) return fail("null tensor pointer");
  ws_point_mutation m{};
  if (mutation) m = *mutation;
  splice_rows_kernel<<<grid_for(N * L, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      parent1, parent2, p1_rows, p2_rows, c1_rows, c2_rows, s1, e1, s2, e2, cx_mask, child1,
      child2, N, (int)L, pad_id, individual_rand, cut, m, mutation ? 1 : 0);
  return launched("splice_rows");
}

extern "C" ws_status ws_mutate_rows(uint8_t* population, const int64_t* rows, int64_t N,
                                    int64_t L, const float* individual_rand, float cut,
                                    const ws_point_mutation* mutation, int32_t pad_id,
                                    void* stream) {
  clear_error();
  if (N < 0 || L < 1 || L > 65535) return fail("mutate_rows: bad shape");
  if (N == 0) return WS_OK;
  if (!population || !rows || !individual_rand || !mutation || !mutation->arities)
    return fail("null tensor pointer");
  mutate_rows_kernel<<<grid_for(N * L, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      population, rows, N, (int)L, individual_rand, cut, *mutation, pad_id);
  return launched("mutate_rows");
}

extern "C" ws_status ws_sbx_constants(const float* constants, const int64_t* p1_rows,
                                      const int64_t* p2_rows, const float* u_sbx,
                                      const float* mask_rand, float* out1, float* out2,
                                      int64_t n_pairs, int64_t K, float eta, void* stream) {
  clear_error();
  if (n_pairs < 0 || K < 0) return fail("sbx_constants: bad shape");
  if (n_pairs == 0 || K == 0) return WS_OK;
  if (!constants || !u_sbx || !mask_rand || !out1 || !out2) return fail("null tensor pointer");
  sbx_kernel<<<grid_for(n_pairs * K, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      constants, p1_rows, p2_rows, u_sbx, mask_rand, out1, out2, n_pairs * K, K, eta);
  return launched("sbx_constants");
}

extern "C" ws_status ws_splice_constants(const uint8_t* population, const int64_t* p1_rows,
                                         const int64_t* p2_rows, const float* consts1,
                                         const float* consts2, const int64_t* s1,
                                         const int64_t* e1, const int64_t* s2, const int64_t* e2,
                                         const uint8_t* cx_mask, float* child_consts,
                                         const int64_t* c1_rows, const int64_t* c2_rows,
                                         int64_t N, int64_t L, int64_t K, int32_t id_C,
                                         void* stream) {
  clear_error();
  if (N < 0 || L < 1 || K < 0 || L > 65535 || K > 65535) return fail("splice_constants: bad shape");
  if (N == 0 || K == 0) return WS_OK;
  if (!population || !consts1 || !consts2 || !s1 || !e1 || !s2 || !e2 || !child_consts)
    return fail("null tensor pointer");
  splice_consts_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      population, p1_rows, p2_rows, consts1, consts2, s1, e1, s2, e2, cx_mask, child_consts,
      c1_rows, c2_rows, N, (int)L, (int)K, id_C);
  return launched("splice_constants");
}

extern "C" ws_status ws_hoist_rows(uint8_t* population, const int64_t* rows, int64_t N,
                                   int64_t L, const int32_t* arities, int32_t vocab,
                                   const int64_t* rand_ints, int32_t pad_id, void* stream) {
  clear_error();
  if (N < 0 || L < 1 || L > 65535) return fail("hoist_rows: bad shape");
  if (N == 0) return WS_OK;
  if (!population || !rows || !arities || !rand_ints) return fail("null tensor pointer");
  if (L <= kHoistStagedL && vocab <= 256) {
    hoist_rows_warp_kernel<<<grid_for(N, kHoistWarps), 32 * kHoistWarps, 0,
                             static_cast<cudaStream_t>(stream)>>>(
        population, rows, N, (int)L, arities, vocab, rand_ints, pad_id);
  } else {
    hoist_rows_kernel<<<grid_for(N, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        population, rows, N, (int)L, arities, vocab, rand_ints, pad_id);
  }
  return launched("hoist_rows");
}
