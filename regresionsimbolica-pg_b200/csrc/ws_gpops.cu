// ws_gpops.cu -- the reference extension's genetic-operator and bookkeeping kernels, restated:
// point mutation from pre-drawn randoms (mutate_population), subtree splicing (crossover_splicing),
// in-place constant perturbation (constant_perturbation), valid random program generation
// (generate_random_rpn) and device-side best tracking (update_best, check_improvement,
// batch_update_best).  Same inputs -> same outputs, bit for bit; the two tracker reductions the
// reference runs across several blocks without ordering are made deterministic (see below).
//
// These are byte / integer passes bound by memory traffic (or, for the generator and the
// trackers, by one thread's serial loop); the launches use grid-stride loops sized to the GPU.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "ws_internal.h"

namespace ws {
namespace {

unsigned grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)device_info().sm_count * 16;
  if (g > cap) g = cap;
  return (unsigned)(g < 1 ? 1 : g);
}

// mutation_kernel (rpn_kernels.cu:772-813): each non-PAD token with rand_floats < rate is
// replaced by arity_k_ids[rand_ints % n_k] of its own arity (tokens outside the table count as
// arity 0).
__global__ void __launch_bounds__(256) mutate_kernel(
    uint8_t* __restrict__ pop, int64_t total, const float* __restrict__ rf,
    const int64_t* __restrict__ ri, const int32_t* __restrict__ arities, int vocab,
    const uint8_t* __restrict__ a0, int n0, const uint8_t* __restrict__ a1, int n1,
    const uint8_t* __restrict__ a2, int n2, float rate, int pad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int tok = pop[i];
    if (tok == pad || !(rf[i] < rate)) continue;
    const int ar = tok < vocab ? arities[tok] : 0;
    const uint64_t r = (uint64_t)ri[i];
    int nt = tok;
    if (ar == 0 && n0 > 0) nt = a0[r % (uint64_t)n0];
    else if (ar == 1 && n1 > 0) nt = a1[r % (uint64_t)n1];
    else if (ar == 2 && n2 > 0) nt = a2[r % (uint64_t)n2];
    pop[i] = (uint8_t)nt;
  }
}

// The same, four tokens per thread: one 4-byte token load, one 16-byte load of their uniforms,
// the replacement ids read only for the tokens that mutate, one 4-byte store when any did
// (total % 4 == 0, the population 4-byte and the uniforms 16-byte aligned).
__global__ void __launch_bounds__(256) mutate4_kernel(
    uint8_t* __restrict__ pop, int64_t total4, const float* __restrict__ rf,
    const int64_t* __restrict__ ri, const int32_t* __restrict__ arities, int vocab,
    const uint8_t* __restrict__ a0, int n0, const uint8_t* __restrict__ a1, int n1,
    const uint8_t* __restrict__ a2, int n2, float rate, int pad) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total4;
       q += (int64_t)gridDim.x * blockDim.x) {
    uint32_t w = reinterpret_cast<const uint32_t*>(pop)[q];
    const float4 f = __ldg(reinterpret_cast<const float4*>(rf) + q);
    const float fr[4] = {f.x, f.y, f.z, f.w};
    uint32_t nw = w;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int tok = (w >> (8 * k)) & 0xFFu;
      if (tok == pad || !(fr[k] < rate)) continue;
      const int ar = tok < vocab ? __ldg(arities + tok) : 0;
      const uint64_t r = (uint64_t)__ldg(reinterpret_cast<const long long*>(ri) + 4 * q + k);
      int nt = tok;
      if (ar == 0 && n0 > 0) nt = a0[r % (uint64_t)n0];
      else if (ar == 1 && n1 > 0) nt = a1[r % (uint64_t)n1];
      else if (ar == 2 && n2 > 0) nt = a2[r % (uint64_t)n2];
      nw = (nw & ~(0xFFu << (8 * k))) | ((uint32_t)nt << (8 * k));
    }
    if (nw != w) reinterpret_cast<uint32_t*>(pop)[q] = nw;
  }
}

// crossover_splicing_kernel (rpn_kernels.cu:927-1016): child1 = p1[0:s1] + p2[s2:e2+1] +
// p1[e1+1:], child2 symmetric; positions whose source index leaves [0, L) are PAD; pairs with a
// false mask copy their parents.
__device__ __forceinline__ uint8_t splice_at(const uint8_t* a, const uint8_t* b, int64_t sa,
                                             int64_t ea, int64_t sb, int64_t eb, int64_t t,
                                             int64_t L, int pad) {
  const int64_t pre = sa, cut = sa + (eb - sb + 1);
  int64_t src;
  const uint8_t* from;
  if (t < pre) {
    src = t;
    from = a;
  } else if (t < cut) {
    src = sb + t - pre;
    from = b;
  } else {
    src = ea + 1 + t - cut;
    from = a;
  }
  return (src >= 0 && src < L) ? from[src] : (uint8_t)pad;
}

__global__ void __launch_bounds__(256) splice_kernel(
    const uint8_t* __restrict__ p1, const uint8_t* __restrict__ p2, int64_t N, int64_t L,
    const int64_t* __restrict__ s1, const int64_t* __restrict__ e1,
    const int64_t* __restrict__ s2, const int64_t* __restrict__ e2,
    const uint8_t* __restrict__ mask, uint8_t* __restrict__ c1, uint8_t* __restrict__ c2,
    int pad) {
  const int64_t total = N * L;
  const bool narrow = total < ((int64_t)1 << 31);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t n, t;
    if (narrow) {  // 32-bit division: the 64-bit one costs more than the copy
      const uint32_t q = (uint32_t)i / (uint32_t)L;
      n = q;
      t = (int64_t)((uint32_t)i - q * (uint32_t)L);
    } else {
      n = i / L;
      t = i - n * L;
    }
    const uint8_t* a = p1 + n * L;
    const uint8_t* b = p2 + n * L;
    if (mask && !mask[n]) {
      c1[i] = a[t];
      c2[i] = b[t];
      continue;
    }
    c1[i] = splice_at(a, b, s1[n], e1[n], s2[n], e2[n], t, L, pad);
    c2[i] = splice_at(b, a, s2[n], e2[n], s1[n], e1[n], t, L, pad);
  }
}

// The same with rows of L % 16 == 0 bytes (L <= 256, 16-byte aligned rows): a pair's two parent
// rows are staged in shared memory by 16-byte loads (S = L / 16 threads per pair), each thread
// builds one 16-byte segment of both children there and writes each with one 16-byte store.
// 8 KB of shared memory per 256-thread block.
__global__ void __launch_bounds__(256) splice16_kernel(
    const uint8_t* __restrict__ p1, const uint8_t* __restrict__ p2, int64_t N, int64_t L,
    const int64_t* __restrict__ s1, const int64_t* __restrict__ e1,
    const int64_t* __restrict__ s2, const int64_t* __restrict__ e2,
    const uint8_t* __restrict__ mask, uint8_t* __restrict__ c1, uint8_t* __restrict__ c2,
    int pad) {
  __shared__ __align__(16) uint8_t sm[256 * 2 * 16];  // [pairs][parent][L]
  const int S = (int)(L >> 4);
  const int P = (int)blockDim.x / S;  // pairs per block step
  const int pr = (int)threadIdx.x / S, seg = (int)threadIdx.x - pr * S;
  uint8_t* ra = sm + (size_t)pr * 2 * L;
  uint8_t* rb = ra + L;
  for (int64_t n0 = (int64_t)blockIdx.x * P; n0 < N; n0 += (int64_t)gridDim.x * P) {
    const int64_t n = n0 + pr;
    const bool act = pr < P && n < N;
    if (act) {
      reinterpret_cast<uint4*>(ra)[seg] = __ldg(reinterpret_cast<const uint4*>(p1 + n * L) + seg);
      reinterpret_cast<uint4*>(rb)[seg] = __ldg(reinterpret_cast<const uint4*>(p2 + n * L) + seg);
    }
    __syncthreads();
    if (act) {
      const bool copy = mask && !mask[n];
      const int64_t as = s1[n], ae = e1[n], bs = s2[n], be = e2[n];
      uint32_t o1[4] = {0u, 0u, 0u, 0u}, o2[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int64_t t = (int64_t)seg * 16 + k;
        const uint32_t x1 = copy ? ra[t] : splice_at(ra, rb, as, ae, bs, be, t, L, pad);
        const uint32_t x2 = copy ? rb[t] : splice_at(rb, ra, bs, be, as, ae, t, L, pad);
        o1[k >> 2] |= x1 << (8 * (k & 3));
        o2[k >> 2] |= x2 << (8 * (k & 3));
      }
      reinterpret_cast<uint4*>(c1 + n * L)[seg] = make_uint4(o1[0], o1[1], o1[2], o1[3]);
      reinterpret_cast<uint4*>(c2 + n * L)[seg] = make_uint4(o2[0], o2[1], o2[2], o2[3]);
    }
    __syncthreads();
  }
}

// constant_perturbation_kernel (rpn_kernels.cu:1455-1499): a row is perturbed when its hashed
// uniform is below `rate`; each of its constants moves by z * (|c| * sigma + 1e-4) with z from
// Box-Muller of two hashed uniforms, then is clamped to [c_min, c_max].  The hash is the
// published 32-bit integer mixer (xor-shift 16/15/16 with multipliers 0x7feb352d, 0x846ca68b).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float unit_open(uint32_t x) {
  return ((mix32(x) >> 8) + 1.0f) * (1.0f / 16777217.0f);
}

template <typename T>
__global__ void __launch_bounds__(256) perturb_kernel(T* __restrict__ c, int64_t B, int64_t K,
                                                      float rate, float sigma, float cmin,
                                                      float cmax, uint32_t seed) {
  // one thread per row: the row's draw decides once whether any of its constants move
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < B;
       row += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t rk = seed ^ ((uint32_t)(row + 1) * 0x9e3779b9u);
    if (unit_open(rk) >= rate) continue;
    T* cr = c + row * K;
    for (int64_t col = 0; col < K; ++col) {
      const uint32_t k1 = rk ^ ((uint32_t)(col + 1) * 0x85ebca6bu);
      const uint32_t k2 = rk ^ ((uint32_t)(col + 1) * 0xc2b2ae35u);
      const float u1 = fmaxf(unit_open(k1), 1e-7f);
      const float u2 = unit_open(k2);
      const float z = sqrtf(-2.0f * logf(u1)) * cosf(6.283185307179586f * u2);
      const float v = (float)cr[col];
      const float scale = fabsf(v) * sigma + 1e-4f;
      float nv = v + z * scale;
      nv = fminf(fmaxf(nv, cmin), cmax);
      cr[col] = (T)nv;
    }
  }
}

// generate_random_rpn_kernel (genrand_kernels.cu:70-175): one program per thread from a
// xorshift64 stream (shifts 13, 7, 17) seeded with seed + b * 6364136223846793005 +
// 1442695040888963407 and advanced twice; at each position the categories that can still close
// the program at depth 1 are weighted (terminal / unary / binary weights), one is drawn, then a
// token of it; the program ends at the first position after the first where the depth is 1; a
// program that cannot close becomes the first terminal alone.
__device__ __forceinline__ float xs_uniform(uint64_t& s) {
  uint64_t x = s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  s = x;
  return (float)(x & 0xFFFFFF) / 16777216.0f;
}
__device__ __forceinline__ int xs_int(uint64_t& s, int n) {
  const int r = (int)(xs_uniform(s) * n);
  return min(r, n - 1);
}

__global__ void __launch_bounds__(128) genrand_kernel(
    uint8_t* __restrict__ pop, int64_t B, int L, const uint8_t* __restrict__ term, int nt,
    const uint8_t* __restrict__ un, int nu, const uint8_t* __restrict__ bin, int nb,
    uint64_t seed, float wt, float wu, float wb) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    uint64_t st = seed + (uint64_t)b * 6364136223846793005ull + 1442695040888963407ull;
    xs_uniform(st);
    xs_uniform(st);
    uint8_t* row = pop + b * L;
    // tokens are packed four to a word and stored a word at a time when rows are 4-byte
    // aligned (byte stores from 32 rows per warp instruction would touch 32 sectors each)
    const bool words = ((L & 3) == 0) && ((((uintptr_t)pop) & 3u) == 0);
    uint32_t word = 0u;
    auto put = [&](int j, uint8_t t) {
      if (!words) {
        row[j] = t;
        return;
      }
      word |= (uint32_t)t << (8 * (j & 3));
      if ((j & 3) == 3) {
        *reinterpret_cast<uint32_t*>(row + (j & ~3)) = word;
        word = 0u;
      }
    };
    int depth = 0;
    bool closed = false;
    for (int j = 0; j < L; ++j) {
      if (closed) {
        put(j, 0);
        continue;
      }
      const int rem = L - j - 1;
      bool ct = (depth + 1 >= 1) && (depth + 1 <= 1 + rem);
      bool cu = nu > 0 && depth >= 1 && depth <= 1 + rem;
      bool cb = nb > 0 && depth - 1 >= 1 && depth - 1 <= 1 + rem;
      if (rem == 0) {
        ct = ct && depth + 1 == 1;
        cu = cu && depth == 1;
        cb = cb && depth - 1 == 1;
      }
      float w_t = ct ? wt : 0.0f;
      const float w_u = cu ? wu : 0.0f;
      const float w_b = cb ? wb : 0.0f;
      float tw = w_t + w_u + w_b;
      if (tw <= 1e-6f) {  // no category can follow: a terminal (operator weights stay)
        w_t = 1.0f;
        tw = 1.0f;
      }
      const float r = xs_uniform(st);
      const float pt = w_t / tw;
      const float pu = w_u / tw;
      uint8_t tok;
      int dd;
      // (the reference indexes an empty operator list here when rounding of pt + pu below 1
      // sends r past it; that read is out of bounds there, a terminal here)
      if (r < pt || (r >= pt + pu ? nb == 0 : nu == 0)) {
        tok = term[xs_int(st, nt)];
        dd = 1;
      } else if (r < pt + pu) {
        tok = un[xs_int(st, nu)];
        dd = 0;
      } else {
        tok = bin[xs_int(st, nb)];
        dd = -1;
      }
      put(j, tok);
      depth += dd;
      if (depth == 1 && j > 0) closed = true;
    }
    if (depth != 1) {
      row[0] = term[0];
      for (int j = 1; j < L; ++j) row[j] = 0;
    }
  }
}

// Best trackers (best_tracker_kernels.cu:47-231): the lowest fitness of the generation by a
// 256-thread block -- each thread keeps the first strictly smaller value of its strided slice,
// the tree keeps the lower thread on ties -- replaces the tracked best when it is lower by more
// than `tolerance`.  The reference's update_best and check_improvement launch up to 256 blocks
// whose first threads each read and write the tracker without ordering, so with more than 256
// programs their outcome depends on block scheduling; here one block reduces all programs, the
// reference's result whenever it is deterministic (B <= 256) and otherwise the global minimum.
__device__ void block_argmin(const float* __restrict__ f, int64_t B, float& v, int& idx) {
  __shared__ float sv[256];
  __shared__ int si[256];
  const int tid = threadIdx.x;
  float m = 1e30f;
  int mi = -1;
  for (int64_t i = tid; i < B; i += blockDim.x) {
    const float x = f[i];
    if (x < m) {
      m = x;
      mi = (int)i;
    }
  }
  sv[tid] = m;
  si[tid] = mi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s && sv[tid + s] < sv[tid]) {
      sv[tid] = sv[tid + s];
      si[tid] = si[tid + s];
    }
    __syncthreads();
  }
  v = sv[0];
  idx = si[0];
}

__global__ void __launch_bounds__(256) update_best_kernel(
    const int64_t* __restrict__ pop, int64_t B, int64_t L, const float* __restrict__ consts,
    int64_t K, const float* __restrict__ fit, int64_t* t_rpn, float* t_consts, float* t_rmse,
    int32_t* t_idx, int32_t* t_gen, int32_t* t_len, int32_t* t_upd, int gen, float tol) {
  float v;
  int bi;
  block_argmin(fit, B, v, bi);
  if (threadIdx.x == 0) {
    if (v < t_rmse[0] - tol) {
      if (bi >= 0 && bi < B) {
        for (int64_t j = 0; j < L && j < 256; ++j) t_rpn[j] = pop[bi * L + j];
        for (int64_t k = 0; k < K && k < 32; ++k) t_consts[k] = consts[bi * K + k];
        t_rmse[0] = v;
        t_idx[0] = bi;
        t_gen[0] = gen;
        t_len[0] = (int32_t)L;
        t_upd[0] = 1;
      }
    } else {
      t_upd[0] = 0;
    }
  }
}

__global__ void __launch_bounds__(256) check_improvement_kernel(const float* __restrict__ fit,
                                                                int64_t B,
                                                                const float* __restrict__ tracked,
                                                                int32_t* improved, float tol) {
  __shared__ float sm[256];
  const int tid = threadIdx.x;
  float m = 1e30f;
  for (int64_t i = tid; i < B; i += blockDim.x) m = fminf(m, fit[i]);
  sm[tid] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s) sm[tid] = fminf(sm[tid], sm[tid + s]);
    __syncthreads();
  }
  if (tid == 0) improved[0] = (sm[0] < tracked[0] - tol) ? 1 : 0;
}

__global__ void __launch_bounds__(256) batch_update_best_kernel(
    const uint8_t* __restrict__ pop, int64_t B, int64_t L, const float* __restrict__ consts,
    int64_t K, const float* __restrict__ fit, uint8_t* b_rpn, float* b_consts, float* b_rmse,
    int32_t* b_idx, float tol) {
  float v;
  int bi;
  block_argmin(fit, B, v, bi);
  if (threadIdx.x == 0 && v < b_rmse[0] - tol && bi >= 0) {
    b_rmse[0] = v;
    b_idx[0] = bi;
    for (int64_t j = 0; j < L; ++j) b_rpn[j] = pop[(int64_t)bi * L + j];
    for (int64_t k = 0; k < K; ++k) b_consts[k] = consts[(int64_t)bi * K + k];
  }
}

ws_status launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, what);
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

ws_status ws_mutate_population(uint8_t* population, int64_t B, int64_t L, const float* rand_floats,
                               const int64_t* rand_ints, const int32_t* token_arities,
                               int64_t vocab_size, const uint8_t* arity0_ids, int64_t n0,
                               const uint8_t* arity1_ids, int64_t n1, const uint8_t* arity2_ids,
                               int64_t n2, float mutation_rate, int32_t pad_id, void* stream) {
  clear_error();
  if (B < 0 || L < 0 || vocab_size < 0 || n0 < 0 || n1 < 0 || n2 < 0) return fail("negative size");
  if (B * L == 0) return WS_OK;
  if (!population || !rand_floats || !rand_ints || (vocab_size > 0 && !token_arities) ||
      (n0 > 0 && !arity0_ids) || (n1 > 0 && !arity1_ids) || (n2 > 0 && !arity2_ids))
    return fail("null tensor pointer");
  const int64_t total = B * L;
  if (total % 4 == 0 && (uintptr_t)population % 4 == 0 && (uintptr_t)rand_floats % 16 == 0)
    mutate4_kernel<<<grid_for(total / 4, 256), 256, 0, (cudaStream_t)stream>>>(
        population, total / 4, rand_floats, rand_ints, token_arities, (int)vocab_size,
        arity0_ids, (int)n0, arity1_ids, (int)n1, arity2_ids, (int)n2, mutation_rate, pad_id);
  else
    mutate_kernel<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(
        population, total, rand_floats, rand_ints, token_arities, (int)vocab_size, arity0_ids,
        (int)n0, arity1_ids, (int)n1, arity2_ids, (int)n2, mutation_rate, pad_id);
  return launched("mutate_population launch");
}

ws_status ws_crossover_splicing(const uint8_t* parent1, const uint8_t* parent2, int64_t N,
                                int64_t L, const int64_t* starts1, const int64_t* ends1,
                                const int64_t* starts2, const int64_t* ends2, uint8_t* child1,
                                uint8_t* child2, int32_t pad_id, const uint8_t* cx_mask,
                                void* stream) {
  clear_error();
  if (N < 0 || L < 0) return fail("negative size");
  if (N * L == 0) return WS_OK;
  if (!parent1 || !parent2 || !starts1 || !ends1 || !starts2 || !ends2 || !child1 || !child2)
    return fail("null tensor pointer");
  const bool rows16 = L % 16 == 0 && L <= 256 &&
                      (((uintptr_t)parent1 | (uintptr_t)parent2 | (uintptr_t)child1 |
                        (uintptr_t)child2) % 16) == 0;
  if (rows16) {
    const int64_t per_block = 256 / (L / 16);
    splice16_kernel<<<grid_for((N + per_block - 1) / per_block * 256, 256), 256, 0,
                      (cudaStream_t)stream>>>(parent1, parent2, N, L, starts1, ends1, starts2,
                                              ends2, cx_mask, child1, child2, pad_id);
  } else {
    splice_kernel<<<grid_for(N * L, 256), 256, 0, (cudaStream_t)stream>>>(
        parent1, parent2, N, L, starts1, ends1, starts2, ends2, cx_mask, child1, child2, pad_id);
  }
  return launched("crossover_splicing launch");
}

ws_status ws_constant_perturbation(int32_t dtype, void* constants, int64_t B, int64_t K,
                                   float rate, float sigma, float c_min, float c_max,
                                   uint32_t seed, void* stream) {
  clear_error();
  if (dtype != WS_F32 && dtype != WS_F64) return fail("constants must be float32 or float64");
  if (B < 0 || K < 0) return fail("negative size");
  if (B * K == 0 || rate <= 0.0f || sigma <= 0.0f) return WS_OK;
  if (!constants) return fail("null tensor pointer");
  const unsigned g = grid_for(B, 256);
  if (dtype == WS_F32)
    perturb_kernel<float><<<g, 256, 0, (cudaStream_t)stream>>>(
        static_cast<float*>(constants), B, K, rate, sigma, c_min, c_max, seed);
  else
    perturb_kernel<double><<<g, 256, 0, (cudaStream_t)stream>>>(
        static_cast<double*>(constants), B, K, rate, sigma, c_min, c_max, seed);
  return launched("constant_perturbation launch");
}

ws_status ws_generate_random_rpn(uint8_t* population, int64_t B, int64_t L,
                                 const uint8_t* terminal_ids, int64_t n_terminals,
                                 const uint8_t* unary_ids, int64_t n_unary,
                                 const uint8_t* binary_ids, int64_t n_binary, uint64_t seed,
                                 float term_weight, float unary_weight, float bin_weight,
                                 void* stream) {
  clear_error();
  if (n_terminals <= 0) return fail("Must have at least one terminal token");
  if (B < 0 || L < 0 || n_unary < 0 || n_binary < 0) return fail("negative size");
  if (B * L == 0) return WS_OK;
  if (!population || !terminal_ids || (n_unary > 0 && !unary_ids) ||
      (n_binary > 0 && !binary_ids))
    return fail("null tensor pointer");
  genrand_kernel<<<grid_for(B, 128), 128, 0, (cudaStream_t)stream>>>(
      population, B, (int)L, terminal_ids, (int)n_terminals, unary_ids, (int)n_unary,
      binary_ids, (int)n_binary, seed, term_weight, unary_weight, bin_weight);
  return launched("generate_random_rpn launch");
}

ws_status ws_update_best(const int64_t* population, int64_t B, int64_t L, const float* constants,
                         int64_t K, const float* fitness, int64_t* tracker_rpn,
                         float* tracker_consts, float* tracker_rmse, int32_t* tracker_idx,
                         int32_t* tracker_gen, int32_t* tracker_len, int32_t* tracker_updated,
                         int32_t current_generation, float tolerance, void* stream) {
  clear_error();
  if (B < 0 || L < 0 || K < 0) return fail("negative size");
  if (B > INT32_MAX) return fail("at most 2^31-1 programs");
  if (!fitness || !tracker_rpn || !tracker_rmse || !tracker_idx || !tracker_gen ||
      !tracker_len || !tracker_updated || (B > 0 && !population) || (K > 0 && !constants))
    return fail("null tensor pointer");
  update_best_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(
      population, B, L, constants, K, fitness, tracker_rpn, tracker_consts, tracker_rmse,
      tracker_idx, tracker_gen, tracker_len, tracker_updated, current_generation, tolerance);
  return launched("update_best launch");
}

ws_status ws_check_improvement(const float* fitness, int64_t B, const float* tracked_rmse,
                               int32_t* improved, float tolerance, void* stream) {
  clear_error();
  if (B < 0) return fail("negative size");
  if (!fitness || !tracked_rmse || !improved) return fail("null tensor pointer");
  check_improvement_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(fitness, B, tracked_rmse,
                                                                improved, tolerance);
  return launched("check_improvement launch");
}

ws_status ws_batch_update_best(const uint8_t* population, int64_t B, int64_t L,
                               const float* constants, int64_t K, const float* fitness,
                               uint8_t* best_rpn, float* best_consts, float* best_rmse,
                               int32_t* best_idx, float tolerance, void* stream) {
  clear_error();
  if (B < 0 || L < 0 || K < 0) return fail("negative size");
  if (B > INT32_MAX) return fail("at most 2^31-1 programs");
  if (!fitness || !best_rpn || !best_rmse || !best_idx || (B > 0 && !population) ||
      (K > 0 && (!constants || !best_consts)))
    return fail("null tensor pointer");
  batch_update_best_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(
      population, B, L, constants, K, fitness, best_rpn, best_consts, best_rmse, best_idx,
      tolerance);
  return launched("batch_update_best launch");
}

}  // extern "C"
