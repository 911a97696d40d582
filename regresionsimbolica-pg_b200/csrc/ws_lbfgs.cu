// ws_lbfgs.cu -- per-program constant fitting with the reference's L-BFGS kernel semantics.
//
// Replaces `lbfgs_optimize` (bindings.cpp:542-563 -> launch_lbfgs_optimize,
// lbfgs_kernels.cu:624-694; kernel :214-621).  What the reference kernel computes, step by step:
//   - fitness: RMSE of the program under its own evaluator (:278-344): literals, variables and C
//     push; every other token is a binary operator (+ - * / pow %; a unary or unknown token is
//     an error); / by |b| <= 1e-12 gives 1e30, pow is powf(|a| + 1e-12, b), % by |b| <= 1e-12
//     gives 0; any failing row makes the fitness 1e30;
//   - gradient: central differences of the RMSE with eps 1e-5 clamped to the box (:348-471),
//     whose evaluator knows only the literals 0, 1, 2, pi, e and the operators + - * / pow, and
//     skips failing rows instead of failing;
//   - iterations: the gradient is evaluated once, at the start: after an accepted step the kernel
//     copies the old gradient over the trial one (:590-593), so the stored curvature pairs are
//     zero, no pair is ever admitted (y's == 0), and each iteration searches along -g0 with
//     Armijo backtracking (step 1, halved up to 20 times, accept on sufficient or any decrease).
//     The reference's two-loop recursion then reads history slots it never wrote; here they are
//     zero, which gives the steepest-descent direction above.
// Since the trial gradients are overwritten unused, they are not computed here: the results are
// the same and a line-search trial costs one fitness evaluation instead of 2K + 1.
//
// B200 layout: one 1024-thread block per program (the reference runs ONE thread per program):
// rows are evaluated in parallel into shared memory (one row per thread at D <= 1024), then
// reduced in the reference's row order (sequential fused multiply-adds, y staged in shared
// memory) so that every RMSE is the reference's bit for bit; the 2K finite-difference sums run
// in parallel, one thread per (constant, sign).  1024 threads rather than 256: the block owns
// its program for the whole optimisation, so the rows are the only parallelism (64 programs x
// 1024 rows x 10 iterations: 3.6 ms with 256 threads, 1.7 ms with 1024).
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "ws_internal.h"

namespace ws {
namespace {

constexpr int kLbMaxK = 32, kLbMaxD = 1024, kLbHistory = 10, kLbStack = 64, kLbMaxL = 256,
              kLbMaxLineSearch = 20;
constexpr int kLbThreads = 1024;

struct LbIds {
  int pad, xs, nvars, id_C, id_pi, id_e;
  int id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10;
  int op_add, op_sub, op_mul, op_div, op_pow, op_mod;
};

// One row.  FULL: the fitness evaluator (lbfgs_kernels.cu:278-335); otherwise the reduced
// evaluator of the finite differences (:380-412).  Returns false when the row fails.
template <typename T, bool FULL>
__device__ bool lb_eval_row(const uint8_t* prog, int L, const T* __restrict__ x, int64_t D, int d,
                            const T* pos, int K, const LbIds& id, T pi_val, T e_val, T& pred) {
  T stack[kLbStack];
  int sp = 0, c_idx = 0;
  bool err = false;
  for (int pc = 0; pc < L && !err; ++pc) {
    const int tok = prog[pc];
    if (tok == id.pad) break;
    T val = (T)0;
    bool push = true;
    if (tok >= id.xs && tok < id.xs + id.nvars) val = x[(int64_t)(tok - id.xs) * D + d];
    else if (tok == id.id_0) val = (T)0.0;
    else if (tok == id.id_1) val = (T)1.0;
    else if (tok == id.id_2) val = (T)2.0;
    else if (FULL && tok == id.id_3) val = (T)3.0;
    else if (FULL && tok == id.id_4) val = (T)4.0;
    else if (FULL && tok == id.id_5) val = (T)5.0;
    else if (FULL && tok == id.id_6) val = (T)6.0;
    else if (FULL && tok == id.id_10) val = (T)10.0;
    else if (tok == id.id_pi) val = pi_val;
    else if (tok == id.id_e) val = e_val;
    else if (tok == id.id_C) {
      const int ri = c_idx < K ? c_idx : K - 1;
      val = ri >= 0 ? pos[ri] : (T)1.0;
      c_idx++;
    } else {
      push = false;
      if (sp < 2) {
        err = true;
        break;
      }
      const T rhs = stack[--sp];
      const T lhs = stack[--sp];
      T res = (T)0.0;
      if (tok == id.op_add) res = lhs + rhs;
      else if (tok == id.op_sub) res = lhs - rhs;
      else if (tok == id.op_mul) res = lhs * rhs;
      else if (tok == id.op_div) res = (fabsf(rhs) > 1e-12f) ? lhs / rhs : (T)1e30;
      else if (tok == id.op_pow) res = powf(fabsf(lhs) + 1e-12f, rhs);
      else if (FULL && tok == id.op_mod) res = (fabsf(rhs) > 1e-12f) ? fmodf(lhs, rhs) : (T)0.0;
      else {
        sp += 2;
        err = true;
      }
      if (!err) stack[sp++] = res;
    }
    if (push && sp < kLbStack) stack[sp++] = val;
  }
  if (err || sp != 1) return false;
  pred = stack[0];
  return pred == pred && !isinf(pred);
}

template <typename T>
struct LbArgs {
  const uint8_t* pop;
  T* consts;
  const T* x;
  const T* y;
  T* out_rmse;
  int64_t B, D;
  int L, K, max_iter;
  T gtol, cmin, cmax, pi_val, e_val;
  LbIds id;
  int kc;  // constants per finite-difference chunk (2 * kc row buffers)
};

template <typename T>
__global__ void __launch_bounds__(kLbThreads) lbfgs_kernel(LbArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* rowbuf = reinterpret_cast<T*>(smem);  // [2 * kc][D] predictions (or skipped rows)
  uint8_t* rowok = reinterpret_cast<uint8_t*>(rowbuf + (size_t)2 * a.kc * a.D);  // [2 kc][D]
  // y staged once: the row-order sums below read it from shared memory, eight rows ahead
  T* s_y = reinterpret_cast<T*>(rowok + ((size_t)2 * a.kc * a.D + 15) / 16 * 16);
  __shared__ uint8_t s_prog[kLbMaxL];
  __shared__ T s_pos[kLbMaxK];     // point being evaluated
  __shared__ T s_pm[2 * kLbMaxK];  // clamped +eps / -eps coordinate per chunk pair
  __shared__ T s_sum[2 * kLbMaxK];
  __shared__ T s_x[kLbMaxK], s_g[kLbMaxK], s_p[kLbMaxK];
  __shared__ T s_f;
  __shared__ int s_fail;
  // curvature memory of the two-loop recursion (thread 0), filled as the reference fills it
  __shared__ T s_hist[kLbHistory][kLbMaxK], y_hist[kLbHistory][kLbMaxK], rho_hist[kLbHistory];
  const int tid = threadIdx.x;
  const int K = a.K, D = (int)a.D;
  for (int d = tid; d < D; d += blockDim.x) s_y[d] = a.y[d];

  for (int64_t b = blockIdx.x; b < a.B; b += gridDim.x) {
    __syncthreads();
    for (int i = tid; i < a.L; i += blockDim.x) s_prog[i] = a.pop[b * a.L + i];
    if (tid < K) {
      s_x[tid] = a.consts[b * K + tid];
      s_pos[tid] = s_x[tid];
    }
    __syncthreads();

    // Fitness of s_pos into s_f (1e30 when a row fails), rows in parallel, summed in row order.
    auto fitness = [&]() {
      if (tid == 0) s_fail = 0;
      __syncthreads();
      for (int d = tid; d < D; d += blockDim.x) {
        T pred;
        const bool ok = lb_eval_row<T, true>(s_prog, a.L, a.x, a.D, d, s_pos, K, a.id, a.pi_val,
                                             a.e_val, pred);
        rowbuf[d] = pred;
        if (!ok) s_fail = 1;
      }
      __syncthreads();
      if (tid == 0) {
        if (s_fail) {
          s_f = (T)1e30;
        } else {
          T mse_sum = (T)0.0;
#pragma unroll 8
          for (int d = 0; d < D; ++d) {
            const T diff = rowbuf[d] - s_y[d];
            mse_sum += diff * diff;
          }
          s_f = sqrtf(mse_sum / (T)D);
        }
      }
      __syncthreads();
    };

    // ---- initial fitness and finite-difference gradient (lbfgs_kernels.cu:271-473) ----
    fitness();
    if (tid < K) s_g[tid] = (T)0.0;
    if (!s_fail) {
      const T eps = (T)1e-5;
      for (int k0 = 0; k0 < K; k0 += a.kc) {
        const int nk = (K - k0) < a.kc ? (K - k0) : a.kc;
        if (tid < 2 * nk) {
          const int k = k0 + (tid >> 1);
          T v = s_x[k];
          if (tid & 1) v -= eps;
          else v += eps;
          s_pm[tid] = fmaxf(a.cmin, fminf(a.cmax, v));
        }
        __syncthreads();
        for (int w = tid; w < 2 * nk * D; w += blockDim.x) {
          const int j = w / D, d = w - j * D;
          T pos[kLbMaxK];
          for (int q = 0; q < K; ++q) pos[q] = s_x[q];
          pos[k0 + (j >> 1)] = s_pm[j];
          T pred;
          const bool ok = lb_eval_row<T, false>(s_prog, a.L, a.x, a.D, d, pos, K, a.id,
                                                a.pi_val, a.e_val, pred);
          rowbuf[(size_t)j * D + d] = pred;
          rowok[(size_t)j * D + d] = ok ? 1 : 0;
        }
        __syncthreads();
        if (tid < 2 * nk) {
          T mse = (T)0.0;
#pragma unroll 8
          for (int d = 0; d < D; ++d) {
            if (!rowok[(size_t)tid * D + d]) continue;
            const T diff = rowbuf[(size_t)tid * D + d] - s_y[d];
            mse += diff * diff;
          }
          s_sum[tid] = sqrtf(mse / (T)D);
        }
        __syncthreads();
        if (tid < nk) {
          const int k = k0 + tid;
          const T actual_eps = s_pm[2 * tid] - s_pm[2 * tid + 1];
          if (actual_eps > 1e-10f) s_g[k] = (s_sum[2 * tid] - s_sum[2 * tid + 1]) / actual_eps;
        }
        __syncthreads();
      }
    }
    T f_curr = s_f;  // every thread holds the same value

    // ---- iterations (lbfgs_kernels.cu:478-611) ----
    if (tid < kLbHistory) {
      rho_hist[tid] = (T)0.0;
      for (int k = 0; k < kLbMaxK; ++k) s_hist[tid][k] = y_hist[tid][k] = (T)0.0;
    }
    __syncthreads();
    T g_norm = (T)0.0;
    for (int k = 0; k < K; ++k) g_norm += s_g[k] * s_g[k];
    g_norm = sqrtf(g_norm);
    int history_ptr = 0, history_count = 0;
    for (int iter = 0; iter < a.max_iter; ++iter) {
      if (g_norm < a.gtol) break;
      if (tid == 0) {
        T q[kLbMaxK], alpha[kLbHistory];
        for (int k = 0; k < K; ++k) q[k] = s_g[k];
        const int num_hist = history_count;
        for (int i = num_hist - 1; i >= 0; --i) {
          const int idx = (history_ptr - num_hist + i + kLbHistory) % kLbHistory;
          T dot = (T)0.0;
          for (int k = 0; k < K; ++k) dot += s_hist[idx][k] * q[k];
          alpha[i] = rho_hist[idx] * dot;
          for (int k = 0; k < K; ++k) q[k] -= alpha[i] * y_hist[idx][k];
        }
        T gamma = (T)1.0;
        if (history_count > 0) {
          const int last = (history_ptr - 1 + kLbHistory) % kLbHistory;
          T yty = (T)0.0, yts = (T)0.0;
          for (int k = 0; k < K; ++k) {
            yty += y_hist[last][k] * y_hist[last][k];
            yts += y_hist[last][k] * s_hist[last][k];
          }
          if (yts > 1e-10f) gamma = yts / yty;
        }
        for (int k = 0; k < K; ++k) q[k] *= gamma;
        for (int i = 0; i < num_hist; ++i) {
          const int idx = (history_ptr - num_hist + i + kLbHistory) % kLbHistory;
          T dot = (T)0.0;
          for (int k = 0; k < K; ++k) dot += y_hist[idx][k] * q[k];
          const T beta = rho_hist[idx] * dot;
          for (int k = 0; k < K; ++k) q[k] += s_hist[idx][k] * (alpha[i] - beta);
        }
        for (int k = 0; k < K; ++k) s_p[k] = -q[k];
      }
      __syncthreads();
      T step = (T)1.0;
      bool accepted = false;
      for (int ls = 0; ls < kLbMaxLineSearch; ++ls) {
        if (tid < K) {
          T v = s_x[tid] + step * s_p[tid];
          if (v < a.cmin) v = a.cmin;
          if (v > a.cmax) v = a.cmax;
          s_pos[tid] = v;
        }
        __syncthreads();
        fitness();
        const T f_trial = s_f;
        if (f_trial <= f_curr - (T)1e-4 * step * g_norm * g_norm || f_trial < f_curr) {
          __syncthreads();
          if (tid < K) s_x[tid] = s_pos[tid];
          f_curr = f_trial;
          accepted = true;
          __syncthreads();
          break;
        }
        step *= (T)0.5;
      }
      if (!accepted) break;
      // history update with x_prev == x_curr and the trial gradient replaced by g_curr
      if (history_count < kLbHistory) history_count++;
      const int idx = history_ptr % kLbHistory;
      T ys = (T)0.0;
      for (int k = 0; k < K; ++k) {
        const T sk = s_x[k] - s_x[k];
        const T yk = s_g[k] - s_g[k];
        ys += yk * sk;
        if (tid == 0) {
          s_hist[idx][k] = sk;
          y_hist[idx][k] = yk;
        }
      }
      if (ys > 1e-10f) {
        if (tid == 0) rho_hist[idx] = (T)1.0 / ys;
        history_ptr++;
      }
      __syncthreads();
    }
    __syncthreads();
    if (tid < K) a.consts[b * K + tid] = s_x[tid];
    if (tid == 0) a.out_rmse[b] = f_curr;
  }
}

template <typename T>
ws_status launch_lbfgs_typed(LbArgs<T> a, cudaStream_t stream) {
  const size_t per_pair = (size_t)a.D * (sizeof(T) + 1);
  const size_t budget = 96 * 1024;
  int kc = (int)(budget / (2 * per_pair));
  if (kc > a.K) kc = a.K;
  if (kc < 1) kc = 1;
  a.kc = kc;
  const size_t smem = 2 * (size_t)kc * per_pair + 16 + (size_t)a.D * sizeof(T) + 16;
  auto kern = lbfgs_kernel<T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return fail_cuda(e, "lbfgs_optimize");
  const int64_t cap = (int64_t)device_info().sm_count * 4;
  const int grid = (int)(a.B < cap ? a.B : cap);
  kern<<<grid, kLbThreads, smem, stream>>>(a);
  e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "lbfgs_optimize");
}

}  // namespace
}  // namespace ws

extern "C" ws_status ws_lbfgs_optimize(int32_t dtype, const uint8_t* population, int64_t B,
                                       int64_t L, void* constants, int64_t K, const void* x,
                                       int64_t num_vars, int64_t D, const void* y_target,
                                       void* out_rmse, int32_t max_iter, int32_t history_size,
                                       float gtol, float const_min, float const_max,
                                       const ws_token_map* ids, void* stream) {
  using namespace ws;
  (void)history_size;  // the reference kernel's history is fixed at 10 entries
  clear_error();
  NvtxRange nvtx("ws_lbfgs_optimize");
  if (!ids) return fail("token map is required");
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  // launch_lbfgs_optimize's checks, in its order (lbfgs_kernels.cu:661-663)
  if (L > kLbMaxL) return fail("Formula length exceeds LBFGS_MAX_L");
  if (K > kLbMaxK) return fail("Constants exceed LBFGS_MAX_K");
  if (D > kLbMaxD) return fail("Data samples exceed LBFGS_MAX_D");
  if (B < 0 || L < 0 || K < 0 || D < 0 || num_vars < 0) return fail("negative dimension");
  if (B == 0) return WS_OK;
  if (D == 0) return fail("lbfgs_optimize needs at least one data sample");
  if (!population || (K > 0 && !constants) || (num_vars > 0 && !x) || !y_target || !out_rmse)
    return fail("null tensor pointer");
  LbIds id{ids->pad_id, ids->id_x_start, (int)num_vars, ids->id_C, ids->id_pi, ids->id_e,
           ids->id_0, ids->id_1, ids->id_2, ids->id_3, ids->id_4, ids->id_5, ids->id_6,
           ids->id_10, ids->op_add, ids->op_sub, ids->op_mul, ids->op_div, ids->op_pow,
           ids->op_mod};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == WS_F32) {
    LbArgs<float> a{population, static_cast<float*>(constants), static_cast<const float*>(x),
                    static_cast<const float*>(y_target), static_cast<float*>(out_rmse), B, D,
                    (int)L, (int)K, max_iter, gtol, const_min, const_max, (float)ids->pi_val,
                    (float)ids->e_val, id, 1};
    return launch_lbfgs_typed<float>(a, s);
  }
  LbArgs<double> a{population, static_cast<double*>(constants), static_cast<const double*>(x),
                   static_cast<const double*>(y_target), static_cast<double*>(out_rmse), B, D,
                   (int)L, (int)K, max_iter, (double)gtol, (double)const_min,
                   (double)const_max, ids->pi_val, ids->e_val, id, 1};
  return launch_lbfgs_typed<double>(a, s);
}
