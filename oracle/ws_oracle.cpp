// ws_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference WarpSymbolic evaluator semantics, used by tests/ as the
// checker of the CUDA kernels and by bench.py as the timed CPU baseline (the reference's own
// device="cpu" path cannot evaluate programs: rpn_kernels.cu:10,382 rejects CPU tensors).
// Nothing in the product links, loads or calls this file.
//
// Every function cites the reference lines it restates (paths relative to the reference
// project root, src/warpsymbolic/gpu/...).  Compiled with IEEE semantics (no -ffast-math,
// -ffp-contract=off); templated on float (parity) and double (the FP64 oracle).
//
// Pinned against: the known-answer vectors of the reference tests (tests/golden/) and the
// outputs of the reference extension itself, built from its sources by oracle/build_ref.sh and
// run on a B200 (tests/golden/make_ref_golden.py).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "../include/warpsym.h"

namespace {

constexpr int kStackSize = 32;  // STACK_SIZE, rpn_kernels.cu:19

// ---------------------------------------------------------------------------------------
// Protected operators, rpn_kernels.cu:27-120.
template <typename T> T p_div(T a, T b, bool&) { return (std::fabs(b) < (T)1e-9) ? a : a / b; }
template <typename T> T p_mod(T a, T b, bool&) {
  if (std::fabs(b) < (T)1e-9) return (T)0.0;
  T r = std::fmod(a, b);
  if ((b > 0 && r < 0) || (b < 0 && r > 0)) r += b;
  return r;
}
template <typename T> T p_log(T a, bool&) { return std::log(std::fabs(a) + (T)1e-9); }
template <typename T> T p_exp(T a, bool&) {
  T x = a;
  if (x < (T)-80.0) x = (T)-80.0;
  if (x > (T)80.0) x = (T)80.0;
  return std::exp(x);
}
template <typename T> T p_sqrt(T a, bool&) { return std::sqrt(std::fabs(a)); }
template <typename T> T p_pow(T a, T b, bool& e) {
  if (a != a || b != b) { e = true; return (T)0.0; }
  if (std::fabs(a) < (T)1e-10 && std::fabs(b) < (T)1e-10) return (T)1.0;
  if (a < (T)0.0) {
    T ib = std::round(b);
    if (std::fabs(b - ib) > (T)1e-3) a = std::fabs(a); else b = ib;
  }
  if (std::fabs(a) > (T)1.0 && b > (T)80.0) b = (T)80.0;
  if (std::fabs(a) > (T)100.0 && b > (T)10.0) b = (T)10.0;
  T res = std::pow(a, b);
  if (res != res || std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}
template <typename T> T p_asin(T a, bool&) {
  if (a < (T)-1.0) a = (T)-1.0;
  if (a > (T)1.0) a = (T)1.0;
  return std::asin(a);
}
template <typename T> T p_acos(T a, bool&) {
  if (a < (T)-1.0) a = (T)-1.0;
  if (a > (T)1.0) a = (T)1.0;
  return std::acos(a);
}
template <typename T> T p_tgamma(T a, bool& e) {
  if (a <= (T)0.0 && std::floor(a) == a) return (T)0.0;
  T res = std::tgamma(a);
  if (res != res || std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}
template <typename T> T p_lgamma(T a, bool& e) {
  if (a <= (T)0.0 && std::floor(a) == a) return (T)0.0;
  T res = std::lgamma(a);
  if (res != res || std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}
// Strict operators, rpn_kernels.cu:126-199.
template <typename T> T s_div(T a, T b, bool& e) {
  if (std::fabs(b) < (T)1e-9) { e = true; return (T)0.0; }
  return a / b;
}
template <typename T> T s_mod(T a, T b, bool& e) {
  if (std::fabs(b) < (T)1e-9) { e = true; return (T)0.0; }
  T r = std::fmod(a, b);
  if ((b > 0 && r < 0) || (b < 0 && r > 0)) r += b;
  return r;
}
template <typename T> T s_log(T a, bool& e) {
  if (a <= (T)0.0) { e = true; return (T)0.0; }
  return std::log(a);
}
template <typename T> T s_exp(T a, bool& e) {
  T res = std::exp(a);
  if (std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}
template <typename T> T s_sqrt(T a, bool& e) {
  if (a < (T)0.0) { e = true; return (T)0.0; }
  return std::sqrt(a);
}
template <typename T> T s_pow(T a, T b, bool& e) {
  if (a != a || b != b) { e = true; return (T)0.0; }
  if (std::fabs(a) < (T)1e-10 && std::fabs(b) < (T)1e-10) return (T)1.0;
  if (a < (T)0.0) {
    T ib = std::round(b);
    if (std::fabs(b - ib) > (T)1e-3) { e = true; return (T)0.0; }
    b = ib;
  }
  T res = std::pow(a, b);
  if (res != res || std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}
template <typename T> T s_asin(T a, bool& e) {
  if (a < (T)-1.0 || a > (T)1.0) { e = true; return (T)0.0; }
  return std::asin(a);
}
template <typename T> T s_acos(T a, bool& e) {
  if (a < (T)-1.0 || a > (T)1.0) { e = true; return (T)0.0; }
  return std::acos(a);
}
template <typename T> T s_tgamma(T a, bool& e) {
  if (a <= (T)0.0 && std::floor(a) == a) { e = true; return (T)0.0; }
  T res = std::tgamma(a);
  if (res != res || std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}
template <typename T> T s_lgamma(T a, bool& e) {
  if (a <= (T)0.0 && std::floor(a) == a) { e = true; return (T)0.0; }
  T res = std::lgamma(a);
  if (res != res || std::isinf(res)) { e = true; return (T)0.0; }
  return res;
}

// Result of interpreting one (program, row): the reference kernels' registers at loop exit.
template <typename T> struct RowState {
  T top;       // stack[sp-1] when sp > 0
  int sp;
  bool error;
};

// One (program, row) interpretation: the loop of rpn_eval_kernel (rpn_kernels.cu:245-350) and,
// with fused_order=true, of rpn_eval_fused_kernel (rpn_kernels.cu:2327-2402), whose only
// difference is the order in which unary operator IDs are compared (it matters only when two
// operators share an ID) and the x<4 register preload, which the fused envelope makes moot.
template <typename T>
RowState<T> interp_row(const uint8_t* prog, int64_t L, const T* x, int64_t num_vars, int64_t D,
                       int64_t d, const T* consts, int64_t K, const ws_token_map& m, int strict,
                       bool fused_order) {
  T stack[kStackSize];
  int sp = 0;
  bool error = false;
  int64_t c_idx = 0;
  for (int64_t pc = 0; pc < L; ++pc) {
    const int64_t token = (int64_t)prog[pc];
    if (token == m.pad_id) break;
    T val = (T)0.0;
    bool is_push = true;
    if (token >= m.id_x_start && token < m.id_x_start + num_vars) {
      val = x[(token - m.id_x_start) * D + d];
    } else if (token == m.id_C) {
      if (K > 0) {
        int64_t r = c_idx;
        if (r >= K) r = K - 1;
        val = consts[r];
        c_idx++;
      } else {
        val = (T)1.0;
      }
    } else if (token == m.id_0) val = (T)0.0;
    else if (token == m.id_1) val = (T)1.0;
    else if (token == m.id_2) val = (T)2.0;
    else if (token == m.id_3) val = (T)3.0;
    else if (token == m.id_4) val = (T)4.0;
    else if (token == m.id_5) val = (T)5.0;
    else if (token == m.id_6) val = (T)6.0;
    else if (token == m.id_10) val = (T)10.0;
    else if (token == m.id_pi) val = (T)m.pi_val;
    else if (token == m.id_e) val = (T)m.e_val;
    else is_push = false;

    if (is_push) {  // push-drop at STACK_SIZE, rpn_kernels.cu:289-293
      if (sp < kStackSize) stack[sp++] = val;
      continue;
    }
    if (token == m.op_add || token == m.op_sub || token == m.op_mul || token == m.op_div ||
        token == m.op_pow || token == m.op_mod) {
      if (sp < 2) { error = true; break; }
      T op2 = stack[--sp];
      T op1 = stack[--sp];
      T res = (T)0.0;
      if (token == m.op_add) res = op1 + op2;
      else if (token == m.op_sub) res = op1 - op2;
      else if (token == m.op_mul) res = op1 * op2;
      else if (token == m.op_div) res = strict ? s_div(op1, op2, error) : p_div(op1, op2, error);
      else if (token == m.op_pow) res = strict ? s_pow(op1, op2, error) : p_pow(op1, op2, error);
      else res = strict ? s_mod(op1, op2, error) : p_mod(op1, op2, error);
      if (error) break;
      stack[sp++] = res;
      continue;
    }
    if (sp < 1) { error = true; break; }
    T a = stack[--sp];
    T res = (T)0.0;
    bool matched = true;
    auto sign = [](T v) { return (v > (T)0.0) ? (T)1.0 : ((v < (T)0.0) ? (T)-1.0 : (T)0.0); };
    if (token == m.op_lgamma) res = strict ? s_lgamma(a, error) : p_lgamma(a, error);
    else if (token == m.op_fact) res = strict ? s_tgamma(a + (T)1.0, error) : p_tgamma(a + (T)1.0, error);
    else if (token == m.op_sqrt) res = strict ? s_sqrt(a, error) : p_sqrt(a, error);
    else if (token == m.op_exp) res = strict ? s_exp(a, error) : p_exp(a, error);
    else if (token == m.op_log) res = strict ? s_log(a, error) : p_log(a, error);
    else if (token == m.op_sin) res = std::sin(a);
    else if (token == m.op_cos) res = std::cos(a);
    else if (token == m.op_tan) res = std::tan(a);
    else if (token == m.op_abs) res = std::fabs(a);
    else if (token == m.op_neg) res = -a;
    else if (!fused_order) {  // rpn_kernels.cu:339-346
      if (token == m.op_floor) res = std::floor(a);
      else if (token == m.op_ceil) res = std::ceil(a);
      else if (token == m.op_sign) res = sign(a);
      else if (token == m.op_asin) res = strict ? s_asin(a, error) : p_asin(a, error);
      else if (token == m.op_acos) res = strict ? s_acos(a, error) : p_acos(a, error);
      else if (token == m.op_atan) res = std::atan(a);
      else if (token == m.op_gamma) res = strict ? s_tgamma(a, error) : p_tgamma(a, error);
      else matched = false;
    } else {  // rpn_kernels.cu:2391-2398
      if (token == m.op_gamma) res = strict ? s_tgamma(a, error) : p_tgamma(a, error);
      else if (token == m.op_asin) res = strict ? s_asin(a, error) : p_asin(a, error);
      else if (token == m.op_acos) res = strict ? s_acos(a, error) : p_acos(a, error);
      else if (token == m.op_atan) res = std::atan(a);
      else if (token == m.op_floor) res = std::floor(a);
      else if (token == m.op_ceil) res = std::ceil(a);
      else if (token == m.op_sign) res = sign(a);
      else matched = false;
    }
    if (!matched) { error = true; break; }
    if (error) break;
    stack[sp++] = res;
  }
  RowState<T> st;
  st.sp = sp;
  st.error = error;
  st.top = (sp > 0) ? stack[sp - 1] : (T)0.0;
  return st;
}

template <typename T> struct Lim;
template <> struct Lim<float> {
  static constexpr float invalid = 1e15f, max_diff = 4e18f;
};
template <> struct Lim<double> {
  static constexpr double invalid = 1e100, max_diff = 1e150;
};

// rpn_eval_kernel outputs (rpn_kernels.cu:353-357).
template <typename T>
void eval_rows(const uint8_t* pop, int64_t B, int64_t L, const T* x, int64_t V, int64_t D,
               const T* c, int64_t K, const ws_token_map* m, int strict, T* preds, int32_t* sp,
               uint8_t* err, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t b = 0; b < B; ++b) {
    for (int64_t d = 0; d < D; ++d) {
      RowState<T> s = interp_row<T>(pop + b * L, L, x, V, D, d, c ? c + b * K : nullptr, K, *m,
                                    strict, false);
      const int64_t i = b * D + d;
      sp[i] = s.sp;
      err[i] = s.error ? 1 : 0;
      preds[i] = s.sp > 0 ? s.top : (T)1e30;
    }
  }
}

// Warp-butterfly sum as done by __shfl_xor_sync(…, 16..1) with lane 0 reading the result
// (rpn_kernels.cu:2439-2443 and 2481-2485): lane l adds lane l^off at every level.
template <typename T> T butterfly_lane0(T v[32]) {
  for (int off = 16; off > 0; off >>= 1) {
    T nv[32];
    for (int l = 0; l < 32; ++l) nv[l] = v[l] + v[l ^ off];
    for (int l = 0; l < 32; ++l) v[l] = nv[l];
  }
  return v[0];
}

// rpn_eval_fused_kernel, block mode (rpn_kernels.cu:2259-2502) with its exact reduction order:
// warp butterflies over blockDim = ceil(D/32)*32 threads, then warp 0 reduces the warp sums.
template <typename T>
void fused_rmse(const uint8_t* pop, int64_t B, int64_t L, const T* x, int64_t V, int64_t D,
                const T* c, int64_t K, const T* y, const ws_token_map* m, int strict, T* out,
                int nthreads) {
  const int64_t nwarps = (D + 31) / 32;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t b = 0; b < B; ++b) {
    std::vector<T> wsum(32, (T)0.0);
    bool any_inv = false, any_ovf = false;
    for (int64_t w = 0; w < nwarps; ++w) {
      T lanes[32];
      for (int l = 0; l < 32; ++l) {
        const int64_t d = w * 32 + l;
        T sq = (T)0.0;
        if (d < D) {
          RowState<T> s = interp_row<T>(pop + b * L, std::min<int64_t>(L, 256), x, V, D, d,
                                        c ? c + b * K : nullptr, K, *m, strict, true);
          bool valid = !s.error && s.sp == 1;
          T pred = valid ? s.top : Lim<T>::invalid;
          valid = valid && !std::isnan(pred) && !std::isinf(pred);
          if (valid) {
            T diff = pred - y[d];
            T ad = diff < (T)0.0 ? -diff : diff;
            bool ovf = std::isnan(diff) || std::isinf(diff) || ad > Lim<T>::max_diff;
            sq = ovf ? (T)0.0 : diff * diff;
            ovf = ovf || std::isnan(sq) || std::isinf(sq);
            if (ovf) sq = (T)0.0;
            any_ovf |= ovf;
          } else {
            sq = Lim<T>::invalid;
            any_inv = true;
          }
        }
        lanes[l] = sq;
      }
      wsum[w] = butterfly_lane0(lanes);
    }
    T lanes[32];
    for (int l = 0; l < 32; ++l) lanes[l] = (l < nwarps) ? wsum[l] : (T)0.0;
    const T total = butterfly_lane0(lanes);
    T rmse;
    if (any_inv) rmse = Lim<T>::invalid;
    else if (any_ovf) rmse = std::sqrt(Lim<T>::invalid);
    else {
      T mse = total / (T)D;
      rmse = std::sqrt(mse);
      if (std::isnan(rmse) || std::isinf(rmse)) rmse = Lim<T>::invalid;
    }
    out[b] = rmse;
  }
}

// General fitness semantics of ws_eval_fitness: per-row evaluation as above; squared errors
// rounded in T and accumulated in FP64; validity and overflow per the chosen policy:
//   WS_POLICY_FUSED   -- rpn_kernels.cu:2405-2430, 2487-2497
//   WS_POLICY_CLASSIC -- evaluation.py:153-189 (invalid rows => program invalid; non-finite
//                        mean => sqrt(INF_VAL))
// An FP64 sum above the T range counts as the overflow of the reference's T accumulator.
template <typename T>
void fitness(const uint8_t* pop, int64_t B, int64_t L, const T* x, int64_t V, int64_t D,
             const T* c, int64_t K, const T* y, const ws_token_map* m, int strict, int policy,
             int loss, double invalid_value, void* out_loss, int32_t* out_ninv, int nthreads) {
  double ymean = 0.0, yvar = 0.0;
  for (int64_t d = 0; d < D; ++d) ymean += (double)y[d];
  ymean /= (double)D;
  for (int64_t d = 0; d < D; ++d) yvar += ((double)y[d] - ymean) * ((double)y[d] - ymean);
  yvar /= (double)D;
  const bool fused = policy == WS_POLICY_FUSED;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t b = 0; b < B; ++b) {
    double sse = 0.0;
    int64_t ninv = 0;
    bool ovf_any = false;
    for (int64_t d = 0; d < D; ++d) {
      RowState<T> s = interp_row<T>(pop + b * L, L, x, V, D, d, c ? c + b * K : nullptr, K, *m,
                                    strict, fused);
      bool valid = !s.error && s.sp == 1 && !std::isnan(s.top) && !std::isinf(s.top);
      if (!valid) { ninv++; continue; }
      T diff = s.top - y[d];
      if (fused) {
        T ad = diff < (T)0.0 ? -diff : diff;
        bool ovf = std::isnan(diff) || std::isinf(diff) || ad > Lim<T>::max_diff;
        T sq = ovf ? (T)0.0 : diff * diff;
        ovf = ovf || std::isnan(sq) || std::isinf(sq);
        if (ovf) { ovf_any = true; continue; }
        sse += (double)sq;
      } else {
        T sq = diff * diff;
        sse += (double)sq;
      }
    }
    if (out_ninv) out_ninv[b] = (int32_t)ninv;
    const double tmax = (double)std::numeric_limits<T>::max();
    if (loss == WS_LOSS_SSE) {
      ((double*)out_loss)[b] = (ninv > 0) ? invalid_value : sse;
      continue;
    }
    const bool invalid = ninv > 0;
    const bool sum_ovf = !(sse <= tmax);
    const bool row_ovf = fused && ovf_any;
    const T iv = (T)invalid_value;
    double outv;
    if (invalid) {
      outv = (loss == WS_LOSS_R2) ? -invalid_value : invalid_value;
    } else if (row_ovf || sum_ovf) {
      // fused: row overflow -> sqrt(INVALID) (rpn_kernels.cu:2491-2492), non-finite mean ->
      // INVALID (:2496); classic: non-finite mean -> sqrt(INF_VAL) (evaluation.py:184-186)
      if (loss == WS_LOSS_RMSE) outv = (fused && !row_ovf) ? (double)iv : (double)std::sqrt(iv);
      else outv = (loss == WS_LOSS_MSE) ? invalid_value : -invalid_value;
    } else {
      const double mse = sse / (double)D;
      const T mse_t = (T)mse;
      if (loss == WS_LOSS_RMSE) {
        T r = std::sqrt(mse_t);
        outv = (std::isnan(r) || std::isinf(r)) ? invalid_value : (double)r;
      } else if (loss == WS_LOSS_MSE) {
        outv = (double)mse_t;
      } else {
        outv = yvar > 0.0 ? 1.0 - mse / yvar : (mse == 0.0 ? 1.0 : -invalid_value);
      }
    }
    if (sizeof(T) == 4) ((float*)out_loss)[b] = (float)outv;
    else ((double*)out_loss)[b] = outv;
  }
}

}  // namespace

extern "C" {

int ws_oracle_threads(void) { return omp_get_max_threads(); }

void ws_oracle_eval_rows_f32(const uint8_t* pop, int64_t B, int64_t L, const float* x, int64_t V,
                             int64_t D, const float* c, int64_t K, const ws_token_map* m,
                             int strict, float* preds, int32_t* sp, uint8_t* err, int nthreads) {
  eval_rows<float>(pop, B, L, x, V, D, c, K, m, strict, preds, sp, err, nthreads);
}
void ws_oracle_eval_rows_f64(const uint8_t* pop, int64_t B, int64_t L, const double* x,
                             int64_t V, int64_t D, const double* c, int64_t K,
                             const ws_token_map* m, int strict, double* preds, int32_t* sp,
                             uint8_t* err, int nthreads) {
  eval_rows<double>(pop, B, L, x, V, D, c, K, m, strict, preds, sp, err, nthreads);
}
void ws_oracle_fused_rmse_f32(const uint8_t* pop, int64_t B, int64_t L, const float* x,
                              int64_t V, int64_t D, const float* c, int64_t K, const float* y,
                              const ws_token_map* m, int strict, float* out, int nthreads) {
  fused_rmse<float>(pop, B, L, x, V, D, c, K, y, m, strict, out, nthreads);
}
void ws_oracle_fused_rmse_f64(const uint8_t* pop, int64_t B, int64_t L, const double* x,
                              int64_t V, int64_t D, const double* c, int64_t K, const double* y,
                              const ws_token_map* m, int strict, double* out, int nthreads) {
  fused_rmse<double>(pop, B, L, x, V, D, c, K, y, m, strict, out, nthreads);
}
void ws_oracle_fitness_f32(const uint8_t* pop, int64_t B, int64_t L, const float* x, int64_t V,
                           int64_t D, const float* c, int64_t K, const float* y,
                           const ws_token_map* m, int strict, int policy, int loss,
                           double invalid_value, void* out, int32_t* ninv, int nthreads) {
  fitness<float>(pop, B, L, x, V, D, c, K, y, m, strict, policy, loss, invalid_value, out, ninv,
                 nthreads);
}
void ws_oracle_fitness_f64(const uint8_t* pop, int64_t B, int64_t L, const double* x, int64_t V,
                           int64_t D, const double* c, int64_t K, const double* y,
                           const ws_token_map* m, int strict, int policy, int loss,
                           double invalid_value, void* out, int32_t* ninv, int nthreads) {
  fitness<double>(pop, B, L, x, V, D, c, K, y, m, strict, policy, loss, invalid_value, out, ninv,
                  nthreads);
}

}  // extern "C"
