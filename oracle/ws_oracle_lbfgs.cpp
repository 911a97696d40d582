// ws_oracle_lbfgs.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Literal CPU restatement of the reference's L-BFGS kernel lbfgs_optimize_kernel
// (src/warpsymbolic/gpu/cuda/lbfgs_kernels.cu:214-621), one program at a time, including the
// finite-difference gradient at every line-search trial (the CUDA kernel of this library skips
// those, since the reference overwrites them unused) and the history slots the reference reads
// before writing, taken as zero.  IEEE libm; the same float conversions as the reference
// (fabsf / powf / fmodf / sqrtf / fmaxf / fminf applied to double values in the FP64 variant).

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../include/warpsym.h"

namespace {

constexpr int kMaxK = 32, kHist = 10, kStack = 64, kMaxLs = 20;

template <typename T, bool FULL>
bool eval_row(const uint8_t* prog, int64_t L, const T* x, int64_t nv, int64_t D, int64_t d,
              const T* pos, int64_t K, const ws_token_map& v, T pi_val, T e_val, T& pred) {
  T stack[kStack];
  int sp = 0;
  int64_t c_idx = 0;
  bool err = false;
  for (int64_t pc = 0; pc < L && !err; ++pc) {
    const int tok = prog[pc];
    if (tok == v.pad_id) break;
    T val = 0;
    bool push = true;
    if (tok >= v.id_x_start && tok < v.id_x_start + nv) val = x[(tok - v.id_x_start) * D + d];
    else if (tok == v.id_0) val = (T)0.0;
    else if (tok == v.id_1) val = (T)1.0;
    else if (tok == v.id_2) val = (T)2.0;
    else if (FULL && tok == v.id_3) val = (T)3.0;
    else if (FULL && tok == v.id_4) val = (T)4.0;
    else if (FULL && tok == v.id_5) val = (T)5.0;
    else if (FULL && tok == v.id_6) val = (T)6.0;
    else if (FULL && tok == v.id_10) val = (T)10.0;
    else if (tok == v.id_pi) val = pi_val;
    else if (tok == v.id_e) val = e_val;
    else if (tok == v.id_C) {
      const int64_t ri = c_idx < K ? c_idx : K - 1;
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
      if (tok == v.op_add) res = lhs + rhs;
      else if (tok == v.op_sub) res = lhs - rhs;
      else if (tok == v.op_mul) res = lhs * rhs;
      else if (tok == v.op_div) res = (fabsf((float)rhs) > 1e-12f) ? lhs / rhs : (T)1e30;
      else if (tok == v.op_pow) res = powf(fabsf((float)lhs) + 1e-12f, (float)rhs);
      else if (FULL && tok == v.op_mod)
        res = (fabsf((float)rhs) > 1e-12f) ? fmodf((float)lhs, (float)rhs) : (T)0.0;
      else {
        sp += 2;
        err = true;
      }
      if (!err) stack[sp++] = res;
    }
    if (push && sp < kStack) stack[sp++] = val;
  }
  if (err || sp != 1) return false;
  pred = stack[0];
  return pred == pred && !std::isinf(pred);
}

template <typename T>
void rmse_and_grad(const uint8_t* prog, int64_t L, const T* x, int64_t nv, int64_t D,
                   const T* y, const T* pos, int64_t K, const ws_token_map& v, T pi_val, T e_val,
                   T cmin, T cmax, T* rmse_out, T* grad_out) {
  T mse_sum = (T)0.0;
  for (int64_t k = 0; k < K; ++k) grad_out[k] = (T)0.0;
  const T eps = (T)1e-5;
  for (int64_t d = 0; d < D; ++d) {
    T pred;
    if (!eval_row<T, true>(prog, L, x, nv, D, d, pos, K, v, pi_val, e_val, pred)) {
      *rmse_out = (T)1e30;
      return;
    }
    const T diff = pred - y[d];
    mse_sum += diff * diff;
  }
  *rmse_out = sqrtf((float)(mse_sum / (T)D));
  for (int64_t k = 0; k < K; ++k) {
    T pp[kMaxK], pm[kMaxK];
    for (int64_t j = 0; j < K; ++j) pp[j] = pm[j] = pos[j];
    pp[k] += eps;
    pm[k] -= eps;
    pp[k] = fmaxf((float)cmin, fminf((float)cmax, (float)pp[k]));
    pm[k] = fmaxf((float)cmin, fminf((float)cmax, (float)pm[k]));
    T mse_p = (T)0.0, mse_m = (T)0.0;
    for (int64_t d = 0; d < D; ++d) {
      T pred;
      if (eval_row<T, false>(prog, L, x, nv, D, d, pp, K, v, pi_val, e_val, pred)) {
        const T diff = pred - y[d];
        mse_p += diff * diff;
      }
      if (eval_row<T, false>(prog, L, x, nv, D, d, pm, K, v, pi_val, e_val, pred)) {
        const T diff = pred - y[d];
        mse_m += diff * diff;
      }
    }
    const T rp = sqrtf((float)(mse_p / (T)D));
    const T rm = sqrtf((float)(mse_m / (T)D));
    const T actual_eps = pp[k] - pm[k];
    if (actual_eps > 1e-10f) grad_out[k] = (rp - rm) / actual_eps;
  }
}

template <typename T>
void lbfgs(const uint8_t* pop, int64_t B, int64_t L, T* consts, int64_t K, const T* x,
           int64_t nv, int64_t D, const T* y, T* out, int max_iter, float gtol_f, float cmin_f,
           float cmax_f, const ws_token_map& v) {
  const T gtol = (T)gtol_f, cmin = (T)cmin_f, cmax = (T)cmax_f;
  const T pi_val = (T)v.pi_val, e_val = (T)v.e_val;
  for (int64_t b = 0; b < B; ++b) {
    const uint8_t* prog = pop + b * L;
    T x_curr[kMaxK], g_curr[kMaxK], x_prev[kMaxK], g_prev[kMaxK];
    T s_hist[kHist][kMaxK], y_hist[kHist][kMaxK], rho_hist[kHist];
    std::memset(s_hist, 0, sizeof(s_hist));
    std::memset(y_hist, 0, sizeof(y_hist));
    std::memset(rho_hist, 0, sizeof(rho_hist));
    int history_ptr = 0, history_count = 0;
    for (int64_t k = 0; k < K; ++k) x_curr[k] = x_prev[k] = consts[b * K + k];
    T f_curr;
    rmse_and_grad<T>(prog, L, x, nv, D, y, x_curr, K, v, pi_val, e_val, cmin, cmax, &f_curr,
                     g_curr);
    for (int iter = 0; iter < max_iter; ++iter) {
      T g_norm = (T)0.0;
      for (int64_t k = 0; k < K; ++k) g_norm += g_curr[k] * g_curr[k];
      g_norm = sqrtf((float)g_norm);
      if (g_norm < gtol) break;
      T q[kMaxK], alpha[kHist];
      for (int64_t k = 0; k < K; ++k) q[k] = g_curr[k];
      const int num_hist = history_count;
      for (int i = num_hist - 1; i >= 0; --i) {
        const int idx = (history_ptr - num_hist + i + kHist) % kHist;
        T dot = (T)0.0;
        for (int64_t k = 0; k < K; ++k) dot += s_hist[idx][k] * q[k];
        alpha[i] = rho_hist[idx] * dot;
        for (int64_t k = 0; k < K; ++k) q[k] -= alpha[i] * y_hist[idx][k];
      }
      T gamma = (T)1.0;
      if (history_count > 0) {
        const int last = (history_ptr - 1 + kHist) % kHist;
        T yty = (T)0.0, yts = (T)0.0;
        for (int64_t k = 0; k < K; ++k) {
          yty += y_hist[last][k] * y_hist[last][k];
          yts += y_hist[last][k] * s_hist[last][k];
        }
        if (yts > 1e-10f) gamma = yts / yty;
      }
      for (int64_t k = 0; k < K; ++k) q[k] *= gamma;
      for (int i = 0; i < num_hist; ++i) {
        const int idx = (history_ptr - num_hist + i + kHist) % kHist;
        T dot = (T)0.0;
        for (int64_t k = 0; k < K; ++k) dot += y_hist[idx][k] * q[k];
        const T beta = rho_hist[idx] * dot;
        for (int64_t k = 0; k < K; ++k) q[k] += s_hist[idx][k] * (alpha[i] - beta);
      }
      T p[kMaxK];
      for (int64_t k = 0; k < K; ++k) p[k] = -q[k];
      T step = (T)1.0;
      bool ok = false;
      for (int ls = 0; ls < kMaxLs; ++ls) {
        for (int64_t k = 0; k < K; ++k) {
          x_prev[k] = x_curr[k] + step * p[k];
          if (x_prev[k] < cmin) x_prev[k] = cmin;
          if (x_prev[k] > cmax) x_prev[k] = cmax;
        }
        T f_trial;
        rmse_and_grad<T>(prog, L, x, nv, D, y, x_prev, K, v, pi_val, e_val, cmin, cmax, &f_trial,
                         g_prev);
        if (f_trial <= f_curr - (T)1e-4 * step * g_norm * g_norm || f_trial < f_curr) {
          for (int64_t k = 0; k < K; ++k) x_curr[k] = x_prev[k];
          for (int64_t k = 0; k < K; ++k) g_prev[k] = g_curr[k];
          f_curr = f_trial;
          ok = true;
          break;
        }
        step *= (T)0.5;
      }
      if (!ok) break;
      if (history_count < kHist) history_count++;
      const int idx = history_ptr % kHist;
      T ys = (T)0.0;
      for (int64_t k = 0; k < K; ++k) {
        s_hist[idx][k] = x_curr[k] - x_prev[k];
        y_hist[idx][k] = g_curr[k] - g_prev[k];
        ys += y_hist[idx][k] * s_hist[idx][k];
      }
      if (ys > 1e-10f) {
        rho_hist[idx] = (T)1.0 / ys;
        history_ptr++;
      }
    }
    for (int64_t k = 0; k < K; ++k) consts[b * K + k] = x_curr[k];
    out[b] = f_curr;
  }
}

}  // namespace

extern "C" {

void ws_oracle_lbfgs_f32(const uint8_t* pop, int64_t B, int64_t L, float* consts, int64_t K,
                         const float* x, int64_t nv, int64_t D, const float* y, float* out,
                         int max_iter, float gtol, float cmin, float cmax, const ws_token_map* m) {
  lbfgs<float>(pop, B, L, consts, K, x, nv, D, y, out, max_iter, gtol, cmin, cmax, *m);
}
void ws_oracle_lbfgs_f64(const uint8_t* pop, int64_t B, int64_t L, double* consts, int64_t K,
                         const double* x, int64_t nv, int64_t D, const double* y, double* out,
                         int max_iter, float gtol, float cmin, float cmax,
                         const ws_token_map* m) {
  lbfgs<double>(pop, B, L, consts, K, x, nv, D, y, out, max_iter, gtol, cmin, cmax, *m);
}

}  // extern "C"
