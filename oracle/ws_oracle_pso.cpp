// ws_oracle_pso.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatements of the reference's particle-swarm pieces, used by tests/ as checkers:
//   pso_update        pso_update_kernel (src/warpsymbolic/gpu/cuda/pso_kernels.cu:29-70)
//   pso_update_bests  pso_update_bests_kernel + pso_update_gbest_kernel (:74-153), including
//                     the warp's lane-strided / shuffle-tree tie rule
//   pso_rmse          the fused PSO's fitness: eval_rpn_single over every row, then RMSE
//                     (fused_pso_kernels.cu:35-197, 330-351), IEEE libm
// The random streams of the fused loop come from curand; they are not restated here.  The fused
// loop is checked against the reference extension itself, and here through properties of its
// result (the reported error is the fitness of the reported constants).

#include <cmath>
#include <cstdint>
#include <vector>

#include "../include/warpsym.h"

namespace {

template <typename T>
void pso_update(T* pos, T* vel, const T* pbest, const T* gbest, const T* r1, const T* r2,
                float w, float c1, float c2, int64_t B, int64_t P, int64_t K) {
  for (int64_t idx = 0; idx < B * P * K; ++idx) {
    const int64_t k = idx % K, b = (idx / K) / P;
    const T nv = (T)w * vel[idx] + (T)c1 * r1[idx] * (pbest[idx] - pos[idx]) +
                 (T)c2 * r2[idx] * (gbest[b * K + k] - pos[idx]);
    vel[idx] = nv;
    pos[idx] = pos[idx] + nv;
  }
}

template <typename T>
void pso_bests(const T* cur_err, T* pb_err, T* pb_pos, const T* cur_pos, T* gb_err, T* gb_pos,
               int64_t B, int64_t P, int64_t K) {
  for (int64_t i = 0; i < B * P; ++i)
    if (cur_err[i] < pb_err[i]) {
      pb_err[i] = cur_err[i];
      for (int64_t k = 0; k < K; ++k) pb_pos[i * K + k] = cur_pos[i * K + k];
    }
  for (int64_t b = 0; b < B; ++b) {
    T best[32];
    int bp[32];
    for (int t = 0; t < 32; ++t) {
      best[t] = (T)1e30;
      bp[t] = -1;
      for (int64_t p = t; p < P; p += 32)
        if (pb_err[b * P + p] < best[t]) {
          best[t] = pb_err[b * P + p];
          bp[t] = (int)p;
        }
    }
    for (int off = 16; off > 0; off >>= 1)  // __shfl_down tree: lane t takes t + off if smaller
      for (int t = 0; t + off < 32; ++t)
        if (best[t + off] < best[t]) {
          best[t] = best[t + off];
          bp[t] = bp[t + off];
        }
    if (bp[0] >= 0 && best[0] < gb_err[b]) {
      gb_err[b] = best[0];
      for (int64_t k = 0; k < K; ++k) gb_pos[b * K + k] = pb_pos[(b * P + bp[0]) * K + k];
    }
  }
}

constexpr float kInf = 1e30f;

float safe_pow(float a, float b) {
  if (a != a || b != b) return kInf;
  const bool is_int = (std::floor(b) == b);
  if (a < 0.0f && !is_int) {
    if (std::fabs(b - std::round(b)) < 1e-4f) b = std::round(b);
    else return kInf;
  }
  if (a == 0.0f && b < 0.0f) return kInf;
  const float res = std::pow(a, b);
  if (res != res || std::isinf(res)) return kInf;
  if (std::fabs(res) > 1e18f) return kInf;
  return res;
}

// eval_rpn_single (fused_pso_kernels.cu:57-197) for one row.
float eval_single(const uint8_t* prog, int64_t L, const float* x, int64_t num_vars, int64_t d,
                  int64_t D, const float* consts, int64_t K, const ws_token_map& v) {
  float stack[32];
  int sp = 0;
  int64_t c_idx = 0;
  const float pi_val = (float)v.pi_val, e_val = (float)v.e_val;
  for (int64_t pc = 0; pc < L; ++pc) {
    const int64_t token = prog[pc];
    if (token == v.pad_id) break;
    float val = 0.0f;
    bool is_push = true;
    if (token >= v.id_x_start && token < v.id_x_start + num_vars)
      val = x[(token - v.id_x_start) * D + d];
    else if (token == v.id_0) val = 0.0f;
    else if (token == v.id_1) val = 1.0f;
    else if (token == v.id_2) val = 2.0f;
    else if (token == v.id_3) val = 3.0f;
    else if (token == v.id_4) val = 4.0f;
    else if (token == v.id_5) val = 5.0f;
    else if (token == v.id_6) val = 6.0f;
    else if (token == v.id_10) val = 10.0f;
    else if (token == v.id_pi) val = pi_val;
    else if (token == v.id_e) val = e_val;
    else if (token == v.id_C) {
      const int64_t r = c_idx < K ? c_idx : K - 1;
      val = r >= 0 ? consts[r] : 1.0f;
      c_idx++;
    } else is_push = false;
    if (is_push) {
      if (sp < 32) stack[sp++] = val;
      continue;
    }
    if (token == v.op_add || token == v.op_sub || token == v.op_mul || token == v.op_div ||
        token == v.op_pow || token == v.op_mod) {
      if (sp < 2) return kInf;
      const float b = stack[--sp], a = stack[--sp];
      float res = 0.0f;
      if (token == v.op_add) res = a + b;
      else if (token == v.op_sub) res = a - b;
      else if (token == v.op_mul) res = a * b;
      else if (token == v.op_div) {
        if (std::fabs(b) < 1e-12f) return kInf;
        res = a / b;
      } else if (token == v.op_pow) {
        res = safe_pow(a, b);
        if (res >= 1e29f) return kInf;
      } else {
        if (std::fabs(b) < 1e-12f) return kInf;
        res = std::fmod(a, b);
      }
      stack[sp++] = res;
      continue;
    }
    if (sp < 1) return kInf;
    const float a = stack[--sp];
    float res = 0.0f;
    if (token == v.op_sin) res = std::sin(a);
    else if (token == v.op_cos) res = std::cos(a);
    else if (token == v.op_tan) res = std::tan(a);
    else if (token == v.op_abs) res = std::fabs(a);
    else if (token == v.op_neg) res = -a;
    else if (token == v.op_sqrt) {
      if (a < 0.0f) return kInf;
      res = std::sqrt(a);
    } else if (token == v.op_log) {
      if (a <= 1e-12f) return kInf;
      res = std::log(a);
    } else if (token == v.op_exp) {
      if (a > 80.0f) return kInf;
      res = a < -80.0f ? 0.0f : std::exp(a);
    } else if (token == v.op_floor) res = std::floor(a);
    else if (token == v.op_ceil) res = std::ceil(a);
    else if (token == v.op_sign) res = a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : 0.0f);
    else if (token == v.op_asin) {
      if (a < -1.0f || a > 1.0f) return kInf;
      res = std::asin(a);
    } else if (token == v.op_acos) {
      if (a < -1.0f || a > 1.0f) return kInf;
      res = std::acos(a);
    } else if (token == v.op_atan) res = std::atan(a);
    else if (token == v.op_fact) {
      if (a <= -1.0f && std::floor(a + 1.0f) == a + 1.0f) return kInf;
      if (a > 50.0f) return kInf;
      res = std::tgamma(a + 1.0f);
      if (res != res || std::isinf(res)) return kInf;
    } else if (token == v.op_gamma) {
      if (a <= 0.0f && std::floor(a) == a) return kInf;
      if (a > 50.0f) return kInf;
      res = std::tgamma(a);
      if (res != res || std::isinf(res)) return kInf;
    } else if (token == v.op_lgamma) {
      if (a <= 0.0f && std::floor(a) == a) return kInf;
      res = std::lgamma(a);
      if (res != res || std::isinf(res)) return kInf;
    }
    if (res != res || std::isinf(res)) return kInf;
    stack[sp++] = res;
  }
  if (sp != 1) return kInf;
  const float r = stack[0];
  return (r != r || std::isinf(r)) ? kInf : r;
}

}  // namespace

extern "C" {

void ws_oracle_pso_update_f32(float* pos, float* vel, const float* pbest, const float* gbest,
                              const float* r1, const float* r2, float w, float c1, float c2,
                              int64_t B, int64_t P, int64_t K) {
  pso_update<float>(pos, vel, pbest, gbest, r1, r2, w, c1, c2, B, P, K);
}
void ws_oracle_pso_update_f64(double* pos, double* vel, const double* pbest, const double* gbest,
                              const double* r1, const double* r2, float w, float c1, float c2,
                              int64_t B, int64_t P, int64_t K) {
  pso_update<double>(pos, vel, pbest, gbest, r1, r2, w, c1, c2, B, P, K);
}
void ws_oracle_pso_bests_f32(const float* ce, float* pe, float* pp, const float* cp, float* ge,
                             float* gp, int64_t B, int64_t P, int64_t K) {
  pso_bests<float>(ce, pe, pp, cp, ge, gp, B, P, K);
}
void ws_oracle_pso_bests_f64(const double* ce, double* pe, double* pp, const double* cp,
                             double* ge, double* gp, int64_t B, int64_t P, int64_t K) {
  pso_bests<double>(ce, pe, pp, cp, ge, gp, B, P, K);
}

// RMSE of program b under the fused PSO's evaluator for constants consts[b, :K] (float32);
// 1e30 when any row fails (fused_pso_kernels.cu:330-351).
void ws_oracle_pso_rmse(const uint8_t* pop, int64_t B, int64_t L, const float* x,
                        int64_t num_vars, int64_t D, const float* consts, int64_t K,
                        const float* y, const ws_token_map* m, float* out) {
  for (int64_t b = 0; b < B; ++b) {
    float mse_sum = 0.0f;
    bool any_error = false;
    for (int64_t d = 0; d < D; ++d) {
      const float pred = eval_single(pop + b * L, L, x, num_vars, d, D, consts + b * K, K, *m);
      if (pred >= 1e29f) {
        any_error = true;
        break;
      }
      const float diff = pred - y[d];
      mse_sum += diff * diff;
    }
    out[b] = any_error ? kInf : std::sqrt(mse_sum / (float)D);
  }
}

}  // extern "C"
