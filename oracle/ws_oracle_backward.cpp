// ws_oracle_backward.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's adjoint kernel rpn_eval_backward_kernel
// (src/warpsymbolic/gpu/cuda/backward_kernels.cu:13-281), one (program, row) at a time with the
// reference's own forward rules, index stack and reverse sweep.  Instead of the reference's
// float atomics, the per-row constant adjoints are summed in double, and the sum of their
// absolute values is returned alongside, so that tests can bound the rounding of any
// summation order (tolerance = rtol * sum|terms|).  IEEE libm, no contraction.
//
// Pinned against: the reference extension's eval_rpn_backward on the same inputs (GPU tests),
// central finite differences and torch autograd on differentiable programs (tests).

#include <cmath>
#include <cstdint>
#include <vector>

#include "../include/warpsym.h"

namespace {

constexpr int kStack = 32;

// With y non-null (loss mode) the root adjoint of row d is (pred - y[d]) * (2 / D) and loss[b]
// receives mean_d (pred - y[d])^2 (infinite for a program without a result): the loss and
// gradient of the per-program L-BFGS (csrc/ws_lbfgs_batch.cu).
template <typename T>
void backward_rows(const uint8_t* pop, int64_t B, int64_t L, const T* x, int64_t num_vars,
                   int64_t D, const T* consts, int64_t K, const T* gout,
                   const ws_token_map& m, double* grad, double* abssum, const T* y = nullptr,
                   double* loss = nullptr) {
  const ws_token_map& v = m;
  std::vector<T> val_tape(L), adj_tape(L);
  std::vector<int> args_left(L), args_right(L), const_index(L);
  const T scale = (T)(2.0 / (double)D);
  for (int64_t b = 0; b < B; ++b) {
    const uint8_t* prog = pop + b * L;
    if (y) loss[b] = 0.0;
    for (int64_t d = 0; d < D; ++d) {
      int idx_stack[kStack];
      int sp = 0, root_pc = -1;
      int64_t c_idx = 0;
      for (int pc = 0; pc < (int)L; ++pc) {
        const int64_t token = prog[pc];
        if (token == v.pad_id) break;
        args_left[pc] = -1;
        args_right[pc] = -1;
        const_index[pc] = -1;
        adj_tape[pc] = (T)0.0;
        T val = (T)0.0;
        bool is_push = true;
        if (token >= v.id_x_start && token < v.id_x_start + num_vars) {
          val = x[(token - v.id_x_start) * D + d];
        } else if (token == v.id_0) val = (T)0.0;
        else if (token == v.id_1) val = (T)1.0;
        else if (token == v.id_2) val = (T)2.0;
        else if (token == v.id_3) val = (T)3.0;
        else if (token == v.id_4) val = (T)4.0;
        else if (token == v.id_5) val = (T)5.0;
        else if (token == v.id_6) val = (T)6.0;
        else if (token == v.id_10) val = (T)10.0;
        else if (token == v.id_pi) val = (T)v.pi_val;
        else if (token == v.id_e) val = (T)v.e_val;
        else if (token == v.id_C) {
          if (K > 0) {
            const int64_t r_idx = (c_idx < K) ? c_idx : (K - 1);
            val = consts[b * K + r_idx];
            const_index[pc] = (int)r_idx;
            c_idx++;
          } else {
            val = (T)1.0;
          }
        } else {
          is_push = false;
        }
        if (is_push) {
          val_tape[pc] = val;
          if (sp < kStack) idx_stack[sp++] = pc;
          root_pc = pc;
          continue;
        }
        if (token == v.op_add || token == v.op_sub || token == v.op_mul || token == v.op_div ||
            token == v.op_pow || token == v.op_mod) {
          if (sp < 2) break;
          const int right_pc = idx_stack[--sp];
          const int left_pc = idx_stack[--sp];
          T op2 = val_tape[right_pc];
          T op1 = val_tape[left_pc];
          args_left[pc] = left_pc;
          args_right[pc] = right_pc;
          if (token == v.op_add) val = op1 + op2;
          else if (token == v.op_sub) val = op1 - op2;
          else if (token == v.op_mul) val = op1 * op2;
          else if (token == v.op_div) {
            if (std::fabs(op2) < (T)1e-9) val = op1; else val = op1 / op2;
          } else if (token == v.op_pow) {
            if (op1 < 0) {
              const T ib = std::round(op2);
              if (std::fabs(op2 - ib) <= (T)1e-3) op2 = ib; else op1 = std::fabs(op1);
            }
            val = std::pow(op1, op2);
          } else if (token == v.op_mod) {
            if (std::fabs(op2) < (T)1e-9) val = 0; else val = std::fmod(op1, op2);
          }
        } else {
          if (sp < 1) break;
          const int left_pc = idx_stack[--sp];
          const T op1 = val_tape[left_pc];
          args_left[pc] = left_pc;
          if (token == v.op_sin) val = std::sin(op1);
          else if (token == v.op_cos) val = std::cos(op1);
          else if (token == v.op_tan) val = std::tan(op1);
          else if (token == v.op_log) val = std::log(std::fabs(op1) + (T)1e-9);
          else if (token == v.op_exp) {
            T cl = op1;
            if (cl < -80.0) cl = (T)-80.0;
            if (cl > 80.0) cl = (T)80.0;
            val = std::exp(cl);
          } else if (token == v.op_sqrt) val = std::sqrt(std::fabs(op1));
          else if (token == v.op_abs) val = std::fabs(op1);
          else if (token == v.op_neg) val = -op1;
        }
        val_tape[pc] = val;
        idx_stack[sp++] = pc;
        root_pc = pc;
      }
      if (root_pc == -1 || sp != 1) {
        if (y) loss[b] = HUGE_VAL;
        continue;
      }
      if (y) {
        const T diff = val_tape[root_pc] - y[d];
        loss[b] += (double)diff * (double)diff;
        adj_tape[root_pc] = diff * scale;
      } else {
        adj_tape[root_pc] = gout[b * D + d];
      }
      for (int pc = root_pc; pc >= 0; --pc) {
        const T adj = adj_tape[pc];
        if (adj == (T)0.0) continue;
        const int64_t token = prog[pc];
        const int l_pc = args_left[pc];
        const int r_pc = args_right[pc];
        if (const_index[pc] != -1) {
          grad[b * K + const_index[pc]] += (double)adj;
          abssum[b * K + const_index[pc]] += std::fabs((double)adj);
          continue;
        }
        if (l_pc == -1) continue;
        const T l_val = val_tape[l_pc];
        if (r_pc != -1) {
          const T r_val = val_tape[r_pc];
          if (token == v.op_add) {
            adj_tape[l_pc] += adj;
            adj_tape[r_pc] += adj;
          } else if (token == v.op_sub) {
            adj_tape[l_pc] += adj;
            adj_tape[r_pc] -= adj;
          } else if (token == v.op_mul) {
            adj_tape[l_pc] += r_val * adj;
            adj_tape[r_pc] += l_val * adj;
          } else if (token == v.op_div) {
            if (std::fabs(r_val) >= (T)1e-9) {
              adj_tape[l_pc] += (1.0 / r_val) * adj;
              adj_tape[r_pc] -= (l_val / (r_val * r_val)) * adj;
            }
          } else if (token == v.op_pow) {
            const T out_val = val_tape[pc];
            if (l_val > 0) {
              adj_tape[l_pc] += (r_val * std::pow((double)l_val, r_val - 1.0)) * adj;
              adj_tape[r_pc] += (out_val * std::log(l_val)) * adj;
            }
          }
        } else {
          if (token == v.op_sin) adj_tape[l_pc] += std::cos(l_val) * adj;
          else if (token == v.op_cos) adj_tape[l_pc] += -std::sin(l_val) * adj;
          else if (token == v.op_log) {
            if (std::fabs(l_val) > (T)1e-9) adj_tape[l_pc] += (1.0 / l_val) * adj;
          } else if (token == v.op_exp) {
            adj_tape[l_pc] += val_tape[pc] * adj;
          } else if (token == v.op_sqrt) {
            if (l_val > (T)1e-9) adj_tape[l_pc] += (0.5 / std::sqrt(l_val)) * adj;
          } else if (token == v.op_neg) {
            adj_tape[l_pc] += -adj;
          }
        }
      }
    }
    if (y) loss[b] /= (double)D;
  }
}

}  // namespace

extern "C" {

// grad / abssum: double [B, K], zeroed here.
void ws_oracle_backward_f32(const uint8_t* pop, int64_t B, int64_t L, const float* x,
                            int64_t num_vars, int64_t D, const float* consts, int64_t K,
                            const float* gout, const ws_token_map* m, double* grad,
                            double* abssum) {
  for (int64_t i = 0; i < B * K; ++i) grad[i] = abssum[i] = 0.0;
  backward_rows<float>(pop, B, L, x, num_vars, D, consts, K, gout, *m, grad, abssum);
}
void ws_oracle_backward_f64(const uint8_t* pop, int64_t B, int64_t L, const double* x,
                            int64_t num_vars, int64_t D, const double* consts, int64_t K,
                            const double* gout, const ws_token_map* m, double* grad,
                            double* abssum) {
  for (int64_t i = 0; i < B * K; ++i) grad[i] = abssum[i] = 0.0;
  backward_rows<double>(pop, B, L, x, num_vars, D, consts, K, gout, *m, grad, abssum);
}

// loss [B], grad / abssum [B, K]: double, written here.
void ws_oracle_loss_grad_f32(const uint8_t* pop, int64_t B, int64_t L, const float* x,
                             int64_t num_vars, int64_t D, const float* consts, int64_t K,
                             const float* y, const ws_token_map* m, double* loss, double* grad,
                             double* abssum) {
  for (int64_t i = 0; i < B * K; ++i) grad[i] = abssum[i] = 0.0;
  backward_rows<float>(pop, B, L, x, num_vars, D, consts, K, nullptr, *m, grad, abssum, y, loss);
}
void ws_oracle_loss_grad_f64(const uint8_t* pop, int64_t B, int64_t L, const double* x,
                             int64_t num_vars, int64_t D, const double* consts, int64_t K,
                             const double* y, const ws_token_map* m, double* loss, double* grad,
                             double* abssum) {
  for (int64_t i = 0; i < B * K; ++i) grad[i] = abssum[i] = 0.0;
  backward_rows<double>(pop, B, L, x, num_vars, D, consts, K, nullptr, *m, grad, abssum, y, loss);
}

}  // extern "C"
