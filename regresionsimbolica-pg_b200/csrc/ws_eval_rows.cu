// ws_eval_rows.cu -- per-(program,row) interpreter with the reference's exact per-row outputs.
//
// Replaces rpn_eval_kernel / launch_rpn_kernel (rpn_kernels.cu:202-429) behind `eval_rpn`:
// writes the stack top (or 1e30), the final stack depth and the error byte of every
// (program, row), which callers of eval_rpn consume directly (cuda_vm.py:84-152).  Those
// outputs depend on where a row stops (its stack at the error), so this kernel keeps the
// reference's stack discipline instead of the compiled tape.  Differences by design: the token
// classification is one shared-memory table lookup instead of a chain of ~40 compares, the
// index space is 64-bit (the reference's `int B*D` overflows beyond 2^31 rows), and launches go
// to the caller's stream.
#include <cuda_runtime.h>
#include <cstdint>

#include "ws_internal.h"

namespace ws {

template <typename T, bool STRICT>
__global__ void __launch_bounds__(256) eval_rows_kernel(
    const uint8_t* __restrict__ pop, int64_t B, int64_t L, const T* __restrict__ x, int64_t D,
    const T* __restrict__ consts, int64_t K, TokenLut lut, T* __restrict__ out_preds,
    int32_t* __restrict__ out_sp, uint8_t* __restrict__ out_err) {
  __shared__ uint8_t s_cls[256];
  __shared__ uint8_t s_arg[256];
  __shared__ T s_lit[N_LITERALS];
  s_cls[threadIdx.x] = lut.cls[threadIdx.x];
  s_arg[threadIdx.x] = lut.arg[threadIdx.x];
  if (threadIdx.x < N_LITERALS) s_lit[threadIdx.x] = (T)lut.lit[threadIdx.x];
  __syncthreads();

  const int64_t total = B * D;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = idx / D, d = idx - b * D;
    const uint8_t* prog = pop + b * L;
    T stack[32];
    int sp = 0;
    bool error = false;
    int64_t c_idx = 0;
    for (int64_t pc = 0; pc < L; ++pc) {
      const int tok = prog[pc];
      const int cls = s_cls[tok];
      if (cls == T_PAD) break;
      if (is_leaf(cls)) {
        T val;
        if (cls == T_VAR) {
          val = x[(int64_t)s_arg[tok] * D + d];
        } else if (cls == T_CONST) {
          if (K > 0) {
            const int64_t r = c_idx < K ? c_idx : K - 1;
            val = consts[b * K + r];
            c_idx++;
          } else {
            val = (T)1.0;
          }
        } else {
          val = s_lit[s_arg[tok]];
        }
        if (sp < 32) stack[sp++] = val;
        continue;
      }
      if (is_binary(cls)) {
        if (sp < 2) { error = true; break; }
        const T op2 = stack[--sp];
        const T op1 = stack[--sp];
        bool e = false;
        const T res = apply_binary<T, STRICT>(cls, op1, op2, e);
        if (e) { error = true; break; }
        stack[sp++] = res;
        continue;
      }
      if (sp < 1) { error = true; break; }
      const T a = stack[--sp];
      if (!is_unary(cls)) { error = true; break; }
      bool e = false;
      const T res = apply_unary<T, STRICT>(cls, a, e);
      if (e) { error = true; break; }
      stack[sp++] = res;
    }
    out_sp[idx] = sp;
    out_err[idx] = error ? 1 : 0;
    out_preds[idx] = sp > 0 ? stack[sp - 1] : Limits<T>::no_value;
  }
}

ws_status launch_eval_rows(int dtype, const uint8_t* pop, int64_t B, int64_t L, const void* x,
                           int64_t D, const void* consts, int64_t K, const TokenLut& lut,
                           void* out_preds, int32_t* out_sp, uint8_t* out_err, int strict,
                           cudaStream_t stream) {
  const int64_t total = B * D;
  if (total == 0) return WS_OK;
  const int threads = 256;
  int64_t blocks = (total + threads - 1) / threads;
  const int64_t cap = (int64_t)device_info().sm_count * 32;
  if (blocks > cap) blocks = cap;
  if (dtype == WS_F32) {
    if (strict)
      eval_rows_kernel<float, true><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const float*)x, D, (const float*)consts, K, lut, (float*)out_preds, out_sp, out_err);
    else
      eval_rows_kernel<float, false><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const float*)x, D, (const float*)consts, K, lut, (float*)out_preds, out_sp, out_err);
  } else {
    if (strict)
      eval_rows_kernel<double, true><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const double*)x, D, (const double*)consts, K, lut, (double*)out_preds, out_sp, out_err);
    else
      eval_rows_kernel<double, false><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const double*)x, D, (const double*)consts, K, lut, (double*)out_preds, out_sp, out_err);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "eval_rows_kernel launch");
  return WS_OK;
}

}  // namespace ws
