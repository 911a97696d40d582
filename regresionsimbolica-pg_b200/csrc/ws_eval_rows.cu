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

// A warp owns a tile of 32 * R rows of one program; lane t carries rows base + t + 32 r
// (r < R), so x reads and output writes stay coalesced.  The interpreter's control flow depends
// on the tokens only (pushes, pops, the push-drop at depth 32, underflow and unknown tokens), so
// the R rows share it and one decode of a token serves them all; a row that the reference would
// stop at an operator's error (a domain error, or what the protected operators report) is frozen
// instead: its depth and stack top at that point are recorded and its later values ignored.
// Each row's outputs are the reference's.
template <typename T, int R>
struct __align__(16) RowVec {
  T v[R];
};

template <typename T, bool STRICT, int R>
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

  const int lane = threadIdx.x & 31;
  const int64_t tile_rows = 32 * (int64_t)R;
  const int64_t tiles_per_prog = (D + tile_rows - 1) / tile_rows;
  const int64_t n_tiles = B * tiles_per_prog;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       tile < n_tiles; tile += warps) {
    const int64_t b = tile / tiles_per_prog;
    const int64_t base = (tile - b * tiles_per_prog) * tile_rows + lane;
    const uint8_t* prog = pop + b * L;
    RowVec<T, R> stack[32];
    int sp = 0;
    int64_t c_idx = 0;
    // per row: frozen at an error (depth and top recorded then)
    bool stopped[R];
    int stop_sp[R];
    T stop_top[R];
#pragma unroll
    for (int r = 0; r < R; ++r) stopped[r] = false;
    bool all_stop = false;  // a token-driven error stops every row at once
    for (int64_t pc = 0; pc < L && !all_stop; ++pc) {
      const int tok = prog[pc];
      const int cls = s_cls[tok];
      if (cls == T_PAD) break;
      if (is_leaf(cls)) {
        RowVec<T, R> val;
        if (cls == T_VAR) {
          const T* xr = x + (int64_t)s_arg[tok] * D;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int64_t d = base + 32 * r;
            val.v[r] = d < D ? xr[d] : (T)0;
          }
        } else {
          T c;
          if (cls == T_CONST) {
            if (K > 0) {
              const int64_t ri = c_idx < K ? c_idx : K - 1;
              c = consts[b * K + ri];
              c_idx++;
            } else {
              c = (T)1.0;
            }
          } else {
            c = s_lit[s_arg[tok]];
          }
#pragma unroll
          for (int r = 0; r < R; ++r) val.v[r] = c;
        }
        if (sp < 32) stack[sp++] = val;
        continue;
      }
      if (is_binary(cls)) {
        if (sp < 2) {
          all_stop = true;
          break;
        }
        const RowVec<T, R> op2 = stack[--sp];
        const RowVec<T, R> op1 = stack[--sp];
        RowVec<T, R> res;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          bool e = false;
          res.v[r] = apply_binary<T, STRICT>(cls, op1.v[r], op2.v[r], e);
          if (e && !stopped[r]) {
            stopped[r] = true;
            stop_sp[r] = sp;
            stop_top[r] = sp > 0 ? stack[sp - 1].v[r] : Limits<T>::no_value;
          }
        }
        stack[sp++] = res;
        continue;
      }
      if (sp < 1) {
        all_stop = true;
        break;
      }
      const RowVec<T, R> a = stack[--sp];
      if (!is_unary(cls)) {
        all_stop = true;
        break;
      }
      RowVec<T, R> res;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        bool e = false;
        res.v[r] = apply_unary<T, STRICT>(cls, a.v[r], e);
        if (e && !stopped[r]) {
          stopped[r] = true;
          stop_sp[r] = sp;
          stop_top[r] = sp > 0 ? stack[sp - 1].v[r] : Limits<T>::no_value;
        }
      }
      stack[sp++] = res;
    }
    // rows still running at a token-driven error or at the end take the current depth and top
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t d = base + 32 * r;
      if (d >= D) continue;
      const int64_t idx = b * D + d;
      if (stopped[r]) {
        out_sp[idx] = stop_sp[r];
        out_err[idx] = 1;
        out_preds[idx] = stop_top[r];
      } else {
        out_sp[idx] = sp;
        out_err[idx] = all_stop ? 1 : 0;
        out_preds[idx] = sp > 0 ? stack[sp - 1].v[r] : Limits<T>::no_value;
      }
    }
  }
}

ws_status launch_eval_rows(int dtype, const uint8_t* pop, int64_t B, int64_t L, const void* x,
                           int64_t D, const void* consts, int64_t K, const TokenLut& lut,
                           void* out_preds, int32_t* out_sp, uint8_t* out_err, int strict,
                           cudaStream_t stream) {
  if (B * D == 0) return WS_OK;
  const int threads = 256;
  constexpr int RF = 4, RD = 2;  // rows per lane (16-byte stack entries): float, double
  const int64_t rows_per_tile = 32 * (int64_t)(dtype == WS_F32 ? RF : RD);
  const int64_t tiles = B * ((D + rows_per_tile - 1) / rows_per_tile);
  int64_t blocks = (tiles + (threads / 32) - 1) / (threads / 32);
  const int64_t cap = (int64_t)device_info().sm_count * 32;
  if (blocks > cap) blocks = cap;
  if (dtype == WS_F32) {
    if (strict)
      eval_rows_kernel<float, true, RF><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const float*)x, D, (const float*)consts, K, lut, (float*)out_preds, out_sp, out_err);
    else
      eval_rows_kernel<float, false, RF><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const float*)x, D, (const float*)consts, K, lut, (float*)out_preds, out_sp, out_err);
  } else {
    if (strict)
      eval_rows_kernel<double, true, RD><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const double*)x, D, (const double*)consts, K, lut, (double*)out_preds, out_sp, out_err);
    else
      eval_rows_kernel<double, false, RD><<<(unsigned)blocks, threads, 0, stream>>>(
          pop, B, L, (const double*)x, D, (const double*)consts, K, lut, (double*)out_preds, out_sp, out_err);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "eval_rows_kernel launch");
  return WS_OK;
}

}  // namespace ws
