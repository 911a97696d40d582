// ws_structure.cu -- integer structure kernels on populations: stack validation, subtree starts,
// tournament selection.  All of them are bit-exact restatements of the reference's kernels:
//
//   validate  : validate_rpn_batch_kernel (rpn_kernels.cu:850-900), plus the two torch variants
//               the reference's Python callers use (operators.py:551-570 with clamped arity
//               lookup, gpu_simplifier.py:513-579 without the contiguity rule);
//   subtrees  : find_subtree_ranges_kernel (rpn_kernels.cu:433-504) and
//               precompute_subtree_starts_kernel (simplify_kernels.cu:612-661);
//   selection : tournament_selection_kernel / tournament_selection_offsets_kernel
//               (rpn_kernels.cu:1535-1668).
//
// These are HBM-bound byte/integer passes: one thread owns one program (the reference's own
// unit of dependence), reads its row once, and the [B, L] int64 outputs -- 8 bytes per token,
// the dominant traffic -- are staged per tile in shared memory and written out row-major by the
// whole block, so every warp store covers 256 contiguous bytes.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "ws_internal.h"

namespace ws {
namespace {

constexpr int kThreads = 128;  // one block = 128 programs
constexpr int kStagedMaxBytes = 96 * 1024;

// Reads one program row as a token stream: 16 or 4 bytes per load when the row allows it.
template <typename Tok>
struct RowReader;

template <>
struct RowReader<uint8_t> {
  const uint8_t* row;
  int64_t L;
  bool vec4;
  bool vec16 = false;  // L % 16 == 0 and a 16-byte aligned row
  template <typename F>
  __device__ __forceinline__ void for_each(F&& f) const {
    if (vec16) {
      const uint4* w = reinterpret_cast<const uint4*>(row);
      for (int64_t i0 = 0; i0 < L; i0 += 16) {
        const uint4 v = __ldg(w + (i0 >> 4));
        const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 16; ++k)
          if (!f(i0 + k, (int64_t)((q[k >> 2] >> (8 * (k & 3))) & 0xFFu))) return;
      }
    } else if (vec4) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(row);
      for (int64_t i0 = 0; i0 < L; i0 += 4) {
        uint32_t v = __ldg(w + (i0 >> 2));
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (!f(i0 + k, (int64_t)((v >> (8 * k)) & 0xFFu))) return;
      }
    } else {
      for (int64_t i = 0; i < L; ++i)
        if (!f(i, (int64_t)__ldg(row + i))) return;
    }
  }
};

template <>
struct RowReader<int64_t> {
  const int64_t* row;
  int64_t L;
  bool vec4;
  template <typename F>
  __device__ __forceinline__ void for_each(F&& f) const {
    for (int64_t i = 0; i < L; ++i)
      if (!f(i, (int64_t)__ldg(reinterpret_cast<const long long*>(row) + i))) return;
  }
};

__device__ __forceinline__ int32_t arity_of(const int32_t* ar, int64_t n_ar, int64_t t) {
  return (t >= 0 && t < n_ar) ? __ldg(ar + t) : 0;
}

__device__ __forceinline__ int32_t arity_clamped(const int32_t* ar, int64_t n_ar, int64_t t) {
  int64_t c = t < 0 ? 0 : (t > n_ar - 1 ? n_ar - 1 : t);
  return __ldg(ar + c);
}

// ---------------------------------------------------------------------------------------------
// Validation.  mode 0: validate_rpn_batch_kernel; 1: operators.py torch fallback (arity looked
// up with the token clamped into the table); 2: gpu_simplifier._validate_batch_stack (no
// contiguity rule, minimum over every position, at least one non-PAD token).
// uint8 tokens: the arity of every byte value is staged in shared memory once per block (the
// rule's lookup: mode 0 zero outside the table, modes 1-2 the clamped entry) and rows are read
// 16 bytes per load when their length and address allow.
template <typename Tok>
__global__ void __launch_bounds__(kThreads)
    validate_kernel(const Tok* __restrict__ pop, int64_t B, int64_t L,
                    const int32_t* __restrict__ ar, int64_t n_ar, int64_t pad, int mode,
                    bool vec4, bool vec16, uint8_t* __restrict__ out) {
  constexpr bool U8 = sizeof(Tok) == 1;
  __shared__ int32_t s_ar[U8 ? 256 : 1];
  if (U8) {
    for (int t = threadIdx.x; t < 256; t += blockDim.x)
      s_ar[t] = mode == 0 ? arity_of(ar, n_ar, t) : arity_clamped(ar, n_ar, t);
    __syncthreads();
  }
  auto arity = [&](int64_t t) -> int64_t {
    if (U8) return s_ar[t];
    return mode == 0 ? arity_of(ar, n_ar, t) : arity_clamped(ar, n_ar, t);
  };
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    RowReader<Tok> rd{pop + b * L, L, vec4};
    if constexpr (U8) rd.vec16 = vec16;
    int64_t stack = 0;
    bool ok = true, pad_seen = false, has_tok = false;
    if (mode != 2) {
      rd.for_each([&](int64_t, int64_t t) {
        if (t == pad) { pad_seen = true; return true; }
        if (pad_seen) { ok = false; return false; }
        stack += 1 - arity(t);
        if (stack < 1) { ok = false; return false; }
        return true;
      });
      ok = ok && stack == 1;
    } else {
      rd.for_each([&](int64_t, int64_t t) {
        if (t != pad) {
          has_tok = true;
          stack += 1 - arity(t);
        }
        if (stack < 1) { ok = false; return false; }
        return true;
      });
      ok = ok && has_tok && stack == 1 && L > 0;
    }
    out[b] = ok ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------------------------
// Subtree starts.  Both kernels compute one row per thread into `srow` (a shared-memory tile row
// with stride `sstride`, or the output row itself when the row is too long to stage), reading
// back only the thread's own earlier results.

// find_subtree_ranges: start[i] is the largest j < i, inside the PAD-free run that ends at i,
// where the reference's backward scan (needed = arity_i; needed += a_j - 1) reaches zero; -1 if
// it never does.  With non-negative arities `needed` falls by at most one per step, so it can
// only reach zero at the start of a complete child: the scan is equivalent to hopping over
// arity_i child subtrees, start[i-1], start[start[i-1]-1], ..., which is O(arity) per token.
// Rows that contain a negative arity use the literal scan for the tokens after it.
template <typename Out>
__device__ __forceinline__ void subtree_ranges_row(const uint8_t* __restrict__ row, int64_t L,
                                                   bool vec4, const int32_t* __restrict__ ar,
                                                   int64_t n_ar, int64_t pad, Out* srow,
                                                   int64_t* __restrict__ out_len, int64_t b) {
  RowReader<uint8_t> rd{row, L, vec4};
  int64_t first_pad = -1;
  bool neg_seen = false;
  rd.for_each([&](int64_t i, int64_t t) {
    if (t == pad) {
      if (first_pad < 0) first_pad = i;
      srow[i] = (Out)-1;
      return true;
    }
    const int32_t a = arity_of(ar, n_ar, t);
    if (a < 0) neg_seen = true;
    int64_t s;
    if (a == 0) {
      s = i;
    } else if (!neg_seen) {
      s = i;
      for (int32_t k = 0; k < a; ++k) {
        if (s == 0) { s = -1; break; }
        s = (int64_t)srow[s - 1];
        if (s < 0) { s = -1; break; }
      }
    } else {
      // literal backward scan (rpn_kernels.cu:478-502)
      int64_t need = a;
      s = -1;
      for (int64_t j = i - 1; j >= 0; --j) {
        const int64_t tj = (int64_t)__ldg(row + j);
        if (tj == pad) break;
        need += (int64_t)arity_of(ar, n_ar, tj) - 1;
        if (need == 0) { s = j; break; }
      }
    }
    srow[i] = (Out)s;
    return true;
  });
  if (out_len != nullptr) out_len[b] = first_pad >= 0 ? first_pad : L;
}

// precompute_subtree_starts: forward subtree-length recurrence of simplify_kernels.cu:627-654
// (rows longer than 256 tokens keep -1 beyond position 255).  The subtree length of an earlier
// position is recovered from its start (length = j - start + 1; -1 stands for length 0).
template <typename Out>
__device__ __forceinline__ void subtree_starts_row(const int64_t* __restrict__ row, int64_t L,
                                                   const int32_t* __restrict__ ar, int64_t n_ar,
                                                   Out* srow) {
  const int64_t actual = L < 256 ? L : 256;
  auto len_at = [&](int64_t j) -> int64_t {
    const int64_t s = (int64_t)srow[j];
    return s < 0 ? 0 : j - s + 1;
  };
  for (int64_t j = 0; j < actual; ++j) {
    const int64_t t = (int64_t)__ldg(reinterpret_cast<const long long*>(row) + j);
    if (t == 0 || t < 0 || t >= n_ar) { srow[j] = (Out)-1; continue; }
    const int32_t a = __ldg(ar + t);
    int64_t len;
    if (a == 0) {
      len = 1;
    } else if (a == 1 && j >= 1) {
      len = 1 + len_at(j - 1);
    } else if (a == 2 && j >= 2) {
      const int64_t right = len_at(j - 1);
      const int64_t left_idx = j - 1 - right;
      len = 1 + right + (left_idx >= 0 ? len_at(left_idx) : 0);
    } else {
      len = 1;
    }
    srow[j] = (Out)(j - len + 1);
  }
  for (int64_t j = actual; j < L; ++j) srow[j] = (Out)-1;
}

struct SubtreeArgs {
  const void* pop;  // uint8 [B, L] (ranges) or int64 [B, L] (starts)
  int64_t B, L;
  const int32_t* ar;
  int64_t n_ar;
  int64_t pad;
  bool vec4;
  int64_t* out;
  int64_t* out_len;
  int sstride;  // shared-memory row stride in int32 (odd: conflict-free per-thread rows)
};

// KIND 0 = find_subtree_ranges, 1 = precompute_subtree_starts.
template <int KIND, bool STAGED>
__global__ void __launch_bounds__(kThreads) subtree_kernel(SubtreeArgs a) {
  extern __shared__ int32_t s_tile[];
  const int64_t n_tiles = (a.B + kThreads - 1) / kThreads;
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t b0 = tile * kThreads;
    const int64_t b = b0 + threadIdx.x;
    const int rows = (int)((a.B - b0) < kThreads ? (a.B - b0) : kThreads);
    if (b < a.B) {
      if (STAGED) {
        int32_t* srow = s_tile + (size_t)threadIdx.x * a.sstride;
        if (KIND == 0)
          subtree_ranges_row(static_cast<const uint8_t*>(a.pop) + b * a.L, a.L, a.vec4, a.ar,
                             a.n_ar, a.pad, srow, a.out_len, b);
        else
          subtree_starts_row(static_cast<const int64_t*>(a.pop) + b * a.L, a.L, a.ar, a.n_ar,
                             srow);
      } else {
        int64_t* orow = a.out + b * a.L;
        if (KIND == 0)
          subtree_ranges_row(static_cast<const uint8_t*>(a.pop) + b * a.L, a.L, a.vec4, a.ar,
                             a.n_ar, a.pad, orow, a.out_len, b);
        else
          subtree_starts_row(static_cast<const int64_t*>(a.pop) + b * a.L, a.L, a.ar, a.n_ar,
                             orow);
      }
    }
    if (STAGED) {
      __syncthreads();
      // Row-major write-out of the tile: consecutive threads store consecutive int64s.
      const int64_t n = (int64_t)rows * a.L;
      const int64_t step_r = kThreads / a.L, step_c = kThreads % a.L;
      int64_t r = threadIdx.x / a.L, c = threadIdx.x % a.L;
      int64_t* dst = a.out + b0 * a.L;
      for (int64_t f = threadIdx.x; f < n; f += kThreads) {
        dst[f] = (int64_t)s_tile[(size_t)r * a.sstride + c];
        r += step_r;
        c += step_c;
        if (c >= a.L) { c -= a.L; ++r; }
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Tournament selection (rpn_kernels.cu:1535-1668).  OFFSETS selects the island-offset variant:
// candidates are base + (offset % span), clamped into [0, B-1].
constexpr int kTourFast = 8;  // tournaments up to this size keep their candidates in registers

// State of one tournament: the incumbent, its value and (once read) its length.
struct TourState {
  const float* lengths;  // null: no parsimony tie-break
  float eps;             // tie epsilon, used only with lengths
  int64_t best = -1;
  float best_val = 0.0f;
  float best_len = 0.0f;
  bool best_len_known = false;
};

// Candidate `c` with value `val` challenges the incumbent with the reference's comparisons
// (rpn_kernels.cu:1603-1668): a strictly smaller value wins; otherwise, with lengths, a value
// within eps of the incumbent's is a tie, won by a strictly shorter program.  A candidate's
// length is only read on a tie (the incumbent's once, then the challenger's); the winner of a
// tie keeps its length known, a strict winner's length is read on a later tie.
__device__ __forceinline__ void tour_challenge(TourState& st, int64_t c, float val) {
  bool improve = val < st.best_val;
  float len = 0.0f;
  const bool tie = !improve && st.lengths != nullptr && fabsf(val - st.best_val) < st.eps;
  if (tie) {
    if (!st.best_len_known) st.best_len = st.lengths[st.best];
    st.best_len_known = true;
    len = st.lengths[c];
    improve = len < st.best_len;
  }
  if (improve) {
    st.best_val = val;
    st.best = c;
    st.best_len = len;
    st.best_len_known = tie;
  }
}

template <bool OFFSETS>
__global__ void __launch_bounds__(256)
    tournament_kernel(const float* __restrict__ fitness, const float* __restrict__ errors,
                      const int64_t* __restrict__ rand_idx, const int32_t* __restrict__ rand_off,
                      const int32_t* __restrict__ rand_cases, int64_t* __restrict__ selected,
                      const float* __restrict__ lengths, const float* __restrict__ mad_eps,
                      int64_t B, int64_t T, int64_t n_data, int island_size, int n_islands) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < B;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int base = 0, span = (int)B;
    if (OFFSETS && n_islands > 1) {
      span = island_size > 1 ? island_size : 1;
      base = (int)(idx / span) * span;
      span = span < (int)B - base ? span : (int)B - base;
      span = span > 1 ? span : 1;
    }
    auto candidate = [&](int64_t k) -> int64_t {
      if (!OFFSETS) return rand_idx[idx * T + k];
      int64_t c = (int64_t)(base + (rand_off[idx * T + k] % span));
      if (c < 0) c = 0;
      if (c >= B) c = B - 1;
      return c;
    };
    const int case_idx = rand_cases != nullptr ? rand_cases[idx] : -1;
    const bool by_case = case_idx >= 0 && errors != nullptr;
    // The tie epsilon is only read when lengths are given (as in the reference).
    float eps = 0.0f;
    if (lengths != nullptr)
      eps = (case_idx >= 0 && mad_eps != nullptr) ? mad_eps[case_idx]
                                                  : (case_idx >= 0 ? 1e-3f : 1e-9f);
    // A candidate's length only matters on a tie (|val - best_val| < eps), so lengths are read
    // there alone: the incumbent's once, then the challenger's.  The comparisons are the
    // reference's, in candidate order, so the winner is the same.
    TourState st;
    st.lengths = lengths;
    st.eps = eps;
    if (T <= kTourFast) {
      // all candidates, then all their values, then the comparisons in candidate order: two
      // rounds of memory latency per program instead of two per candidate
      int64_t cs[kTourFast];
      float vals[kTourFast];
      if (!OFFSETS && (T % 2) == 0 && (reinterpret_cast<uintptr_t>(rand_idx) & 15) == 0) {
        // even T on a 16-byte aligned base: every row of rand_idx starts on a 16-byte boundary
        const longlong2* row = reinterpret_cast<const longlong2*>(rand_idx + idx * T);
#pragma unroll
        for (int k = 0; k < kTourFast; k += 2) {
          if (k < T) {
            const longlong2 v = row[k / 2];
            cs[k] = v.x;
            cs[k + 1] = v.y;
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < kTourFast; ++k)
          if (k < T) cs[k] = candidate(k);
      }
#pragma unroll
      for (int k = 0; k < kTourFast; ++k)
        if (k < T) vals[k] = by_case ? errors[cs[k] * n_data + case_idx] : fitness[cs[k]];
      st.best = cs[0];
      st.best_val = vals[0];
#pragma unroll
      for (int k = 1; k < kTourFast; ++k) {
        if (k >= T) break;
        tour_challenge(st, cs[k], vals[k]);
      }
      selected[idx] = st.best;
      continue;
    }
    st.best = candidate(0);
    st.best_val = by_case ? errors[st.best * n_data + case_idx] : fitness[st.best];
    for (int64_t k = 1; k < T; ++k) {
      const int64_t c = candidate(k);
      tour_challenge(st, c, by_case ? errors[c * n_data + case_idx] : fitness[c]);
    }
    selected[idx] = st.best;
  }
}

int grid_for(int64_t units, int threads, int per_sm) {
  const int64_t want = (units + threads - 1) / threads;
  const int64_t cap = (int64_t)device_info().sm_count * per_sm;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

template <int KIND>
ws_status launch_subtree(SubtreeArgs a, cudaStream_t stream, const char* what) {
  if (a.B == 0 || a.L == 0) {
    if (a.B > 0 && a.out_len != nullptr) {
      cudaError_t e = cudaMemsetAsync(a.out_len, 0, (size_t)a.B * sizeof(int64_t), stream);
      if (e != cudaSuccess) return fail_cuda(e, what);
    }
    return WS_OK;
  }
  a.sstride = (int)((a.L % 2 == 0) ? a.L + 1 : a.L);
  const size_t smem = (size_t)kThreads * a.sstride * sizeof(int32_t);
  const bool staged = a.L <= 16384 && smem <= (size_t)kStagedMaxBytes &&
                      smem <= device_info().smem_optin;
  const int64_t n_tiles = (a.B + kThreads - 1) / kThreads;
  cudaError_t e;
  if (staged) {
    auto kern = subtree_kernel<KIND, true>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail_cuda(e, what);
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (e != cudaSuccess) return fail_cuda(e, what);
    if (per_sm < 1) per_sm = 1;
    const int64_t cap = (int64_t)device_info().sm_count * per_sm;
    const int grid = (int)(n_tiles < cap ? n_tiles : cap);
    kern<<<grid, kThreads, smem, stream>>>(a);
  } else {
    const int grid = grid_for(a.B, kThreads, 16);
    subtree_kernel<KIND, false><<<grid, kThreads, 0, stream>>>(a);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, what);
}

ws_status check_arity_table(const int32_t* ar, int64_t n_ar, bool clamped) {
  if (n_ar < 0) return fail("token_arities must have a non-negative length");
  if (n_ar > 0 && ar == nullptr) return fail("token_arities is NULL");
  if (clamped && n_ar == 0) return fail("token_arities must be non-empty");
  return WS_OK;
}

ws_status check_tournament(const float* fitness, int64_t B, const float* errors, int64_t n_data,
                           const void* cand, int64_t T, int64_t* selected) {
  if (B < 0) return fail("fitness must have a non-negative length");
  if (B > 0 && T < 1) return fail("tournament size must be at least 1");
  if (errors != nullptr && n_data < 1) return fail("errors must have at least one column");
  if (B > 0 && (fitness == nullptr || cand == nullptr || selected == nullptr))
    return fail("fitness, candidates and selected_idx must be device pointers");
  return WS_OK;
}

ws_status launch_tournament(const float* fitness, int64_t B, const float* errors, int64_t n_data,
                            const int64_t* rand_idx, const int32_t* rand_off, int64_t T,
                            const int32_t* rand_cases, const float* lengths, const float* mad_eps,
                            int island_size, int n_islands, int64_t* selected,
                            cudaStream_t stream) {
  if (B == 0) return WS_OK;
  // one program per thread: every program's gathers are in flight at once
  const int grid = grid_for(B, 256, 64);
  if (rand_off != nullptr)
    tournament_kernel<true><<<grid, 256, 0, stream>>>(fitness, errors, nullptr, rand_off,
                                                      rand_cases, selected, lengths, mad_eps, B, T,
                                                      n_data, island_size, n_islands);
  else
    tournament_kernel<false><<<grid, 256, 0, stream>>>(fitness, errors, rand_idx, nullptr,
                                                       rand_cases, selected, lengths, mad_eps, B,
                                                       T, n_data, island_size, n_islands);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "tournament_selection");
}

}  // namespace
}  // namespace ws

// ---------------------------------------------------------------------------------------------
// C ABI (include/warpsym.h).

extern "C" ws_status ws_validate_rpn_batch(const void* population, int32_t token_bytes,
                                           int64_t B, int64_t L, const int32_t* token_arities,
                                           int64_t n_arities, int32_t pad_id, int32_t mode,
                                           uint8_t* out_valid, void* stream) {
  using namespace ws;
  clear_error();
  NvtxRange nvtx("ws_validate_rpn_batch");
  if (B < 0 || L < 0) return fail("population must have non-negative shape");
  if (token_bytes != 1 && token_bytes != 8) return fail("token_bytes must be 1 or 8");
  if (mode < WS_VALIDATE_KERNEL || mode > WS_VALIDATE_STACK)
    return fail("validation mode must be WS_VALIDATE_KERNEL, _CLAMPED or _STACK");
  ws_status st = check_arity_table(token_arities, n_arities, mode != WS_VALIDATE_KERNEL);
  if (st != WS_OK) return st;
  if (B > 0 && (out_valid == nullptr || (L > 0 && population == nullptr)))
    return fail("population and out_valid must be device pointers");
  if (B == 0) return WS_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int grid = grid_for(B, kThreads, 16);
  if (token_bytes == 1) {
    const bool vec4 = (L % 4 == 0) && ((uintptr_t)population % 4 == 0);
    const bool vec16 = (L % 16 == 0) && ((uintptr_t)population % 16 == 0);
    validate_kernel<uint8_t><<<grid, kThreads, 0, s>>>(static_cast<const uint8_t*>(population),
                                                       B, L, token_arities, n_arities, pad_id,
                                                       mode, vec4, vec16, out_valid);
  } else {
    validate_kernel<int64_t><<<grid, kThreads, 0, s>>>(static_cast<const int64_t*>(population),
                                                       B, L, token_arities, n_arities, pad_id,
                                                       mode, false, false, out_valid);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "validate_rpn_batch");
}

extern "C" ws_status ws_find_subtree_ranges(const uint8_t* population, int64_t B, int64_t L,
                                            const int32_t* token_arities, int64_t n_arities,
                                            int32_t pad_id, int64_t* out_starts,
                                            int64_t* out_lengths, void* stream) {
  using namespace ws;
  clear_error();
  if (B < 0 || L < 0) return fail("population must have non-negative shape");
  ws_status st = check_arity_table(token_arities, n_arities, false);
  if (st != WS_OK) return st;
  if (B > 0 && L > 0 && (population == nullptr || out_starts == nullptr))
    return fail("population and out_starts must be device pointers");
  const bool vec4 = (L % 4 == 0) && ((uintptr_t)population % 4 == 0);
  SubtreeArgs a{population, B, L, token_arities, n_arities, pad_id, vec4, out_starts,
                out_lengths, 0};
  return launch_subtree<0>(a, static_cast<cudaStream_t>(stream), "find_subtree_ranges");
}

extern "C" ws_status ws_precompute_subtree_starts(const int64_t* population, int64_t B, int64_t L,
                                                  const int32_t* arities, int64_t n_arities,
                                                  int64_t* out_starts, void* stream) {
  using namespace ws;
  clear_error();
  if (B < 0 || L < 0) return fail("population must have non-negative shape");
  ws_status st = check_arity_table(arities, n_arities, false);
  if (st != WS_OK) return st;
  if (B > 0 && L > 0 && (population == nullptr || out_starts == nullptr))
    return fail("population and out_starts must be device pointers");
  SubtreeArgs a{population, B, L, arities, n_arities, 0, false, out_starts, nullptr, 0};
  return launch_subtree<1>(a, static_cast<cudaStream_t>(stream), "precompute_subtree_starts");
}

extern "C" ws_status ws_tournament_select(const float* fitness, int64_t B, const float* errors,
                                          int64_t n_data, const int64_t* rand_idx,
                                          int64_t tour_size, const int32_t* rand_cases,
                                          const float* lengths, const float* mad_eps,
                                          int64_t* selected_idx, void* stream) {
  using namespace ws;
  clear_error();
  ws_status st = check_tournament(fitness, B, errors, n_data, rand_idx, tour_size, selected_idx);
  if (st != WS_OK) return st;
  return launch_tournament(fitness, B, errors, n_data, rand_idx, nullptr, tour_size, rand_cases,
                           lengths, mad_eps, 0, 1, selected_idx,
                           static_cast<cudaStream_t>(stream));
}

extern "C" ws_status ws_tournament_select_offsets(const float* fitness, int64_t B,
                                                  const float* errors, int64_t n_data,
                                                  const int32_t* rand_offsets, int64_t tour_size,
                                                  const int32_t* rand_cases, const float* lengths,
                                                  const float* mad_eps, int32_t island_size,
                                                  int32_t n_islands, int64_t* selected_idx,
                                                  void* stream) {
  using namespace ws;
  clear_error();
  ws_status st =
      check_tournament(fitness, B, errors, n_data, rand_offsets, tour_size, selected_idx);
  if (st != WS_OK) return st;
  if (B > INT32_MAX) return fail("island tournament supports at most 2^31-1 programs");
  return launch_tournament(fitness, B, errors, n_data, nullptr, rand_offsets, tour_size,
                           rand_cases, lengths, mad_eps, island_size, n_islands, selected_idx,
                           static_cast<cudaStream_t>(stream));
}
