// ws_fitness.cu -- batched RPN evaluation fused with the per-program loss (the hot path).
//
// Replaces rpn_eval_fused_kernel (rpn_kernels.cu:2259-2502) and the classic chunked path of
// GPUEvaluator.evaluate_batch (rpn_eval_kernel + torch reductions, evaluation.py:128-198) with
// one pipeline that has neither the fused envelope (<=4 variables, D<=1024) nor the classic
// path's [B, D] materialisation:
//
//   1. compile_kernel  -- one thread per program: tokens -> accumulator-machine tape
//                         (ws_compile.cuh), constant slots baked, constants folded.
//   2. fitness_kernel  -- persistent CTAs pull work items (a block of PB programs x a range of
//                         row chunks).  Per chunk the CTA stages X[:, rows] and y[rows] in shared
//                         memory once; its warps then take programs of the block one at a time
//                         and run the program's tape over the chunk in passes of 32*R rows
//                         (R rows per lane, 16-byte shared loads, conflict-free), accumulating
//                         squared errors in FP64.  Per-program partials are combined in a fixed
//                         order, so results do not depend on the schedule or on what else is in
//                         the batch (up to FP64 rounding of the sum).
//
// Per-row values are bit-identical to the reference kernels when this file is compiled with
// the reference's flags (--use_fast_math): same operator code (ws_ops.cuh), same FP32 rounding
// of pred - y and of its square.  Only the order of the sum differs (FP64 here, FP32 warp
// butterflies in the reference).
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cfloat>
#include <mutex>
#include <map>
#include <tuple>

#include "ws_internal.h"
#include "ws_compile.cuh"

namespace ws {

struct alignas(16) PartRec {
  double sse;
  int32_t ninv;
  int32_t ovf;
};

// ---------------------------------------------------------------------------------------
// 1. compile
template <typename T, bool STRICT, int LMAX>
__global__ void __launch_bounds__(128) compile_kernel(const uint8_t* __restrict__ pop, int64_t B,
                                                      int L, const T* __restrict__ consts, int K,
                                                      TokenLut lut, Instr<T>* __restrict__ tape,
                                                      int Lcap, ProgHdr* __restrict__ hdr,
                                                      unsigned* __restrict__ prog_cnt,
                                                      unsigned* __restrict__ misc, int S) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) misc[0] = 0u;  // work-queue head of the evaluator launch that follows
  if (p >= B) return;
  ProgHdr h = compile_program<T, STRICT, true, LMAX>(pop + p * (int64_t)L, L,
                                                      K > 0 ? consts + p * (int64_t)K : nullptr,
                                                      K, lut, tape + p * (int64_t)Lcap);
  if (h.status == PROG_OK && h.n_slots > S) {  // cannot happen (Sethi-Ullman bound); guard
    h.status = PROG_INVALID;
    atomicAdd(&misc[1], 1u);
  }
  hdr[p] = h;
  prog_cnt[p] = 0u;
}

// FP64 variance of y (population variance, same rows as the loss) for WS_LOSS_R2.
template <typename T>
__global__ void __launch_bounds__(256) yvar_kernel(const T* __restrict__ y, int64_t D,
                                                   double* __restrict__ out) {
  __shared__ double s1[256], s2[256];
  double a = 0.0, b = 0.0;
  for (int64_t i = threadIdx.x; i < D; i += blockDim.x) {
    const double v = (double)y[i];
    a += v;
    b += v * v;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double m = s1[0] / (double)D;
    double v = s2[0] / (double)D - m * m;
    out[0] = v > 0.0 ? v : 0.0;
  }
}

// ---------------------------------------------------------------------------------------
// 2. evaluate
template <typename T>
struct FitParams {
  const Instr<T>* tape;
  const ProgHdr* hdr;
  int Lcap;
  const T* x;
  const T* y;
  int V;
  int64_t D;
  int64_t B;
  int RC;            // rows per chunk (multiple of 32*R)
  int64_t n_chunks;
  int PB;            // programs per block
  int64_t n_blocks;
  int n_splits;      // chunk ranges per block
  int64_t cps;       // chunks per split
  int64_t n_items;
  int S;             // spill slots per warp
  int policy, loss;
  double invalid_value;
  void* out_loss;
  int32_t* out_ninv;
  PartRec* part;
  unsigned* prog_cnt;
  unsigned* work;
  const double* yvar;
};

template <typename T> struct Vec16;
template <> struct Vec16<float> {
  static constexpr int N = 4;
  __device__ static void load(float* d, const float* s) {
    const float4 t = *reinterpret_cast<const float4*>(s);
    d[0] = t.x; d[1] = t.y; d[2] = t.z; d[3] = t.w;
  }
  __device__ static void store(float* s, const float* d) {
    *reinterpret_cast<float4*>(s) = make_float4(d[0], d[1], d[2], d[3]);
  }
};
template <> struct Vec16<double> {
  static constexpr int N = 2;
  __device__ static void load(double* d, const double* s) {
    const double2 t = *reinterpret_cast<const double2*>(s);
    d[0] = t.x; d[1] = t.y;
  }
  __device__ static void store(double* s, const double* d) {
    *reinterpret_cast<double2*>(s) = make_double2(d[0], d[1]);
  }
};

// Loads R values of one lane: group g holds rows g*32N + lane*N + [0,N) of the pass.
template <typename T, int R>
__device__ __forceinline__ void lane_load(T (&d)[R], const T* s) {
  constexpr int N = Vec16<T>::N;
#pragma unroll
  for (int g = 0; g < R / N; ++g) Vec16<T>::load(&d[g * N], s + g * 32 * N);
}
template <typename T, int R>
__device__ __forceinline__ void lane_store(T* s, const T (&d)[R]) {
  constexpr int N = Vec16<T>::N;
#pragma unroll
  for (int g = 0; g < R / N; ++g) Vec16<T>::store(s + g * 32 * N, &d[g * N]);
}

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Runs one program tape over one pass of 32*R rows.  xp: X tile at this pass and lane
// (variable v at xp + v*RC); sp: this warp's spill slots at this lane.
template <typename T, int R, bool STRICT>
__device__ __forceinline__ void run_tape(const Instr<T>* __restrict__ tp, int n,
                                         const T* __restrict__ xp, int RC, T* __restrict__ sp,
                                         T (&acc)[R], uint32_t& err) {
  constexpr int SLOT = 32 * R;
  err = 0u;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const Instr<T> ins = tp[i];
    const uint32_t c = ins.ctrl;
    if (c & F_SPILL) lane_store<T, R>(sp + ((c >> SH_SLOT) & 31u) * SLOT, acc);
    const uint32_t la = (c >> SH_LA) & 3u;
    if (la == LA_X) {
      lane_load<T, R>(acc, xp + ((c >> SH_LA_IDX) & 63u) * RC);
    } else if (la != LA_NONE) {  // immediate (parameters are not used by the baked tape)
#pragma unroll
      for (int k = 0; k < R; ++k) acc[k] = ins.imm;
    }
    const uint32_t ok = (c >> SH_OPK) & 3u;
    const uint32_t oi = (c >> SH_OP_IDX) & 63u;
    T v[R];
    T s = ins.imm;
    if (ok == OK_X) lane_load<T, R>(v, xp + oi * RC);
    else if (ok == OK_SLOT) lane_load<T, R>(v, sp + oi * SLOT);

#define WS_ROWS(BODY) _Pragma("unroll") for (int k = 0; k < R; ++k) { BODY; } break
#define WS_ERR(EXPR) { bool e_ = false; acc[k] = (EXPR); err |= (uint32_t)e_ << k; }
#define WS_BIN4(CLS, F)                                                                  \
  case CASE_BIN + 4 * (CLS - T_ADD) + FORM_AV: WS_ROWS(F(acc[k], v[k]));                \
  case CASE_BIN + 4 * (CLS - T_ADD) + FORM_VA: WS_ROWS(F(v[k], acc[k]));                \
  case CASE_BIN + 4 * (CLS - T_ADD) + FORM_AS: WS_ROWS(F(acc[k], s));                   \
  case CASE_BIN + 4 * (CLS - T_ADD) + FORM_SA: WS_ROWS(F(s, acc[k]));
#define F_ADD(a, b) acc[k] = (a) + (b)
#define F_SUB(a, b) acc[k] = (a) - (b)
#define F_MUL(a, b) acc[k] = (a) * (b)
#define F_DIV(a, b) WS_ERR((op_div<T, STRICT>((a), (b), e_)))
#define F_POW(a, b) WS_ERR((op_pow<T, STRICT>((a), (b), e_)))
#define F_MOD(a, b) WS_ERR((op_mod<T, STRICT>((a), (b), e_)))
    switch (c & CASE_MASK) {
      case CASE_NOP: break;
      WS_BIN4(T_ADD, F_ADD)
      WS_BIN4(T_SUB, F_SUB)
      WS_BIN4(T_MUL, F_MUL)
      WS_BIN4(T_DIV, F_DIV)
      WS_BIN4(T_POW, F_POW)
      WS_BIN4(T_MOD, F_MOD)
      case T_SIN: WS_ROWS(acc[k] = m_sin(acc[k]));
      case T_COS: WS_ROWS(acc[k] = m_cos(acc[k]));
      case T_TAN: WS_ROWS(acc[k] = m_tan(acc[k]));
      case T_LOG: WS_ROWS(WS_ERR((op_log<T, STRICT>(acc[k], e_))));
      case T_EXP: WS_ROWS(WS_ERR((op_exp<T, STRICT>(acc[k], e_))));
      case T_SQRT: WS_ROWS(WS_ERR((op_sqrt<T, STRICT>(acc[k], e_))));
      case T_ABS: WS_ROWS(acc[k] = m_abs(acc[k]));
      case T_NEG: WS_ROWS(acc[k] = -acc[k]);
      case T_FACT: WS_ROWS(WS_ERR((op_tgamma<T, STRICT>(acc[k] + (T)1.0, e_))));
      case T_FLOOR: WS_ROWS(acc[k] = m_floor(acc[k]));
      case T_CEIL: WS_ROWS(acc[k] = m_ceil(acc[k]));
      case T_SIGN: WS_ROWS(acc[k] = op_sign<T>(acc[k]));
      case T_GAMMA: WS_ROWS(WS_ERR((op_tgamma<T, STRICT>(acc[k], e_))));
      case T_LGAMMA: WS_ROWS(WS_ERR((op_lgamma<T, STRICT>(acc[k], e_))));
      case T_ASIN: WS_ROWS(WS_ERR((op_asin<T, STRICT>(acc[k], e_))));
      case T_ACOS: WS_ROWS(WS_ERR((op_acos<T, STRICT>(acc[k], e_))));
      case T_ATAN: WS_ROWS(acc[k] = m_atan(acc[k]));
      default: err = 0xFFFFFFFFu; break;  // malformed tape: every row invalid
    }
#undef F_ADD
#undef F_SUB
#undef F_MUL
#undef F_DIV
#undef F_POW
#undef F_MOD
#undef WS_BIN4
#undef WS_ERR
#undef WS_ROWS
  }
}

// Final loss of one program from its combined record.  Classification mirrors the
// reference epilogues:
//   WS_POLICY_FUSED (rpn_kernels.cu:2487-2497): invalid row -> iv; per-row metric overflow ->
//     sqrt(iv); non-finite mean (sum overflow) -> iv.
//   WS_POLICY_CLASSIC (evaluation.py:182-189): invalid row -> iv; non-finite mean -> sqrt(iv).
// An FP64 sum above the T range stands for the overflow of the reference's T accumulator.
// MSE uses the same classification (any overflow -> iv); R2 writes -iv for both.
template <typename T>
__device__ void write_final(const FitParams<T>& P, int64_t p, const PartRec& r) {
  if (P.out_ninv) P.out_ninv[p] = r.ninv;
  const double tmax = (double)(sizeof(T) == 4 ? FLT_MAX : DBL_MAX);
  if (P.loss == WS_LOSS_SSE) {
    ((double*)P.out_loss)[p] = (r.ninv > 0) ? P.invalid_value : r.sse;
    return;
  }
  const bool fused = P.policy == WS_POLICY_FUSED;
  const bool invalid = r.ninv > 0;
  const bool sum_ovf = !(r.sse <= tmax);
  const bool row_ovf = fused && r.ovf;
  const T iv = (T)P.invalid_value;
  double out;
  if (invalid) {
    out = (P.loss == WS_LOSS_R2) ? -P.invalid_value : P.invalid_value;
  } else if (row_ovf || sum_ovf) {
    if (P.loss == WS_LOSS_RMSE) out = (fused && !row_ovf) ? (double)iv : (double)m_sqrt(iv);
    else out = (P.loss == WS_LOSS_MSE) ? P.invalid_value : -P.invalid_value;
  } else {
    const double mse = r.sse / (double)P.D;
    const T mse_t = (T)mse;
    if (P.loss == WS_LOSS_RMSE) {
      const T q = m_sqrt(mse_t);
      out = (m_isnan(q) || m_isinf(q)) ? P.invalid_value : (double)q;
    } else if (P.loss == WS_LOSS_MSE) {
      out = (double)mse_t;
    } else {
      const double vy = *P.yvar;
      out = vy > 0.0 ? 1.0 - mse / vy : (mse == 0.0 ? 1.0 : -P.invalid_value);
    }
  }
  if (sizeof(T) == 4) ((float*)P.out_loss)[p] = (float)out;
  else ((double*)P.out_loss)[p] = out;
}

template <typename T, int R, bool STRICT>
__global__ void __launch_bounds__(256) fitness_kernel(const FitParams<T> P) {
  constexpr int N = Vec16<T>::N;
  constexpr int PASS = 32 * R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* xs = reinterpret_cast<T*>(smem_raw);
  T* ys = xs + (size_t)P.V * P.RC;
  T* spill = ys + P.RC;
  Instr<T>* tapes = reinterpret_cast<Instr<T>*>(spill + (size_t)W * P.S * PASS);
  PartRec* acc_s = reinterpret_cast<PartRec*>(tapes + (size_t)W * P.Lcap);
  __shared__ int64_t s_item;
  __shared__ int s_next;

  T* sp_w = spill + (size_t)warp * P.S * PASS + lane * N;
  Instr<T>* tape_w = tapes + (size_t)warp * P.Lcap;
  const bool fused_policy = P.policy == WS_POLICY_FUSED;

  for (;;) {
    if (threadIdx.x == 0) s_item = (int64_t)atomicAdd(P.work, 1u);
    __syncthreads();
    const int64_t item = s_item;
    if (item >= P.n_items) break;
    const int64_t blk = item / P.n_splits;
    const int split = (int)(item % P.n_splits);
    const int64_t p0 = blk * P.PB;
    const int np = (int)min((int64_t)P.PB, P.B - p0);
    const int64_t c0 = (int64_t)split * P.cps;
    const int64_t c1 = min(P.n_chunks, c0 + P.cps);
    for (int q = threadIdx.x; q < np; q += blockDim.x) acc_s[q] = PartRec{0.0, 0, 0};

    for (int64_t c = c0; c < c1; ++c) {
      __syncthreads();  // previous chunk fully consumed; accumulators initialised
      const int64_t row0 = c * P.RC;
      const int rows = (int)min((int64_t)P.RC, P.D - row0);
      for (int v = 0; v < P.V; ++v) {
        const T* src = P.x + (size_t)v * P.D + row0;
        T* dst = xs + (size_t)v * P.RC;
        for (int r = threadIdx.x; r < P.RC; r += blockDim.x) dst[r] = (r < rows) ? src[r] : (T)0;
      }
      for (int r = threadIdx.x; r < P.RC; r += blockDim.x) ys[r] = (r < rows) ? P.y[row0 + r] : (T)0;
      if (threadIdx.x == 0) s_next = 0;
      __syncthreads();
      const int npass = (rows + PASS - 1) / PASS;

      for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(&s_next, 1);
        q = __shfl_sync(0xFFFFFFFFu, q, 0);
        if (q >= np) break;
        const int64_t p = p0 + q;
        const ProgHdr h = P.hdr[p];
        if (h.status != PROG_OK) {
          if (lane == 0) acc_s[q].ninv += rows;
          continue;
        }
        const Instr<T>* tg = P.tape + p * (int64_t)P.Lcap;
        for (int i = lane; i < h.n_instr; i += 32) tape_w[i] = tg[i];
        __syncwarp();
        double sse = 0.0;
        int ninv = 0;
        bool ovf = false;
        for (int pass = 0; pass < npass; ++pass) {
          T a[R];
          uint32_t err;
          const T* xp = xs + pass * PASS + lane * N;
          run_tape<T, R, STRICT>(tape_w, h.n_instr, xp, P.RC, sp_w, a, err);
          T yv[R];
          lane_load<T, R>(yv, ys + pass * PASS + lane * N);
#pragma unroll
          for (int k = 0; k < R; ++k) {
            const int row = pass * PASS + (k / N) * 32 * N + lane * N + (k % N);
            if (row < rows) {
              const T pv = a[k];
              if (((err >> k) & 1u) || m_isnan(pv) || m_isinf(pv)) {
                ninv++;
              } else {
                const T diff = pv - yv[k];
                if (fused_policy) {
                  const T ad = diff < (T)0 ? -diff : diff;
                  bool o = m_isnan(diff) || m_isinf(diff) || ad > Limits<T>::max_diff;
                  const T sq = o ? (T)0 : mul_rn(diff, diff);
                  o = o || m_isnan(sq) || m_isinf(sq);
                  if (o) ovf = true;
                  else sse += (double)sq;
                } else {
                  sse += (double)mul_rn(diff, diff);
                }
              }
            }
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          sse += __shfl_xor_sync(0xFFFFFFFFu, sse, o);
          ninv += __shfl_xor_sync(0xFFFFFFFFu, ninv, o);
        }
        const bool any_ovf = __any_sync(0xFFFFFFFFu, ovf);
        if (lane == 0) {
          acc_s[q].sse += sse;
          acc_s[q].ninv += ninv;
          acc_s[q].ovf |= any_ovf ? 1 : 0;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
      const int64_t p = p0 + q;
      const PartRec r = acc_s[q];
      if (P.n_splits == 1) {
        write_final<T>(P, p, r);
      } else {
        P.part[p * P.n_splits + split] = r;
        __threadfence();
        const unsigned done = atomicAdd(&P.prog_cnt[p], 1u);
        if (done == (unsigned)P.n_splits - 1u) {
          __threadfence();
          PartRec t{0.0, 0, 0};
          for (int s2 = 0; s2 < P.n_splits; ++s2) {
            const PartRec* pr = &P.part[p * P.n_splits + s2];
            t.sse += __ldcg(&pr->sse);
            t.ninv += __ldcg(&pr->ninv);
            t.ovf |= __ldcg(&pr->ovf);
          }
          write_final<T>(P, p, t);
          P.prog_cnt[p] = 0u;  // ready for an evaluate-only rerun on the same tape
        }
      }
    }
    // the next item's accumulator reset waits on the __syncthreads() at the loop top
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// host side
namespace {

constexpr int kR = 8;       // rows per lane per pass
constexpr int kW = 8;       // warps per CTA
constexpr int kPBMax = 64;  // programs per block (upper bound)
constexpr size_t kSmemBudget = 72 * 1024;

// Largest dynamic shared memory the kernel may request (opt-in limit minus its static shared
// memory); the attribute is raised to it once per device.
template <typename T, int R, bool STRICT>
size_t max_dynamic_smem() {
  static std::mutex mu;
  static size_t cache[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> g(mu);
  if (cache[dev] == 0) {
    cudaFuncAttributes fa;
    size_t stat = 0;
    if (cudaFuncGetAttributes(&fa, fitness_kernel<T, R, STRICT>) == cudaSuccess)
      stat = fa.sharedSizeBytes;
    size_t lim = device_info().smem_optin > stat ? device_info().smem_optin - stat : 0;
    if (cudaFuncSetAttribute(fitness_kernel<T, R, STRICT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim) != cudaSuccess) {
      (void)cudaGetLastError();  // clear our own failed attribute call; fall back to 48 KB
      lim = 48 * 1024 - stat;
    }
    cache[dev] = lim;
  }
  return cache[dev];
}

template <typename T, int R, bool STRICT>
int occupancy_for(size_t smem, int threads) {
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > max_dynamic_smem<T, R, STRICT>()) return 0;
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(dev, smem);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fitness_kernel<T, R, STRICT>, threads,
                                                    smem) != cudaSuccess) {
    (void)cudaGetLastError();
    occ = 0;
  }
  cache[key] = occ;
  return occ;
}

template <typename T, bool STRICT>
ws_status launch_typed(const FitnessRequest& rq) {
  const FitnessWorkspace lay = fitness_workspace_layout(rq.B, rq.L, rq.dtype);
  unsigned char* wsb = static_cast<unsigned char*>(rq.workspace);
  ProgHdr* hdr = reinterpret_cast<ProgHdr*>(wsb + lay.hdr_off);
  Instr<T>* tape = reinterpret_cast<Instr<T>*>(wsb + lay.tape_off);
  PartRec* part = reinterpret_cast<PartRec*>(wsb + lay.part_off);
  unsigned* cnt = reinterpret_cast<unsigned*>(wsb + lay.cnt_off);
  unsigned* misc = reinterpret_cast<unsigned*>(wsb + lay.misc_off);
  double* yvar = reinterpret_cast<double*>(wsb + lay.misc_off + 16);

  const int L = (int)rq.L;
  const int Lcap = L > 1 ? L : 1;
  const int S = spill_slots_bound(L);
  const T* consts = static_cast<const T*>(rq.consts);

  // 1. compile
  if (rq.phase != WS_PHASE_EVALUATE) {
    const int threads = 128;
    const unsigned grid = (unsigned)((rq.B + threads - 1) / threads);
    if (L <= 64)
      compile_kernel<T, STRICT, 64><<<grid, threads, 0, rq.stream>>>(
          rq.pop, rq.B, L, consts, (int)rq.K, rq.lut, tape, Lcap, hdr, cnt, misc, S);
    else
      compile_kernel<T, STRICT, 256><<<grid, threads, 0, rq.stream>>>(
          rq.pop, rq.B, L, consts, (int)rq.K, rq.lut, tape, Lcap, hdr, cnt, misc, S);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "compile_kernel launch");
  }
  if (rq.phase == WS_PHASE_COMPILE) return WS_OK;
  if (rq.phase == WS_PHASE_EVALUATE) {  // the compile kernel is what resets the queue head
    cudaError_t e = cudaMemsetAsync(misc, 0, 16, rq.stream);
    if (e != cudaSuccess) return fail_cuda(e, "work-queue reset");
  }
  if (rq.loss == WS_LOSS_R2) {
    yvar_kernel<T><<<1, 256, 0, rq.stream>>>(static_cast<const T*>(rq.y), rq.D, yvar);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "yvar_kernel launch");
  }

  // 2. schedule
  constexpr int R = kR;
  constexpr int PASS = 32 * R;
  const int W = kW;
  const int threads = W * 32;
  const size_t szT = sizeof(T);
  const size_t fixed = (size_t)W * S * PASS * szT + (size_t)W * Lcap * sizeof(Instr<T>) +
                       (size_t)kPBMax * sizeof(PartRec);
  const size_t per_row = (size_t)(rq.V + 1) * szT;
  const int64_t d_pad = (rq.D + PASS - 1) / PASS * PASS;
  int64_t rc_cap = kSmemBudget > fixed + per_row * PASS
                       ? (int64_t)((kSmemBudget - fixed) / per_row) / PASS * PASS
                       : PASS;
  const size_t optin = max_dynamic_smem<T, R, STRICT>();
  if (fixed + per_row * PASS > optin) return fail("too many variables for the shared-memory tile");
  int RC = (int)(d_pad < rc_cap ? d_pad : rc_cap);
  if (RC < PASS) RC = PASS;
  size_t smem = fixed + per_row * (size_t)RC;
  const int occ = occupancy_for<T, R, STRICT>(smem, threads);
  if (occ <= 0) return fail("fitness kernel cannot be resident with this tile size");
  const int64_t n_ctas = (int64_t)occ * device_info().sm_count;

  const int64_t n_chunks = (rq.D + RC - 1) / RC;
  int PB = kPBMax;
  int64_t n_blocks = (rq.B + PB - 1) / PB;
  while (PB > W && n_blocks * n_chunks < 2 * n_ctas) {
    PB >>= 1;
    n_blocks = (rq.B + PB - 1) / PB;
  }
  int64_t n_splits = 1;
  if (n_blocks < 2 * n_ctas) {
    n_splits = (2 * n_ctas + n_blocks - 1) / n_blocks;
    if (n_splits > n_chunks) n_splits = n_chunks;
    const int64_t cap = lay.max_partials / (rq.B > 0 ? rq.B : 1);
    if (n_splits > cap) n_splits = cap > 0 ? cap : 1;
  }
  const int64_t cps = (n_chunks + n_splits - 1) / n_splits;
  n_splits = (n_chunks + cps - 1) / cps;

  FitParams<T> P;
  P.tape = tape;
  P.hdr = hdr;
  P.Lcap = Lcap;
  P.x = static_cast<const T*>(rq.x);
  P.y = static_cast<const T*>(rq.y);
  P.V = (int)rq.V;
  P.D = rq.D;
  P.B = rq.B;
  P.RC = RC;
  P.n_chunks = n_chunks;
  P.PB = PB;
  P.n_blocks = n_blocks;
  P.n_splits = (int)n_splits;
  P.cps = cps;
  P.n_items = n_blocks * n_splits;
  P.S = S;
  P.policy = rq.policy;
  P.loss = rq.loss;
  P.invalid_value = rq.invalid_value;
  P.out_loss = rq.out_loss;
  P.out_ninv = rq.out_ninv;
  P.part = part;
  P.prog_cnt = cnt;
  P.work = misc;
  P.yvar = yvar;
  const int64_t grid = P.n_items < n_ctas ? P.n_items : n_ctas;
  fitness_kernel<T, R, STRICT><<<(unsigned)grid, threads, smem, rq.stream>>>(P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "fitness_kernel launch");
  return WS_OK;
}

}  // namespace

FitnessWorkspace fitness_workspace_layout(int64_t B, int64_t L, int dtype) {
  FitnessWorkspace w;
  const size_t instr = dtype == WS_F64 ? sizeof(Instr<double>) : sizeof(Instr<float>);
  const int64_t Lcap = L > 1 ? L : 1;
  size_t off = 0;
  w.hdr_off = off;
  off = align_up(off + (size_t)B * sizeof(ProgHdr), 256);
  w.tape_off = off;
  off = align_up(off + (size_t)B * Lcap * instr, 256);
  w.max_partials = B > 65536 ? B : 65536;
  w.part_off = off;
  off = align_up(off + (size_t)w.max_partials * sizeof(PartRec), 256);
  w.cnt_off = off;
  off = align_up(off + (size_t)B * sizeof(unsigned), 256);
  w.misc_off = off;
  off = align_up(off + 256, 256);
  w.total = off;
  return w;
}

ws_status launch_fitness(const FitnessRequest& rq) {
  if (rq.dtype == WS_F32)
    return rq.strict ? launch_typed<float, true>(rq) : launch_typed<float, false>(rq);
  return rq.strict ? launch_typed<double, true>(rq) : launch_typed<double, false>(rq);
}

}  // namespace ws
