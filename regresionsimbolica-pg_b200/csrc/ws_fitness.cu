// ws_fitness.cu -- batched RPN evaluation fused with the per-program loss (the hot path).
//
// Replaces rpn_eval_fused_kernel (rpn_kernels.cu:2259-2502) and the classic chunked path of
// GPUEvaluator.evaluate_batch (rpn_eval_kernel + torch reductions, evaluation.py:128-198) with
// one pipeline that has neither the fused envelope (<=4 variables, D<=1024) nor the classic
// path's [B, D] materialisation:
//
//   1. compile_kernel  -- one thread per program: tokens -> accumulator-machine tape
//                         (ws_compile.cuh), constant slots baked, constants folded; programs
//                         are taken in token-count order (count_kernel + a counting sort), so
//                         a warp's threads parse programs of similar length.
//   2. sort_*_kernel   -- counting sort of the programs by tape length (longest first).
//   3. fitness_kernel  -- persistent CTAs pull work items (a block of PB length-sorted programs
//                         x a range of row chunks).  The block's tapes are staged in shared memory
//                         once; X[:, rows] and y[rows] of each chunk stream into a second shared
//                         tile (cp.async) while the current one is evaluated.  Warp w runs programs
//                         w, w+W, ... of the block (balanced: similar lengths) over the chunk in
//                         passes of 32*R rows (R rows per lane, 16-byte conflict-free shared
//                         loads), accumulating squared errors in FP64 per lane.  Per-lane
//                         partials live in shared memory across chunks and are combined once per
//                         block in a fixed order, so results do not depend on the schedule or on
//                         what else is in the batch (up to FP64 rounding of the sum).
//                         Programs whose spill slots all fit in shared memory (all but ~0.2% of
//                         random 64-token programs) run an FP32 interpreter that addresses its
//                         operands, spill slots and tape words as 32-bit shared addresses.
//
// Per-row values are bit-identical to the reference kernels when this file is compiled with
// the reference's flags (--use_fast_math): same operator code (ws_ops.cuh), same FP32 rounding
// of pred - y and of its square.  Only the order of the sum differs: each lane sums the R
// squared errors of a pass in T (two interleaved partial sums for FP32), passes and lanes are
// combined in FP64 (the reference sums in FP32 warp butterflies).
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cfloat>
#include <mutex>
#include <map>
#include <tuple>
#include <algorithm>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "ws_internal.h"
#include "ws_compile.cuh"

namespace ws {

struct alignas(16) PartRec {
  double sse;
  int32_t ninv;
  int32_t ovf;
};
// per-program per-lane partial sums: row stride of 33 doubles (conflict-free column reads)
constexpr int kLaneStride = 33;
// shared meta word of a staged program: tape length, and a flag for global spill slots
constexpr int kMetaLenMask = 0xFFFF;
constexpr int kMetaGlobalSpill = 1 << 16;

// ---------------------------------------------------------------------------------------
// Problem descriptors.  One launch evaluates the programs of one or many problems (each with
// its own population, constants, data set, token map and outputs).  The programs of all
// problems form one index space [0, sum of B): problem p owns [prog0, prog0 + B); its work
// items (blocks of PB programs x ranges of row chunks) are [item0, item0 + n_blocks * n_splits).
template <typename T>
struct ProbDesc {
  const uint8_t* pop;   // [B, L]
  const T* consts;      // [B, K] or null
  const T* x;           // [V, D]
  const T* y;           // [D]
  void* out_loss;       // [B]
  int32_t* out_ninv;    // [B] or null
  int64_t B, D, prog0, item0, n_chunks, cps, part0;
  int V, K, RC, xmul, n_splits, count, async_stage;
  int single;  // 1: one staging tile spanning both buffers (many variables), no prefetch
};

// Index of the problem whose range [start, next start) holds `i` (starts ascending, n >= 1).
template <typename T>
__device__ __forceinline__ int find_problem(const ProbDesc<T>* __restrict__ d, int n, int64_t i,
                                            bool by_item) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int64_t st = by_item ? d[mid].item0 : d[mid].prog0;
    if (st <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ---------------------------------------------------------------------------------------
// 1. compile (one thread per program of any problem)
// Pre-pass of the compile: a program's token count before its first PAD as the sort key (in
// hdr[g].n_instr, status OK) and its problem.  Compiling in that order puts programs of similar
// length in a warp, so its threads run their parse and emit loops for similar trip counts.
template <typename T>
__global__ void __launch_bounds__(256) count_kernel(const ProbDesc<T>* __restrict__ desc,
                                                   int n_prob, const TokenLut* __restrict__ luts,
                                                   int64_t total_B, int L,
                                                   ProgHdr* __restrict__ hdr,
                                                   int32_t* __restrict__ prob_of) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total_B;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int pi = find_problem(desc, n_prob, g, false);
    const ProbDesc<T>& d = desc[pi];
    const uint8_t* row = d.pop + (g - d.prog0) * (int64_t)L;
    const uint8_t* cls = luts[pi].cls;
    int n = 0;
    while (n < L && cls[row[n]] != T_PAD) ++n;
    ProgHdr h;
    h.n_instr = n;
    h.status = PROG_OK;
    h.n_slots = 0;
    h.n_tok = n;
    hdr[g] = h;
    prob_of[g] = pi;
  }
}

// One thread per program, programs taken in `perm` order (by token count): tokens ->
// accumulator-machine tape and header.
template <typename T, bool STRICT, int LMAX>
__global__ void __launch_bounds__(128) compile_kernel(
    const ProbDesc<T>* __restrict__ desc, const TokenLut* __restrict__ luts, int64_t total_B,
    int L, Instr<T>* __restrict__ tape, int Lcap, ProgHdr* __restrict__ hdr,
    const int32_t* __restrict__ prob_of, const int64_t* __restrict__ perm,
    unsigned* __restrict__ prog_cnt, unsigned* __restrict__ misc, int S) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) misc[0] = 0u;  // work-queue head of the evaluator launch that follows
  if (i >= total_B) return;
  const int64_t g = perm[i];
  const int pi = prob_of[g];
  const ProbDesc<T>& d = desc[pi];
  const int64_t p = g - d.prog0;
  ProgHdr h = compile_program_v2<T, STRICT, true, LMAX>(
      d.pop + p * (int64_t)L, L, d.K > 0 ? d.consts + p * (int64_t)d.K : nullptr, d.K, luts[pi],
      tape + g * (int64_t)Lcap, d.xmul);
  // Neither can happen (Sethi-Ullman bound; chunk size chosen for the offsets): guard anyway.
  if ((h.status == PROG_OK && h.n_slots > S) || h.status == PROG_UNREPRESENTABLE) {
    h.status = PROG_INVALID;
    atomicAdd(&misc[1], 1u);
  }
  hdr[g] = h;
  prog_cnt[g] = 0u;
}

// Copies one problem's descriptor and token table into device memory: the single-problem entry
// points write their descriptor this way (a kernel argument), so their launch sequence stays a
// pure sequence of kernels and memsets that a CUDA graph can capture.
template <typename T>
__global__ void write_desc_kernel(const ProbDesc<T> d, const TokenLut lut, ProbDesc<T>* dst,
                                  TokenLut* lut_dst) {
  if (threadIdx.x == 0) *dst = d;
  const unsigned* s = reinterpret_cast<const unsigned*>(&lut);
  unsigned* o = reinterpret_cast<unsigned*>(lut_dst);
  for (int i = threadIdx.x; i < (int)(sizeof(TokenLut) / 4); i += blockDim.x) o[i] = s[i];
}

// Up to kUploadChunk descriptors and token tables of a batch, passed as one kernel argument and
// copied into the workspace: batch plans reach the device in stream order, without a host-side
// copy that would wait for the work already queued.
constexpr int kUploadChunk = 16;
template <typename T>
struct DescChunk {
  int n, base;
  ProbDesc<T> d[kUploadChunk];
  TokenLut lut[kUploadChunk];
};
template <typename T>
__global__ void __launch_bounds__(128) upload_desc_kernel(const DescChunk<T> c,
                                                          ProbDesc<T>* __restrict__ dst,
                                                          TokenLut* __restrict__ lut_dst) {
  const int nd = c.n * (int)(sizeof(ProbDesc<T>) / 4), nl = c.n * (int)(sizeof(TokenLut) / 4);
  const unsigned* sd = reinterpret_cast<const unsigned*>(c.d);
  const unsigned* sl = reinterpret_cast<const unsigned*>(c.lut);
  unsigned* od = reinterpret_cast<unsigned*>(dst + c.base);
  unsigned* ol = reinterpret_cast<unsigned*>(lut_dst + c.base);
  for (int i = threadIdx.x; i < nd; i += blockDim.x) od[i] = sd[i];
  for (int i = threadIdx.x; i < nl; i += blockDim.x) ol[i] = sl[i];
}

// FP64 variance of y (population variance, same rows as the loss) for WS_LOSS_R2; one block per
// problem.
template <typename T>
__global__ void __launch_bounds__(256) yvar_kernel(const ProbDesc<T>* __restrict__ desc,
                                                   double* __restrict__ out) {
  __shared__ double s1[256], s2[256];
  const ProbDesc<T>& d = desc[blockIdx.x];
  double a = 0.0, b = 0.0;
  for (int64_t i = threadIdx.x; i < d.D; i += blockDim.x) {
    const double v = (double)d.y[i];
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
    const double m = s1[0] / (double)d.D;
    double v = s2[0] / (double)d.D - m * m;
    out[blockIdx.x] = v > 0.0 ? v : 0.0;
  }
}

// ---------------------------------------------------------------------------------------
// 2. evaluate
template <typename T>
struct FitParams {
  const ProbDesc<T>* desc;  // problems, ascending item0 / prog0
  int n_prob;
  const Instr<T>* tape;     // [sum B, Lcap]
  const ProgHdr* hdr;       // [sum B]
  int Lcap;
  int PB;                   // programs per block
  int64_t n_items;
  int64_t tile_cap;         // elements per staging buffer (a single-buffered tile spans two)
  int S;                    // spill slots per warp
  int policy, loss;
  double invalid_value;
  PartRec* part;
  unsigned* prog_cnt;
  unsigned* work;
  const double* yvar;       // [n_prob] (WS_LOSS_R2)
  const int64_t* perm;      // programs in evaluation order: by problem, then tape length
  T* gspill;                // per-warp scratch for spill slots beyond the shared ones
  const int32_t* cancel;    // optional: nonzero -> take no further work items
};

// The next work item of a persistent evaluator, or n_items (no more work) once the launch's
// cancel flag reads nonzero: the flag is polled once per item, so a cancelled launch ends after
// the items in flight, without any wait.
__device__ __forceinline__ int64_t next_item(unsigned* work, const int32_t* cancel,
                                             int64_t n_items) {
  if (cancel && *reinterpret_cast<const volatile int32_t*>(cancel) != 0) return n_items;
  return (int64_t)atomicAdd(work, 1u);
}

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
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float m_max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double m_max(double a, double b) { return fmax(a, b); }

// Paired FP32 arithmetic (sm_100 f32x2): two rows per instruction, each lane rounded exactly as
// the scalar add / sub / mul of this translation unit (round to nearest, subnormals flushed, as
// --use_fast_math compiles them), so pairing changes instruction counts, not results.
#define WS_PAIR_ASM(OP)                                                                   \
  asm("{\n .reg .b64 p, q;\n mov.b64 p, {%0, %1};\n mov.b64 q, {%2, %3};\n " OP      \
      " p, p, q;\n mov.b64 {%0, %1}, p;\n}"                                             \
      : "+f"(a0), "+f"(a1)                                                                \
      : "f"(b0), "f"(b1))
__device__ __forceinline__ void pair_add(float& a0, float& a1, float b0, float b1) {
  WS_PAIR_ASM("add.rn.ftz.f32x2");
}
__device__ __forceinline__ void pair_sub(float& a0, float& a1, float b0, float b1) {
  WS_PAIR_ASM("sub.rn.ftz.f32x2");
}
__device__ __forceinline__ void pair_mul(float& a0, float& a1, float b0, float b1) {
  WS_PAIR_ASM("mul.rn.ftz.f32x2");
}
#undef WS_PAIR_ASM

// a = a OP b (REV: a = b OP a) for rows k, k+1; OPK 0 add, 1 sub, 2 mul.
template <int OPK, bool REV>
__device__ __forceinline__ void pair_apply(float& a0, float& a1, float b0, float b1) {
  if (OPK == 0) {
    pair_add(a0, a1, b0, b1);
  } else if (OPK == 2) {
    pair_mul(a0, a1, b0, b1);
  } else if (!REV) {
    pair_sub(a0, a1, b0, b1);
  } else {
    float t0 = b0, t1 = b1;
    pair_sub(t0, t1, a0, a1);
    a0 = t0;
    a1 = t1;
  }
}

// ---- shared-memory access by 32-bit address ------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void lds4(float (&d)[4], uint32_t a) {
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
               : "r"(a));
}
__device__ __forceinline__ void sts4(uint32_t a, float d0, float d1, float d2, float d3) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(d0), "f"(d1), "f"(d2),
               "f"(d3)
               : "memory");
}
__device__ __forceinline__ void lds_word(uint32_t& c, uint32_t& imm, uint32_t a) {
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(c), "=r"(imm) : "r"(a));
}

// Vector-operand loaders: group g (16 bytes) of this lane's rows of operand V.
template <typename T>
struct GenericOperand {  // V anywhere (shared X tile, shared or global spill slot)
  const T* vp;
  __device__ __forceinline__ void load(T (&v)[Vec16<T>::N], int g) const {
    Vec16<T>::load(v, vp + g * 32 * Vec16<T>::N);
  }
};
struct SharedOperand {  // V in shared memory at a 32-bit address (FP32)
  uint32_t va;
  __device__ __forceinline__ void load(float (&v)[4], int g) const { lds4(v, va + g * 512); }
};

// One tape instruction's operator over this lane's R rows: ACC = ACC o V / V o ACC / ACC o s /
// s o ACC for binary cases, ACC = f(ACC) for unary ones.  A fetched operand is read group by
// group inside its case (16-byte loads), so only one group of it is live at a time: registers
// go to the R accumulators instead.
template <typename T, int R, bool STRICT, class LD>
__device__ __forceinline__ void exec_case(uint32_t cs, T s, const LD& ld, T (&acc)[R],
                                          uint32_t& err) {
  constexpr int N = Vec16<T>::N;
  constexpr bool PAIR = sizeof(T) == 4;
#define WS_ROWS(BODY) _Pragma("unroll") for (int k = 0; k < R; ++k) { BODY; } break
// rows with a fetched operand: group g of the operand is loaded, then used as v[q]
#define WS_ROWS_V(BODY)                                                        \
  _Pragma("unroll") for (int g = 0; g < R / N; ++g) {                          \
    T v[N];                                                                    \
    ld.load(v, g);                                                             \
    _Pragma("unroll") for (int q = 0; q < N; ++q) { const int k = g * N + q; BODY; } \
  }                                                                            \
  break
#define WS_PAIRS_V(OPK, REV)                                                   \
  _Pragma("unroll") for (int g = 0; g < R / N; ++g) {                          \
    T v[N];                                                                    \
    ld.load(v, g);                                                             \
    _Pragma("unroll") for (int q = 0; q < N; q += 2)                           \
      pair_apply<OPK, REV>(*(float*)&acc[g * N + q], *(float*)&acc[g * N + q + 1], \
                           *(float*)&v[q], *(float*)&v[q + 1]);                \
  }                                                                            \
  break
#define WS_PAIRS_S(OPK, REV)                                                   \
  _Pragma("unroll") for (int k = 0; k < R; k += 2)                             \
    pair_apply<OPK, REV>(*(float*)&acc[k], *(float*)&acc[k + 1], (float)s, (float)s); \
  break
#define WS_ERR(EXPR) { bool e_ = false; acc[k] = (EXPR); err |= (uint32_t)e_ << k; }
#define WS_BIN4(CLS, F)                                                          \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_AV: WS_ROWS_V(F(acc[k], v[q]));      \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_VA: WS_ROWS_V(F(v[q], acc[k]));      \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_AS: WS_ROWS(F(acc[k], s));           \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_SA: WS_ROWS(F(s, acc[k]));
// + - *: paired when T is float
#define WS_BIN4P(CLS, F, OPK)                                                    \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_AV:                                  \
    if (PAIR) { WS_PAIRS_V(OPK, false); } else { WS_ROWS_V(F(acc[k], v[q])); }   \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_VA:                                  \
    if (PAIR) { WS_PAIRS_V(OPK, true); } else { WS_ROWS_V(F(v[q], acc[k])); }    \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_AS:                                  \
    if (PAIR) { WS_PAIRS_S(OPK, false); } else { WS_ROWS(F(acc[k], s)); }        \
  case PCASE_BIN + 4 * (CLS - T_ADD) + FORM_SA:                                  \
    if (PAIR) { WS_PAIRS_S(OPK, true); } else { WS_ROWS(F(s, acc[k])); }
#define F_ADD(a, b) acc[k] = (a) + (b)
#define F_SUB(a, b) acc[k] = (a) - (b)
#define F_MUL(a, b) acc[k] = (a) * (b)
#define F_DIV(a, b) WS_ERR((op_div<T, STRICT>((a), (b), e_)))
#define F_POW(a, b) WS_ERR((op_pow<T, STRICT>((a), (b), e_)))
#define F_MOD(a, b) WS_ERR((op_mod<T, STRICT>((a), (b), e_)))
#define U_(CLS) (PCASE_UNARY0 + (CLS - T_SIN))
  switch (cs) {
    case PCASE_NOP: break;
    WS_BIN4P(T_ADD, F_ADD, 0)
    WS_BIN4P(T_SUB, F_SUB, 1)
    WS_BIN4P(T_MUL, F_MUL, 2)
    WS_BIN4(T_DIV, F_DIV)
    WS_BIN4(T_POW, F_POW)
    WS_BIN4(T_MOD, F_MOD)
    case U_(T_SIN): WS_ROWS(acc[k] = m_sin(acc[k]));
    case U_(T_COS): WS_ROWS(acc[k] = m_cos(acc[k]));
    case U_(T_TAN): WS_ROWS(acc[k] = m_tan(acc[k]));
    case U_(T_LOG): WS_ROWS(WS_ERR((op_log<T, STRICT>(acc[k], e_))));
    case U_(T_EXP): WS_ROWS(WS_ERR((op_exp<T, STRICT>(acc[k], e_))));
    case U_(T_SQRT): WS_ROWS(WS_ERR((op_sqrt<T, STRICT>(acc[k], e_))));
    case U_(T_ABS): WS_ROWS(acc[k] = m_abs(acc[k]));
    case U_(T_NEG): WS_ROWS(acc[k] = -acc[k]);
    case U_(T_FACT): WS_ROWS(WS_ERR((op_tgamma<T, STRICT>(acc[k] + (T)1.0, e_))));
    case U_(T_FLOOR): WS_ROWS(acc[k] = m_floor(acc[k]));
    case U_(T_CEIL): WS_ROWS(acc[k] = m_ceil(acc[k]));
    case U_(T_SIGN): WS_ROWS(acc[k] = op_sign<T>(acc[k]));
    case U_(T_GAMMA): WS_ROWS(WS_ERR((op_tgamma<T, STRICT>(acc[k], e_))));
    case U_(T_LGAMMA): WS_ROWS(WS_ERR((op_lgamma<T, STRICT>(acc[k], e_))));
    case U_(T_ASIN): WS_ROWS(WS_ERR((op_asin<T, STRICT>(acc[k], e_))));
    case U_(T_ACOS): WS_ROWS(WS_ERR((op_acos<T, STRICT>(acc[k], e_))));
    case U_(T_ATAN): WS_ROWS(acc[k] = m_atan(acc[k]));
    // the compiler emits only the cases above (the tape's case field is 6 bits; 42..63 unused)
    default: __builtin_unreachable();
  }
#undef U_
#undef F_ADD
#undef F_SUB
#undef F_MUL
#undef F_DIV
#undef F_POW
#undef F_MOD
#undef WS_BIN4
#undef WS_BIN4P
#undef WS_PAIRS_V
#undef WS_PAIRS_S
#undef WS_ERR
#undef WS_ROWS_V
#undef WS_ROWS
}

// Runs one program tape over one pass of 32*R rows (any T, any spill depth).  xb: the X tile
// at this pass and lane; sb / gb: this warp's shared / global spill slots at this lane.  Tape
// offsets are in units of one pass.
template <typename T, int R, bool STRICT>
__device__ __forceinline__ void run_tape(const Instr<T>* __restrict__ tp, int n,
                                         const T* __restrict__ xb, T* __restrict__ sb,
                                         T* __restrict__ gb, T (&acc)[R], uint32_t& err,
                                         uint32_t x_lim, uint32_t n_deep) {
  constexpr int PASS = 32 * R;
  err = 0u;
  // The next tape word is loaded while the current one executes (reading one word past the end
  // of a tape stays inside the block's shared memory and is never used).
  Instr<T> nxt = tp[0];
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const Instr<T> ins = nxt;
    nxt = tp[i + 1];
    const uint32_t c = __shfl_sync(0xFFFFFFFFu, ins.ctrl, 0);  // warp-uniform by construction
    // vector operand: an X row of the tile or a shared spill slot (dereferenced only by the
    // cases that read it)
    const T* vp = ((c & P_FETCH_SLOT) ? sb : xb) + (c >> P_SH_V) * PASS;
#ifdef WS_BOUNDS_CHECK
    if (pcase_fetches(c & P_CASE_MASK) && !(c & P_FETCH_SLOT) &&
        !WS_BC((c >> P_SH_V) < x_lim, BC_FIT_X, c >> P_SH_V))
      vp = xb;
#endif
    if (c & P_SLOW) {  // spill, accumulator load, deep spill slot: rare
      if (c & P_SPILL) {
        const uint32_t sl = (c >> P_SH_SLOT) & 7u;
        if (sl < (uint32_t)kSharedSlots) lane_store<T, R>(sb + sl * PASS, acc);
        else if (WS_BC(sl - kSharedSlots < n_deep, BC_FIT_SLOT, sl))
          lane_store<T, R>(gb + (sl - kSharedSlots) * PASS, acc);
      }
      if (c & P_LOADA_X) {
        const uint32_t la = (c >> P_SH_LA) & P_OFF_MASK;
        if (WS_BC(la < x_lim, BC_FIT_X, la)) lane_load<T, R>(acc, xb + la * PASS);
      } else if (c & P_LOADA_S) {
#pragma unroll
        for (int k = 0; k < R; ++k) acc[k] = ins.imm;
      }
      const uint32_t off = c >> P_SH_V;
      if ((c & P_FETCH_SLOT) && off >= (uint32_t)kSharedSlots)
        vp = WS_BC(off - kSharedSlots < n_deep, BC_FIT_SLOT, off) ? gb + (off - kSharedSlots) * PASS
                                                                   : sb;
    }
    exec_case<T, R, STRICT>(c & P_CASE_MASK, ins.imm, GenericOperand<T>{vp}, acc, err);
  }
}

// The FP32 interpreter for programs whose spill slots are all in shared memory (every program
// but the deepest 0.2%): operands, spill slots and tape words are addressed as 32-bit shared
// addresses.  xa: X tile at this pass and lane; sa: this warp's spill slot 0 at this lane; ta:
// the tape.  One pass is 32*R rows = PASS*4 bytes = 1 << PSH.  Each iteration reads its tape
// word (a broadcast load), takes lane 0's copy (warp-uniform by construction), and dispatches;
// a software-pipelined decode (next word in flight while the current one executes) measured
// 5% more instructions per tape word on this loop and no faster, so the loop stays plain.
template <int R, bool STRICT>
__device__ __forceinline__ void run_tape_shared(uint32_t ta, int n, uint32_t xa, uint32_t sa,
                                                float (&acc)[R], uint32_t& err, uint32_t x_lim) {
  static_assert(R == 8 || R == 16 || R == 32, "pass size");
  constexpr int PSH = R == 8 ? 10 : (R == 16 ? 11 : 12);
  err = 0u;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    uint32_t c0, ni;
    lds_word(c0, ni, ta + 8u * (uint32_t)i);
    const uint32_t c = __shfl_sync(0xFFFFFFFFu, c0, 0);
    const float s = __uint_as_float(ni);
    uint32_t va = ((c & P_FETCH_SLOT) ? sa : xa) + ((c >> P_SH_V) << PSH);
#ifdef WS_BOUNDS_CHECK
    if (pcase_fetches(c & P_CASE_MASK) &&
        !((c & P_FETCH_SLOT) ? WS_BC((c >> P_SH_V) < (uint32_t)kSharedSlots, BC_FIT_SLOT, c >> P_SH_V)
                             : WS_BC((c >> P_SH_V) < x_lim, BC_FIT_X, c >> P_SH_V)))
      va = xa;
#endif
    if (c & P_SLOW) {  // spill, accumulator load: rare
      if ((c & P_SPILL) &&
          WS_BC(((c >> P_SH_SLOT) & 7u) < (uint32_t)kSharedSlots, BC_FIT_SLOT, (c >> P_SH_SLOT) & 7u)) {
        const uint32_t a = sa + (((c >> P_SH_SLOT) & 7u) << PSH);
#pragma unroll
        for (int g = 0; g < R / 4; ++g)
          sts4(a + g * 512, acc[4 * g], acc[4 * g + 1], acc[4 * g + 2], acc[4 * g + 3]);
      }
      if ((c & P_LOADA_X) &&
          WS_BC(((c >> P_SH_LA) & P_OFF_MASK) < x_lim, BC_FIT_X, (c >> P_SH_LA) & P_OFF_MASK)) {
        const uint32_t a = xa + (((c >> P_SH_LA) & P_OFF_MASK) << PSH);
#pragma unroll
        for (int g = 0; g < R / 4; ++g) {
          float v[4];
          lds4(v, a + g * 512);
          acc[4 * g] = v[0]; acc[4 * g + 1] = v[1]; acc[4 * g + 2] = v[2]; acc[4 * g + 3] = v[3];
        }
      } else if (c & P_LOADA_S) {
#pragma unroll
        for (int k = 0; k < R; ++k) acc[k] = s;
      }
    }
    exec_case<float, R, STRICT>(c & P_CASE_MASK, s, SharedOperand{va}, acc, err);
  }
}

// Per-pass epilogue: squared errors of this lane's rows, summed in T (then widened by the
// caller), invalid-row count and per-row metric-overflow flag (WS_POLICY_FUSED only).
template <typename T, int R, bool FUSED>
__device__ __forceinline__ T pass_epilogue(const T (&a)[R], uint32_t err, const T* __restrict__ yb,
                                           int lane, int first_row, int rows, int& ninv,
                                           bool& ovf) {
  constexpr int N = Vec16<T>::N;
  constexpr int PASS = 32 * R;
  constexpr T tmax = sizeof(T) == 4 ? (T)3.4028234663852886e38 : (T)1.7976931348623157e308;
  T yv[R];
  lane_load<T, R>(yv, yb);
  const bool full = first_row + PASS <= rows;
  T part = (T)0;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int row = first_row + (k / N) * 32 * N + lane * N + (k % N);
    const bool act = full || row < rows;
    const T pv = a[k];
    const bool bad = ((err >> k) & 1u) || !(m_abs(pv) <= tmax);  // error, NaN or inf
    const T diff = pv - yv[k];
    T sq;
    if (FUSED) {
      const bool o = !(m_abs(diff) <= Limits<T>::max_diff);  // NaN / inf / > 4e18
      const T q = mul_rn(diff, diff);
      const bool o2 = o || !(m_abs(q) <= tmax);
      ovf = ovf || (act && !bad && o2);
      sq = (bad || o2) ? (T)0 : q;
    } else {
      sq = bad ? (T)0 : mul_rn(diff, diff);
    }
    ninv += (act && bad) ? 1 : 0;
    part += act ? sq : (T)0;
  }
  return part;
}

// Fast per-pass epilogue for a pass whose rows are all inside the chunk, when per-row invalid
// counts are not requested: squared errors summed in T; validity tracked without branches --
// fma(pred, 0, acc) turns acc into NaN iff some prediction is NaN or infinite, and for the fused
// policy fma(diff, 0, .) and max |diff| flag the metric overflow.  Rows that are invalid or
// overflow only decide the program's class, never a value, so they need no masking here.
template <typename T, int R, bool FUSED>
__device__ __forceinline__ T pass_fast(const T (&a)[R], const T* __restrict__ yb, T& nanacc,
                                       T& ovfacc, T& dmax) {
  T yv[R];
  lane_load<T, R>(yv, yb);
  T part = (T)0;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const T diff = a[k] - yv[k];
    part = part + mul_rn(diff, diff);
    nanacc = fma_rn(a[k], (T)0, nanacc);
    if (FUSED) {
      ovfacc = fma_rn(diff, (T)0, ovfacc);
      dmax = m_max(dmax, m_abs(diff));
    }
  }
  return part;
}

// Paired fast epilogue (FP32, classic policy): diff, square and the running sums two rows per
// instruction, each row rounded as the scalar code rounds it.  A non-finite prediction makes
// the pass sum non-finite (NaN, or +inf: squares are >= 0), so rows are only re-examined then.
template <int R>
__device__ __forceinline__ float pass_fast_pairs(const float (&a)[R], const float* __restrict__ yb,
                                                 bool& bad) {
  float yv[R];
  lane_load<float, R>(yv, yb);
  float p0 = 0.f, p1 = 0.f;
#pragma unroll
  for (int k = 0; k < R; k += 2) {
    float d0 = a[k], d1 = a[k + 1];
    pair_sub(d0, d1, yv[k], yv[k + 1]);
    pair_mul(d0, d1, d0, d1);
    pair_add(p0, p1, d0, d1);
  }
  const float part = p0 + p1;
  if (!(part <= 3.4028234663852886e38f)) {
#pragma unroll
    for (int k = 0; k < R; ++k) bad = bad || !(fabsf(a[k]) <= 3.4028234663852886e38f);
  }
  return part;
}

// Final loss of one program from its combined record.  Classification mirrors the
// reference epilogues:
//   WS_POLICY_FUSED (rpn_kernels.cu:2487-2497): invalid row -> iv; per-row metric overflow ->
//     sqrt(iv); non-finite mean (sum overflow) -> iv.
//   WS_POLICY_CLASSIC (evaluation.py:182-189): invalid row -> iv; non-finite mean -> sqrt(iv).
// An FP64 sum above the T range stands for the overflow of the reference's T accumulator.
// MSE uses the same classification (any overflow -> iv); R2 writes -iv for both.
template <typename T>
__device__ void write_final(const FitParams<T>& P, const ProbDesc<T>& d, double yvar, int64_t p,
                            const PartRec& r) {
  if (d.out_ninv) d.out_ninv[p] = r.ninv;
  const double tmax = (double)(sizeof(T) == 4 ? FLT_MAX : DBL_MAX);
  if (P.loss == WS_LOSS_SSE) {
    ((double*)d.out_loss)[p] = (r.ninv > 0) ? P.invalid_value : r.sse;
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
    const double mse = r.sse / (double)d.D;
    const T mse_t = (T)mse;
    if (P.loss == WS_LOSS_RMSE) {
      const T q = m_sqrt(mse_t);
      out = (m_isnan(q) || m_isinf(q)) ? P.invalid_value : (double)q;
    } else if (P.loss == WS_LOSS_MSE) {
      out = (double)mse_t;
    } else {
      out = yvar > 0.0 ? 1.0 - mse / yvar : (mse == 0.0 ? 1.0 : -P.invalid_value);
    }
  }
  if (sizeof(T) == 4) ((float*)d.out_loss)[p] = (float)out;
  else ((double*)d.out_loss)[p] = out;
}

// ---- chunk staging: 16-byte asynchronous copies (cp.async) into a shared tile ---------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issues the copy of chunk c (X rows of every variable, then y) into tile `tb` and commits one
// cp.async group.  With async_stage the copies are 16-byte cp.async (rows of X are 16-byte
// aligned: D is a multiple of 16/sizeof(T)); otherwise plain loads/stores with zero fill.
template <typename T>
__device__ __forceinline__ void stage_chunk(const ProbDesc<T>& d, int64_t c, T* tb, int tid,
                                            int nthreads) {
  constexpr int VE = 16 / (int)sizeof(T);
  const int64_t row0 = c * d.RC;
  const int rows = (int)min((int64_t)d.RC, d.D - row0);
  if (d.async_stage) {
    const int nvec = rows / VE;
    for (int v = 0; v <= d.V; ++v) {
      const T* src = (v < d.V ? d.x + (size_t)v * d.D : d.y) + row0;
      T* dst = tb + (size_t)v * d.RC;
      for (int i = tid; i < nvec; i += nthreads) cp_async16(dst + i * VE, src + i * VE);
    }
  } else {
    for (int v = 0; v <= d.V; ++v) {
      const T* src = (v < d.V ? d.x + (size_t)v * d.D : d.y) + row0;
      T* dst = tb + (size_t)v * d.RC;
      for (int r = tid; r < d.RC; r += nthreads) dst[r] = (r < rows) ? src[r] : (T)0;
    }
  }
  cp_async_commit();
}

template <typename T, int R, bool STRICT>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 && R <= 16) ? 3 : 2)
    fitness_kernel(const FitParams<T> P) {
  constexpr int N = Vec16<T>::N;
  constexpr int PASS = 32 * R;
  constexpr bool F32 = sizeof(T) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x >> 5;
  // warp index broadcast from lane 0: the compiler then treats it (and the tape addresses
  // derived from it) as warp-uniform
  const int warp = __shfl_sync(0xFFFFFFFFu, (int)(threadIdx.x >> 5), 0);
  const int lane = threadIdx.x & 31;
  // two tiles of X[:, chunk] and y[chunk] (double-buffered staging), per-warp spill slots, the
  // block's tapes, per-program records, per-program per-lane FP64 partial sums
  T* tiles = reinterpret_cast<T*>(smem_raw);
  T* spill = tiles + 2 * P.tile_cap;
  Instr<T>* tapes = reinterpret_cast<Instr<T>*>(spill + (size_t)W * kSharedSlots * PASS);
  PartRec* acc_s = reinterpret_cast<PartRec*>(tapes + (size_t)P.PB * P.Lcap);
  double* lane_sse = reinterpret_cast<double*>(acc_s + P.PB);  // [PB][kLaneStride]
  int* meta_s = reinterpret_cast<int*>(lane_sse + (size_t)P.PB * kLaneStride);
  __shared__ int64_t s_item;
  __shared__ ProbDesc<T> s_desc;
  __shared__ double s_yvar;

  T* sp_w = spill + (size_t)warp * kSharedSlots * PASS + lane * N;
  const int deep = P.S > kSharedSlots ? P.S - kSharedSlots : 0;
  T* gsp_w = P.gspill + ((size_t)blockIdx.x * W + warp) * (size_t)deep * PASS + lane * N;
  const bool fused_policy = P.policy == WS_POLICY_FUSED;

  for (;;) {
    if (threadIdx.x == 0) {
      const int64_t it = next_item(P.work, P.cancel, P.n_items);
      s_item = it;
      if (it < P.n_items) {
        const int pi = find_problem(P.desc, P.n_prob, it, true);
        s_desc = P.desc[pi];
        s_yvar = P.yvar ? P.yvar[pi] : 0.0;
      }
    }
    __syncthreads();
    const int64_t item = s_item;
    if (item >= P.n_items) break;
    const ProbDesc<T>& d = s_desc;
    const int64_t local = item - d.item0;
    const int64_t blk = local / d.n_splits;
    const int split = (int)(local % d.n_splits);
    const int64_t p0 = d.prog0 + blk * P.PB;  // position in perm
    const int np = (int)min((int64_t)P.PB, d.B - blk * P.PB);
    const int64_t c0 = (int64_t)split * d.cps;
    const int64_t c1 = min(d.n_chunks, c0 + d.cps);
    const size_t tile_elems = (size_t)(d.V + 1) * d.RC;
    // stage the block's tapes once for all its chunks (programs arrive sorted by tape length,
    // so a static warp assignment is balanced)
    for (int q = warp; q < np; q += W) {
      const int64_t g = P.perm[p0 + q];
      ProgHdr h = P.hdr[g];
      if (!WS_BC(h.n_instr <= P.Lcap, BC_FIT_TAPE_LEN, h.n_instr)) h.status = PROG_INVALID;
      const Instr<T>* tg = P.tape + g * (int64_t)P.Lcap;
      for (int i = lane; i < h.n_instr && WS_BC(i < P.Lcap, BC_FIT_TAPE_LEN, i); i += 32)
        tapes[(size_t)q * P.Lcap + i] = tg[i];
      lane_sse[q * kLaneStride + lane] = 0.0;
      if (lane == 0) {
        // n_instr, kMetaGlobalSpill if a spill slot lives in global memory; -1: invalid
        meta_s[q] = h.status == PROG_OK
                        ? (h.n_instr | (h.n_slots > kSharedSlots ? kMetaGlobalSpill : 0))
                        : -1;
        acc_s[q] = PartRec{0.0, 0, 0};
      }
    }

    int buf = 0;
    const bool single = d.single != 0;
    stage_chunk<T>(d, c0, tiles, threadIdx.x, blockDim.x);
    for (int64_t c = c0; c < c1; ++c) {
      T* xs = tiles + (size_t)buf * P.tile_cap;
      T* ys = xs + (size_t)d.V * d.RC;
      if (!single && c + 1 < c1) {  // the next chunk streams in while this one is evaluated
        stage_chunk<T>(d, c + 1, tiles + (size_t)(buf ^ 1) * P.tile_cap, threadIdx.x, blockDim.x);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      const int64_t row0 = c * d.RC;
      const int rows = (int)min((int64_t)d.RC, d.D - row0);
      if (d.async_stage && rows < d.RC) {  // zero the rows past the end of the data
        for (int v = 0; v <= d.V; ++v)
          for (int r = rows + threadIdx.x; r < d.RC; r += blockDim.x) xs[(size_t)v * d.RC + r] = (T)0;
      }
      __syncthreads();  // chunk c visible to all warps; tapes and accumulators ready
      const int npass = (rows + PASS - 1) / PASS;
      const bool count = d.count != 0;

      for (int q = warp; q < np; q += W) {
        const int meta = meta_s[q];
        if (meta < 0) {
          if (lane == 0) acc_s[q].ninv += rows;
          continue;
        }
        const int n_instr = meta & kMetaLenMask;
        const bool shared_only = F32 && !(meta & kMetaGlobalSpill);
        const Instr<T>* tape_q = tapes + (size_t)q * P.Lcap;
        double sse = 0.0;
        int ninv = 0;
        bool ovf = false, nonfinite = false;
        uint32_t errany = 0u;
        T nanacc = (T)0, ovfacc = (T)0, dmax = (T)0;
        for (int pass = 0; pass < npass; ++pass) {
          T a[R];
          uint32_t err;
          // variable operands lie below this offset (in passes) from the pass's X row
          const uint32_t x_lim = (uint32_t)(d.V * (d.RC / PASS) - pass);
          if constexpr (F32) {
            if (shared_only)
              run_tape_shared<R, STRICT>(smem_u32(tape_q), n_instr,
                                         smem_u32(xs + pass * PASS + lane * N), smem_u32(sp_w),
                                         *reinterpret_cast<float(*)[R]>(&a), err, x_lim);
            else
              run_tape<T, R, STRICT>(tape_q, n_instr, xs + pass * PASS + lane * N, sp_w, gsp_w,
                                     a, err, x_lim, (uint32_t)deep);
          } else {
            run_tape<T, R, STRICT>(tape_q, n_instr, xs + pass * PASS + lane * N, sp_w, gsp_w, a,
                                   err, x_lim, (uint32_t)deep);
          }
          const T* yb = ys + pass * PASS + lane * N;
          T part;
          if (!count && (pass + 1) * PASS <= rows) {
            errany |= err;
            if (fused_policy) {
              part = pass_fast<T, R, true>(a, yb, nanacc, ovfacc, dmax);
            } else if constexpr (F32) {
              part = pass_fast_pairs<R>(*reinterpret_cast<const float(*)[R]>(&a),
                                        reinterpret_cast<const float*>(yb), nonfinite);
            } else {
              part = pass_fast<T, R, false>(a, yb, nanacc, ovfacc, dmax);
            }
          } else {
            part = fused_policy
                ? pass_epilogue<T, R, true>(a, err, yb, lane, pass * PASS, rows, ninv, ovf)
                : pass_epilogue<T, R, false>(a, err, yb, lane, pass * PASS, rows, ninv, ovf);
          }
          sse += (double)part;
        }
        // this lane's partial sum of the program, in a fixed per-lane order across chunks
        lane_sse[q * kLaneStride + lane] += sse;
        // without per-row counts only "ninv > 0" matters
        if (errany != 0u || nonfinite || m_isnan(nanacc)) ninv += 1;
        if (count) {
          const unsigned tot = __reduce_add_sync(0xFFFFFFFFu, (unsigned)ninv);
          if (lane == 0 && tot) acc_s[q].ninv += (int)tot;
        } else if (__any_sync(0xFFFFFFFFu, ninv > 0)) {
          if (lane == 0) acc_s[q].ninv += 1;
        }
        if (fused_policy) {
          ovf = ovf || m_isnan(ovfacc) || dmax > Limits<T>::max_diff;
          if (__any_sync(0xFFFFFFFFu, ovf) && lane == 0) acc_s[q].ovf = 1;
        }
      }
      __syncthreads();  // every warp is done with this tile before it is refilled
      if (single) {
        if (c + 1 < c1) stage_chunk<T>(d, c + 1, tiles, threadIdx.x, blockDim.x);
      } else {
        buf ^= 1;
      }
    }
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
      const int64_t g = P.perm[p0 + q];
      const int64_t pl = g - d.prog0;  // index within the problem
      PartRec r = acc_s[q];
      double t = 0.0;  // lanes combined in a fixed order
      for (int l = 0; l < 32; ++l) t += lane_sse[q * kLaneStride + l];
      r.sse = t;
      if (d.n_splits == 1) {
        write_final<T>(P, d, s_yvar, pl, r);
      } else {
        PartRec* pr0 = P.part + d.part0 + pl * d.n_splits;
        pr0[split] = r;
        __threadfence();
        const unsigned done = atomicAdd(&P.prog_cnt[g], 1u);
        if (done == (unsigned)d.n_splits - 1u) {
          __threadfence();
          PartRec t2{0.0, 0, 0};
          for (int s2 = 0; s2 < d.n_splits; ++s2) {
            t2.sse += __ldcg(&pr0[s2].sse);
            t2.ninv += __ldcg(&pr0[s2].ninv);
            t2.ovf |= __ldcg(&pr0[s2].ovf);
          }
          write_final<T>(P, d, s_yvar, pl, t2);
          P.prog_cnt[g] = 0u;  // ready for an evaluate-only rerun on the same tape
        }
      }
    }
    // the next item's staging (and the descriptor) waits on the __syncthreads() at the loop top
    __syncthreads();
  }
}

// ---- small data sets: several programs per warp ---------------------------------------------
// With D <= 128 rows, a warp of fitness_kernel would carry mostly padding rows (one pass is
// 32*R >= 256 rows; at D = 20, 92% of the lanes idle).  Here a warp holds PW = 32 / S programs,
// S lanes each, and lane t of a subgroup carries rows [4t, 4t + 4) of the data set zero-padded
// to DP = 4S rows, which every CTA stages once.  The subgroups of a warp run different tapes, so
// their dispatches diverge; the tape-word load and the operand-address arithmetic still run once
// for the whole warp, which makes one warp step advance PW programs.  Programs arrive sorted by
// tape length, so the subgroups of a warp finish together.  All spill slots live in shared memory
// (`NS` per lane, 16 or 32 bytes each).
//
// Per-row values are those of fitness_kernel (same compiler, same operator code).  A program's
// loss sums its rows in order within a lane (in T), then the S lanes of its subgroup in FP64 by a
// fixed butterfly: the order depends on D only, never on the other programs of the launch.

// Operand loader for 4 contiguous rows of a lane (16-byte groups).
template <typename T>
struct ContigOperand {
  const T* vp;
  __device__ __forceinline__ void load(T (&v)[Vec16<T>::N], int g) const {
    Vec16<T>::load(v, vp + g * Vec16<T>::N);
  }
};

// One program tape over this lane's 4 rows.  xb: the staged data set at this lane's rows (one
// variable every DP elements); sb: this lane's spill slot 0 (one slot every 32*4 elements).
template <typename T, int DP, bool STRICT>
__device__ __forceinline__ void run_tape_small(const Instr<T>* __restrict__ tp, int n,
                                               const T* __restrict__ xb, T* __restrict__ sb,
                                               T (&acc)[4], uint32_t& err, uint32_t n_vars,
                                               uint32_t n_slots) {
  constexpr int N = Vec16<T>::N;
  constexpr int SLOT = 32 * 4;
  err = 0u;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const Instr<T> ins = tp[i];
    const uint32_t c = ins.ctrl;
    const uint32_t off = c >> P_SH_V;
    const T* vp = (c & P_FETCH_SLOT) ? sb + off * SLOT : xb + off * DP;
#ifdef WS_BOUNDS_CHECK
    if (pcase_fetches(c & P_CASE_MASK) &&
        !((c & P_FETCH_SLOT) ? WS_BC(off < n_slots, BC_SMALL_SLOT, off)
                             : WS_BC(off < n_vars, BC_SMALL_X, off)))
      vp = xb;
#endif
    if (c & P_SLOW) {  // spill, accumulator load
      if ((c & P_SPILL) &&
          WS_BC(((c >> P_SH_SLOT) & 7u) < n_slots, BC_SMALL_SLOT, (c >> P_SH_SLOT) & 7u)) {
        T* dst = sb + ((c >> P_SH_SLOT) & 7u) * SLOT;
#pragma unroll
        for (int g = 0; g < 4 / N; ++g) Vec16<T>::store(dst + g * N, &acc[g * N]);
      }
      if ((c & P_LOADA_X) &&
          WS_BC(((c >> P_SH_LA) & P_OFF_MASK) < n_vars, BC_SMALL_X, (c >> P_SH_LA) & P_OFF_MASK)) {
        const T* src = xb + ((c >> P_SH_LA) & P_OFF_MASK) * DP;
#pragma unroll
        for (int g = 0; g < 4 / N; ++g) Vec16<T>::load(&acc[g * N], src + g * N);
      } else if (c & P_LOADA_S) {
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] = ins.imm;
      }
    }
    exec_case<T, 4, STRICT>(c & P_CASE_MASK, ins.imm, ContigOperand<T>{vp}, acc, err);
  }
}

// Squared errors of a lane's 4 contiguous rows (row index first_row + k), summed in T in row
// order, with the invalid-row count and the per-row metric-overflow flag of pass_epilogue.
template <typename T, bool FUSED>
__device__ __forceinline__ T small_epilogue(const T (&a)[4], uint32_t err, const T* __restrict__ yb,
                                            int first_row, int rows, int& ninv, bool& ovf) {
  constexpr T tmax = sizeof(T) == 4 ? (T)3.4028234663852886e38 : (T)1.7976931348623157e308;
  T part = (T)0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const bool act = first_row + k < rows;
    const T pv = a[k];
    const bool bad = ((err >> k) & 1u) || !(m_abs(pv) <= tmax);  // error, NaN or inf
    const T diff = pv - yb[k];
    T sq;
    if (FUSED) {
      const bool o = !(m_abs(diff) <= Limits<T>::max_diff);
      const T q = mul_rn(diff, diff);
      const bool o2 = o || !(m_abs(q) <= tmax);
      ovf = ovf || (act && !bad && o2);
      sq = (bad || o2) ? (T)0 : q;
    } else {
      sq = bad ? (T)0 : mul_rn(diff, diff);
    }
    ninv += (act && bad) ? 1 : 0;
    part += act ? sq : (T)0;
  }
  return part;
}

// P.PB = W * PW programs per work item (one problem, P.desc[0]); P.S = spill slots per lane.
template <typename T, int S, bool STRICT>
__global__ void __launch_bounds__(256) fitness_small_kernel(const FitParams<T> P) {
  constexpr int PW = 32 / S;
  constexpr int DP = 4 * S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / S, t = lane % S;
  __shared__ ProbDesc<T> s_desc;
  __shared__ int64_t s_item;
  if (threadIdx.x == 0) s_desc = P.desc[0];
  __syncthreads();
  const ProbDesc<T>& d = s_desc;
  const int V = d.V;
  const int rows = (int)d.D;
  const int tstride = P.Lcap + 1;  // odd word stride: the subgroups' tape words hit distinct banks
  // data set [V + 1][DP] (y last), spill slots [W][S][32][4], tapes [PB][Lcap + 1], meta [PB]
  T* xs = reinterpret_cast<T*>(smem_raw);
  T* spill = xs + (size_t)(V + 1) * DP;
  Instr<T>* tapes = reinterpret_cast<Instr<T>*>(spill + (size_t)W * P.S * 32 * 4);
  int* meta_s = reinterpret_cast<int*>(tapes + (size_t)P.PB * tstride);
  for (int i = threadIdx.x; i < (V + 1) * DP; i += blockDim.x) {
    const int v = i / DP, r = i - v * DP;
    xs[i] = r < rows ? (v < V ? d.x[(size_t)v * rows + r] : d.y[r]) : (T)0;
  }
  const T* xb = xs + t * 4;
  const T* yb = xs + (size_t)V * DP + t * 4;
  T* sb = spill + ((size_t)warp * P.S * 32 + lane) * 4;
  const bool fused_policy = P.policy == WS_POLICY_FUSED;
  const double yvar = P.yvar ? P.yvar[0] : 0.0;

  for (;;) {
    if (threadIdx.x == 0) s_item = next_item(P.work, P.cancel, P.n_items);
    __syncthreads();  // also: the data set is staged, the previous item's tapes are consumed
    const int64_t item = s_item;
    if (item >= P.n_items) break;
    const int64_t p0 = item * P.PB;
    const int np = (int)min((int64_t)P.PB, d.B - p0);
    for (int q = warp; q < np; q += W) {  // warp-cooperative tape copies
      const int64_t g = P.perm[p0 + q];
      ProgHdr h = P.hdr[g];
      if (!WS_BC(h.n_instr <= P.Lcap, BC_SMALL_TAPE_LEN, h.n_instr)) h.status = PROG_INVALID;
      const Instr<T>* tg = P.tape + g * (int64_t)P.Lcap;
      for (int i = lane; i < h.n_instr && WS_BC(i < P.Lcap, BC_SMALL_TAPE_LEN, i); i += 32)
        tapes[(size_t)q * tstride + i] = tg[i];
      if (lane == 0) meta_s[q] = h.status == PROG_OK ? h.n_instr : -1;
    }
    __syncthreads();
    const int q = warp * PW + sub;  // consecutive (similar-length) programs share a warp
    const bool active = q < np;
    const int meta = active ? meta_s[q] : -1;
    T a[4];
    uint32_t err = 0u;
    if (meta >= 0) {
      run_tape_small<T, DP, STRICT>(tapes + (size_t)q * tstride, meta, xb, sb, a, err,
                                    (uint32_t)V, (uint32_t)P.S);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = (T)0;
      err = active ? 0xFu : 0u;  // a statically invalid program: every row is invalid
    }
    int ninv = 0;
    bool ovf = false;
    T part = (T)0;
    if (active) {
      part = fused_policy ? small_epilogue<T, true>(a, err, yb, t * 4, rows, ninv, ovf)
                          : small_epilogue<T, false>(a, err, yb, t * 4, rows, ninv, ovf);
    }
    // the subgroup's sums, by a fixed butterfly over its S lanes (every lane takes part)
    double sse = (double)part;
    int ovf_i = ovf ? 1 : 0;
#pragma unroll
    for (int o = S / 2; o >= 1; o >>= 1) {
      sse += __shfl_xor_sync(0xFFFFFFFFu, sse, o);
      ninv += __shfl_xor_sync(0xFFFFFFFFu, ninv, o);
      ovf_i |= __shfl_xor_sync(0xFFFFFFFFu, ovf_i, o);
    }
    if (active && t == 0) {
      const int64_t pl = P.perm[p0 + q] - d.prog0;
      write_final<T>(P, d, yvar, pl, PartRec{sse, ninv, ovf_i});
    }
  }
}

// ---- length-sorted schedule: counting sort of programs by (problem, tape length) -----------
// Bins are problem-major; within a problem tape lengths descend and invalid programs come last,
// so problem p's programs occupy perm[prog0, prog0 + B) longest first.
constexpr int kSortBins = 258;  // tape lengths 0..256, plus invalid programs

__device__ __forceinline__ int sort_key(const ProgHdr& v) {
  return v.status == PROG_OK ? min(v.n_instr, 256) : 257;
}

// Each block counts a contiguous range of programs; counts of the problem that opens the range
// go through a shared-memory histogram, the (rare) others straight to global memory.
__global__ void __launch_bounds__(256) sort_hist_kernel(const ProgHdr* __restrict__ hdr,
                                                        const int32_t* __restrict__ prob_of,
                                                        int64_t total_B, int64_t per_block,
                                                        unsigned* __restrict__ bins) {
  __shared__ unsigned h[kSortBins];
  for (int i = threadIdx.x; i < kSortBins; i += blockDim.x) h[i] = 0u;
  const int64_t g0 = (int64_t)blockIdx.x * per_block;
  const int64_t g1 = min(total_B, g0 + per_block);
  const int pb = g0 < total_B ? prob_of[g0] : 0;
  __syncthreads();
  for (int64_t g = g0 + threadIdx.x; g < g1; g += blockDim.x) {
    const int key = sort_key(hdr[g]);
    const int pi = prob_of[g];
    if (pi == pb) atomicAdd(&h[key], 1u);
    else atomicAdd(&bins[(size_t)pi * kSortBins + key], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kSortBins; i += blockDim.x)
    if (h[i]) atomicAdd(&bins[(size_t)pb * kSortBins + i], h[i]);
}

// Exclusive offsets over all bins in evaluation order (problem ascending; within a problem tape
// length descending, invalid last).  One block of 1024 threads.
__device__ __forceinline__ int sort_bin_at(int j) {
  const int p = j / kSortBins, r = j - p * kSortBins;
  return p * kSortBins + (r < 257 ? 256 - r : 257);
}
__global__ void __launch_bounds__(1024) sort_scan_kernel(unsigned* __restrict__ bins, int n_prob) {
  __shared__ unsigned wsum[32];
  const int n = n_prob * kSortBins;
  const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
  const int j0 = min(n, (int)threadIdx.x * per), j1 = min(n, j0 + per);
  unsigned sum = 0u;
  for (int j = j0; j < j1; ++j) sum += bins[sort_bin_at(j)];
  // block exclusive scan of the per-thread sums
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int nw = (int)blockDim.x >> 5;
    unsigned v = lane < nw ? wsum[lane] : 0u;
    unsigned iv = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xFFFFFFFFu, iv, o);
      if (lane >= o) iv += t;
    }
    if (lane < nw) wsum[lane] = iv - v;  // exclusive warp offsets
  }
  __syncthreads();
  unsigned run = wsum[warp] + (incl - sum);
  for (int j = j0; j < j1; ++j) {
    const int b = sort_bin_at(j);
    const unsigned c = bins[b];
    bins[b] = run;
    run += c;
  }
}

// Each block scatters the contiguous range the histogram block counted, one tile of its threads
// at a time: the tile's programs of the tile's first problem are ranked within their key by a
// shared-memory atomic and every key reserves its range of the output with ONE global atomic
// per tile (programs of a later problem in the tile, at problem boundaries, reserve one by one):
// a few dozen global atomics per tile instead of one per program on a few dozen addresses.
__global__ void __launch_bounds__(256) sort_scatter_kernel(const ProgHdr* __restrict__ hdr,
                                                           const int32_t* __restrict__ prob_of,
                                                           int64_t total_B, int64_t per_block,
                                                           unsigned* __restrict__ bins,
                                                           int64_t* __restrict__ perm) {
  __shared__ unsigned h[kSortBins], base[kSortBins];
  const int64_t g0 = (int64_t)blockIdx.x * per_block;
  const int64_t g1 = min(total_B, g0 + per_block);
  for (int64_t t0 = g0; t0 < g1; t0 += blockDim.x) {
    for (int i = threadIdx.x; i < kSortBins; i += blockDim.x) h[i] = 0u;
    __syncthreads();
    const int pb = prob_of[t0];
    const int64_t g = t0 + threadIdx.x;
    const bool act = g < g1;
    int key = 0, pi = pb;
    unsigned rank = 0u;
    if (act) {
      key = sort_key(hdr[g]);
      pi = prob_of[g];
      if (pi == pb) rank = atomicAdd(&h[key], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSortBins; i += blockDim.x)
      if (h[i]) base[i] = atomicAdd(&bins[(size_t)pb * kSortBins + i], h[i]);
    __syncthreads();
    if (act) {
      const unsigned pos = pi == pb ? base[key] + rank
                                    : atomicAdd(&bins[(size_t)pi * kSortBins + key], 1u);
      perm[pos] = g;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// host side
namespace {


// Compiled schedules: rows per lane per pass (R), warps per CTA (W), shared-memory budget per
// CTA.  Index 0 = choose automatically; the Python autotuner times the others.
struct Sched {
  int R, W, PB;
  size_t smem_budget;
};
constexpr Sched kSched[] = {
    {16, 8, 24, 75 * 1024},   // 0: auto placeholder (resolved by pick_schedule)
    {8, 8, 32, 72 * 1024},    // 1
    {16, 4, 16, 56 * 1024},   // 2
    {16, 8, 24, 75 * 1024},   // 3
    {16, 8, 32, 100 * 1024},  // 4
    {8, 8, 64, 100 * 1024},   // 5
    {16, 4, 32, 72 * 1024},   // 6
    {32, 8, 32, 100 * 1024},  // 7
    {32, 4, 16, 100 * 1024},  // 8
    {32, 8, 32, 140 * 1024},  // 9
    {16, 8, 16, 72 * 1024},   // 10
    {16, 8, 16, 100 * 1024},  // 11
};
constexpr int kNumSched = (int)(sizeof(kSched) / sizeof(kSched[0]));
// schedules of the small-data-set evaluator, numbered after kSched (single-problem calls only)
constexpr int kNumSmall = 5;

Sched pick_schedule(int idx, int64_t D) {
  if (idx > 0 && idx < kNumSched) return kSched[idx];
  return D >= 2048 ? kSched[3] : kSched[1];
}

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
  static std::map<std::tuple<int, size_t, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > max_dynamic_smem<T, R, STRICT>()) return 0;
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_tuple(dev, smem, threads);
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

// ---- plans -----------------------------------------------------------------------------
// A plan fixes, for one schedule and one set of problems, the chunk size of every problem, the
// programs per block, the row splits and the order of the work items (heaviest items first, so
// that the persistent CTAs finish together).
struct ProbPlan {
  int RC = 0, xmul = 0, n_splits = 1, async_stage = 0, single = 0;
  int64_t n_chunks = 0, cps = 0, n_blocks = 0, item0 = 0, prog0 = 0, part0 = 0;
};
struct Plan {
  int R = 16, W = 8, PB = 8, S = 0, Lcap = 1;
  size_t smem = 0;
  int64_t n_ctas = 0, n_items = 0, total_B = 0, n_part = 0, tile_cap = 0;
  std::vector<int> order;    // descriptor index -> problem index (problems with B > 0 only)
  std::vector<ProbPlan> pp;  // by problem index
};

template <typename T, int R, bool STRICT>
ws_status make_plan(const ProblemRequest* probs, int n, int64_t L, const Sched& sc,
                    int64_t part_cap, size_t gspill_bytes, Plan& pl) {
  constexpr int PASS = 32 * R;
  constexpr int64_t VE = 16 / (int64_t)sizeof(T);
  const size_t szT = sizeof(T);
  pl.R = R;
  pl.W = sc.W;
  pl.Lcap = tape_capacity(L < 256 ? (int)L : 256);
  pl.S = spill_slots_bound((int)L);
  const int threads = pl.W * 32;
  // programs per block: as the schedule says, but the staged tapes stay within 24 KB (long
  // programs get fewer per block; at least one per warp)
  int PBmax = sc.PB;
  {
    const int fit = (int)((24 * 1024) / ((size_t)pl.Lcap * sizeof(Instr<T>)));
    if (PBmax > fit) PBmax = fit > pl.W ? fit : pl.W;
  }
  const size_t fixed = (size_t)pl.W * kSharedSlots * PASS * szT +
                       (size_t)PBmax * pl.Lcap * sizeof(Instr<T>) +
                       (size_t)PBmax * (sizeof(PartRec) + sizeof(int) + kLaneStride * sizeof(double));
  // Staging tiles: a problem whose two tiles of one pass fit the schedule's budget is
  // double-buffered; one with more variables gets a single tile spanning both buffers (staged
  // after each chunk instead of during it), so that it does not force the whole launch to a
  // larger tile and a lower occupancy.
  int64_t vmax = 0;
  for (int i = 0; i < n; ++i) vmax = probs[i].V > vmax ? probs[i].V : vmax;
  const size_t single_max = (size_t)(vmax + 1) * PASS * szT;
  const size_t optin = max_dynamic_smem<T, R, STRICT>();
  if (fixed + single_max > optin) return fail("too many variables for the shared-memory tile");
  size_t avail = sc.smem_budget > fixed ? sc.smem_budget - fixed : 0;
  if (avail < single_max) avail = single_max;
  pl.pp.assign(n, ProbPlan());
  pl.tile_cap = 0;
  int64_t region = 0;  // elements of the staging region (both buffers)
  for (int i = 0; i < n; ++i) {
    const ProblemRequest& q = probs[i];
    ProbPlan& pp = pl.pp[i];
    pp.single = 2 * (size_t)(q.V + 1) * PASS * szT > avail ? 1 : 0;
    const size_t per_row = (pp.single ? 1 : 2) * (size_t)(q.V + 1) * szT;
    int64_t rc = (int64_t)(avail / per_row) / PASS * PASS;
    const int64_t d_pad = (q.D + PASS - 1) / PASS * PASS;
    if (rc > d_pad) rc = d_pad;
    // tape offsets: variable v at v * (RC / PASS) must fit 9 bits
    const int64_t xmul_cap = q.V > 0 ? (int64_t)P_OFF_MASK / q.V : (int64_t)P_OFF_MASK;
    if (rc / PASS > xmul_cap) rc = xmul_cap * PASS;
    if (rc < PASS) rc = PASS;
    pp.RC = (int)rc;
    pp.xmul = (int)(rc / PASS);
    pp.n_chunks = (q.D + rc - 1) / rc;
    const int64_t tile = (q.V + 1) * rc;
    const int64_t need = pp.single ? tile : 2 * tile;
    if (need > region) region = need;
    pp.async_stage = (q.D % VE == 0) && (((uintptr_t)q.x & 15u) == 0) &&
                     (((uintptr_t)q.y & 15u) == 0) ? 1 : 0;
  }
  pl.tile_cap = ((region + 1) / 2 + 3) / 4 * 4;  // per-buffer stride (16-byte aligned)
  pl.smem = fixed + 2 * (size_t)pl.tile_cap * szT;
  const int occ = occupancy_for<T, R, STRICT>(pl.smem, threads);
  if (occ <= 0) return fail("fitness kernel cannot be resident with this tile size");
  pl.n_ctas = (int64_t)occ * device_info().sm_count;
  const int deep = pl.S > kSharedSlots ? pl.S - kSharedSlots : 0;
  if (deep > 0) {  // one global spill area per resident warp: cap the persistent grid to it
    const int64_t fit = (int64_t)(gspill_bytes / ((size_t)pl.W * deep * PASS * szT));
    if (fit < 1) return fail("workspace too small for the spill scratch of this schedule");
    if (pl.n_ctas > fit) pl.n_ctas = fit;
  }
  // programs per block: halve while the whole launch has fewer than two units per CTA
  auto units = [&](int pb) {
    int64_t u = 0;
    for (int i = 0; i < n; ++i) u += (probs[i].B + pb - 1) / pb * pl.pp[i].n_chunks;
    return u;
  };
  int PB = PBmax;
  while (PB > pl.W && units(PB) < 2 * pl.n_ctas) PB >>= 1;
  pl.PB = PB;
  // Row splits per problem, from the problem's own shape only (its programs per block at the
  // schedule's PB and a nominal three CTAs per SM, as if it ran alone): the summation order of a
  // program's loss -- and so the loss, bit for bit -- does not depend on what else shares the
  // launch.  Small problems are cut into enough items to fill the GPU by themselves.
  const int64_t nominal_ctas = 3 * (int64_t)device_info().sm_count;
  for (int i = 0; i < n; ++i) {
    ProbPlan& pp = pl.pp[i];
    const int64_t B = probs[i].B;
    pp.n_blocks = (B + PB - 1) / PB;
    const int64_t own_blocks = (B + PBmax - 1) / PBmax;
    int64_t ns = own_blocks > 0 ? (2 * nominal_ctas + own_blocks - 1) / own_blocks : 1;
    if (ns < 1) ns = 1;
    if (ns > pp.n_chunks) ns = pp.n_chunks;
    if (part_cap >= 0 && ns > 1 && B * ns > part_cap) ns = B > 0 && part_cap / B > 1 ? part_cap / B : 1;
    pp.cps = (pp.n_chunks + ns - 1) / ns;
    pp.n_splits = (int)((pp.n_chunks + pp.cps - 1) / pp.cps);
  }
  // evaluation order: heaviest work items first
  pl.order.clear();
  for (int i = 0; i < n; ++i)
    if (probs[i].B > 0) pl.order.push_back(i);
  auto cost = [&](int i) {
    const ProbPlan& pp = pl.pp[i];
    return (double)(probs[i].B < pl.PB ? probs[i].B : pl.PB) * (double)pp.cps * (double)pp.RC;
  };
  std::stable_sort(pl.order.begin(), pl.order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  pl.total_B = pl.n_items = pl.n_part = 0;
  for (int i : pl.order) {
    ProbPlan& pp = pl.pp[i];
    pp.prog0 = pl.total_B;
    pp.item0 = pl.n_items;
    pp.part0 = pl.n_part;
    pl.total_B += probs[i].B;
    pl.n_items += pp.n_blocks * pp.n_splits;
    if (pp.n_splits > 1) pl.n_part += probs[i].B * pp.n_splits;
  }
  if (part_cap >= 0 && pl.n_part > part_cap) return fail("partial-record area too small");
  return WS_OK;
}

template <typename T>
ProbDesc<T> make_desc(const ProblemRequest& q, const ProbPlan& pp) {
  ProbDesc<T> d;
  d.pop = q.pop;
  d.consts = static_cast<const T*>(q.consts);
  d.x = static_cast<const T*>(q.x);
  d.y = static_cast<const T*>(q.y);
  d.out_loss = q.out_loss;
  d.out_ninv = q.out_ninv;
  d.B = q.B;
  d.D = q.D;
  d.prog0 = pp.prog0;
  d.item0 = pp.item0;
  d.n_chunks = pp.n_chunks;
  d.cps = pp.cps;
  d.part0 = pp.part0;
  d.V = (int)q.V;
  d.K = q.consts ? (int)q.K : 0;
  d.RC = pp.RC;
  d.xmul = pp.xmul;
  d.n_splits = pp.n_splits;
  d.count = q.out_ninv != nullptr ? 1 : 0;
  d.async_stage = pp.async_stage;
  d.single = pp.single;
  return d;
}

struct RunArgs {
  int64_t L;
  int n_desc;
  int phase, policy, loss;
  double invalid_value;
  cudaStream_t stream;
  const int32_t* cancel = nullptr;  // see FitParams::cancel
};

// Compile + length sort of the programs of the descriptors in the workspace (unless
// evaluate-only), and the work-queue reset of an evaluate-only launch.  Kernels and memsets only.
template <typename T, bool STRICT>
ws_status compile_and_sort(int64_t total_B, int Lcap, int S, const FitnessWorkspace& lay,
                           unsigned char* wsb, const RunArgs& a) {
  NvtxRange nvtx("compile_and_sort");
  ProgHdr* hdr = reinterpret_cast<ProgHdr*>(wsb + lay.hdr_off);
  Instr<T>* tape = reinterpret_cast<Instr<T>*>(wsb + lay.tape_off);
  unsigned* cnt = reinterpret_cast<unsigned*>(wsb + lay.cnt_off);
  unsigned* misc = reinterpret_cast<unsigned*>(wsb + lay.misc_off);
  int64_t* perm = reinterpret_cast<int64_t*>(wsb + lay.perm_off);
  unsigned* bins = reinterpret_cast<unsigned*>(wsb + lay.bins_off);
  const ProbDesc<T>* desc = reinterpret_cast<const ProbDesc<T>*>(wsb + lay.desc_off);
  const TokenLut* luts = reinterpret_cast<const TokenLut*>(wsb + lay.lut_off);
  int32_t* prob_of = reinterpret_cast<int32_t*>(wsb + lay.probof_off);
  if (a.phase != WS_PHASE_EVALUATE) {
    int64_t hgrid = (total_B + 4095) / 4096;
    if (hgrid < 1) hgrid = 1;
    if (hgrid > (int64_t)device_info().sm_count * 8) hgrid = (int64_t)device_info().sm_count * 8;
    const int64_t per_block = (total_B + hgrid - 1) / hgrid;
    // order programs by the key in hdr (per problem, descending, invalid last) into perm
    auto sort = [&]() -> ws_status {
      cudaError_t e0 = cudaMemsetAsync(bins, 0, (size_t)a.n_desc * kSortBins * sizeof(unsigned),
                                       a.stream);
      if (e0 != cudaSuccess) return fail_cuda(e0, "sort-bin reset");
      sort_hist_kernel<<<(unsigned)hgrid, 256, 0, a.stream>>>(hdr, prob_of, total_B, per_block,
                                                              bins);
      sort_scan_kernel<<<1, 1024, 0, a.stream>>>(bins, a.n_desc);
      sort_scatter_kernel<<<(unsigned)hgrid, 256, 0, a.stream>>>(hdr, prob_of, total_B,
                                                                 per_block, bins, perm);
      const cudaError_t e = cudaGetLastError();
      return e == cudaSuccess ? WS_OK : fail_cuda(e, "sort kernels launch");
    };
    // 1. token counts, ordered: the compile takes programs of similar length per warp
    const int64_t cg = (total_B + 255) / 256;
    count_kernel<T><<<(unsigned)(cg < 4096 ? cg : 4096), 256, 0, a.stream>>>(
        desc, a.n_desc, luts, total_B, (int)a.L, hdr, prob_of);
    ws_status st = sort();
    if (st != WS_OK) return st;
    // 2. compile in that order
    const int ct = 128;
    const unsigned grid = (unsigned)((total_B + ct - 1) / ct);
    if (a.L <= 64)
      compile_kernel<T, STRICT, 64><<<grid, ct, 0, a.stream>>>(
          desc, luts, total_B, (int)a.L, tape, Lcap, hdr, prob_of, perm, cnt, misc, S);
    else
      compile_kernel<T, STRICT, 256><<<grid, ct, 0, a.stream>>>(
          desc, luts, total_B, (int)a.L, tape, Lcap, hdr, prob_of, perm, cnt, misc, S);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "compile_kernel launch");
    // 3. evaluation order: tape length (measured 2% faster on the scale workload than token
    // count: the tape, not the token count, is what a warp runs)
    st = sort();
    if (st != WS_OK) return st;
  }
  if (a.phase == WS_PHASE_EVALUATE) {  // the compile kernel is what resets the queue head
    cudaError_t e = cudaMemsetAsync(misc, 0, 16, a.stream);
    if (e != cudaSuccess) return fail_cuda(e, "work-queue reset");
    // a cancelled launch can leave split counters mid-count (the last split of a program is
    // what zeroes its counter): with a cancel flag attached they are reset every launch
    if (a.cancel) {
      e = cudaMemsetAsync(cnt, 0, (size_t)total_B * sizeof(unsigned), a.stream);
      if (e != cudaSuccess) return fail_cuda(e, "split-counter reset");
    }
  }
  return WS_OK;
}

// The launch sequence of a plan whose descriptors and token tables are in the workspace:
// compile + length sort (unless evaluate-only), then the evaluator.  Kernels and memsets only,
// so a CUDA graph can capture it.
template <typename T, int R, bool STRICT>
ws_status run_plan(const Plan& pl, const FitnessWorkspace& lay, unsigned char* wsb,
                   const RunArgs& a) {
  ProgHdr* hdr = reinterpret_cast<ProgHdr*>(wsb + lay.hdr_off);
  Instr<T>* tape = reinterpret_cast<Instr<T>*>(wsb + lay.tape_off);
  PartRec* part = reinterpret_cast<PartRec*>(wsb + lay.part_off);
  unsigned* cnt = reinterpret_cast<unsigned*>(wsb + lay.cnt_off);
  unsigned* misc = reinterpret_cast<unsigned*>(wsb + lay.misc_off);
  int64_t* perm = reinterpret_cast<int64_t*>(wsb + lay.perm_off);
  T* gspill = reinterpret_cast<T*>(wsb + lay.gspill_off);
  const ProbDesc<T>* desc = reinterpret_cast<const ProbDesc<T>*>(wsb + lay.desc_off);
  double* yvar = reinterpret_cast<double*>(wsb + lay.yvar_off);
  if (pl.total_B == 0) return WS_OK;

  // 1. compile, then order the programs by (problem, tape length)
  ws_status st = compile_and_sort<T, STRICT>(pl.total_B, pl.Lcap, pl.S, lay, wsb, a);
  if (st != WS_OK || a.phase == WS_PHASE_COMPILE) return st;
  if (a.loss == WS_LOSS_R2) {
    yvar_kernel<T><<<a.n_desc, 256, 0, a.stream>>>(desc, yvar);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "yvar_kernel launch");
  }

  // 2. evaluate
  NvtxRange nvtx("evaluate");
  FitParams<T> P;
  P.desc = desc;
  P.n_prob = a.n_desc;
  P.tape = tape;
  P.hdr = hdr;
  P.Lcap = pl.Lcap;
  P.PB = pl.PB;
  P.n_items = pl.n_items;
  P.tile_cap = pl.tile_cap;
  P.S = pl.S;
  P.policy = a.policy;
  P.loss = a.loss;
  P.invalid_value = a.invalid_value;
  P.part = part;
  P.prog_cnt = cnt;
  P.work = misc;
  P.yvar = a.loss == WS_LOSS_R2 ? yvar : nullptr;
  P.perm = perm;
  P.gspill = gspill;
  P.cancel = a.cancel;
  const int64_t grid = pl.n_items < pl.n_ctas ? pl.n_items : pl.n_ctas;
  if (grid <= 0) return WS_OK;
  fitness_kernel<T, R, STRICT><<<(unsigned)grid, pl.W * 32, pl.smem, a.stream>>>(P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "fitness_kernel launch");
  return WS_OK;
}

// Calls f(TypeTag<T>, integral_constant<int, R>, integral_constant<bool, STRICT>) for the
// element type, operator mode and rows per lane of a request.  FP64 runs R = 8 (16 doubles per
// operand array would spill registers); 32-row passes are compiled for the protected operators
// only.
template <class T> struct TypeTag { using type = T; };
template <int R> using RowsTag = std::integral_constant<int, R>;
template <class F>
ws_status dispatch(int dtype, bool strict, const Sched& sc, F&& f) {
  if (dtype == WS_F64) {
    if (strict) return f(TypeTag<double>(), RowsTag<8>(), std::true_type());
    return f(TypeTag<double>(), RowsTag<8>(), std::false_type());
  }
  if (strict) {
    if (sc.R == 8) return f(TypeTag<float>(), RowsTag<8>(), std::true_type());
    return f(TypeTag<float>(), RowsTag<16>(), std::true_type());
  }
  if (sc.R == 8) return f(TypeTag<float>(), RowsTag<8>(), std::false_type());
  if (sc.R == 32) return f(TypeTag<float>(), RowsTag<32>(), std::false_type());
  return f(TypeTag<float>(), RowsTag<16>(), std::false_type());
}
#define WS_DISPATCH_TYPES                        \
  using T = typename decltype(tt_)::type;        \
  constexpr int R = decltype(rr_)::value;        \
  constexpr bool S = decltype(ss_)::value;

// Opaque batch handle behind the ws_batch_* entry points.
struct BatchState {
  int dtype = WS_F32, strict = 0, n_desc = 0;
  int policy = WS_POLICY_CLASSIC, loss = WS_LOSS_MSE;
  double invalid_value = 0.0;
  int64_t L = 0;
  Sched sc{};
  Plan plan;
  FitnessWorkspace lay{};
  unsigned char* wsb = nullptr;
  const int32_t* cancel = nullptr;  // ws_batch_set_cancel
};

}  // namespace

int schedule_count() { return kNumSched + kNumSmall; }

FitnessWorkspace fitness_workspace_layout(int64_t total_B, int64_t L, int dtype, int64_t n_prob,
                                          int64_t n_part) {
  FitnessWorkspace w;
  const size_t instr = dtype == WS_F64 ? sizeof(Instr<double>) : sizeof(Instr<float>);
  const int64_t Lcap = tape_capacity(L < 0 ? 0 : (L > 256 ? 256 : (int)L));
  if (n_prob < 1) n_prob = 1;
  size_t off = 0;
  w.hdr_off = off;
  off = align_up(off + (size_t)total_B * sizeof(ProgHdr), 256);
  w.tape_off = off;
  off = align_up(off + (size_t)total_B * Lcap * instr, 256);
  w.max_partials = n_part;
  w.part_off = off;
  off = align_up(off + (size_t)n_part * sizeof(PartRec), 256);
  w.cnt_off = off;
  off = align_up(off + (size_t)total_B * sizeof(unsigned), 256);
  w.misc_off = off;
  off = align_up(off + 256, 256);
  w.perm_off = off;
  off = align_up(off + (size_t)total_B * sizeof(int64_t), 256);
  w.bins_off = off;
  off = align_up(off + (size_t)n_prob * kSortBins * sizeof(unsigned), 256);
  w.probof_off = off;
  off = align_up(off + (size_t)total_B * sizeof(int32_t), 256);
  w.desc_off = off;
  off = align_up(off + (size_t)n_prob * sizeof(ProbDesc<double>), 256);
  w.lut_off = off;
  off = align_up(off + (size_t)n_prob * sizeof(TokenLut), 256);
  w.yvar_off = off;
  off = align_up(off + (size_t)n_prob * sizeof(double), 256);
  // deep spill slots: 32 resident warps per SM (the schedules run at most that many; the
  // launcher caps its grid otherwise), one pass of 512 rows per slot
  const int Lc = L < 0 ? 0 : (L > 256 ? 256 : (int)L);
  const int deep = spill_slots_bound(Lc) > kSharedSlots ? spill_slots_bound(Lc) - kSharedSlots : 0;
  const size_t tsz = dtype == WS_F64 ? sizeof(double) : sizeof(float);
  w.gspill_bytes = (size_t)device_info().sm_count * 32 * (size_t)deep * 512 * tsz;
  w.gspill_off = off;
  off = align_up(off + w.gspill_bytes, 256);
  w.total = off;
  return w;
}

FitnessWorkspace fitness_workspace_layout(int64_t B, int64_t L, int dtype) {
  return fitness_workspace_layout(B, L, dtype, 1, B > 65536 ? B : 65536);
}

// ---- small data sets (fitness_small_kernel) --------------------------------------------------
// Schedule index kNumSched + j runs the small-data-set evaluator with S = 2 << j lanes per program
// (rows per program 4S = 8, 16, 32, 64, 128); the automatic choice (index 0) takes it for
// 1 <= D <= 128 with the smallest S that covers D.
int small_lanes(int schedule, int64_t D) {
  if (schedule >= kNumSched && schedule < kNumSched + kNumSmall) return 2 << (schedule - kNumSched);
  if (schedule == 0 && D >= 1 && D <= 128) {
    int s = 2;
    while (4 * s < D) s <<= 1;
    return s;
  }
  return 0;
}

template <typename T, int S, bool STRICT>
size_t small_max_dynamic_smem() {
  static std::mutex mu;
  static size_t cache[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> g(mu);
  if (cache[dev] == 0) {
    cudaFuncAttributes fa;
    size_t stat = 0;
    if (cudaFuncGetAttributes(&fa, fitness_small_kernel<T, S, STRICT>) == cudaSuccess)
      stat = fa.sharedSizeBytes;
    size_t lim = device_info().smem_optin > stat ? device_info().smem_optin - stat : 0;
    if (cudaFuncSetAttribute(fitness_small_kernel<T, S, STRICT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim) != cudaSuccess) {
      (void)cudaGetLastError();
      lim = 48 * 1024 - stat;
    }
    cache[dev] = lim;
  }
  return cache[dev];
}

template <typename T, int S, bool STRICT>
ws_status launch_small(const FitnessRequest& rq, const ProblemRequest& pr,
                       const FitnessWorkspace& lay) {
  constexpr int PW = 32 / S;
  if (4 * (int64_t)S < rq.D) return fail("this schedule covers fewer rows than the data set");
  unsigned char* wsb = static_cast<unsigned char*>(rq.workspace);
  const int W = S <= 4 ? 4 : 8;
  const int Lcap = tape_capacity(rq.L < 256 ? (int)rq.L : 256);
  int NS = spill_slots_bound((int)rq.L);
  if (NS < 1) NS = 1;
  const int PB = W * PW;
  const int64_t n_items = (rq.B + PB - 1) / PB;
  const size_t smem = (size_t)(rq.V + 1) * 4 * S * sizeof(T) + (size_t)W * NS * 32 * 4 * sizeof(T) +
                      (size_t)PB * (Lcap + 1) * sizeof(Instr<T>) + (size_t)PB * sizeof(int);
  if (smem > small_max_dynamic_smem<T, S, STRICT>())
    return fail("too many variables for the small-data-set evaluator");
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fitness_small_kernel<T, S, STRICT>,
                                                    W * 32, smem) != cudaSuccess) {
    (void)cudaGetLastError();
    occ = 0;
  }
  if (occ <= 0) return fail("small-data-set evaluator cannot be resident");
  ProbPlan pp;
  pp.RC = 4 * S;
  pp.xmul = 1;  // tape operand offsets count variables (rows of 4S elements)
  pp.n_chunks = 1;
  pp.cps = 1;
  pp.n_splits = 1;
  pp.n_blocks = n_items;
  const ProbDesc<T> d = make_desc<T>(pr, pp);
  write_desc_kernel<T><<<1, 128, 0, rq.stream>>>(
      d, pr.lut, reinterpret_cast<ProbDesc<T>*>(wsb + lay.desc_off),
      reinterpret_cast<TokenLut*>(wsb + lay.lut_off));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "descriptor write");
  if (rq.B == 0) return WS_OK;
  RunArgs a{rq.L, 1, rq.phase, rq.policy, rq.loss, rq.invalid_value, rq.stream};
  ws_status st = compile_and_sort<T, STRICT>(rq.B, Lcap, NS, lay, wsb, a);
  if (st != WS_OK || rq.phase == WS_PHASE_COMPILE) return st;
  const ProbDesc<T>* desc = reinterpret_cast<const ProbDesc<T>*>(wsb + lay.desc_off);
  double* yvar = reinterpret_cast<double*>(wsb + lay.yvar_off);
  if (rq.loss == WS_LOSS_R2) {
    yvar_kernel<T><<<1, 256, 0, rq.stream>>>(desc, yvar);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "yvar_kernel launch");
  }
  NvtxRange nvtx("evaluate");
  FitParams<T> P{};
  P.desc = desc;
  P.n_prob = 1;
  P.tape = reinterpret_cast<const Instr<T>*>(wsb + lay.tape_off);
  P.hdr = reinterpret_cast<const ProgHdr*>(wsb + lay.hdr_off);
  P.Lcap = Lcap;
  P.PB = PB;
  P.n_items = n_items;
  P.S = NS;
  P.policy = rq.policy;
  P.loss = rq.loss;
  P.invalid_value = rq.invalid_value;
  P.work = reinterpret_cast<unsigned*>(wsb + lay.misc_off);
  P.yvar = rq.loss == WS_LOSS_R2 ? yvar : nullptr;
  P.perm = reinterpret_cast<const int64_t*>(wsb + lay.perm_off);
  const int64_t cap = (int64_t)occ * device_info().sm_count;
  const int64_t grid = n_items < cap ? n_items : cap;
  fitness_small_kernel<T, S, STRICT><<<(unsigned)grid, W * 32, smem, rq.stream>>>(P);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "fitness_small_kernel launch");
  return WS_OK;
}

template <typename T, bool STRICT>
ws_status launch_small_s(int S, const FitnessRequest& rq, const ProblemRequest& pr,
                         const FitnessWorkspace& lay) {
  switch (S) {
    case 2: return launch_small<T, 2, STRICT>(rq, pr, lay);
    case 4: return launch_small<T, 4, STRICT>(rq, pr, lay);
    case 8: return launch_small<T, 8, STRICT>(rq, pr, lay);
    case 16: return launch_small<T, 16, STRICT>(rq, pr, lay);
    default: return launch_small<T, 32, STRICT>(rq, pr, lay);
  }
}

ws_status launch_fitness(const FitnessRequest& rq) {
  NvtxRange nvtx("ws_eval_fitness");
  const FitnessWorkspace lay = fitness_workspace_layout(rq.B, rq.L, rq.dtype);
  ProblemRequest pr;
  pr.pop = rq.pop;
  pr.B = rq.B;
  pr.x = rq.x;
  pr.V = rq.V;
  pr.D = rq.D;
  pr.consts = rq.consts;
  pr.K = rq.K;
  pr.y = rq.y;
  pr.out_loss = rq.out_loss;
  pr.out_ninv = rq.out_ninv;
  pr.lut = rq.lut;
  const int small = small_lanes(rq.schedule, rq.D);
  if (small > 0) {
    if (rq.dtype == WS_F64)
      return rq.strict ? launch_small_s<double, true>(small, rq, pr, lay)
                       : launch_small_s<double, false>(small, rq, pr, lay);
    return rq.strict ? launch_small_s<float, true>(small, rq, pr, lay)
                     : launch_small_s<float, false>(small, rq, pr, lay);
  }
  const Sched sc = pick_schedule(rq.schedule, rq.D);
  unsigned char* wsb = static_cast<unsigned char*>(rq.workspace);
  return dispatch(rq.dtype, rq.strict != 0, sc, [&](auto tt_, auto rr_, auto ss_) -> ws_status {
    WS_DISPATCH_TYPES
    Plan pl;
    ws_status st = make_plan<T, R, S>(&pr, 1, rq.L, sc, lay.max_partials, lay.gspill_bytes, pl);
    if (st != WS_OK) return st;
    const ProbDesc<T> d = make_desc<T>(pr, pl.pp[0]);
    write_desc_kernel<T><<<1, 128, 0, rq.stream>>>(
        d, pr.lut, reinterpret_cast<ProbDesc<T>*>(wsb + lay.desc_off),
        reinterpret_cast<TokenLut*>(wsb + lay.lut_off));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "descriptor write");
    RunArgs a{rq.L, 1, rq.phase, rq.policy, rq.loss, rq.invalid_value, rq.stream};
    return run_plan<T, R, S>(pl, lay, wsb, a);
  });
}

// ---- batches of problems (one launch sequence for all of them) --------------------------------
static Sched batch_schedule(const ProblemRequest* probs, int n, int schedule) {
  int64_t dmax = 0;
  for (int i = 0; i < n; ++i) dmax = probs[i].D > dmax ? probs[i].D : dmax;
  return pick_schedule(schedule, dmax);
}

ws_status batch_workspace_bytes(int dtype, const ProblemRequest* probs, int n, int64_t L,
                                int strict, int schedule, size_t* out) {
  if (schedule >= kNumSched) return fail("the small-data-set schedules take one problem per call");
  const Sched sc = batch_schedule(probs, n, schedule);
  return dispatch(dtype, strict != 0, sc, [&](auto tt_, auto rr_, auto ss_) -> ws_status {
    WS_DISPATCH_TYPES
    int64_t tb = 0;
    for (int i = 0; i < n; ++i) tb += probs[i].B;
    // the spill scratch does not depend on the plan: size it first, then plan against it
    const FitnessWorkspace probe = fitness_workspace_layout(tb, L, dtype, n, 0);
    Plan pl;
    ws_status st = make_plan<T, R, S>(probs, n, L, sc, -1, probe.gspill_bytes, pl);
    if (st != WS_OK) return st;
    *out = fitness_workspace_layout(tb, L, dtype, n, pl.n_part).total;
    return WS_OK;
  });
}

ws_status batch_create(int dtype, const ProblemRequest* probs, int n, int64_t L, int strict,
                       int policy, int loss, int schedule, double invalid_value, void* workspace,
                       size_t workspace_bytes, cudaStream_t stream, void** out) {
  if (schedule >= kNumSched) return fail("the small-data-set schedules take one problem per call");
  const Sched sc = batch_schedule(probs, n, schedule);
  BatchState* bs = new BatchState();
  bs->dtype = dtype;
  bs->strict = strict;
  bs->policy = policy;
  bs->loss = loss;
  bs->invalid_value = invalid_value;
  bs->L = L;
  bs->sc = sc;
  bs->wsb = static_cast<unsigned char*>(workspace);
  ws_status st = dispatch(dtype, strict != 0, sc, [&](auto tt_, auto rr_, auto ss_) -> ws_status {
    WS_DISPATCH_TYPES
    int64_t tb = 0;
    for (int i = 0; i < n; ++i) tb += probs[i].B;
    const FitnessWorkspace probe = fitness_workspace_layout(tb, L, dtype, n, 0);
    ws_status s2 = make_plan<T, R, S>(probs, n, L, sc, -1, probe.gspill_bytes, bs->plan);
    if (s2 != WS_OK) return s2;
    bs->n_desc = (int)bs->plan.order.size();
    bs->lay = fitness_workspace_layout(tb, L, dtype, n, bs->plan.n_part);
    if (!workspace || workspace_bytes < bs->lay.total) {
      set_error("workspace of " + std::to_string(bs->lay.total) + " bytes required (got " +
                std::to_string(workspace_bytes) + ")");
      return WS_ERR_WORKSPACE;
    }
    if (((uintptr_t)workspace & 255u) != 0) {
      set_error("workspace must be 256-byte aligned");
      return WS_ERR_WORKSPACE;
    }
    std::vector<ProbDesc<T>> descs;
    std::vector<TokenLut> luts;
    for (int i : bs->plan.order) {
      descs.push_back(make_desc<T>(probs[i], bs->plan.pp[i]));
      luts.push_back(probs[i].lut);
    }
    for (size_t b0 = 0; b0 < descs.size(); b0 += kUploadChunk) {
      DescChunk<T> ch;
      std::memset(&ch, 0, sizeof(ch));
      ch.base = (int)b0;
      ch.n = (int)std::min(descs.size() - b0, (size_t)kUploadChunk);
      for (int j = 0; j < ch.n; ++j) {
        ch.d[j] = descs[b0 + j];
        ch.lut[j] = luts[b0 + j];
      }
      upload_desc_kernel<T><<<1, 128, 0, stream>>>(
          ch, reinterpret_cast<ProbDesc<T>*>(bs->wsb + bs->lay.desc_off),
          reinterpret_cast<TokenLut*>(bs->wsb + bs->lay.lut_off));
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return fail_cuda(e, "batch descriptor upload");
    }
    return WS_OK;
  });
  if (st != WS_OK) {
    delete bs;
    return st;
  }
  *out = bs;
  return WS_OK;
}

ws_status batch_eval(void* handle, int phase, cudaStream_t stream) {
  NvtxRange nvtx("ws_batch_eval");
  BatchState* bs = static_cast<BatchState*>(handle);
  return dispatch(bs->dtype, bs->strict != 0, bs->sc, [&](auto tt_, auto rr_, auto ss_) -> ws_status {
    WS_DISPATCH_TYPES
    RunArgs a{bs->L, bs->n_desc, phase, bs->policy, bs->loss, bs->invalid_value, stream,
              bs->cancel};
    return run_plan<T, R, S>(bs->plan, bs->lay, bs->wsb, a);
  });
}

void batch_set_cancel(void* handle, const int32_t* flag) {
  static_cast<BatchState*>(handle)->cancel = flag;
}

void batch_destroy(void* handle) { delete static_cast<BatchState*>(handle); }

int64_t batch_info(void* handle, int what) {
  const BatchState* bs = static_cast<const BatchState*>(handle);
  switch (what) {
    case 0: return bs->plan.n_items;
    case 1: return bs->plan.R;
    case 2: return bs->plan.PB;
    case 3: return (int64_t)bs->plan.smem;
    case 4: return bs->plan.n_ctas;
    case 5: return bs->plan.total_B;
    default: return -1;
  }
}

}  // namespace ws
