// ws_fitness.cu -- batched RPN evaluation fused with the per-program loss (the hot path).
//
// Replaces rpn_eval_fused_kernel (rpn_kernels.cu:2259-2502) and the classic chunked path of
// GPUEvaluator.evaluate_batch (rpn_eval_kernel + torch reductions, evaluation.py:128-198) with
// one pipeline that has neither the fused envelope (<=4 variables, D<=1024) nor the classic
// path's [B, D] materialisation:
//
//   1. compile_kernel  -- one thread per program: tokens -> accumulator-machine tape
//                         (ws_compile.cuh), constant slots baked, constants folded.
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
// per-program per-lane partial sums: row stride of 33 doubles (conflict-free column reads)
constexpr int kLaneStride = 33;
// shared meta word of a staged program: tape length, and a flag for global spill slots
constexpr int kMetaLenMask = 0xFFFF;
constexpr int kMetaGlobalSpill = 1 << 16;

// ---------------------------------------------------------------------------------------
// 1. compile
template <typename T, bool STRICT, int LMAX>
__global__ void __launch_bounds__(128) compile_kernel(const uint8_t* __restrict__ pop, int64_t B,
                                                      int L, const T* __restrict__ consts, int K,
                                                      TokenLut lut, Instr<T>* __restrict__ tape,
                                                      int Lcap, ProgHdr* __restrict__ hdr,
                                                      unsigned* __restrict__ prog_cnt,
                                                      unsigned* __restrict__ misc, int S,
                                                      int xmul) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) misc[0] = 0u;  // work-queue head of the evaluator launch that follows
  if (p >= B) return;
  ProgHdr h = compile_program<T, STRICT, true, LMAX>(pop + p * (int64_t)L, L,
                                                      K > 0 ? consts + p * (int64_t)K : nullptr,
                                                      K, lut, tape + p * (int64_t)Lcap, xmul);
  // Neither can happen (Sethi-Ullman bound; chunk size chosen for the offsets): guard anyway.
  if ((h.status == PROG_OK && h.n_slots > S) || h.status == PROG_UNREPRESENTABLE) {
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
  const int64_t* perm;  // programs in evaluation order (sorted by tape length)
  T* gspill;            // per-warp scratch for spill slots beyond the shared ones
  int count;            // 1: exact per-row invalid counts (out_ninv requested)
  int async_stage;      // 1: chunk rows are 16-byte aligned -> cp.async staging
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
                                         T* __restrict__ gb, T (&acc)[R], uint32_t& err) {
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
    if (c & P_SLOW) {  // spill, accumulator load, deep spill slot: rare
      if (c & P_SPILL) {
        const uint32_t sl = (c >> P_SH_SLOT) & 7u;
        if (sl < (uint32_t)kSharedSlots) lane_store<T, R>(sb + sl * PASS, acc);
        else lane_store<T, R>(gb + (sl - kSharedSlots) * PASS, acc);
      }
      if (c & P_LOADA_X) {
        lane_load<T, R>(acc, xb + ((c >> P_SH_LA) & P_OFF_MASK) * PASS);
      } else if (c & P_LOADA_S) {
#pragma unroll
        for (int k = 0; k < R; ++k) acc[k] = ins.imm;
      }
      const uint32_t off = c >> P_SH_V;
      if ((c & P_FETCH_SLOT) && off >= (uint32_t)kSharedSlots) vp = gb + (off - kSharedSlots) * PASS;
    }
    exec_case<T, R, STRICT>(c & P_CASE_MASK, ins.imm, GenericOperand<T>{vp}, acc, err);
  }
}

// The FP32 interpreter for programs whose spill slots are all in shared memory (every program
// but the deepest 0.2%): operands, spill slots and tape words are addressed as 32-bit shared
// addresses.  xa: X tile at this pass and lane; sa: this warp's spill slot 0 at this lane; ta:
// the tape.  One pass is 32*R rows = PASS*4 bytes = 1 << PSH.
template <int R, bool STRICT>
__device__ __forceinline__ void run_tape_shared(uint32_t ta, int n, uint32_t xa, uint32_t sa,
                                                float (&acc)[R], uint32_t& err) {
  static_assert(R == 8 || R == 16 || R == 32, "pass size");
  constexpr int PSH = R == 8 ? 10 : (R == 16 ? 11 : 12);
  err = 0u;
  // software-pipelined decode: the next word is broadcast and its operand address computed
  // while the current case executes; the word after it is already in flight
  uint32_t nc, ni, c1, n1;
  lds_word(c1, n1, ta);
  lds_word(nc, ni, ta + 8u);
  uint32_t cn = __shfl_sync(0xFFFFFFFFu, c1, 0);  // warp-uniform by construction
  float sn = __uint_as_float(n1);
  uint32_t van = ((cn & P_FETCH_SLOT) ? sa : xa) + ((cn >> P_SH_V) << PSH);
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const uint32_t c = cn;
    const float s = sn;
    const uint32_t va = van;
    cn = __shfl_sync(0xFFFFFFFFu, nc, 0);
    sn = __uint_as_float(ni);
    van = ((cn & P_FETCH_SLOT) ? sa : xa) + ((cn >> P_SH_V) << PSH);
    ta += 8u;
    lds_word(nc, ni, ta + 8u);  // up to two words past the end: inside the block's smem
    if (c & P_SLOW) {  // spill, accumulator load: rare
      if (c & P_SPILL) {
        const uint32_t a = sa + (((c >> P_SH_SLOT) & 7u) << PSH);
#pragma unroll
        for (int g = 0; g < R / 4; ++g)
          sts4(a + g * 512, acc[4 * g], acc[4 * g + 1], acc[4 * g + 2], acc[4 * g + 3]);
      }
      if (c & P_LOADA_X) {
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
__device__ __forceinline__ void stage_chunk(const FitParams<T>& P, int64_t c, T* tb, int tid,
                                            int nthreads) {
  constexpr int VE = 16 / (int)sizeof(T);
  const int64_t row0 = c * P.RC;
  const int rows = (int)min((int64_t)P.RC, P.D - row0);
  if (P.async_stage) {
    const int nvec = rows / VE;
    for (int v = 0; v <= P.V; ++v) {
      const T* src = (v < P.V ? P.x + (size_t)v * P.D : P.y) + row0;
      T* dst = tb + (size_t)v * P.RC;
      for (int i = tid; i < nvec; i += nthreads) cp_async16(dst + i * VE, src + i * VE);
    }
  } else {
    for (int v = 0; v <= P.V; ++v) {
      const T* src = (v < P.V ? P.x + (size_t)v * P.D : P.y) + row0;
      T* dst = tb + (size_t)v * P.RC;
      for (int r = tid; r < P.RC; r += nthreads) dst[r] = (r < rows) ? src[r] : (T)0;
    }
  }
  cp_async_commit();
}

template <typename T, int R, bool STRICT>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 && R <= 16) ? 3 : 2) fitness_kernel(const FitParams<T> P) {
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
  const size_t tile_elems = (size_t)(P.V + 1) * P.RC;
  T* tiles = reinterpret_cast<T*>(smem_raw);
  T* spill = tiles + 2 * tile_elems;
  Instr<T>* tapes = reinterpret_cast<Instr<T>*>(spill + (size_t)W * kSharedSlots * PASS);
  PartRec* acc_s = reinterpret_cast<PartRec*>(tapes + (size_t)P.PB * P.Lcap);
  double* lane_sse = reinterpret_cast<double*>(acc_s + P.PB);  // [PB][kLaneStride]
  int* meta_s = reinterpret_cast<int*>(lane_sse + (size_t)P.PB * kLaneStride);
  __shared__ int64_t s_item;

  T* sp_w = spill + (size_t)warp * kSharedSlots * PASS + lane * N;
  const int deep = P.S > kSharedSlots ? P.S - kSharedSlots : 0;
  T* gsp_w = P.gspill + ((size_t)blockIdx.x * W + warp) * (size_t)deep * PASS + lane * N;
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
    // stage the block's tapes once for all its chunks (programs arrive sorted by tape length,
    // so a static warp assignment is balanced)
    for (int q = warp; q < np; q += W) {
      const int64_t p = P.perm[p0 + q];
      const ProgHdr h = P.hdr[p];
      const Instr<T>* tg = P.tape + p * (int64_t)P.Lcap;
      for (int i = lane; i < h.n_instr; i += 32) tapes[(size_t)q * P.Lcap + i] = tg[i];
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
    stage_chunk<T>(P, c0, tiles, threadIdx.x, blockDim.x);
    for (int64_t c = c0; c < c1; ++c) {
      T* xs = tiles + (size_t)buf * tile_elems;
      T* ys = xs + (size_t)P.V * P.RC;
      if (c + 1 < c1) {  // the next chunk streams in while this one is evaluated
        stage_chunk<T>(P, c + 1, tiles + (size_t)(buf ^ 1) * tile_elems, threadIdx.x, blockDim.x);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      const int64_t row0 = c * P.RC;
      const int rows = (int)min((int64_t)P.RC, P.D - row0);
      if (P.async_stage && rows < P.RC) {  // zero the rows past the end of the data
        for (int v = 0; v <= P.V; ++v)
          for (int r = rows + threadIdx.x; r < P.RC; r += blockDim.x) xs[(size_t)v * P.RC + r] = (T)0;
      }
      __syncthreads();  // chunk c visible to all warps; tapes and accumulators ready
      const int npass = (rows + PASS - 1) / PASS;

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
          if constexpr (F32) {
            if (shared_only)
              run_tape_shared<R, STRICT>(smem_u32(tape_q), n_instr,
                                         smem_u32(xs + pass * PASS + lane * N), smem_u32(sp_w),
                                         *reinterpret_cast<float(*)[R]>(&a), err);
            else
              run_tape<T, R, STRICT>(tape_q, n_instr, xs + pass * PASS + lane * N, sp_w, gsp_w,
                                     a, err);
          } else {
            run_tape<T, R, STRICT>(tape_q, n_instr, xs + pass * PASS + lane * N, sp_w, gsp_w, a,
                                   err);
          }
          const T* yb = ys + pass * PASS + lane * N;
          T part;
          if (!P.count && (pass + 1) * PASS <= rows) {
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
        if (P.count) {
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
      buf ^= 1;
    }
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
      const int64_t p = P.perm[p0 + q];
      PartRec r = acc_s[q];
      double t = 0.0;  // lanes combined in a fixed order
      for (int l = 0; l < 32; ++l) t += lane_sse[q * kLaneStride + l];
      r.sse = t;
      if (P.n_splits == 1) {
        write_final<T>(P, p, r);
      } else {
        P.part[p * P.n_splits + split] = r;
        __threadfence();
        const unsigned done = atomicAdd(&P.prog_cnt[p], 1u);
        if (done == (unsigned)P.n_splits - 1u) {
          __threadfence();
          PartRec t2{0.0, 0, 0};
          for (int s2 = 0; s2 < P.n_splits; ++s2) {
            const PartRec* pr = &P.part[p * P.n_splits + s2];
            t2.sse += __ldcg(&pr->sse);
            t2.ninv += __ldcg(&pr->ninv);
            t2.ovf |= __ldcg(&pr->ovf);
          }
          write_final<T>(P, p, t2);
          P.prog_cnt[p] = 0u;  // ready for an evaluate-only rerun on the same tape
        }
      }
    }
    // the next item's staging waits on the __syncthreads() at the loop top
    __syncthreads();
  }
}

// ---- length-sorted schedule: counting sort of programs by tape length (longest first) ------
constexpr int kSortBins = 258;  // tape lengths 0..256, plus invalid programs

__global__ void __launch_bounds__(256) sort_hist_kernel(const ProgHdr* __restrict__ hdr, int64_t B,
                                                        unsigned* __restrict__ bins) {
  __shared__ unsigned h[kSortBins];
  for (int i = threadIdx.x; i < kSortBins; i += blockDim.x) h[i] = 0u;
  __syncthreads();
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < B;
       p += (int64_t)gridDim.x * blockDim.x) {
    const ProgHdr v = hdr[p];
    const int key = v.status == PROG_OK ? min(v.n_instr, 256) : 257;
    atomicAdd(&h[key], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kSortBins; i += blockDim.x)
    if (h[i]) atomicAdd(&bins[i], h[i]);
}

// Exclusive offsets in descending tape length, invalid programs last (single block).
__global__ void __launch_bounds__(32) sort_scan_kernel(unsigned* __restrict__ bins) {
  if (threadIdx.x == 0) {
    unsigned run = 0u;
    for (int key = 256; key >= 0; --key) {
      const unsigned c = bins[key];
      bins[key] = run;
      run += c;
    }
    bins[257] = run;
  }
}

__global__ void __launch_bounds__(256) sort_scatter_kernel(const ProgHdr* __restrict__ hdr,
                                                           int64_t B, unsigned* __restrict__ bins,
                                                           int64_t* __restrict__ perm) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < B;
       p += (int64_t)gridDim.x * blockDim.x) {
    const ProgHdr v = hdr[p];
    const int key = v.status == PROG_OK ? min(v.n_instr, 256) : 257;
    const unsigned pos = atomicAdd(&bins[key], 1u);
    perm[pos] = p;
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
    {16, 8, 24, 72 * 1024},   // 0: auto placeholder (resolved by pick_schedule)
    {8, 8, 32, 72 * 1024},    // 1
    {16, 4, 16, 56 * 1024},   // 2
    {16, 8, 24, 72 * 1024},   // 3
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

template <typename T, int R, bool STRICT>
ws_status launch_typed(const FitnessRequest& rq, const Sched& sc) {
  const FitnessWorkspace lay = fitness_workspace_layout(rq.B, rq.L, rq.dtype);
  unsigned char* wsb = static_cast<unsigned char*>(rq.workspace);
  ProgHdr* hdr = reinterpret_cast<ProgHdr*>(wsb + lay.hdr_off);
  Instr<T>* tape = reinterpret_cast<Instr<T>*>(wsb + lay.tape_off);
  PartRec* part = reinterpret_cast<PartRec*>(wsb + lay.part_off);
  unsigned* cnt = reinterpret_cast<unsigned*>(wsb + lay.cnt_off);
  unsigned* misc = reinterpret_cast<unsigned*>(wsb + lay.misc_off);
  double* yvar = reinterpret_cast<double*>(wsb + lay.misc_off + 16);

  const int L = (int)rq.L;
  const int Lcap = tape_capacity(L < 256 ? L : 256);  // tape words per program
  const int S = spill_slots_bound(L);
  constexpr int PASS = 32 * R;
  const int W = sc.W;
  const int threads = W * 32;

  // ---- schedule: chunk rows RC (multiple of the pass), programs per block, splits ----------
  const size_t szT = sizeof(T);
  // programs per block: as the schedule says, but the staged tapes stay within 24 KB (long
  // programs get fewer per block; at least one per warp)
  int PBmax = sc.PB;
  {
    const int fit = (int)((24 * 1024) / ((size_t)Lcap * sizeof(Instr<T>)));
    if (PBmax > fit) PBmax = fit > W ? fit : W;
  }
  const size_t fixed = (size_t)W * kSharedSlots * PASS * szT +
                       (size_t)PBmax * Lcap * sizeof(Instr<T>) +
                       (size_t)PBmax * (sizeof(PartRec) + sizeof(int) + kLaneStride * sizeof(double));
  const size_t per_row = 2 * (size_t)(rq.V + 1) * szT;  // two tiles (double buffering)
  const size_t optin = max_dynamic_smem<T, R, STRICT>();
  if (fixed + per_row * PASS > optin) return fail("too many variables for the shared-memory tile");
  const size_t budget = sc.smem_budget > fixed + per_row * PASS ? sc.smem_budget
                                                                : fixed + per_row * PASS;
  int64_t rc = (int64_t)((budget - fixed) / per_row) / PASS * PASS;
  const int64_t d_pad = (rq.D + PASS - 1) / PASS * PASS;
  if (rc > d_pad) rc = d_pad;
  // tape offsets: variable v at v * (RC / PASS) must fit 9 bits
  const int64_t xmul_cap = rq.V > 0 ? (int64_t)P_OFF_MASK / rq.V : (int64_t)P_OFF_MASK;
  if (rc / PASS > xmul_cap) rc = xmul_cap * PASS;
  if (rc < PASS) rc = PASS;
  const int RC = (int)rc;
  const int xmul = RC / PASS;
  const size_t smem = fixed + per_row * (size_t)RC;
  const int occ = occupancy_for<T, R, STRICT>(smem, threads);
  if (occ <= 0) return fail("fitness kernel cannot be resident with this tile size");
  int64_t n_ctas = (int64_t)occ * device_info().sm_count;

  const T* consts = static_cast<const T*>(rq.consts);
  int64_t* perm = reinterpret_cast<int64_t*>(wsb + lay.perm_off);
  unsigned* bins = reinterpret_cast<unsigned*>(wsb + lay.bins_off);
  T* gspill = reinterpret_cast<T*>(wsb + lay.gspill_off);
  const int deep = S > kSharedSlots ? S - kSharedSlots : 0;
  if (deep > 0) {  // one global spill area per resident warp: cap the persistent grid to it
    const int64_t fit = (int64_t)(lay.gspill_bytes / ((size_t)W * deep * PASS * szT));
    if (fit < 1) return fail("workspace too small for the spill scratch of this schedule");
    if (n_ctas > fit) n_ctas = fit;
  }
  // 1. compile, then order the programs by tape length
  if (rq.phase != WS_PHASE_EVALUATE) {
    cudaError_t e0 = cudaMemsetAsync(bins, 0, kSortBins * sizeof(unsigned), rq.stream);
    if (e0 != cudaSuccess) return fail_cuda(e0, "sort-bin reset");
    const int ct = 128;
    const unsigned grid = (unsigned)((rq.B + ct - 1) / ct);
    if (L <= 64)
      compile_kernel<T, STRICT, 64><<<grid, ct, 0, rq.stream>>>(
          rq.pop, rq.B, L, consts, (int)rq.K, rq.lut, tape, Lcap, hdr, cnt, misc, S, xmul);
    else
      compile_kernel<T, STRICT, 256><<<grid, ct, 0, rq.stream>>>(
          rq.pop, rq.B, L, consts, (int)rq.K, rq.lut, tape, Lcap, hdr, cnt, misc, S, xmul);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "compile_kernel launch");
    int sgrid = (int)((rq.B + 255) / 256);
    if (sgrid > device_info().sm_count * 8) sgrid = device_info().sm_count * 8;
    sort_hist_kernel<<<sgrid, 256, 0, rq.stream>>>(hdr, rq.B, bins);
    sort_scan_kernel<<<1, 32, 0, rq.stream>>>(bins);
    sort_scatter_kernel<<<sgrid, 256, 0, rq.stream>>>(hdr, rq.B, bins, perm);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "sort kernels launch");
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

  // 2. evaluate
  const int64_t n_chunks = (rq.D + RC - 1) / RC;
  int PB = PBmax;
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
  P.perm = perm;
  P.gspill = gspill;
  P.count = rq.out_ninv != nullptr ? 1 : 0;
  {
    constexpr int64_t VE = 16 / (int64_t)sizeof(T);
    P.async_stage = (rq.D % VE == 0) && (((uintptr_t)rq.x & 15u) == 0) &&
                    (((uintptr_t)rq.y & 15u) == 0) ? 1 : 0;
  }
  const int64_t grid = P.n_items < n_ctas ? P.n_items : n_ctas;
  fitness_kernel<T, R, STRICT><<<(unsigned)grid, threads, smem, rq.stream>>>(P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "fitness_kernel launch");
  return WS_OK;
}

template <typename T, bool STRICT>
ws_status launch_sched(const FitnessRequest& rq) {
  Sched sc = pick_schedule(rq.schedule, rq.D);
  if constexpr (sizeof(T) == 8) {
    sc.R = 8;  // 16 doubles per operand array would spill registers
    return launch_typed<T, 8, STRICT>(rq, sc);
  } else {
    if (sc.R == 8) return launch_typed<T, 8, STRICT>(rq, sc);
    if constexpr (!STRICT) {
      if (sc.R == 32) return launch_typed<T, 32, STRICT>(rq, sc);
    }
    sc.R = 16;  // 32-row passes are compiled for the protected operators only
    return launch_typed<T, 16, STRICT>(rq, sc);
  }
}

}  // namespace

int schedule_count() { return kNumSched; }

FitnessWorkspace fitness_workspace_layout(int64_t B, int64_t L, int dtype) {
  FitnessWorkspace w;
  const size_t instr = dtype == WS_F64 ? sizeof(Instr<double>) : sizeof(Instr<float>);
  const int64_t Lcap = tape_capacity(L < 0 ? 0 : (L > 256 ? 256 : (int)L));
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
  w.perm_off = off;
  off = align_up(off + (size_t)B * sizeof(int64_t), 256);
  w.bins_off = off;
  off = align_up(off + kSortBins * sizeof(unsigned), 256);
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

ws_status launch_fitness(const FitnessRequest& rq) {
  if (rq.dtype == WS_F32)
    return rq.strict ? launch_sched<float, true>(rq) : launch_sched<float, false>(rq);
  return rq.strict ? launch_sched<double, true>(rq) : launch_sched<double, false>(rq);
}

}  // namespace ws
