// ws_backward.cu -- adjoint (reverse-mode) gradient of program outputs w.r.t. their constants.
//
// Replaces rpn_eval_backward_kernel / launch_rpn_backward (backward_kernels.cu:13-335) behind
// `eval_rpn_backward`: for every program b and constant slot k,
//     grad_constants[b, k] += sum_d  dL/dpred[b, d] * dpred[b, d] / dC_k
// with the reference's own forward rules (its simplified protected operators, the 32-entry
// index stack, C-slot clamping, unknown tokens acting as unary zero) and its adjoint rules
// (no gradient through %, tan, abs and the remaining unary operators; guarded div/log/sqrt/pow).
// Per-row arithmetic follows the reference expression by expression, including its mixed
// float/double promotions, so per-row adjoints are the reference's bit for bit.
//
// B200 layout: one block owns one program for a range of rows.  The program is parsed once per
// block into a shared-memory tape of its OPERATORS only, each naming its operands (an earlier
// operator, a variable, a literal or a constant slot) and whether its value reaches the root;
// terminals are read where they are used.  Every thread evaluates rows: operator values and
// adjoints live in shared memory as [operator][thread] (all lanes touch the same operator at the
// same time: conflict-free).  The program is a tree, so each node receives exactly one adjoint
// contribution: a child's slot is written with the value the reference's `+=` leaves in it
// (`0 + contribution`, or 0 where the reference adds nothing), and constant adjoints go straight
// into per-thread FP64 accumulators.  The reduction over rows is a fixed-order block
// sum, written without atomics when one block covers all rows of a program; only programs
// split across blocks use one atomic per (block, slot) -- the reference issues one atomic per
// (row, constant node).
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <cmath>
#include <type_traits>

#include "ws_internal.h"

namespace ws {
namespace {

enum : uint8_t { BK_PAD = 0, BK_VAR, BK_LIT, BK_CONST, BK_BIN, BK_UN };
// forward operator codes (reference comparison order, backward_kernels.cu:135-188)
enum : uint8_t { FO_NONE = 0, FO_ADD, FO_SUB, FO_MUL, FO_DIV, FO_POW, FO_MOD,
                 FO_SIN, FO_COS, FO_TAN, FO_LOG, FO_EXP, FO_SQRT, FO_ABS, FO_NEG };
// adjoint operator codes (backward_kernels.cu:222-278)
enum : uint8_t { BO_NONE = 0, BO_ADD, BO_SUB, BO_MUL, BO_DIV, BO_POW,
                 BO_SIN, BO_COS, BO_LOG, BO_EXP, BO_SQRT, BO_NEG };

struct BwdLut {
  uint8_t kind[256], arg[256], fop[256], bop[256];
  double lit[10];
};

// Operand kinds of a tape operator.
enum : uint8_t { OPD_OP = 0, OPD_VAR, OPD_LIT, OPD_CONST };

struct BOp {
  uint8_t fop, bop;   // forward and adjoint operator codes
  uint8_t ka, kb;     // operand kinds (kb unused for unary operators)
  uint16_t a, b;      // operand: operator index, variable, literal index (10 = 1.0), constant slot
  uint8_t binary, reach;  // reach: the value flows into the root
  uint16_t pad;
};

struct BRoot {
  int n_ops;          // operators in the tape (0: the program is one terminal)
  uint8_t kind;       // root operand kind (OPD_OP: the last operator)
  uint16_t idx;
  int valid;          // the reference's forward pass yields a root (final depth 1)
};

constexpr int kMaxL = 256;

__host__ __device__ constexpr size_t al16(size_t v) { return (v + 15) / 16 * 16; }
constexpr int kStack = 32;  // STACK_SIZE, backward_kernels.cu:6

template <typename T>
struct BwdParams {
  const uint8_t* pop;
  int64_t B, L;
  const T* x;
  int64_t D;
  const T* consts;
  int64_t K;
  const T* gout;
  T* grad;
  int64_t n_splits, rows_per_split, n_items;
  int tape_stride;  // threads per block (row dimension of the tapes)
  // loss mode: the root adjoint of row d is dL/dpred = 2 (pred - y[d]) / D, L = mean (pred - y)^2;
  // each (program, row range) item writes its partial sums (no atomics, fixed order)
  const T* y;
  const int32_t* active;  // optional: programs with 0 are skipped
  int64_t V;              // variables; with stage_x each thread copies its rows of x to shared
  int stage_x;            // memory once per row group
  int tape_ops;           // operator slots of the tape (>= every program's operator count)
  const int32_t* list;        // optional: the programs of this launch (a bucket) ...
  const int32_t* list_count;  // ... and how many there are (read on the device)
  double* part_loss;      // [n_items]   sum over the item's rows of (pred - y)^2
  double* part_grad;      // [n_items, K] sum over the item's rows of the constant adjoints
};

// Walks program b as the reference's forward loop does (backward_kernels.cu:84-195): PAD ends
// it, an operator that finds too few operands ends it (the prefix is the program), pushes beyond
// depth 32 are dropped, C takes slot min(c_idx, K-1) (1.0 without constants).  Operands are kept
// on the stack as (kind, index) pairs, so terminals never enter the tape.
__device__ BRoot parse_program(const uint8_t* __restrict__ prog, int64_t L, int64_t K,
                               const uint8_t* s_tab, BOp* ops) {
  const uint8_t* t_kind = s_tab;
  const uint8_t* t_fop = s_tab + 256;
  const uint8_t* t_bop = s_tab + 512;
  const uint8_t* t_arg = s_tab + 768;
  uint8_t sk[kStack];
  uint16_t si[kStack];
  int sp = 0, n_ops = 0;
  int64_t c_idx = 0;
  for (int pc = 0; pc < (int)L; ++pc) {
    const int tok = prog[pc];
    const uint8_t kind = t_kind[tok];
    if (kind == BK_PAD) break;
    if (kind == BK_VAR || kind == BK_LIT || kind == BK_CONST) {
      uint8_t k = kind == BK_VAR ? OPD_VAR : OPD_LIT;
      uint16_t ix = t_arg[tok];
      if (kind == BK_CONST) {
        if (K > 0) {
          k = OPD_CONST;
          ix = (uint16_t)(c_idx < K ? c_idx : K - 1);
          c_idx++;
        } else {
          ix = 10;  // C without constants pushes 1.0 and takes no gradient
        }
      }
      if (sp < kStack) {
        sk[sp] = k;
        si[sp] = ix;
        ++sp;
      }
      continue;
    }
    BOp o;
    o.fop = t_fop[tok];
    o.bop = t_bop[tok];
    o.reach = 0;
    o.pad = 0;
    o.kb = OPD_LIT;
    o.b = 0;
    if (kind == BK_BIN) {
      if (sp < 2) break;
      --sp;
      o.kb = sk[sp];
      o.b = si[sp];
      --sp;
      o.ka = sk[sp];
      o.a = si[sp];
      o.binary = 1;
    } else {
      if (sp < 1) break;
      --sp;
      o.ka = sk[sp];
      o.a = si[sp];
      o.binary = 0;
    }
    ops[n_ops] = o;
    sk[sp] = OPD_OP;  // an operator always finds room: it just freed one or two slots
    si[sp] = (uint16_t)n_ops;
    ++sp;
    ++n_ops;
  }
  BRoot r;
  r.n_ops = n_ops;
  r.valid = sp == 1 ? 1 : 0;
  r.kind = sp >= 1 ? sk[0] : OPD_LIT;
  r.idx = sp >= 1 ? si[0] : 0;
  if (r.valid && r.kind == OPD_OP) {  // mark the operators whose value reaches the root
    ops[r.idx].reach = 1;
    for (int o = r.idx; o >= 0; --o) {
      if (!ops[o].reach) continue;
      if (ops[o].ka == OPD_OP) ops[ops[o].a].reach = 1;
      if (ops[o].binary && ops[o].kb == OPD_OP) ops[ops[o].b].reach = 1;
    }
  }
  return r;
}

// ---- forward values (backward_kernels.cu:146-188) ------------------------------------------
template <typename T>
__device__ __forceinline__ T fwd_binary(uint8_t op, T op1, T op2) {
  const T tiny = (T)1e-9;
  switch (op) {
    case FO_ADD: return op1 + op2;
    case FO_SUB: return op1 - op2;
    case FO_MUL: return op1 * op2;
    case FO_DIV: return (fabs(op2) < tiny) ? op1 : op1 / op2;
    case FO_POW: {
      if (op1 < 0) {
        const T ib = round(op2);
        if (fabs(op2 - ib) <= (T)1e-3) op2 = ib;
        else op1 = fabs(op1);
      }
      return pow(op1, op2);
    }
    case FO_MOD: return (fabs(op2) < tiny) ? (T)0 : fmod(op1, op2);
    default: return (T)0;
  }
}

template <typename T>
__device__ __forceinline__ T fwd_unary(uint8_t op, T op1) {
  switch (op) {
    case FO_SIN: return sin(op1);
    case FO_COS: return cos(op1);
    case FO_TAN: return tan(op1);
    case FO_LOG: return log(fabs(op1) + (T)1e-9);
    case FO_EXP: {
      T cl = op1;
      if (cl < -80.0) cl = (T)-80.0;
      if (cl > 80.0) cl = (T)80.0;
      return exp(cl);
    }
    case FO_SQRT: return sqrt(fabs(op1));
    case FO_ABS: return fabs(op1);
    case FO_NEG: return -op1;
    default: return (T)0;  // operators without a forward rule here evaluate to 0
  }
}

// ---- adjoint rules (backward_kernels.cu:222-278) -------------------------------------------
// The reference writes e.g. `adj_tape[l] += (1.0 / r_val) * adj`: for float that expression is
// evaluated in double (a double constant promotes it) and the multiply-add contracts into one
// fused operation before the store rounds back to float.  acc_d / acc_t spell those two shapes.
template <typename T>
__device__ __forceinline__ void acc_d(T& dst, double coef, T adj) {
  dst = (T)fma(coef, (double)adj, (double)dst);
}
template <typename T>
__device__ __forceinline__ void acc_t(T& dst, T coef, T adj) {
  dst = fma(coef, adj, dst);
}

// ---- the adjoint kernel ---------------------------------------------------------------------
// One block owns one program for a range of rows; every thread carries R consecutive rows
// through each tape step, so one decode of an operator (a broadcast shared-memory load and a
// block-uniform branch) serves R rows, and the R rows' arithmetic is independent work for the
// pipelines.  One tape slot per operator and thread ([op][thread][R] values, vector loads and
// stores) holds the operator's values after the forward sweep and its adjoints during the reverse
// sweep: the program is a tree, so the only reader of a value is the operator's parent, which
// reads it before it writes the adjoint into the same slot; exp and pow, whose adjoint rules use
// their own output, recompute it from their operands bit for bit.  The previous operator's values
// and the adjoint handed to it stay in registers (BOp::pad bit 0 / bit 1: the left / right operand
// is operator o-1), and constant adjoints are summed in registers when K <= kRegSlots (the slot of
// a delivery is the same for the whole block, so the register is chosen by a uniform switch).
//
// LOSS = false (ws_eval_rpn_backward): the root adjoint of row d is grad_output[b, d] and every
// per-row expression is the reference's, double promotions included (acc_d / acc_t), so per-row
// adjoints are bit-identical to the reference's; per-row constant adjoints are summed in FP64.
// LOSS = true (ws_loss_grad): the root adjoint is 2 (pred - y[d]) / D and the arithmetic is in T;
// the loss is summed per thread in FP64.  Both skip the contributions of zero adjoints.
constexpr int kRegSlots = 8;

template <typename T, int R>
__device__ __forceinline__ void ld_vec(const T* p, T (&o)[R]) {
  if constexpr (R * sizeof(T) == 16) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    const T* q = reinterpret_cast<const T*>(&v);
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = q[r];
  } else if constexpr (R * sizeof(T) == 8) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    const T* q = reinterpret_cast<const T*>(&v);
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = q[r];
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = p[r];
  }
}

template <typename T, int R>
__device__ __forceinline__ void st_vec(T* p, const T (&v)[R]) {
  if constexpr (R * sizeof(T) == 16) {
    float4 w;
    T* q = reinterpret_cast<T*>(&w);
#pragma unroll
    for (int r = 0; r < R; ++r) q[r] = v[r];
    *reinterpret_cast<float4*>(p) = w;
  } else if constexpr (R * sizeof(T) == 8) {
    float2 w;
    T* q = reinterpret_cast<T*>(&w);
#pragma unroll
    for (int r = 0; r < R; ++r) q[r] = v[r];
    *reinterpret_cast<float2*>(p) = w;
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) p[r] = v[r];
  }
}

// The R values of one operand: an earlier operator's (tape), a variable's (rows past d_end read
// as 0), a constant's or a literal's.
template <typename T, int R>
__device__ __forceinline__ void operand_vec(uint8_t k, uint16_t i, const T* tape, int TS, int tid,
                                            const T* x, int64_t D, int64_t d0, int64_t d_end,
                                            const T* s_lit, const T* cst, const T* xs,
                                            T (&o)[R]) {
  switch (k) {
    case OPD_OP: ld_vec<T, R>(tape + ((size_t)i * TS + tid) * R, o); break;
    case OPD_VAR: {
      if (xs) {  // this thread's rows, staged at the start of the row group
        ld_vec<T, R>(xs + ((size_t)i * TS + tid) * R, o);
        break;
      }
      const T* xr = x + (int64_t)i * D;
#pragma unroll
      for (int r = 0; r < R; ++r) o[r] = d0 + r < d_end ? xr[d0 + r] : (T)0;
      break;
    }
    case OPD_CONST: {
      const T c = cst[i];
#pragma unroll
      for (int r = 0; r < R; ++r) o[r] = c;
      break;
    }
    default: {
      const T c = i < 10 ? s_lit[i] : (T)1.0;
#pragma unroll
      for (int r = 0; r < R; ++r) o[r] = c;
    }
  }
}

#define WS_FOR_R for (int r = 0; r < R; ++r)

template <typename T, int R>
__device__ __forceinline__ void fwd_binary_vec(uint8_t op, const T (&a)[R], const T (&b)[R],
                                               T (&v)[R]) {
  switch (op) {
    case FO_ADD: WS_FOR_R v[r] = a[r] + b[r]; break;
    case FO_SUB: WS_FOR_R v[r] = a[r] - b[r]; break;
    case FO_MUL: WS_FOR_R v[r] = a[r] * b[r]; break;
    default: WS_FOR_R v[r] = fwd_binary<T>(op, a[r], b[r]); break;
  }
}

template <typename T, int R>
__device__ __forceinline__ void fwd_unary_vec(uint8_t op, const T (&a)[R], T (&v)[R]) {
  switch (op) {
    case FO_SIN: WS_FOR_R v[r] = sin(a[r]); break;
    case FO_COS: WS_FOR_R v[r] = cos(a[r]); break;
    case FO_NEG: WS_FOR_R v[r] = -a[r]; break;
    default: WS_FOR_R v[r] = fwd_unary<T>(op, a[r]); break;
  }
}

template <typename T>
__device__ __forceinline__ void creg_add(T (&cr)[kRegSlots], int i, T c) {
  switch (i) {
    case 0: cr[0] += c; break;
    case 1: cr[1] += c; break;
    case 2: cr[2] += c; break;
    case 3: cr[3] += c; break;
    case 4: cr[4] += c; break;
    case 5: cr[5] += c; break;
    case 6: cr[6] += c; break;
    default: cr[7] += c; break;
  }
}

// Constant-slot accumulator: FP64 per row for the reference path, T for the loss path.
template <typename T, bool LOSS>
using CAcc = typename std::conditional<LOSS, T, double>::type;

template <typename T, int R, bool LOSS, bool KREG>
__device__ __forceinline__ void deliver_vec(uint8_t k, uint16_t i, const T (&c)[R], bool to_carry,
                                            T (&carry)[R], bool& have, T* tape, int TS, int tid,
                                            CAcc<T, LOSS> (&cr)[kRegSlots], double* cacc,
                                            int* touched) {
  if (k == OPD_OP) {
    if (to_carry) {
      WS_FOR_R carry[r] = c[r];
      have = true;
    } else {
      st_vec<T, R>(tape + ((size_t)i * TS + tid) * R, c);
    }
  } else if (k == OPD_CONST) {
    using A = CAcc<T, LOSS>;
    A s = (A)0;
    bool any = false;
    WS_FOR_R {
      if (c[r] != (T)0) {
        s += (A)c[r];
        any = true;
      }
    }
    if (any) {
      if (KREG) creg_add<A>(cr, i, s);
      else cacc[(size_t)i * TS + tid] += (double)s;
      if (!LOSS) touched[i] = 1;
    }
  }
}

template <typename T, int R, bool LOSS, bool KREG>
__global__ void __launch_bounds__(128) adj_kernel(BwdParams<T> p, BwdLut lut) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int TS = p.tape_stride;
  // shared memory: operators | touched flags | (K > kRegSlots) FP64 constant accumulators |
  // work: the tape and staged x during the rows, the block reduction after them
  BOp* ops = reinterpret_cast<BOp*>(smem);
  int* touched = reinterpret_cast<int*>(smem + al16((size_t)p.tape_ops * sizeof(BOp)));
  double* cacc = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(touched) +
                                           al16((size_t)p.K * sizeof(int)));
  unsigned char* work = reinterpret_cast<unsigned char*>(cacc + (KREG ? 0 : (size_t)p.K * TS));
  T* tape = reinterpret_cast<T*>(work);
  T* xs = p.stage_x ? tape + (size_t)p.tape_ops * TS * R : nullptr;  // [V][thread][R]
  __shared__ BRoot s_root;
  __shared__ int64_t s_prog;
  __shared__ T s_lit[10];
  __shared__ uint8_t s_tab[1024];  // kind, forward op, adjoint op, argument per token byte
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    s_tab[t] = lut.kind[t];
    s_tab[256 + t] = lut.fop[t];
    s_tab[512 + t] = lut.bop[t];
    s_tab[768 + t] = lut.arg[t];
  }
  if (threadIdx.x < 10) s_lit[threadIdx.x] = (T)lut.lit[threadIdx.x];
  if (threadIdx.x == 0) s_prog = -1;
  const int tid = threadIdx.x;
  const T loss_scale = LOSS ? (T)(2.0 / (double)p.D) : (T)0;
  using A = CAcc<T, LOSS>;

  const int64_t n_items = p.list ? (int64_t)(*p.list_count) * p.n_splits : p.n_items;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t li = item / p.n_splits;
    const int64_t split = item - li * p.n_splits;
    const int64_t b = p.list ? (int64_t)p.list[li] : li;
    const int64_t slot = b * p.n_splits + split;  // partial sums of (program, row range)
    if (LOSS && p.active && p.active[b] == 0) continue;  // uniform over the block
    __syncthreads();
    if (tid == 0 && s_prog != b) {
      BRoot rt0 = parse_program(p.pop + b * p.L, p.L, p.K, s_tab, ops);
      for (int o = 0; o < rt0.n_ops; ++o) {
        uint16_t f = 0;
        if (ops[o].ka == OPD_OP && (int)ops[o].a == o - 1) f |= 1;
        if (ops[o].binary && ops[o].kb == OPD_OP && (int)ops[o].b == o - 1) f |= 2;
        ops[o].pad = f;
      }
      s_root = rt0;
      s_prog = b;
    }
    for (int64_t k = tid; k < p.K; k += blockDim.x) touched[k] = 0;
    if (!KREG)
      for (int64_t k = 0; k < p.K; ++k) cacc[k * TS + tid] = 0.0;
    __syncthreads();
    const BRoot rt = s_root;
    if (!rt.valid) {
      if (LOSS) {  // no prediction: infinite loss, no gradient
        if (tid == 0) p.part_loss[slot] = __longlong_as_double(0x7ff0000000000000ll);
        for (int64_t k = tid; k < p.K; k += blockDim.x) p.part_grad[slot * p.K + k] = 0.0;
      }
      continue;
    }
    const int64_t d_begin = split * p.rows_per_split;
    int64_t d_end = d_begin + p.rows_per_split;
    if (d_end > p.D) d_end = p.D;
    const T* xcol = p.x;
    const T* cst = p.consts + b * p.K;
    const int n = rt.n_ops;
    A cr[kRegSlots];
#pragma unroll
    for (int k = 0; k < kRegSlots; ++k) cr[k] = (A)0;
    double lacc = 0.0;

    for (int64_t d0 = d_begin + (int64_t)tid * R; d0 < d_end; d0 += (int64_t)TS * R) {
      // this thread's rows: x staged (only this thread reads them: no barrier), the root
      // adjoint's inputs loaded now so that their latency overlaps the forward sweep
      if (xs) {
        for (int64_t v = 0; v < p.V; ++v) {
          const T* xr = xcol + v * p.D;
          T xv[R];
          WS_FOR_R xv[r] = d0 + r < d_end ? xr[d0 + r] : (T)0;
          st_vec<T, R>(xs + ((size_t)v * TS + tid) * R, xv);
        }
      }
      T ext[R];  // y (loss) or grad_output (reference path) of the R rows
      WS_FOR_R ext[r] = d0 + r < d_end ? (LOSS ? p.y[d0 + r] : p.gout[b * p.D + d0 + r]) : (T)0;
      // forward: operator values
      T last[R];
      WS_FOR_R last[r] = (T)0;
      for (int o = 0; o < n; ++o) {
        const BOp op = ops[o];
        T va[R], v[R];
        if (op.pad & 1) {
          WS_FOR_R va[r] = last[r];
        } else {
          operand_vec<T, R>(op.ka, op.a, tape, TS, tid, xcol, p.D, d0, d_end, s_lit, cst, xs, va);
        }
        if (op.binary) {
          T vb[R];
          if (op.pad & 2) {
            WS_FOR_R vb[r] = last[r];
          } else {
            operand_vec<T, R>(op.kb, op.b, tape, TS, tid, xcol, p.D, d0, d_end, s_lit, cst, xs, vb);
          }
          fwd_binary_vec<T, R>(op.fop, va, vb, v);
        } else {
          fwd_unary_vec<T, R>(op.fop, va, v);
        }
        st_vec<T, R>(tape + ((size_t)o * TS + tid) * R, v);
        WS_FOR_R last[r] = v[r];
      }
      // root adjoints
      T g_root[R];
      if (LOSS) {
        T pred[R];
        if (rt.kind == OPD_OP && (int)rt.idx == n - 1) {
          WS_FOR_R pred[r] = last[r];
        } else {
          operand_vec<T, R>(rt.kind, rt.idx, tape, TS, tid, xcol, p.D, d0, d_end, s_lit, cst, xs,
                            pred);
        }
        WS_FOR_R {
          const T diff = d0 + r < d_end ? pred[r] - ext[r] : (T)0;
          lacc += (double)diff * (double)diff;
          g_root[r] = diff * loss_scale;
        }
      } else {
        WS_FOR_R g_root[r] = ext[r];
      }
      T carry[R];
      bool have = false;
      if (rt.kind != OPD_OP) {  // a one-terminal program
        deliver_vec<T, R, LOSS, KREG>(rt.kind, rt.idx, g_root, false, carry, have, tape, TS, tid,
                                      cr, cacc, touched);
        continue;
      }
      if ((int)rt.idx == n - 1) {
        WS_FOR_R carry[r] = g_root[r];
        have = true;
      } else {
        st_vec<T, R>(tape + ((size_t)rt.idx * TS + tid) * R, g_root);
      }
      // reverse: each operator hands its adjoint to its operands
      for (int o = n - 1; o >= 0; --o) {
        const BOp op = ops[o];
        if (!op.reach) {
          have = false;
          continue;
        }
        T g[R];
        if (have) {
          WS_FOR_R g[r] = carry[r];
        } else {
          ld_vec<T, R>(tape + ((size_t)o * TS + tid) * R, g);
        }
        have = false;
        T lv[R], ca[R], cb[R];
        operand_vec<T, R>(op.ka, op.a, tape, TS, tid, xcol, p.D, d0, d_end, s_lit, cst, xs, lv);
        WS_FOR_R { ca[r] = (T)0; cb[r] = (T)0; }
        if (op.binary) {
          T rv[R];
          operand_vec<T, R>(op.kb, op.b, tape, TS, tid, xcol, p.D, d0, d_end, s_lit, cst, xs, rv);
          switch (op.bop) {
            case BO_ADD: WS_FOR_R { ca[r] += g[r]; cb[r] += g[r]; } break;
            case BO_SUB: WS_FOR_R { ca[r] += g[r]; cb[r] -= g[r]; } break;
            case BO_MUL:
              if (LOSS) WS_FOR_R { ca[r] = rv[r] * g[r]; cb[r] = lv[r] * g[r]; }
              else WS_FOR_R { acc_t(ca[r], rv[r], g[r]); acc_t(cb[r], lv[r], g[r]); }
              break;
            case BO_DIV:
              WS_FOR_R {
                if (fabs(rv[r]) >= (T)1e-9) {
                  if (LOSS) {
                    ca[r] = g[r] / rv[r];
                    cb[r] = -(lv[r] / (rv[r] * rv[r])) * g[r];
                  } else {
                    acc_d(ca[r], 1.0 / rv[r], g[r]);
                    acc_t(cb[r], -(lv[r] / (rv[r] * rv[r])), g[r]);
                  }
                }
              }
              break;
            case BO_POW:
              WS_FOR_R {
                if (lv[r] > 0) {
                  const T out_val = fwd_binary<T>(op.fop, lv[r], rv[r]);
                  if (LOSS) {
                    ca[r] = rv[r] * pow(lv[r], rv[r] - (T)1) * g[r];
                    cb[r] = out_val * log(lv[r]) * g[r];
                  } else {
                    acc_d(ca[r], (double)rv[r] * pow((double)lv[r], (double)rv[r] - 1.0), g[r]);
                    acc_t(cb[r], out_val * log(lv[r]), g[r]);
                  }
                }
              }
              break;
            default: break;
          }
          WS_FOR_R if (g[r] == (T)0) cb[r] = (T)0;
          // the right operand sits later in the program: its constants first, as the
          // reference's reverse walk meets them
          deliver_vec<T, R, LOSS, KREG>(op.kb, op.b, cb, (op.pad & 2) != 0, carry, have, tape, TS,
                                        tid, cr, cacc, touched);
        } else {
          switch (op.bop) {
            case BO_SIN:
              if (LOSS) WS_FOR_R ca[r] = cos(lv[r]) * g[r];
              else WS_FOR_R acc_t(ca[r], cos(lv[r]), g[r]);
              break;
            case BO_COS:
              if (LOSS) WS_FOR_R ca[r] = -sin(lv[r]) * g[r];
              else WS_FOR_R acc_t(ca[r], -sin(lv[r]), g[r]);
              break;
            case BO_LOG:
              WS_FOR_R {
                if (fabs(lv[r]) > (T)1e-9) {
                  if (LOSS) ca[r] = g[r] / lv[r];
                  else acc_d(ca[r], 1.0 / lv[r], g[r]);
                }
              }
              break;
            case BO_EXP:
              if (LOSS) WS_FOR_R ca[r] = fwd_unary<T>(op.fop, lv[r]) * g[r];
              else WS_FOR_R acc_t(ca[r], fwd_unary<T>(op.fop, lv[r]), g[r]);
              break;
            case BO_SQRT:
              WS_FOR_R {
                if (lv[r] > (T)1e-9) {
                  if (LOSS) ca[r] = (T)0.5 / sqrt(lv[r]) * g[r];
                  else acc_d(ca[r], 0.5 / sqrt(lv[r]), g[r]);
                }
              }
              break;
            case BO_NEG: WS_FOR_R ca[r] += -g[r]; break;
            default: break;
          }
        }
        WS_FOR_R if (g[r] == (T)0) ca[r] = (T)0;
        deliver_vec<T, R, LOSS, KREG>(op.ka, op.a, ca, (op.pad & 1) != 0, carry, have, tape, TS,
                                      tid, cr, cacc, touched);
      }
    }
    __syncthreads();  // the tape is free: the reduction reuses its memory
    double* cred = KREG ? reinterpret_cast<double*>(work) : cacc;
    double* lacc_s = reinterpret_cast<double*>(work) + (KREG ? (size_t)p.K * TS : 0);
    if (KREG) {
#pragma unroll
      for (int k = 0; k < kRegSlots; ++k)
        if (k < p.K) cred[(size_t)k * TS + tid] = (double)cr[k];
    }
    if (LOSS) lacc_s[tid] = lacc;
    __syncthreads();
    // fixed-order reduction over the block's threads, one thread per slot
    for (int64_t k = tid; k < p.K; k += blockDim.x) {
      double s = 0.0;
      for (int t = 0; t < (int)blockDim.x; ++t) s += cred[k * TS + t];
      if (LOSS) {
        p.part_grad[slot * p.K + k] = s;
      } else if (touched[k]) {
        T* dst = p.grad + b * p.K + k;
        if (p.n_splits == 1) *dst = *dst + (T)s;
        else atomicAdd(dst, (T)s);
      }
    }
    if (LOSS && tid == 0) {
      double s = 0.0;
      for (int t = 0; t < (int)blockDim.x; ++t) s += lacc_s[t];
      p.part_loss[slot] = s;
    }
  }
}

#undef WS_FOR_R

// Programs grouped by operator count, so that each group runs with a tape sized for it: a
// program's count of operator tokens before its first PAD bounds its tape length.  Programs with
// active[b] == 0 are left out.  lists: [n_buckets, B]; the order inside a bucket does not matter
// (every (program, row range) writes its own partial sums).
constexpr int kMaxBuckets = 9;
constexpr int kBucketOps[kMaxBuckets] = {8, 16, 24, 32, 48, 64, 96, 128, 256};
__constant__ int c_bucket_ops[kMaxBuckets] = {8, 16, 24, 32, 48, 64, 96, 128, 256};

__global__ void __launch_bounds__(256) bucket_kernel(const uint8_t* __restrict__ pop, int64_t B,
                                                     int64_t L, BwdLut lut,
                                                     const int32_t* __restrict__ active,
                                                     int n_buckets, int32_t* counts,
                                                     int32_t* lists) {
  __shared__ uint8_t s_kind[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) s_kind[t] = lut.kind[t];
  __syncthreads();
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    if (active && active[b] == 0) continue;
    const uint8_t* row = pop + b * L;
    int n = 0;
    for (int64_t t = 0; t < L; ++t) {
      const uint8_t k = s_kind[row[t]];
      if (k == BK_PAD) break;
      n += (k == BK_BIN || k == BK_UN) ? 1 : 0;
    }
    int j = 0;
    while (j < n_buckets - 1 && n > c_bucket_ops[j]) ++j;
    const int pos = atomicAdd(counts + j, 1);
    lists[(int64_t)j * B + pos] = (int32_t)b;
  }
}

// Loss mode, second launch: a program's partials summed in row-range order; loss = sum / D.
template <typename T>
__global__ void __launch_bounds__(256) loss_grad_reduce_kernel(const double* __restrict__ part_loss,
                                                               const double* __restrict__ part_grad,
                                                               const int32_t* __restrict__ active,
                                                               int64_t B, int64_t K,
                                                               int64_t n_splits, int64_t D,
                                                               double* __restrict__ loss,
                                                               T* __restrict__ grad) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    if (active && active[b] == 0) continue;
    double l = 0.0;
    for (int64_t s = 0; s < n_splits; ++s) l += part_loss[b * n_splits + s];
    loss[b] = l / (double)D;
    for (int64_t k = 0; k < K; ++k) {
      double g = 0.0;
      for (int64_t s = 0; s < n_splits; ++s) g += part_grad[(b * n_splits + s) * K + k];
      grad[b * K + k] = (T)g;
    }
  }
}

BwdLut build_bwd_lut(const ws_token_map& m, int64_t num_vars) {
  BwdLut lut;
  const int lit_ids[10] = {m.id_0, m.id_1, m.id_2, m.id_3, m.id_4,
                           m.id_5, m.id_6, m.id_10, m.id_pi, m.id_e};
  const double lit_val[10] = {0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 10.0, m.pi_val, m.e_val};
  for (int i = 0; i < 10; ++i) lut.lit[i] = lit_val[i];
  const int bin_ids[6] = {m.op_add, m.op_sub, m.op_mul, m.op_div, m.op_pow, m.op_mod};
  const uint8_t bin_f[6] = {FO_ADD, FO_SUB, FO_MUL, FO_DIV, FO_POW, FO_MOD};
  const uint8_t bin_b[6] = {BO_ADD, BO_SUB, BO_MUL, BO_DIV, BO_POW, BO_NONE};
  const int un_f_ids[8] = {m.op_sin, m.op_cos, m.op_tan, m.op_log,
                           m.op_exp, m.op_sqrt, m.op_abs, m.op_neg};
  const uint8_t un_f[8] = {FO_SIN, FO_COS, FO_TAN, FO_LOG, FO_EXP, FO_SQRT, FO_ABS, FO_NEG};
  const int un_b_ids[6] = {m.op_sin, m.op_cos, m.op_log, m.op_exp, m.op_sqrt, m.op_neg};
  const uint8_t un_b[6] = {BO_SIN, BO_COS, BO_LOG, BO_EXP, BO_SQRT, BO_NEG};
  for (int t = 0; t < 256; ++t) {
    uint8_t kind = BK_UN, arg = 0, fo = FO_NONE, bo = BO_NONE;
    bool lit = false;
    if (t == m.pad_id) {
      kind = BK_PAD;
    } else if ((int64_t)t >= (int64_t)m.id_x_start &&
               (int64_t)t < (int64_t)m.id_x_start + num_vars) {
      kind = BK_VAR;
      arg = (uint8_t)(t - m.id_x_start);
    } else {
      for (int i = 0; i < 10 && !lit; ++i)
        if (t == lit_ids[i]) { kind = BK_LIT; arg = (uint8_t)i; lit = true; }
      if (!lit) {
        if (t == m.id_C) {
          kind = BK_CONST;
        } else {
          int bi = -1;
          for (int i = 0; i < 6 && bi < 0; ++i)
            if (t == bin_ids[i]) bi = i;
          if (bi >= 0) {
            kind = BK_BIN;
            fo = bin_f[bi];
            // the adjoint pass compares add, sub, mul, div, pow in that order
            for (int i = 0; i < 5; ++i)
              if (t == bin_ids[i]) { bo = bin_b[i]; break; }
          } else {
            kind = BK_UN;
            for (int i = 0; i < 8; ++i)
              if (t == un_f_ids[i]) { fo = un_f[i]; break; }
            for (int i = 0; i < 6; ++i)
              if (t == un_b_ids[i]) { bo = un_b[i]; break; }
          }
        }
      }
    }
    lut.kind[t] = kind;
    lut.arg[t] = arg;
    lut.fop[t] = fo;
    lut.bop[t] = bo;
  }
  return lut;
}

constexpr int64_t kStageMaxVars = 16;  // x is staged in shared memory up to this many variables

template <typename T>
size_t backward_smem(int64_t M, int64_t K, int64_t V, int threads, int R) {
  const int64_t vs = V <= kStageMaxVars ? V : 0;
  const bool kreg = K <= kRegSlots;
  const size_t tape = (size_t)(M + vs) * threads * R * sizeof(T);
  const size_t red = (size_t)((kreg ? K : 0) + 1) * threads * sizeof(double);
  return al16((size_t)M * sizeof(BOp)) + al16((size_t)K * sizeof(int)) +
         (kreg ? 0 : (size_t)K * threads * sizeof(double)) + (tape > red ? tape : red);
}

// Block size, rows per thread, shared memory and the split of rows into ranges for one launch.
// Rows are split only when there are too few programs to fill the GPU; the split depends on
// (B, L, K, D) and the device alone.
struct BwdPlan {
  int threads, R;
  size_t smem;
  int64_t n_splits, rows, grid;
};

template <typename T>
constexpr int kRowsMax = sizeof(T) == 4 ? 4 : 2;

template <typename T, bool LOSS, int RR>
void (*adj_pick(bool kreg))(BwdParams<T>, BwdLut) {
  return kreg ? adj_kernel<T, RR, LOSS, true> : adj_kernel<T, RR, LOSS, false>;
}

template <typename T, bool LOSS>
void (*adj_fn(int R, bool kreg))(BwdParams<T>, BwdLut) {
  if constexpr (kRowsMax<T> >= 4) {
    if (R == 4) return adj_pick<T, LOSS, 4>(kreg);
  }
  if (R == 2) return adj_pick<T, LOSS, 2>(kreg);
  return adj_pick<T, LOSS, 1>(kreg);
}

// Block size, rows per thread and shared memory for a tape of M operator slots: the shape
// with the most resident threads per SM.
template <typename T, bool LOSS>
ws_status backward_shape(int64_t M, int64_t K, int64_t V, BwdPlan* out, int* per_sm_out) {
  const DeviceInfo& dev = device_info();
  const size_t budget = dev.smem_optin < (size_t)200 * 1024 ? dev.smem_optin : 200 * 1024;
  const bool kreg = K <= kRegSlots;
  // every (rows per thread, block size) shape that fits, scored by the rows its resident warps
  // carry, with warps counted up to 32 per SM (measured: 2 rows per thread at twice the warps
  // is no faster than 4 rows per thread, so rows are weighted fully)
  double best_score = -1.0;
  int best_threads = 0, best_per_sm = 0, best_r = 1;
  for (int R = kRowsMax<T>; R >= 1; R /= 2) {
    auto kern = adj_fn<T, LOSS>(R, kreg);
    for (int threads = 128; threads >= 32; threads /= 2) {
      const size_t smem = backward_smem<T>(M, K, V, threads, R);
      if (smem > budget) continue;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return fail_cuda(e, "eval_rpn_backward");
      int per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
      if (e != cudaSuccess) return fail_cuda(e, "eval_rpn_backward");
      if (per_sm < 1) continue;
      double warps = (double)per_sm * threads / 32.0;
      if (warps > 32.0) warps = 32.0;
      const double score = warps * (double)R;
      if (score > best_score + 1e-9) {
        best_score = score;
        best_threads = threads;
        best_per_sm = per_sm;
        best_r = R;
      }
    }
  }
  if (best_threads == 0)
    return fail("backward: " + std::to_string(K) + " constants and " + std::to_string(M) +
                " operators need more shared memory than a block has");
  const size_t smem = backward_smem<T>(M, K, V, best_threads, best_r);
  cudaError_t e = cudaFuncSetAttribute(adj_fn<T, LOSS>(best_r, kreg),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail_cuda(e, "eval_rpn_backward");
  out->threads = best_threads;
  out->R = best_r;
  out->smem = smem;
  *per_sm_out = best_per_sm;
  return WS_OK;
}

// Rows are split into ranges only when there are too few programs to fill the GPU; ranges are
// multiples of 512 rows (a whole number of row groups of every block shape).  The split depends
// on (B, L, K, V, D) and the device alone.
template <typename T, bool LOSS>
ws_status backward_plan(int64_t B, int64_t L, int64_t D, int64_t K, int64_t V,
                        BwdPlan* out) {
  int per_sm = 0;
  ws_status st = backward_shape<T, LOSS>(L, K, V, out, &per_sm);
  if (st != WS_OK) return st;
  const int64_t slots = (int64_t)device_info().sm_count * per_sm;
  const int64_t group = 512;
  int64_t n_splits = (2 * slots + B - 1) / B;
  const int64_t max_splits = (D + group - 1) / group;
  if (n_splits > max_splits) n_splits = max_splits;
  if (n_splits < 1) n_splits = 1;
  int64_t rows = (D + n_splits - 1) / n_splits;
  rows = (rows + group - 1) / group * group;
  n_splits = (D + rows - 1) / rows;
  out->n_splits = n_splits;
  out->rows = rows;
  const int64_t n_items = B * n_splits;
  out->grid = n_items < slots ? n_items : slots;
  return WS_OK;
}

template <typename T, bool LOSS>
BwdParams<T> backward_params(const uint8_t* pop, int64_t B, int64_t L, const void* x, int64_t V,
                             int64_t D,
                             const void* consts, int64_t K, const BwdPlan& plan) {
  BwdParams<T> prm;
  prm.pop = pop;
  prm.B = B;
  prm.L = L;
  prm.x = static_cast<const T*>(x);
  prm.D = D;
  prm.consts = static_cast<const T*>(consts);
  prm.K = K;
  prm.gout = nullptr;
  prm.grad = nullptr;
  prm.n_splits = plan.n_splits;
  prm.rows_per_split = plan.rows;
  prm.n_items = B * plan.n_splits;
  prm.tape_stride = plan.threads;
  prm.V = V;
  prm.stage_x = V <= kStageMaxVars ? 1 : 0;
  prm.tape_ops = (int)L;
  prm.list = nullptr;
  prm.list_count = nullptr;
  prm.y = nullptr;
  prm.active = nullptr;
  prm.part_loss = nullptr;
  prm.part_grad = nullptr;
  return prm;
}

template <typename T>
ws_status launch_backward_typed(const uint8_t* pop, int64_t B, int64_t L, const void* x,
                                int64_t V, int64_t D, const void* consts, int64_t K,
                                const void* gout,
                                void* grad, const BwdLut& lut, cudaStream_t stream) {
  BwdPlan plan;
  ws_status st = backward_plan<T, false>(B, L, D, K, V, &plan);
  if (st != WS_OK) return st;
  BwdParams<T> prm = backward_params<T, false>(pop, B, L, x, V, D, consts, K, plan);
  prm.gout = static_cast<const T*>(gout);
  prm.grad = static_cast<T*>(grad);
  adj_fn<T, false>(plan.R, K <= kRegSlots)<<<(unsigned)plan.grid, plan.threads, plan.smem,
                                              stream>>>(prm, lut);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "eval_rpn_backward");
}

}  // namespace

// Loss-and-gradient launch shared by ws_loss_grad and the batched L-BFGS: partial sums into
// part_loss [B * n_splits] and part_grad [B * n_splits, K] (double), then, when loss / grad
// are given, the reduce launch.
template <typename T>
ws_status launch_loss_grad(const uint8_t* pop, int64_t B, int64_t L, const void* x, int64_t D,
                           const void* consts, int64_t K, const void* y, const int32_t* active,
                           const ws_token_map& ids, int64_t num_vars, double* part_loss,
                           double* part_grad, double* loss, void* grad, int32_t* buckets,
                           int64_t* n_splits_out, cudaStream_t stream) {
  BwdPlan plan;
  ws_status st = backward_plan<T, true>(B, L, D, K, num_vars, &plan);
  if (st != WS_OK) return st;
  if (n_splits_out) *n_splits_out = plan.n_splits;
  if (!part_loss) return WS_OK;  // plan query only
  const BwdLut lut = build_bwd_lut(ids, num_vars);
  BwdParams<T> prm = backward_params<T, true>(pop, B, L, x, num_vars, D, consts, K, plan);
  prm.y = static_cast<const T*>(y);
  prm.active = active;
  prm.part_loss = part_loss;
  prm.part_grad = part_grad;
  cudaError_t e;
  if (!buckets) {
    adj_fn<T, true>(plan.R, K <= kRegSlots)<<<(unsigned)plan.grid, plan.threads, plan.smem,
                                               stream>>>(prm, lut);
  } else {
    // buckets[0..15]: counts; buckets + 16: lists [n_buckets, B]
    int nb = 0;
    while (nb < kMaxBuckets && (nb == 0 || kBucketOps[nb - 1] < L - 1)) ++nb;
    int32_t* counts = buckets;
    int32_t* lists = buckets + 16;
    e = cudaMemsetAsync(counts, 0, 16 * sizeof(int32_t), stream);
    if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
    const int64_t cb = (B + 255) / 256;
    bucket_kernel<<<(unsigned)(cb < 2048 ? cb : 2048), 256, 0, stream>>>(pop, B, L, lut, active,
                                                                         nb, counts, lists);
    for (int j = 0; j < nb; ++j) {
      const int64_t M = kBucketOps[j] < L ? kBucketOps[j] : L;
      BwdPlan pj;
      int per_sm = 0;
      st = backward_shape<T, true>(M, K, num_vars, &pj, &per_sm);
      if (st != WS_OK) return st;
      BwdParams<T> q = prm;
      q.tape_stride = pj.threads;
      q.tape_ops = (int)M;
      q.list = lists + (int64_t)j * B;
      q.list_count = counts + j;
      const int64_t slots = (int64_t)device_info().sm_count * per_sm;
      const int64_t items = B * plan.n_splits;
      const int64_t grid = items < slots ? items : slots;
      adj_fn<T, true>(pj.R, K <= kRegSlots)<<<(unsigned)grid, pj.threads, pj.smem, stream>>>(
          q, lut);
    }
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
  if (loss) {
    const int64_t blocks = (B + 255) / 256;
    loss_grad_reduce_kernel<T><<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, stream>>>(
        part_loss, part_grad, active, B, K, plan.n_splits, D, loss, static_cast<T*>(grad));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
  }
  return WS_OK;
}

// Device scratch of the operator-count buckets of launch_loss_grad (counts and program lists).
size_t loss_grad_bucket_bytes(int64_t B) {
  return (size_t)(16 + (int64_t)kMaxBuckets * B) * sizeof(int32_t);
}

template ws_status launch_loss_grad<float>(const uint8_t*, int64_t, int64_t, const void*,
                                           int64_t, const void*, int64_t, const void*,
                                           const int32_t*, const ws_token_map&, int64_t, double*,
                                           double*, double*, void*, int32_t*, int64_t*,
                                           cudaStream_t);
template ws_status launch_loss_grad<double>(const uint8_t*, int64_t, int64_t, const void*,
                                            int64_t, const void*, int64_t, const void*,
                                            const int32_t*, const ws_token_map&, int64_t, double*,
                                            double*, double*, void*, int32_t*, int64_t*,
                                            cudaStream_t);
}  // namespace ws

extern "C" ws_status ws_eval_rpn_backward(int32_t dtype, const uint8_t* population, int64_t B,
                                          int64_t L, const void* x, int64_t num_vars, int64_t D,
                                          const void* constants, int64_t K,
                                          const void* grad_output, void* grad_constants,
                                          const ws_token_map* ids, void* stream) {
  using namespace ws;
  clear_error();
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (!ids) return fail("token map is required");
  if (B < 0 || L < 0 || D < 0 || K < 0 || num_vars < 0) return fail("negative dimension");
  if (L > kMaxL) return fail("backward supports programs of at most 256 tokens");
  if (K > 0xFFFF) return fail("backward supports at most 65535 constants per program");
  if (num_vars > 255) return fail("at most 255 variables are addressable by uint8 tokens");
  if (B == 0 || D == 0 || K == 0 || L == 0) return WS_OK;  // nothing to accumulate
  if (!population || !constants || !grad_output || !grad_constants || (num_vars > 0 && !x))
    return fail("null tensor pointer");
  const BwdLut lut = build_bwd_lut(*ids, num_vars);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == WS_F32)
    return launch_backward_typed<float>(population, B, L, x, num_vars, D, constants, K,
                                        grad_output,
                                        grad_constants, lut, s);
  return launch_backward_typed<double>(population, B, L, x, num_vars, D, constants, K,
                                       grad_output,
                                       grad_constants, lut, s);
}

namespace {
ws_status loss_grad_check(int32_t dtype, int64_t B, int64_t L, int64_t D, int64_t K,
                          int64_t num_vars) {
  using namespace ws;
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (B < 0 || L < 0 || D < 0 || K < 0 || num_vars < 0) return fail("negative dimension");
  if (L > kMaxL) return fail("loss_grad supports programs of at most 256 tokens");
  if (K > 0xFFFF) return fail("loss_grad supports at most 65535 constants per program");
  if (num_vars > 255) return fail("at most 255 variables are addressable by uint8 tokens");
  return WS_OK;
}
}  // namespace

extern "C" ws_status ws_loss_grad_workspace_bytes(int32_t dtype, int64_t B, int64_t L,
                                                  int64_t num_vars, int64_t D, int64_t K,
                                                  size_t* bytes) {
  using namespace ws;
  clear_error();
  ws_status st = loss_grad_check(dtype, B, L, D, K, num_vars);
  if (st != WS_OK) return st;
  if (!bytes) return fail("null output pointer");
  *bytes = 0;
  if (B == 0 || D == 0 || L == 0) return WS_OK;
  int64_t n_splits = 1;
  st = dtype == WS_F32
           ? launch_loss_grad<float>(nullptr, B, L, nullptr, D, nullptr, K, nullptr, nullptr,
                                     ws_token_map{}, num_vars, nullptr, nullptr, nullptr,
                                     nullptr, nullptr, &n_splits, nullptr)
           : launch_loss_grad<double>(nullptr, B, L, nullptr, D, nullptr, K, nullptr, nullptr,
                                      ws_token_map{}, num_vars, nullptr, nullptr, nullptr,
                                      nullptr, nullptr, &n_splits, nullptr);
  if (st != WS_OK) return st;
  *bytes = (size_t)(B * n_splits) * (size_t)(K + 1) * sizeof(double) + 256 +
           loss_grad_bucket_bytes(B);
  return WS_OK;
}

extern "C" ws_status ws_loss_grad(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                                  const void* x, int64_t num_vars, int64_t D,
                                  const void* constants, int64_t K, const void* y,
                                  const int32_t* active, double* out_loss, void* out_grad,
                                  const ws_token_map* ids, void* workspace, size_t workspace_bytes,
                                  void* stream) {
  using namespace ws;
  clear_error();
  ws_status st = loss_grad_check(dtype, B, L, D, K, num_vars);
  if (st != WS_OK) return st;
  if (!ids) return fail("token map is required");
  if (B == 0) return WS_OK;
  if (D == 0 || L == 0) return fail("loss_grad needs at least one row and one token");
  if (!population || !y || !out_loss || (K > 0 && (!constants || !out_grad)) ||
      (num_vars > 0 && !x) || !workspace)
    return fail("null tensor pointer");
  size_t need = 0;
  st = ws_loss_grad_workspace_bytes(dtype, B, L, num_vars, D, K, &need);
  if (st != WS_OK) return st;
  if (workspace_bytes < need) return fail("loss_grad workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part_loss = static_cast<double*>(workspace);
  int64_t n_splits = 1;
  st = dtype == WS_F32
           ? launch_loss_grad<float>(nullptr, B, L, nullptr, D, nullptr, K, nullptr, nullptr,
                                     *ids, num_vars, nullptr, nullptr, nullptr, nullptr,
                                     nullptr, &n_splits, nullptr)
           : launch_loss_grad<double>(nullptr, B, L, nullptr, D, nullptr, K, nullptr, nullptr,
                                      *ids, num_vars, nullptr, nullptr, nullptr, nullptr,
                                      nullptr, &n_splits, nullptr);
  if (st != WS_OK) return st;
  double* part_grad = part_loss + B * n_splits;
  int32_t* buckets = reinterpret_cast<int32_t*>(part_grad + B * n_splits * K);
  if (dtype == WS_F32)
    return launch_loss_grad<float>(population, B, L, x, D, constants, K, y, active, *ids,
                                   num_vars, part_loss, part_grad, out_loss, out_grad, buckets,
                                   nullptr, s);
  return launch_loss_grad<double>(population, B, L, x, D, constants, K, y, active, *ids,
                                  num_vars, part_loss, part_grad, out_loss, out_grad, buckets,
                                  nullptr, s);
}
