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
// B200 layout: one block owns one program for a range of rows.  Thread 0 parses the program once
// per block (parse_loss_program) into a shared-memory tape whose operands are resolved to
// addresses: operators, constant leaves and the program's distinct variables own [thread][R]
// slots, constants and literals sit in a broadcast scalar table, so neither sweep branches on an
// operand's kind.  The program is a tree, so the only reader of a value is its parent, which
// reads it before writing the adjoint into the same slot.  Two kernels share this tape:
//   ref_kernel  (ws_eval_rpn_backward): values forward, the reference's adjoint expressions
//               backward (the operator's rule, from the operand values), constant-leaf rows
//               summed in FP64 in the order the reference's reverse walk meets them; a
//               fixed-order block sum writes grad_constants without atomics when one block covers
//               all rows of a program, one atomic per (block, slot) otherwise -- the reference
//               issues one atomic per (row, constant node);
//   loss_kernel (ws_loss_grad, the batched L-BFGS): the forward sweep also stores each operand's
//               local derivative in the operand's slot, so the reverse sweep is the same multiply
//               for every operator; programs are grouped by tape size, one launch per group.
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
  int64_t V;              // variables
  int tape_ops;           // tape slots (>= every program's operators; loss_kernel: operators,
                          // constant leaves and staged variables)
  const int32_t* list;        // optional: the programs of this launch (a bucket) ...
  const int32_t* list_count;  // ... and how many there are (read on the device)
  double* part_loss;      // [n_items]   sum over the item's rows of (pred - y)^2
  double* part_grad;      // [n_items, K] sum over the item's rows of the constant adjoints
};

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

// ---- helpers of the adjoint kernels ---------------------------------------------------------
// Every thread carries R consecutive rows through each tape step, so one decode of an operator
// serves R rows; a tape slot holds [thread][R] values (16-byte vector accesses).  Constant
// adjoints are summed in registers when K <= kRegSlots (the slot of a delivery is the same for
// the whole block, so the register is chosen by a uniform switch).
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

// ---- loss mode: the loss and its gradient with respect to the constants ---------------------
// The root adjoint of row d is dL/dpred = 2 (pred - y[d]) / D and the arithmetic is in T.  Every
// operand that carries a gradient -- an earlier operator or a constant leaf -- owns a tape slot.
// The forward sweep evaluates operator o from its operands, stores the value in slot o and writes
// the local derivative of o with respect to each operand into that operand's slot, whose value o
// has just consumed (the program is a tree: o is its only reader), or into a sink slot for an
// operand without a gradient.  The reverse sweep is then the same steps for every operator
// whatever its rule: load its adjoint, multiply each operand's derivative by it and store the
// product where the derivative was.  A constant leaf's slot thus ends the row group holding its
// adjoint, summed into the constant's accumulator by a short epilogue.  No rule is evaluated
// twice, neither sweep branches on an operand's kind, and operand kinds are resolved once per
// program, at parse time, into shared-memory addresses: a tape slot read at the thread's own
// offset, or an entry of the program's scalar table (R copies of a constant or literal) read by
// every thread at the same address.  The derivatives are the reference's adjoint rules with the
// adjoint factored out (backward_kernels.cu:222-278), in T: + and - hand on +-1, * the other
// operand, / 1/b and -(a/b^2) when |b| >= 1e-9, pow b*a^(b-1) and a^b*log(a) when a > 0, sin
// cos(a), cos -sin(a), log 1/a when |a| > 1e-9, exp its value, sqrt 0.5/sqrt(a) when a > 1e-9,
// neg -1, the other operators 0; zero adjoints hand on nothing.  Against the reference's
// adjoint / b (and adjoint / a for log) the reciprocal rounds once more, and flushes to zero for
// |b| > 2^126, where the contribution is below 2^-126 times the adjoint.
enum : uint8_t {
  LF_BIN = 1,     // binary operator
  LF_A_VEC = 2,   // the left operand is a tape slot (else a scalar-table entry)
  LF_B_VEC = 4,
  LF_A_GRAD = 8,  // the left operand carries a gradient (LOp::fa is its slot)
  LF_B_GRAD = 16,
  LF_REACH = 32,  // the value flows into the root
};
// LOp::code: the adjoint code when the token's forward and adjoint rules are the pair of one
// operator (every token of a real grammar), else kCodeGeneric (value by fop, derivatives by bop)
constexpr uint8_t kCodeGeneric = 0xFF;

// One operator of a loss-mode tape.  Addresses are in 16-byte units from the start of the
// block's dynamic shared memory.
struct __align__(16) LOp {
  uint16_t a, b;    // operands (a unary operator reads its operand twice)
  uint16_t fa, fb;  // where each operand's derivative goes: its slot, or the sink slot
  uint16_t self;    // this operator's slot
  uint8_t code, fop, bop, flags;
  uint16_t pad;
};

// Shared memory of a loss-mode block (bytes): operators | staged-variable list | constant-leaf
// slots and list | scalar table (one 16-byte entry per terminal token at most) | (K > kRegSlots) FP64
// constant accumulators | work: the tape (M slots and the sink) during the rows, the block
// reduction after them.
struct LossLayout {
  size_t ops, stage, leaf, scal, touched, cacc, work, bytes;
};

// `touched`: room for the per-constant "received a contribution" flags (the reference-mode
// kernel writes only those slots).
__host__ __device__ inline LossLayout loss_layout(int64_t M, int64_t L, int64_t K, int threads,
                                                  size_t vec_bytes, bool kreg,
                                                  bool touched = false) {
  LossLayout l;
  l.ops = 0;
  l.stage = al16((size_t)M * sizeof(LOp));
  l.leaf = l.stage + al16((size_t)M);
  l.scal = l.leaf + al16((size_t)2 * M * sizeof(uint32_t));
  l.touched = l.scal + (size_t)L * 16;
  l.cacc = l.touched + (touched ? al16((size_t)K * sizeof(int)) : 0);
  l.work = l.cacc + (kreg ? 0 : (size_t)K * threads * sizeof(double));
  const size_t tape = (size_t)(M + 1) * threads * vec_bytes;
  const size_t red = (size_t)((kreg ? K : 0) + 1) * threads * sizeof(double);
  l.bytes = l.work + (tape > red ? tape : red);
  return l;
}

template <typename T>
struct LRoot {
  int n_ops;      // operators in the tape
  int valid;      // the reference's forward pass yields a root (final depth 1)
  int n_stage;    // distinct variables staged per row group ...
  int stage0;     // ... in the slots from this address on (16-byte units, one slot apart)
  int n_leaf;     // entries of the constant-leaf list (leaves whose parent reaches the root)
  uint16_t kind;  // OPD_OP, OPD_VAR, OPD_LIT or OPD_CONST
  uint16_t at;    // address of the root's slot (OPD_OP, OPD_VAR)
  uint16_t ck;    // constant slot (OPD_CONST)
  T scalar;       // value of a literal or constant root
};

__device__ __forceinline__ uint8_t loss_code(uint8_t fop, uint8_t bop) {
  const uint8_t pair_fop[12] = {FO_NONE, FO_ADD, FO_SUB, FO_MUL, FO_DIV, FO_POW,
                                FO_SIN,  FO_COS, FO_LOG, FO_EXP, FO_SQRT, FO_NEG};
  return (bop != BO_NONE && bop < 12 && pair_fop[bop] == fop) ? bop : kCodeGeneric;
}

// Addresses of one block's tape (16-byte units): slot s sits at tape + s * slot, the sink is
// slot M, the scalar table starts at scal.
struct LossAddr {
  uint32_t tape, slot, scal, sink;
};

// Walks program b with parse_program's rules (the reference's forward loop) and resolves each
// operand into an address: operators take slots 0..n_ops-1, constant leaves the next slots, each
// distinct variable the slots after them (x staged there once per row group); constants and
// literals take scalar-table entries, filled here.  Slots in use <= operators + constant tokens +
// distinct variables <= tokens.  leaf[0, M) holds each constant leaf's constant slot, leaf[M, 2M)
// receives (address | constant slot << 16) of the leaves whose parent reaches the root, in the
// order a reverse walk meets them.
template <typename T, int R>
__device__ LRoot<T> parse_loss_program(const uint8_t* __restrict__ prog, int64_t L, int64_t K,
                                       const uint8_t* s_tab, const T* s_lit,
                                       const T* __restrict__ cst, int64_t V,
                                       const LossAddr& ad, unsigned char* smem, LOp* ops,
                                       uint8_t* stage, uint32_t* leaf) {
  const uint8_t* t_kind = s_tab;
  const uint8_t* t_fop = s_tab + 256;
  const uint8_t* t_bop = s_tab + 512;
  const uint8_t* t_arg = s_tab + 768;
  constexpr int kPer = 16 / (int)sizeof(T);  // values per scalar-table entry
  T* scal = reinterpret_cast<T*>(smem + ((size_t)ad.scal << 4));
  uint8_t sk[kStack];   // operand kind
  uint16_t si[kStack];  // operator index, variable ordinal or scalar-table entry
  uint16_t sl[kStack];  // constant-leaf ordinal of a constant
  int sp = 0, n_ops = 0, n_leaf = 0, n_stage = 0, n_scal = 0;
  int64_t c_idx = 0;
  bool bad = false;  // an array bound was hit (bounds-checked build only)
  const int M = (int)ad.sink;
  for (int pc = 0; pc < (int)L; ++pc) {
    const int tok = prog[pc];
    const uint8_t kind = t_kind[tok];
    if (kind == BK_PAD) break;
    if (kind == BK_VAR || kind == BK_LIT || kind == BK_CONST) {
      uint8_t k = kind == BK_VAR ? OPD_VAR : OPD_LIT;
      uint16_t ix = t_arg[tok], c = 0;
      if (kind == BK_VAR && !WS_BC(ix < V, BC_ADJ_PARSE, ix)) {
        bad = true;
        break;
      }
      if (kind == BK_CONST) {
        if (K > 0) {
          k = OPD_CONST;
          c = (uint16_t)(c_idx < K ? c_idx : K - 1);
          c_idx++;
        } else {
          ix = 10;  // C without constants pushes 1.0 and takes no gradient
        }
      }
      if (sp < kStack) {
        uint16_t lo = 0;
        if (k == OPD_VAR) {
          int j = 0;
          while (j < n_stage && stage[j] != ix) ++j;
          if (j == n_stage) {
            if (!WS_BC(n_stage < M, BC_ADJ_PARSE, n_stage)) {
              bad = true;
              break;
            }
            stage[n_stage++] = (uint8_t)ix;
          }
          ix = (uint16_t)j;
        } else {
          if (!WS_BC(n_scal < (int)L && (k != OPD_CONST || n_leaf < M), BC_ADJ_PARSE, n_scal)) {
            bad = true;
            break;
          }
          const T v = k == OPD_CONST ? cst[c] : (ix < 10 ? s_lit[ix] : (T)1.0);
          for (int r = 0; r < R; ++r) scal[(size_t)n_scal * kPer + r] = v;
          if (k == OPD_CONST) {
            lo = (uint16_t)n_leaf;
            leaf[n_leaf++] = c;
          }
          ix = (uint16_t)n_scal++;
        }
        sk[sp] = k;
        si[sp] = ix;
        sl[sp] = lo;
        ++sp;
      }
      continue;
    }
    LOp o;
    o.fop = t_fop[tok];
    o.bop = t_bop[tok];
    o.code = loss_code(o.fop, o.bop);
    o.flags = 0;
    o.a = o.b = o.fa = o.fb = 0;
    o.self = (uint16_t)n_ops;
    o.pad = 0;
    const int n_in = kind == BK_BIN ? 2 : 1;
    if (sp < n_in) break;
    if (n_in == 2) o.flags |= LF_BIN;
    for (int side = n_in - 1; side >= 0; --side) {  // the right operand is on top
      --sp;
      const uint8_t k = sk[sp];
      uint8_t fl = 0;
      uint16_t f = 0;
      if (k == OPD_OP) {
        fl = LF_A_VEC | LF_A_GRAD;
      } else if (k == OPD_VAR) {
        fl = LF_A_VEC;
      } else if (k == OPD_CONST) {
        fl = LF_A_GRAD;
        f = sl[sp];
      }
      if (side == 0) {
        o.a = si[sp], o.fa = f;
        o.flags |= fl;
      } else {
        o.b = si[sp], o.fb = f;
        o.flags |= (uint8_t)(fl << 1);  // the B flags are the A flags shifted by one
      }
    }
    if (!WS_BC(n_ops < M, BC_ADJ_PARSE, n_ops)) {
      bad = true;
      break;
    }
    ops[n_ops] = o;
    sk[sp] = OPD_OP;  // an operator always finds room: it just freed one or two slots
    si[sp] = (uint16_t)n_ops;
    ++sp;
    ++n_ops;
  }
  if (!WS_BC(n_ops + n_leaf + n_stage <= M, BC_ADJ_PARSE, n_ops + n_leaf + n_stage)) bad = true;
  const uint32_t stage_first = (uint32_t)(n_ops + n_leaf);
  const uint16_t sink = (uint16_t)(ad.tape + ad.sink * ad.slot);
  LRoot<T> r;
  r.n_ops = n_ops;
  r.valid = (sp == 1 && !bad) ? 1 : 0;
  r.n_stage = n_stage;
  r.stage0 = (int)(ad.tape + stage_first * ad.slot);
  r.kind = sp >= 1 ? sk[0] : OPD_LIT;
  r.at = 0;
  r.ck = 0;
  r.scalar = (T)0;
  r.n_leaf = 0;
  if (bad) return r;
  if (sp >= 1) {
    if (r.kind == OPD_OP) r.at = (uint16_t)(ad.tape + si[0] * ad.slot);
    else if (r.kind == OPD_VAR) r.at = (uint16_t)(ad.tape + (stage_first + si[0]) * ad.slot);
    else r.scalar = scal[(size_t)si[0] * kPer];
    if (r.kind == OPD_CONST) r.ck = (uint16_t)leaf[sl[0]];
  }
  constexpr uint8_t kOpA = LF_A_VEC | LF_A_GRAD, kOpB = LF_B_VEC | LF_B_GRAD;
  uint32_t* live = leaf + M;
  int n_live = 0;
  if (r.valid && r.kind == OPD_OP) {  // mark the operators whose value reaches the root
    ops[si[0]].flags |= LF_REACH;
    for (int o = si[0]; o >= 0; --o) {
      const LOp& q = ops[o];
      if (!(q.flags & LF_REACH)) continue;
      if ((q.flags & kOpA) == kOpA) ops[q.a].flags |= LF_REACH;
      if ((q.flags & kOpB) == kOpB) ops[q.b].flags |= LF_REACH;
      // the constant leaves of the operators that reach, in the order a reverse walk meets
      // them (operators from the last, the right operand first): (slot | constant slot << 16)
      if ((q.flags & kOpB) == LF_B_GRAD)
        live[n_live++] = (ad.tape + (uint32_t)(n_ops + q.fb) * ad.slot) | (leaf[q.fb] << 16);
      if ((q.flags & kOpA) == LF_A_GRAD)
        live[n_live++] = (ad.tape + (uint32_t)(n_ops + q.fa) * ad.slot) | (leaf[q.fa] << 16);
    }
  }
  for (int o = 0; o < n_ops; ++o) {  // indices to addresses
    LOp& q = ops[o];
    for (int side = 0; side < 2; ++side) {
      const uint8_t fl = side ? (uint8_t)(q.flags >> 1) : q.flags;
      uint16_t& x = side ? q.b : q.a;
      uint16_t& f = side ? q.fb : q.fa;
      if (side == 1 && !(q.flags & LF_BIN)) {  // a unary operator reads its operand twice
        x = q.a;
        f = sink;
        if (q.flags & LF_A_VEC) q.flags |= LF_B_VEC;
        continue;
      }
      if ((fl & kOpA) == kOpA) {
        x = (uint16_t)(ad.tape + x * ad.slot);
        f = x;
      } else if (fl & LF_A_VEC) {
        x = (uint16_t)(ad.tape + (stage_first + x) * ad.slot);
        f = sink;
      } else {
        x = (uint16_t)(ad.scal + x);
        f = (fl & LF_A_GRAD) ? (uint16_t)(ad.tape + (n_ops + f) * ad.slot) : sink;
      }
    }
    q.self = (uint16_t)(ad.tape + o * ad.slot);
  }
  r.n_leaf = n_live;
  return r;
}

// The derivatives of an adjoint rule (bop) at operands a, b and value v: the fallback of
// op_with_derivs for tokens whose forward and adjoint rules are not one operator's pair.
template <typename T>
__device__ __forceinline__ void derivs_generic(uint8_t bop, T a, T b, T v, T& da, T& db) {
  da = (T)0;
  db = (T)0;
  switch (bop) {
    case BO_ADD: da = (T)1; db = (T)1; break;
    case BO_SUB: da = (T)1; db = (T)-1; break;
    case BO_MUL: da = b; db = a; break;
    case BO_DIV:
      if (fabs(b) >= (T)1e-9) { da = (T)1 / b; db = -(a / (b * b)); }
      break;
    case BO_POW:
      if (a > 0) { da = b * pow(a, b - (T)1); db = v * log(a); }
      break;
    case BO_SIN: da = cos(a); break;
    case BO_COS: da = -sin(a); break;
    case BO_LOG: if (fabs(a) > (T)1e-9) da = (T)1 / a; break;
    case BO_EXP: da = v; break;
    case BO_SQRT: if (a > (T)1e-9) da = (T)0.5 / sqrt(a); break;
    case BO_NEG: da = (T)-1; break;
    default: break;
  }
}

// Value and the local derivatives with respect to both operands of one operator, R rows.
template <typename T, int R>
__device__ __forceinline__ void op_with_derivs(const LOp& op, const T (&a)[R], const T (&b)[R],
                                               T (&v)[R], T (&da)[R], T (&db)[R]) {
  WS_FOR_R db[r] = (T)0;
  switch (op.code) {
    case BO_ADD: WS_FOR_R { v[r] = a[r] + b[r]; da[r] = (T)1; db[r] = (T)1; } break;
    case BO_SUB: WS_FOR_R { v[r] = a[r] - b[r]; da[r] = (T)1; db[r] = (T)-1; } break;
    case BO_MUL: WS_FOR_R { v[r] = a[r] * b[r]; da[r] = b[r]; db[r] = a[r]; } break;
    case BO_DIV:
      WS_FOR_R {
        v[r] = fwd_binary<T>(FO_DIV, a[r], b[r]);
        const bool ok = fabs(b[r]) >= (T)1e-9;
        da[r] = ok ? (T)1 / b[r] : (T)0;
        db[r] = ok ? -(a[r] / (b[r] * b[r])) : (T)0;
      }
      break;
    case BO_POW:
      WS_FOR_R {
        v[r] = fwd_binary<T>(FO_POW, a[r], b[r]);
        da[r] = (T)0;
        if (a[r] > 0) {
          da[r] = b[r] * pow(a[r], b[r] - (T)1);
          db[r] = v[r] * log(a[r]);
        }
      }
      break;
    case BO_SIN: WS_FOR_R { v[r] = sin(a[r]); da[r] = cos(a[r]); } break;
    case BO_COS: WS_FOR_R { v[r] = cos(a[r]); da[r] = -sin(a[r]); } break;
    case BO_LOG:
      WS_FOR_R {
        v[r] = fwd_unary<T>(FO_LOG, a[r]);
        da[r] = fabs(a[r]) > (T)1e-9 ? (T)1 / a[r] : (T)0;
      }
      break;
    case BO_EXP: WS_FOR_R { v[r] = fwd_unary<T>(FO_EXP, a[r]); da[r] = v[r]; } break;
    case BO_SQRT:
      WS_FOR_R {
        v[r] = fwd_unary<T>(FO_SQRT, a[r]);
        da[r] = a[r] > (T)1e-9 ? (T)0.5 / sqrt(a[r]) : (T)0;
      }
      break;
    case BO_NEG: WS_FOR_R { v[r] = -a[r]; da[r] = (T)-1; } break;
    default:
      WS_FOR_R {
        v[r] = (op.flags & LF_BIN) ? fwd_binary<T>(op.fop, a[r], b[r]) : fwd_unary<T>(op.fop, a[r]);
        derivs_generic<T>(op.bop, a[r], b[r], v[r], da[r], db[r]);
      }
      break;
  }
}

template <typename T, int R, bool KREG>
__global__ void __launch_bounds__(128) loss_kernel(BwdParams<T> p, BwdLut lut) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int TS = p.tape_stride;
  const int M = p.tape_ops;  // tape slots, the sink not counted
  const LossLayout lay = loss_layout(M, p.L, p.K, TS, R * sizeof(T), KREG);
  LOp* ops = reinterpret_cast<LOp*>(smem + lay.ops);
  uint8_t* stage = smem + lay.stage;
  uint32_t* leaf = reinterpret_cast<uint32_t*>(smem + lay.leaf);
  double* cacc = reinterpret_cast<double*>(smem + lay.cacc);
  unsigned char* work = smem + lay.work;
  LossAddr ad;
  ad.tape = (uint32_t)(lay.work >> 4);
  ad.slot = (uint32_t)((size_t)TS * R * sizeof(T) >> 4);
  ad.scal = (uint32_t)(lay.scal >> 4);
  ad.sink = (uint32_t)M;
  __shared__ LRoot<T> s_root;
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
  const uint32_t my = (uint32_t)tid * (uint32_t)(R * sizeof(T));  // this thread's part of a slot
  // a tape slot (this thread's R values) or a scalar-table entry, by its 16-byte address
#define WS_AT(addr, mine) reinterpret_cast<T*>(smem + ((uint32_t)(addr) << 4) + ((mine) ? my : 0u))
  const T loss_scale = (T)(2.0 / (double)p.D);

  const int64_t n_items = p.list ? (int64_t)(*p.list_count) * p.n_splits : p.n_items;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t li = item / p.n_splits;
    const int64_t split = item - li * p.n_splits;
    const int64_t b = p.list ? (int64_t)p.list[li] : li;
    const int64_t slot = b * p.n_splits + split;  // partial sums of (program, row range)
    if (p.active && p.active[b] == 0) continue;  // uniform over the block
    __syncthreads();
    if (tid == 0 && s_prog != b) {
      s_root = parse_loss_program<T, R>(p.pop + b * p.L, p.L, p.K, s_tab, s_lit,
                                        p.consts + b * p.K, p.V, ad, smem, ops, stage, leaf);
      s_prog = b;
    }
    if (!KREG)
      for (int64_t k = 0; k < p.K; ++k) cacc[k * TS + tid] = 0.0;
    __syncthreads();
    const LRoot<T> rt = s_root;
    if (!rt.valid) {  // no prediction: infinite loss, no gradient
      if (tid == 0) p.part_loss[slot] = __longlong_as_double(0x7ff0000000000000ll);
      for (int64_t k = tid; k < p.K; k += blockDim.x) p.part_grad[slot * p.K + k] = 0.0;
      continue;
    }
    const int64_t d_begin = split * p.rows_per_split;
    int64_t d_end = d_begin + p.rows_per_split;
    if (d_end > p.D) d_end = p.D;
    const int n = rt.n_ops;
    T cr[kRegSlots];
#pragma unroll
    for (int k = 0; k < kRegSlots; ++k) cr[k] = (T)0;
    double lacc = 0.0;

    for (int64_t d0 = d_begin + (int64_t)tid * R; d0 < d_end; d0 += (int64_t)TS * R) {
      // this thread's rows of the program's variables (only this thread reads them: no barrier)
      for (int j = 0; j < rt.n_stage; ++j) {
        const T* xr = p.x + (int64_t)stage[j] * p.D;
        T xv[R];
        WS_FOR_R xv[r] = d0 + r < d_end ? xr[d0 + r] : (T)0;
        st_vec<T, R>(WS_AT(rt.stage0 + j * ad.slot, true), xv);
      }
      T yv[R];
      WS_FOR_R yv[r] = d0 + r < d_end ? p.y[d0 + r] : (T)0;
      // forward: values, and each operand's derivative where the operand was
      for (int o = 0; o < n; ++o) {
        const LOp op = ops[o];
        T a[R], bv[R], v[R], da[R], db[R];
        ld_vec<T, R>(WS_AT(op.a, op.flags & LF_A_VEC), a);
        ld_vec<T, R>(WS_AT(op.b, op.flags & LF_B_VEC), bv);
        op_with_derivs<T, R>(op, a, bv, v, da, db);
        st_vec<T, R>(WS_AT(op.self, true), v);
        st_vec<T, R>(WS_AT(op.fa, true), da);
        st_vec<T, R>(WS_AT(op.fb, true), db);
      }
      // the root: prediction, loss, root adjoint
      T pred[R];
      if (rt.kind == OPD_OP || rt.kind == OPD_VAR) {
        ld_vec<T, R>(WS_AT(rt.at, true), pred);
      } else {
        WS_FOR_R pred[r] = rt.scalar;
      }
      T g[R];
      WS_FOR_R {
        const T diff = d0 + r < d_end ? pred[r] - yv[r] : (T)0;
        lacc += (double)diff * (double)diff;
        g[r] = diff * loss_scale;
      }
      if (rt.kind == OPD_CONST) {  // a one-constant program
        T s = (T)0;
        WS_FOR_R s += g[r];
        if (KREG) creg_add<T>(cr, rt.ck, s);
        else cacc[(size_t)rt.ck * TS + tid] += (double)s;
        continue;
      }
      if (rt.kind != OPD_OP) continue;  // a variable or a literal: no constant to move
      st_vec<T, R>(WS_AT(rt.at, true), g);
      // reverse: each operator's adjoint times the derivative in each operand's slot, stored
      // back there (the right operand first, as the reference's reverse walk meets it)
      for (int o = n - 1; o >= 0; --o) {
        const LOp op = ops[o];
        if (!(op.flags & LF_REACH)) continue;
        T ga[R];
        ld_vec<T, R>(WS_AT(op.self, true), ga);
        if (op.flags & LF_B_GRAD) {
          T* q = WS_AT(op.fb, true);
          T f[R];
          ld_vec<T, R>(q, f);
          WS_FOR_R f[r] = ga[r] == (T)0 ? (T)0 : f[r] * ga[r];
          st_vec<T, R>(q, f);
        }
        if (op.flags & LF_A_GRAD) {
          T* q = WS_AT(op.fa, true);
          T f[R];
          ld_vec<T, R>(q, f);
          WS_FOR_R f[r] = ga[r] == (T)0 ? (T)0 : f[r] * ga[r];
          st_vec<T, R>(q, f);
        }
      }
      // the constant leaves' adjoints into their constants' accumulators
      for (int j = 0; j < rt.n_leaf; ++j) {
        const uint32_t e = leaf[M + j];
        T c[R];
        ld_vec<T, R>(WS_AT(e & 0xFFFFu, true), c);
        T s = (T)0;
        WS_FOR_R s += c[r];
        if (KREG) creg_add<T>(cr, (int)(e >> 16), s);
        else cacc[(size_t)(e >> 16) * TS + tid] += (double)s;
      }
    }
#undef WS_AT
    __syncthreads();  // the tape is free: the reduction reuses its memory
    double* cred = KREG ? reinterpret_cast<double*>(work) : cacc;
    double* lacc_s = reinterpret_cast<double*>(work) + (KREG ? (size_t)p.K * TS : 0);
    if (KREG) {
#pragma unroll
      for (int k = 0; k < kRegSlots; ++k)
        if (k < p.K) cred[(size_t)k * TS + tid] = (double)cr[k];
    }
    lacc_s[tid] = lacc;
    __syncthreads();
    // fixed-order reduction over the block's threads, one thread per slot
    for (int64_t k = tid; k < p.K; k += blockDim.x) {
      double s = 0.0;
      for (int t = 0; t < (int)blockDim.x; ++t) s += cred[k * TS + t];
      p.part_grad[slot * p.K + k] = s;
    }
    if (tid == 0) {
      double s = 0.0;
      for (int t = 0; t < (int)blockDim.x; ++t) s += lacc_s[t];
      p.part_loss[slot] = s;
    }
  }
}

// ---- reference mode on the resolved tape (ws_eval_rpn_backward) ------------------------------
// The program parsed as for the loss mode (operands as shared-memory addresses, constant leaves
// with their own slots), but the forward sweep stores values only: the reverse sweep evaluates
// the reference's own adjoint expressions (backward_kernels.cu:222-278, double promotions
// included: acc_d / acc_t) from the operand values, which sit in the operands' slots until the
// operator writes their adjoints there.  A constant leaf's contribution goes to its slot and an
// epilogue adds the leaves' rows to their constants' FP64 accumulators in the order the reverse
// walk met them, so every per-row term and every sum is the one of the direct formulation.
template <typename T, int R, bool KREG>
__global__ void __launch_bounds__(128) ref_kernel(BwdParams<T> p, BwdLut lut) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int TS = p.tape_stride;
  const int M = p.tape_ops;
  const LossLayout lay = loss_layout(M, p.L, p.K, TS, R * sizeof(T), KREG, true);
  LOp* ops = reinterpret_cast<LOp*>(smem + lay.ops);
  uint8_t* stage = smem + lay.stage;
  uint32_t* leaf = reinterpret_cast<uint32_t*>(smem + lay.leaf);
  int* touched = reinterpret_cast<int*>(smem + lay.touched);
  double* cacc = reinterpret_cast<double*>(smem + lay.cacc);
  unsigned char* work = smem + lay.work;
  LossAddr ad;
  ad.tape = (uint32_t)(lay.work >> 4);
  ad.slot = (uint32_t)((size_t)TS * R * sizeof(T) >> 4);
  ad.scal = (uint32_t)(lay.scal >> 4);
  ad.sink = (uint32_t)M;
  __shared__ LRoot<T> s_root;
  __shared__ int64_t s_prog;
  __shared__ T s_lit[10];
  __shared__ uint8_t s_tab[1024];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    s_tab[t] = lut.kind[t];
    s_tab[256 + t] = lut.fop[t];
    s_tab[512 + t] = lut.bop[t];
    s_tab[768 + t] = lut.arg[t];
  }
  if (threadIdx.x < 10) s_lit[threadIdx.x] = (T)lut.lit[threadIdx.x];
  if (threadIdx.x == 0) s_prog = -1;
  const int tid = threadIdx.x;
  const uint32_t my = (uint32_t)tid * (uint32_t)(R * sizeof(T));
#define WS_AT(addr, mine) reinterpret_cast<T*>(smem + ((uint32_t)(addr) << 4) + ((mine) ? my : 0u))

  const int64_t n_items = p.list ? (int64_t)(*p.list_count) * p.n_splits : p.n_items;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t li = item / p.n_splits;
    const int64_t split = item - li * p.n_splits;
    const int64_t b = p.list ? (int64_t)p.list[li] : li;
    __syncthreads();
    if (tid == 0 && s_prog != b) {
      s_root = parse_loss_program<T, R>(p.pop + b * p.L, p.L, p.K, s_tab, s_lit,
                                        p.consts + b * p.K, p.V, ad, smem, ops, stage, leaf);
      s_prog = b;
    }
    for (int64_t k = tid; k < p.K; k += blockDim.x) touched[k] = 0;
    if (!KREG)
      for (int64_t k = 0; k < p.K; ++k) cacc[k * TS + tid] = 0.0;
    __syncthreads();
    const LRoot<T> rt = s_root;
    if (!rt.valid) continue;
    const int64_t d_begin = split * p.rows_per_split;
    int64_t d_end = d_begin + p.rows_per_split;
    if (d_end > p.D) d_end = p.D;
    const int n = rt.n_ops;
    double cr[kRegSlots];
#pragma unroll
    for (int k = 0; k < kRegSlots; ++k) cr[k] = 0.0;
    auto add_const = [&](int ck, const T (&c)[R]) {
      double s = 0.0;
      bool any = false;
      WS_FOR_R {
        if (c[r] != (T)0) {
          s += (double)c[r];
          any = true;
        }
      }
      if (any) {
        if (KREG) creg_add<double>(cr, ck, s);
        else cacc[(size_t)ck * TS + tid] += s;
        touched[ck] = 1;
      }
    };

    for (int64_t d0 = d_begin + (int64_t)tid * R; d0 < d_end; d0 += (int64_t)TS * R) {
      for (int j = 0; j < rt.n_stage; ++j) {
        const T* xr = p.x + (int64_t)stage[j] * p.D;
        T xv[R];
        WS_FOR_R xv[r] = d0 + r < d_end ? xr[d0 + r] : (T)0;
        st_vec<T, R>(WS_AT(rt.stage0 + j * ad.slot, true), xv);
      }
      T g[R];  // grad_output of the R rows
      WS_FOR_R g[r] = d0 + r < d_end ? p.gout[b * p.D + d0 + r] : (T)0;
      // forward: values
      for (int o = 0; o < n; ++o) {
        const LOp op = ops[o];
        T a[R], v[R];
        ld_vec<T, R>(WS_AT(op.a, op.flags & LF_A_VEC), a);
        if (op.flags & LF_BIN) {
          T bv[R];
          ld_vec<T, R>(WS_AT(op.b, op.flags & LF_B_VEC), bv);
          fwd_binary_vec<T, R>(op.fop, a, bv, v);
        } else {
          fwd_unary_vec<T, R>(op.fop, a, v);
        }
        st_vec<T, R>(WS_AT(op.self, true), v);
      }
      if (rt.kind == OPD_CONST) {  // a one-constant program
        add_const(rt.ck, g);
        continue;
      }
      if (rt.kind != OPD_OP) continue;  // a variable or a literal: no constant to move
      st_vec<T, R>(WS_AT(rt.at, true), g);
      // reverse: the reference's rules from the operand values, adjoints into the operands'
      // slots (the right operand first)
      for (int o = n - 1; o >= 0; --o) {
        const LOp op = ops[o];
        if (!(op.flags & LF_REACH)) continue;
        T ga[R], lv[R], ca[R], cb[R];
        ld_vec<T, R>(WS_AT(op.self, true), ga);
        ld_vec<T, R>(WS_AT(op.a, op.flags & LF_A_VEC), lv);
        WS_FOR_R { ca[r] = (T)0; cb[r] = (T)0; }
        if (op.flags & LF_BIN) {
          T rv[R];
          ld_vec<T, R>(WS_AT(op.b, op.flags & LF_B_VEC), rv);
          switch (op.bop) {
            case BO_ADD: WS_FOR_R { ca[r] += ga[r]; cb[r] += ga[r]; } break;
            case BO_SUB: WS_FOR_R { ca[r] += ga[r]; cb[r] -= ga[r]; } break;
            case BO_MUL: WS_FOR_R { acc_t(ca[r], rv[r], ga[r]); acc_t(cb[r], lv[r], ga[r]); } break;
            case BO_DIV:
              WS_FOR_R {
                if (fabs(rv[r]) >= (T)1e-9) {
                  acc_d(ca[r], 1.0 / rv[r], ga[r]);
                  acc_t(cb[r], -(lv[r] / (rv[r] * rv[r])), ga[r]);
                }
              }
              break;
            case BO_POW:
              WS_FOR_R {
                if (lv[r] > 0) {
                  const T out_val = fwd_binary<T>(op.fop, lv[r], rv[r]);
                  acc_d(ca[r], (double)rv[r] * pow((double)lv[r], (double)rv[r] - 1.0), ga[r]);
                  acc_t(cb[r], out_val * log(lv[r]), ga[r]);
                }
              }
              break;
            default: break;
          }
          WS_FOR_R if (ga[r] == (T)0) cb[r] = (T)0;
          if (op.flags & LF_B_GRAD) st_vec<T, R>(WS_AT(op.fb, true), cb);
        } else {
          switch (op.bop) {
            case BO_SIN: WS_FOR_R acc_t(ca[r], cos(lv[r]), ga[r]); break;
            case BO_COS: WS_FOR_R acc_t(ca[r], -sin(lv[r]), ga[r]); break;
            case BO_LOG:
              WS_FOR_R if (fabs(lv[r]) > (T)1e-9) acc_d(ca[r], 1.0 / lv[r], ga[r]);
              break;
            case BO_EXP: WS_FOR_R acc_t(ca[r], fwd_unary<T>(op.fop, lv[r]), ga[r]); break;
            case BO_SQRT:
              WS_FOR_R if (lv[r] > (T)1e-9) acc_d(ca[r], 0.5 / sqrt(lv[r]), ga[r]);
              break;
            case BO_NEG: WS_FOR_R ca[r] += -ga[r]; break;
            default: break;
          }
        }
        WS_FOR_R if (ga[r] == (T)0) ca[r] = (T)0;
        if (op.flags & LF_A_GRAD) st_vec<T, R>(WS_AT(op.fa, true), ca);
      }
      for (int j = 0; j < rt.n_leaf; ++j) {
        const uint32_t e = leaf[M + j];
        T c[R];
        ld_vec<T, R>(WS_AT(e & 0xFFFFu, true), c);
        add_const((int)(e >> 16), c);
      }
    }
#undef WS_AT
    __syncthreads();  // the tape is free: the reduction reuses its memory
    double* cred = KREG ? reinterpret_cast<double*>(work) : cacc;
    if (KREG) {
#pragma unroll
      for (int k = 0; k < kRegSlots; ++k)
        if (k < p.K) cred[(size_t)k * TS + tid] = cr[k];
    }
    __syncthreads();
    // fixed-order reduction over the block's threads, one thread per slot
    for (int64_t k = tid; k < p.K; k += blockDim.x) {
      if (!touched[k]) continue;
      double s = 0.0;
      for (int t = 0; t < (int)blockDim.x; ++t) s += cred[k * TS + t];
      T* dst = p.grad + b * p.K + k;
      if (p.n_splits == 1) *dst = *dst + (T)s;
      else atomicAdd(dst, (T)s);
    }
  }
}

#undef WS_FOR_R

// Programs grouped by tape slots, so that each group runs with a tape sized for it: a program's
// operator tokens, constant tokens (when there are constant slots) and distinct variables before
// its first PAD bound the slots parse_loss_program gives it.  Programs with active[b] == 0 are
// left out.  lists: [n_buckets, B]; the order inside a bucket does not matter (every (program,
// row range) writes its own partial sums).
constexpr int kMaxBuckets = 13;
static_assert(kMaxBuckets <= 16, "the bucket counts take 16 entries of the scratch");
constexpr int kBucketSlots[kMaxBuckets] = {8, 12, 16, 20, 24, 28, 32, 40, 48, 64, 96, 128, 256};
__constant__ int c_bucket_slots[kMaxBuckets] = {8,  12, 16, 20, 24,  28, 32,
                                                40, 48, 64, 96, 128, 256};

__global__ void __launch_bounds__(256) bucket_kernel(const uint8_t* __restrict__ pop, int64_t B,
                                                     int64_t L, int64_t K, BwdLut lut,
                                                     const int32_t* __restrict__ active,
                                                     int n_buckets, int32_t* counts,
                                                     int32_t* lists) {
  __shared__ uint8_t s_kind[256], s_arg[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    s_kind[t] = lut.kind[t];
    s_arg[t] = lut.arg[t];
  }
  __syncthreads();
  // whole warps step through the programs together (the bucket counters are claimed per warp)
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t b_end = (B + 31) / 32 * 32;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < b_end; b += stride) {
    const bool take = b < B && !(active && active[b] == 0);
    const uint8_t* row = pop + (take ? b : 0) * L;
    int n = 0;
    uint64_t seen = 0;  // variables 0..63; higher ones are counted at every use (a bound)
    for (int64_t t = 0; take && t < L; ++t) {
      const uint8_t k = s_kind[row[t]];
      if (k == BK_PAD) break;
      if (k == BK_BIN || k == BK_UN || (k == BK_CONST && K > 0)) {
        ++n;
      } else if (k == BK_VAR) {
        const int v = s_arg[row[t]];
        if (v >= 64) {
          ++n;
        } else if (!((seen >> v) & 1)) {
          seen |= 1ull << v;
          ++n;
        }
      }
    }
    int j = 0;
    while (j < n_buckets - 1 && n > c_bucket_slots[j]) ++j;
    // one atomic per bucket per warp: the lowest lane of each group of lanes with the same
    // bucket claims the group's slots, the others take theirs by rank
    const unsigned taking = __ballot_sync(0xFFFFFFFFu, take);
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, take ? j : -1) & taking;
    if (take) {
      const int lane = threadIdx.x & 31;
      const int leader = __ffs(peers) - 1;
      int pos0 = 0;
      if (lane == leader) pos0 = atomicAdd(counts + j, __popc(peers));
      pos0 = __shfl_sync(peers, pos0, leader);
      const int rank = __popc(peers & ((1u << lane) - 1u));
      lists[(int64_t)j * B + pos0 + rank] = (int32_t)b;
    }
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

// Rows are split into ranges only when there are too few programs to fill the GPU; ranges are
// multiples of 512 rows (a whole number of row groups of every block shape).  The split depends
// on (B, D), the resident blocks per SM of the launch's shape and the device alone.
void split_rows(int64_t B, int64_t D, int per_sm, BwdPlan* out) {
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
}

// Resolved-tape kernels (REF: the reference-mode ref_kernel, else loss_kernel): shared memory of
// a block whose tape has M slots, and the shape with the most resident rows per SM: every
// (rows per thread, block size) that fits, scored by the rows its resident warps carry, warps
// counted up to 32 per SM.
template <typename T, bool REF>
size_t loss_smem(int64_t M, int64_t L, int64_t K, int threads, int R) {
  return loss_layout(M, L, K, threads, (size_t)R * sizeof(T), K <= kRegSlots, REF).bytes;
}

template <typename T, bool REF, int RR>
void (*loss_pick(bool kreg))(BwdParams<T>, BwdLut) {
  if constexpr (REF) return kreg ? ref_kernel<T, RR, true> : ref_kernel<T, RR, false>;
  return kreg ? loss_kernel<T, RR, true> : loss_kernel<T, RR, false>;
}

template <typename T, bool REF = false>
void (*loss_fn(int R, bool kreg))(BwdParams<T>, BwdLut) {
  if constexpr (kRowsMax<T> >= 4) {
    if (R == 4) return loss_pick<T, REF, 4>(kreg);
  }
  if (R == 2) return loss_pick<T, REF, 2>(kreg);
  return loss_pick<T, REF, 1>(kreg);
}

template <typename T, bool REF = false>
ws_status loss_shape(int64_t M, int64_t L, int64_t K, BwdPlan* out, int* per_sm_out) {
  const DeviceInfo& dev = device_info();
  const size_t budget = dev.smem_optin < (size_t)200 * 1024 ? dev.smem_optin : 200 * 1024;
  const bool kreg = K <= kRegSlots;
  double best_score = -1.0;
  int best_threads = 0, best_per_sm = 0, best_r = 1;
  for (int R = kRowsMax<T>; R >= 1; R /= 2) {
    auto kern = loss_fn<T, REF>(R, kreg);
    for (int threads = 128; threads >= 32; threads /= 2) {
      const size_t smem = loss_smem<T, REF>(M, L, K, threads, R);
      if (smem > budget) continue;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
      int per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
      if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
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
    return fail("loss_grad: " + std::to_string(K) + " constants and " + std::to_string(M) +
                " tape slots need more shared memory than a block has");
  const size_t smem = loss_smem<T, REF>(M, L, K, best_threads, best_r);
  cudaError_t e = cudaFuncSetAttribute(loss_fn<T, REF>(best_r, kreg),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
  out->threads = best_threads;
  out->R = best_r;
  out->smem = smem;
  *per_sm_out = best_per_sm;
  return WS_OK;
}

template <typename T>
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
  prm.tape_ops = (int)L;
  prm.list = nullptr;
  prm.list_count = nullptr;
  prm.y = nullptr;
  prm.active = nullptr;
  prm.part_loss = nullptr;
  prm.part_grad = nullptr;
  return prm;
}

// buckets (optional, loss_grad_bucket_bytes(B) of scratch): programs grouped by tape slots and
// one launch per group with a tape sized for it, as in the loss path; without it one launch
// sized for L.
template <typename T>
ws_status launch_backward_typed(const uint8_t* pop, int64_t B, int64_t L, const void* x,
                                int64_t V, int64_t D, const void* consts, int64_t K,
                                const void* gout, void* grad, const BwdLut& lut,
                                int32_t* buckets, cudaStream_t stream) {
  BwdPlan plan;
  int per_sm = 0;
  ws_status st = loss_shape<T, true>(L, L, K, &plan, &per_sm);
  if (st != WS_OK) return st;
  split_rows(B, D, per_sm, &plan);
  BwdParams<T> prm = backward_params<T>(pop, B, L, x, V, D, consts, K, plan);
  prm.gout = static_cast<const T*>(gout);
  prm.grad = static_cast<T*>(grad);
  const bool kreg = K <= kRegSlots;
  if (!buckets) {
    loss_fn<T, true>(plan.R, kreg)<<<(unsigned)plan.grid, plan.threads, plan.smem, stream>>>(
        prm, lut);
  } else {
    int nb = 0;
    while (nb < kMaxBuckets && (nb == 0 || kBucketSlots[nb - 1] < L)) ++nb;
    int32_t* counts = buckets;
    int32_t* lists = buckets + 16;
    cudaError_t e = cudaMemsetAsync(counts, 0, 16 * sizeof(int32_t), stream);
    if (e != cudaSuccess) return fail_cuda(e, "eval_rpn_backward");
    const int64_t cb = (B + 255) / 256;
    bucket_kernel<<<(unsigned)(cb < 2048 ? cb : 2048), 256, 0, stream>>>(pop, B, L, K, lut,
                                                                         nullptr, nb, counts,
                                                                         lists);
    for (int j = 0; j < nb; ++j) {
      const int64_t M = kBucketSlots[j] < L ? kBucketSlots[j] : L;
      BwdPlan pj;
      int pj_per_sm = 0;
      st = loss_shape<T, true>(M, L, K, &pj, &pj_per_sm);
      if (st != WS_OK) return st;
      BwdParams<T> q = prm;
      q.tape_stride = pj.threads;
      q.tape_ops = (int)M;
      q.list = lists + (int64_t)j * B;
      q.list_count = counts + j;
      const int64_t slots = (int64_t)device_info().sm_count * pj_per_sm;
      const int64_t grid = prm.n_items < slots ? prm.n_items : slots;
      loss_fn<T, true>(pj.R, kreg)<<<(unsigned)grid, pj.threads, pj.smem, stream>>>(q, lut);
    }
  }
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
  int per_sm = 0;
  ws_status st = loss_shape<T>(L, L, K, &plan, &per_sm);
  if (st != WS_OK) return st;
  split_rows(B, D, per_sm, &plan);
  if (n_splits_out) *n_splits_out = plan.n_splits;
  if (!part_loss) return WS_OK;  // plan query only
  const BwdLut lut = build_bwd_lut(ids, num_vars);
  BwdParams<T> prm = backward_params<T>(pop, B, L, x, num_vars, D, consts, K, plan);
  prm.y = static_cast<const T*>(y);
  prm.active = active;
  prm.part_loss = part_loss;
  prm.part_grad = part_grad;
  const bool kreg = K <= kRegSlots;
  cudaError_t e;
  if (!buckets) {
    loss_fn<T>(plan.R, kreg)<<<(unsigned)plan.grid, plan.threads, plan.smem, stream>>>(prm, lut);
  } else {
    // buckets[0..15]: counts; buckets + 16: lists [n_buckets, B]
    int nb = 0;
    while (nb < kMaxBuckets && (nb == 0 || kBucketSlots[nb - 1] < L)) ++nb;
    int32_t* counts = buckets;
    int32_t* lists = buckets + 16;
    e = cudaMemsetAsync(counts, 0, 16 * sizeof(int32_t), stream);
    if (e != cudaSuccess) return fail_cuda(e, "loss_grad");
    const int64_t cb = (B + 255) / 256;
    bucket_kernel<<<(unsigned)(cb < 2048 ? cb : 2048), 256, 0, stream>>>(pop, B, L, K, lut, active,
                                                                         nb, counts, lists);
    for (int j = 0; j < nb; ++j) {
      const int64_t M = kBucketSlots[j] < L ? kBucketSlots[j] : L;
      BwdPlan pj;
      int pj_per_sm = 0;
      st = loss_shape<T>(M, L, K, &pj, &pj_per_sm);
      if (st != WS_OK) return st;
      BwdParams<T> q = prm;
      q.tape_stride = pj.threads;
      q.tape_ops = (int)M;
      q.list = lists + (int64_t)j * B;
      q.list_count = counts + j;
      const int64_t slots = (int64_t)device_info().sm_count * pj_per_sm;
      const int64_t items = B * plan.n_splits;
      const int64_t grid = items < slots ? items : slots;
      loss_fn<T>(pj.R, kreg)<<<(unsigned)grid, pj.threads, pj.smem, stream>>>(q, lut);
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

namespace {
// The checks and launch shared by ws_eval_rpn_backward and its workspace form (buckets: null, or
// the program-group scratch in the caller's workspace).
ws_status eval_rpn_backward_impl(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                                 const void* x, int64_t num_vars, int64_t D,
                                 const void* constants, int64_t K, const void* grad_output,
                                 void* grad_constants, const ws_token_map* ids, int32_t* buckets,
                                 void* stream) {
  using namespace ws;
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
                                        grad_output, grad_constants, lut, buckets, s);
  return launch_backward_typed<double>(population, B, L, x, num_vars, D, constants, K,
                                       grad_output, grad_constants, lut, buckets, s);
}
}  // namespace

extern "C" ws_status ws_eval_rpn_backward(int32_t dtype, const uint8_t* population, int64_t B,
                                          int64_t L, const void* x, int64_t num_vars, int64_t D,
                                          const void* constants, int64_t K,
                                          const void* grad_output, void* grad_constants,
                                          const ws_token_map* ids, void* stream) {
  ws::clear_error();
  ws::NvtxRange nvtx("ws_eval_rpn_backward");
  return eval_rpn_backward_impl(dtype, population, B, L, x, num_vars, D, constants, K,
                                grad_output, grad_constants, ids, nullptr, stream);
}

extern "C" ws_status ws_eval_rpn_backward_workspace_bytes(int64_t B, size_t* bytes) {
  ws::clear_error();
  if (B < 0) return ws::fail("negative dimension");
  if (!bytes) return ws::fail("null output pointer");
  *bytes = ws::loss_grad_bucket_bytes(B);
  return WS_OK;
}

extern "C" ws_status ws_eval_rpn_backward_ws(int32_t dtype, const uint8_t* population, int64_t B,
                                             int64_t L, const void* x, int64_t num_vars,
                                             int64_t D, const void* constants, int64_t K,
                                             const void* grad_output, void* grad_constants,
                                             const ws_token_map* ids, void* workspace,
                                             size_t workspace_bytes, void* stream) {
  ws::clear_error();
  ws::NvtxRange nvtx("ws_eval_rpn_backward");
  if (B > 0 && (!workspace || workspace_bytes < ws::loss_grad_bucket_bytes(B)))
    return ws::fail("eval_rpn_backward workspace too small");
  return eval_rpn_backward_impl(dtype, population, B, L, x, num_vars, D, constants, K,
                                grad_output, grad_constants, ids,
                                static_cast<int32_t*>(workspace), stream);
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
  NvtxRange nvtx("ws_loss_grad");
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
