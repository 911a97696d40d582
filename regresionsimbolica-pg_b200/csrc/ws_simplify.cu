// ws_simplify.cu -- rule-based simplification of RPN programs, in place.
//
// Replaces `simplify_batch` (bindings.cpp:505 -> launch_simplify_batch,
// simplify_kernels.cu:665-713; kernel :100-601).  The rewrite rules, their order, the way a pass
// sees the edits of the previous rule (positions are PAD-ed in place and compacted only at the
// end of each phase; the commutative normalisation swaps operands without refreshing the
// operand bounds the later rules of the same position use), the nearest-literal constant folding
// (first literal strictly closest, accepted below 1e-5) and the pass loop are the reference's, so
// the output programs are identical.  Per pass:
//   phase 1 (unary / chain), left to right from position 1:
//     neg neg -> (nothing);  x 2 pow sqrt -> x abs;  known constant arguments (sin 0, tan 0,
//     abs 0, log 1, lgamma 1, lgamma 2 -> 0; cos 0, exp 0, gamma 1, gamma 2 -> 1); a unary
//     operator on a literal folds to the nearest literal;  x x' neg + -> 0 when x == x';
//   compact;
//   phase 2 (binary), left to right from position 2, for operators of arity 2:
//     x+0, x-0, x*1, x/1, x^1 -> x;  x^0, 1^x -> 1;  0+x, 1*x -> x;  x*0, 0*x -> 0;
//     0-x -> neg x;  + and * operands ordered (literal < single token < subtree, then lower ID,
//     then shorter);  a x * b x * + -> a b + x * (and x a * x b * +);  x (x y +) + and
//     x (y x +) + -> 2 x * y + (single-token x);  two literal operands fold to a literal;
//   compact;  stop when nothing changed.
// One thread rewrites one program (the rules are sequential within a program).  The working
// program lives in shared memory as 16-bit tokens, position-major across the block's threads
// (position i of thread t at [i * blockDim + t]: a warp at one position reads one 64-byte line),
// so the rule scans run at shared-memory latency; the reference keeps 2 x 256 int64 per thread in
// local memory, which at a few hundred threads per SM spills out of L1 into L2.  A row holding a
// token outside the 16-bit range (possible only for tokens outside the vocabulary) is rewritten
// from a thread-local int64 copy instead, with the same code.  The operand swap of + and * and
// the y move of the x (x y +) + rule are done in place (a rotation by three reversals; a
// downward copy), which gives the same program as the reference's copy through a scratch row.
// Literal table and arity table in shared memory.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "ws_internal.h"

namespace ws {
namespace {

constexpr int kMaxFormula = 256;  // MAX_FORMULA_LEN (simplify_kernels.cu:33)
constexpr int kMaxLits = 64;      // MAX_LITERALS (:35)
constexpr int64_t kPad = 0;       // PAD_ID_CONST (:38)
constexpr int64_t kNone = -999;   // "operand is not a single token"

struct SimplifyIds {
  int op_plus, op_minus, op_mult, op_div, op_neg, op_mod, op_pow;
  int op_sin, op_cos, op_tan, op_asin, op_acos, op_atan;
  int op_log, op_exp, op_sqrt, op_abs, op_gamma, op_lgamma, op_floor, op_ceil, op_sign;
  int id_0, id_1, id_2, id_3, id_4, id_5, id_6;
};

struct SimplifyArgs {
  int64_t* pop;
  const int32_t* ar;
  const float* vt;  // value of each literal token, NaN otherwise
  const int64_t* lit_ids;
  const float* lit_vals;
  int n_lits;
  int max_id;
  int64_t B;
  int L;
  int max_passes;
  SimplifyIds id;
};

// Position i of a thread's working program: 16-bit tokens in shared memory ...
struct SmemRow {
  int16_t* base;
  int stride;
  __device__ int16_t& operator[](int i) const { return base[i * stride]; }
};
// ... or int64 tokens in thread-local memory (rows with tokens outside the 16-bit range).
struct LocalRow {
  int64_t* base;
  __device__ int64_t& operator[](int i) const { return base[i]; }
};

template <class Row>
struct Program {
  Row f;
  int n;  // positions considered (min(L, 256))
  const int32_t* ar;
  int max_id;

  __device__ bool foreign(int64_t t) const { return t == kPad || t < 0 || t >= max_id; }

  // Start of the subtree ending at `end` (backward balance scan; -1 outside the row; the end
  // itself for PAD / out-of-table tokens; 0 when the scan runs off the front).
  __device__ int subtree_start(int end) const {
    if (end < 0 || end >= n) return -1;
    if (foreign(f[end])) return end;
    int balance = 1;
    for (int k = end; k >= 0; --k) {
      const int64_t t = f[k];
      if (foreign(t)) balance -= 1;
      else balance += ar[(int)t < max_id - 1 ? (int)t : max_id - 1] - 1;
      if (balance == 0) return k;
    }
    return 0;
  }

  __device__ void compact() {
    int w = 0;
    for (int r = 0; r < n; ++r) {
      const int64_t t = f[r];
      if (t != kPad) f[w++] = t;
    }
    for (int i = w; i < n; ++i) f[i] = kPad;
  }

  __device__ void blank(int from, int to) {  // f[from..to] = PAD
    for (int k = from; k <= to; ++k) f[k] = kPad;
  }

  __device__ bool same(int a, int b, int len) const {
    for (int k = 0; k < len; ++k)
      if (f[a + k] != f[b + k]) return false;
    return true;
  }

  __device__ void reverse(int lo, int hi) {  // f[lo..hi] reversed
    for (; lo < hi; ++lo, --hi) {
      const int64_t t = f[lo];
      f[lo] = f[hi];
      f[hi] = t;
    }
  }

  // f[s1..s2-1] f[s2..e-1]  ->  f[s2..e-1] f[s1..s2-1]
  __device__ void swap_segments(int s1, int s2, int e) {
    reverse(s1, s2 - 1);
    reverse(s2, e - 1);
    reverse(s1, e - 1);
  }
};

// Nearest literal to `res` (first strictly closest); its token or -1 when none is within 1e-5.
__device__ int64_t nearest_literal(float res, const int64_t* ids, const float* vals, int n) {
  if (isnan(res) || isinf(res)) return -1;
  float best = 1e30f;
  int bi = -1;
  for (int i = 0; i < n; ++i) {
    const float d = fabsf(res - vals[i]);
    if (d < best) {
      best = d;
      bi = i;
    }
  }
  return (bi >= 0 && best < 1e-5f) ? ids[bi] : -1;
}

__device__ float fold_unary(int64_t tok, float v, const SimplifyIds& o) {
  const float nan = nanf("");
  if (tok == o.op_sin) return sinf(v);
  if (tok == o.op_cos) return cosf(v);
  if (tok == o.op_tan) return tanf(v);
  if (tok == o.op_log) return v > 0 ? logf(v) : nan;
  if (tok == o.op_exp) return v < 80.0f ? expf(v) : nan;
  if (tok == o.op_sqrt) return v >= 0 ? sqrtf(v) : nan;
  if (tok == o.op_abs) return fabsf(v);
  if (tok == o.op_neg) return -v;
  if (tok == o.op_floor) return floorf(v);
  if (tok == o.op_ceil) return ceilf(v);
  if (tok == o.op_sign) return (v > 0) ? 1.0f : ((v < 0) ? -1.0f : 0.0f);
  if (tok == o.op_asin) return fabsf(v) <= 1.0f ? asinf(v) : nan;
  if (tok == o.op_acos) return fabsf(v) <= 1.0f ? acosf(v) : nan;
  if (tok == o.op_atan) return atanf(v);
  if (tok == o.op_gamma) return (v > 0 && v < 20.0f) ? expf(lgammaf(v)) : nan;
  if (tok == o.op_lgamma) return v > 0 ? lgammaf(v) : nan;
  return nan;
}

__device__ float fold_binary(int64_t op, float v1, float v2, const SimplifyIds& o) {
  if (op == o.op_plus) return v1 + v2;
  if (op == o.op_minus) return v1 - v2;
  if (op == o.op_mult) return v1 * v2;
  if (op == o.op_div && fabsf(v2) > 1e-9f) return v1 / v2;
  if (op == o.op_pow) return powf(v1, v2);
  if (op == o.op_mod && fabsf(v2) > 1e-9f) return fmodf(v1, v2);
  return nanf("");
}

// Phase 1 at position j (simplify_kernels.cu:144-251).  True when a rule rewrote.
template <class Row>
__device__ bool phase1_at(Program<Row>& p, int j, const SimplifyArgs& a, const int64_t* lit_ids,
                          const float* lit_vals, int n_lits) {
  const SimplifyIds& o = a.id;
  const Row f = p.f;
  const int64_t tok = f[j];
  const int64_t prev = f[j - 1];
  if (tok == o.op_neg && prev == o.op_neg) {
    f[j] = f[j - 1] = kPad;
    return true;
  }
  if (j >= 2 && tok == o.op_sqrt && prev == o.op_pow && f[j - 2] == o.id_2 && o.op_abs != -1) {
    f[j] = o.op_abs;
    f[j - 1] = f[j - 2] = kPad;
    return true;
  }
  if (tok > 0 && tok < a.max_id && p.ar[tok] == 1 && prev != kPad) {
    const bool z = prev == o.id_0, one = prev == o.id_1, two = prev == o.id_2;
    const bool to_zero = (z && (tok == o.op_sin || tok == o.op_tan || tok == o.op_abs)) ||
                         (one && (tok == o.op_log || tok == o.op_lgamma)) ||
                         (two && tok == o.op_lgamma);
    if (to_zero && o.id_0 != -1) {
      f[j - 1] = o.id_0;
      f[j] = kPad;
      return true;
    }
    const bool to_one = (z && (tok == o.op_cos || tok == o.op_exp)) ||
                        ((one || two) && tok == o.op_gamma);
    if (to_one && o.id_1 != -1) {
      f[j - 1] = o.id_1;
      f[j] = kPad;
      return true;
    }
    if (n_lits > 0 && prev > 0 && prev < a.max_id) {
      const float v = a.vt[prev];
      if (!isnan(v)) {
        const int64_t lit = nearest_literal(fold_unary(tok, v, o), lit_ids, lit_vals, n_lits);
        if (lit >= 0) {
          f[j - 1] = lit;
          f[j] = kPad;
          return true;
        }
      }
    }
  }
  if (j >= 3 && tok == o.op_plus && f[j - 1] == o.op_neg) {
    const int s_arg = p.subtree_start(j - 2);
    const int e_first = s_arg - 1;
    if (e_first >= 0 && s_arg >= 0) {
      const int s_first = p.subtree_start(e_first);
      if (s_first >= 0) {
        const int len1 = e_first - s_first + 1, len2 = (j - 2) - s_arg + 1;
        if (len1 == len2 && len1 > 0 && p.same(s_first, s_arg, len1) && o.id_0 != -1) {
          f[s_first] = o.id_0;
          p.blank(s_first + 1, j);
          return true;
        }
      }
    }
  }
  return false;
}

// Phase 2 at binary position j (simplify_kernels.cu:257-591).
template <class Row>
__device__ bool phase2_at(Program<Row>& p, int j, const SimplifyArgs& a, const int64_t* lit_ids,
                          const float* lit_vals, int n_lits) {
  const SimplifyIds& o = a.id;
  const Row f = p.f;
  const int64_t op = f[j];
  const int s2 = p.subtree_start(j - 1);
  const int s1 = p.subtree_start(s2 - 1);
  if (s1 < 0 || s2 < 0) return false;
  const int len1 = s2 - s1, len2 = j - s2;
  const int64_t arg2 = (s2 == j - 1) ? f[j - 1] : kNone;
  const int64_t arg1 = (s1 == s2 - 1) ? f[s2 - 1] : kNone;
  const bool a2_zero = arg2 == o.id_0, a2_one = arg2 == o.id_1;
  const bool a1_zero = arg1 == o.id_0, a1_one = arg1 == o.id_1;
  const bool is_pow = op == o.op_pow;

  if ((op == o.op_plus || op == o.op_minus) && a2_zero) {
    f[j - 1] = f[j] = kPad;
    return true;
  }
  if ((op == o.op_mult || op == o.op_div || is_pow) && a2_one) {
    f[j - 1] = f[j] = kPad;
    return true;
  }
  if (is_pow && (a2_zero || a1_one) && o.id_1 != -1) {
    p.blank(s1, j);
    f[s1] = o.id_1;
    return true;
  }
  if ((op == o.op_plus && a1_zero) || (op == o.op_mult && a1_one)) {
    f[s2 - 1] = f[j] = kPad;
    return true;
  }
  if (op == o.op_mult && (a2_zero || a1_zero) && o.id_0 != -1) {
    p.blank(s1, j);
    f[s1] = o.id_0;
    return true;
  }
  if (op == o.op_minus && a1_zero && o.op_neg != -1) {
    f[s2 - 1] = kPad;
    f[j] = o.op_neg;
    return true;
  }
  // operand order of + and *: no change flag, and the bounds above stay as they were
  if (op == o.op_plus || op == o.op_mult) {
    const bool leaf1 = len1 == 1, leaf2 = len2 == 1;
    const bool c1 = leaf1 && arg1 > 0 && arg1 < a.max_id && !isnan(a.vt[arg1]);
    const bool c2 = leaf2 && arg2 > 0 && arg2 < a.max_id && !isnan(a.vt[arg2]);
    const int sc1 = c1 ? 0 : (leaf1 ? 1 : 2), sc2 = c2 ? 0 : (leaf2 ? 1 : 2);
    bool swap = sc2 < sc1;
    if (sc1 == sc2 && sc1 < 2 && arg2 != kNone && arg1 != kNone && arg2 < arg1) swap = true;
    if (sc1 == 2 && sc2 == 2 && len2 < len1) swap = true;
    if (swap) {
      if (leaf1 && leaf2) {
        f[s2 - 1] = arg2;
        f[j - 1] = arg1;
      } else {
        p.swap_segments(s1, s2, j);
      }
    }
  }
  // a x * b x * +  ->  a b + x *   (and  x a * x b * +)
  if (op == o.op_plus && j >= 6) {
    const int64_t v1 = f[j - 1], v2 = f[j - 2], v3 = f[j - 3], v4 = f[j - 4], v5 = f[j - 5],
                  v6 = f[j - 6];
    auto term = [&](int64_t t) { return t >= 0 && t < a.max_id && p.ar[t] == 0; };
    if (f[j] == o.op_plus && v1 == o.op_mult && v4 == o.op_mult) {
      int64_t ka = 0, kb = 0, kx = 0;
      bool hit = false;
      if (v5 == v2 && v5 != kPad && term(v5) && term(v6) && term(v3)) {
        ka = v6; kb = v3; kx = v5; hit = true;
      } else if (v6 == v3 && v6 != kPad && term(v6) && term(v5) && term(v2)) {
        ka = v5; kb = v2; kx = v6; hit = true;
      }
      if (hit) {
        f[j - 6] = ka;
        f[j - 5] = kb;
        f[j - 4] = o.op_plus;
        f[j - 3] = kx;
        f[j - 2] = o.op_mult;
        f[j - 1] = f[j] = kPad;
        return true;
      }
    }
  }
  // x (x y +) +  and  x (y x +) +  ->  2 x * y +   (single-token x)
  if (op == o.op_plus && o.id_2 != -1 && j >= 4 && f[j - 1] == o.op_plus) {
    const int s_ir = p.subtree_start(j - 2);
    if (s_ir >= 1) {
      const int e_il = s_ir - 1;
      const int s_il = p.subtree_start(e_il);
      if (s_il >= 1) {
        const int e_o1 = s_il - 1;
        const int s_o1 = p.subtree_start(e_o1);
        if (s_o1 >= 0) {
          const bool o1_single = s_o1 == e_o1;
          int y_from = -1, y_len = 0;
          if (o1_single && s_il == e_il && f[s_o1] == f[s_il] && f[s_o1] != kPad) {
            y_from = s_ir;
            y_len = (j - 2) - s_ir + 1;
          }
          if (y_from < 0 || 4 + y_len > j - s_o1 + 1) {
            y_from = -1;
            const int ir_len = (j - 2) - s_ir + 1;
            if (o1_single && ir_len == 1 && f[s_o1] == f[s_ir] && f[s_o1] != kPad) {
              y_from = s_il;
              y_len = e_il - s_il + 1;
            }
          }
          if (y_from >= 0 && 4 + y_len <= j - s_o1 + 1) {
            // y starts at s_o1 + 1 or s_o1 + 2 and moves up to s_o1 + 3: copied downwards, every
            // source token is read before its position is written
            const int64_t x_tok = f[s_o1];
            for (int k = y_len - 1; k >= 0; --k) f[s_o1 + 3 + k] = f[y_from + k];
            f[s_o1] = o.id_2;
            f[s_o1 + 1] = x_tok;
            f[s_o1 + 2] = o.op_mult;
            int w = s_o1 + 3 + y_len;
            f[w++] = o.op_plus;
            p.blank(w, j);
            return true;
          }
        }
      }
    }
  }
  // two literal operands
  if (n_lits > 0 && arg1 != kNone && arg2 != kNone && arg1 > 0 && arg1 < a.max_id && arg2 > 0 &&
      arg2 < a.max_id) {
    const float v1 = a.vt[arg1], v2 = a.vt[arg2];
    if (!isnan(v1) && !isnan(v2)) {
      const int64_t lit = nearest_literal(fold_binary(op, v1, v2, o), lit_ids, lit_vals, n_lits);
      if (lit >= 0) {
        f[s1] = lit;
        p.blank(s1 + 1, j);
        return true;
      }
    }
  }
  return false;
}

template <class Row>
__device__ void simplify_program(Program<Row>& p, const SimplifyArgs& a, const int64_t* lit_ids,
                                 const float* lit_vals, int n_lits) {
  for (int pass = 0; pass < a.max_passes; ++pass) {
    bool changed = false;
    for (int j = 1; j < p.n; ++j) {
      if (p.f[j] == kPad) continue;
      if (phase1_at(p, j, a, lit_ids, lit_vals, n_lits)) changed = true;
    }
    p.compact();
    for (int j = 2; j < p.n; ++j) {
      const int64_t op = p.f[j];
      if (op == kPad || op < 0 || op >= a.max_id || p.ar[op] != 2) continue;
      if (phase2_at(p, j, a, lit_ids, lit_vals, n_lits)) changed = true;
    }
    p.compact();
    if (!changed) break;
  }
}

constexpr int kSimpThreads = 128;
constexpr int kStagedArities = 1024;  // arity tables up to this length are read from shared memory

// narrow != 0: every id fits a 16-bit token and dynamic shared memory holds n x blockDim of them.
__global__ void __launch_bounds__(kSimpThreads) simplify_kernel(SimplifyArgs a, int narrow) {
  extern __shared__ int16_t s_rows[];
  __shared__ int64_t s_lit_ids[kMaxLits];
  __shared__ float s_lit_vals[kMaxLits];
  __shared__ int32_t s_ar[kStagedArities];
  const int n_lits = a.n_lits < kMaxLits ? a.n_lits : kMaxLits;
  bool lits_fit = true;
  for (int i = threadIdx.x; i < n_lits; i += blockDim.x) {
    const int64_t id = a.lit_ids[i];
    s_lit_ids[i] = id;
    s_lit_vals[i] = a.lit_vals[i];
    lits_fit = lits_fit && id == (int64_t)(int16_t)id;
  }
  const bool staged_ar = a.max_id <= kStagedArities;
  if (staged_ar)
    for (int i = threadIdx.x; i < a.max_id; i += blockDim.x) s_ar[i] = a.ar[i];
  const bool use_smem = __syncthreads_and(lits_fit) && narrow != 0;
  const int32_t* ar = staged_ar ? s_ar : a.ar;
  const int n = a.L < kMaxFormula ? a.L : kMaxFormula;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < a.B;
       b += (int64_t)gridDim.x * blockDim.x) {
    int64_t* row = a.pop + b * a.L;
    bool fits = use_smem;
    if (fits) {
      const SmemRow sr{s_rows + threadIdx.x, (int)blockDim.x};
      for (int i = 0; i < n; ++i) {
        const int64_t t = row[i];
        sr[i] = (int16_t)t;
        fits = fits && t == (int64_t)(int16_t)t;
      }
      if (fits) {
        Program<SmemRow> p{sr, n, ar, a.max_id};
        simplify_program(p, a, s_lit_ids, s_lit_vals, n_lits);
        for (int i = 0; i < n; ++i) row[i] = sr[i];
      }
    }
    if (!fits) {
      int64_t loc[kMaxFormula];
      for (int i = 0; i < n; ++i) loc[i] = row[i];
      Program<LocalRow> p{LocalRow{loc}, n, ar, a.max_id};
      simplify_program(p, a, s_lit_ids, s_lit_vals, n_lits);
      for (int i = 0; i < n; ++i) row[i] = loc[i];
    }
  }
}

}  // namespace
}  // namespace ws

extern "C" ws_status ws_simplify_batch(int64_t* population, int64_t B, int64_t L,
                                       const int32_t* arities, int64_t max_id,
                                       const float* val_table, const int64_t* literal_ids,
                                       const float* literal_vals, int64_t n_literals,
                                       int32_t max_passes, const ws_simplify_ids* ids,
                                       void* stream) {
  using namespace ws;
  clear_error();
  NvtxRange nvtx("ws_simplify_batch");
  if (!ids) return fail("simplify ids are required");
  if (B < 0 || L < 0 || max_id < 0 || n_literals < 0) return fail("negative dimension");
  if (B == 0 || L == 0 || max_passes <= 0) return WS_OK;
  if (max_id == 0) return fail("arities must be non-empty");
  if (!population || !arities || !val_table || (n_literals > 0 && (!literal_ids || !literal_vals)))
    return fail("null tensor pointer");
  SimplifyArgs a;
  a.pop = population;
  a.ar = arities;
  a.vt = val_table;
  a.lit_ids = literal_ids;
  a.lit_vals = literal_vals;
  a.n_lits = (int)(n_literals < kMaxLits ? n_literals : kMaxLits);
  a.max_id = (int)max_id;
  a.B = B;
  a.L = (int)L;
  a.max_passes = max_passes;
  a.id = SimplifyIds{ids->op_plus,  ids->op_minus, ids->op_mult,  ids->op_div,   ids->op_neg,
                     ids->op_mod,   ids->op_pow,   ids->op_sin,   ids->op_cos,   ids->op_tan,
                     ids->op_asin,  ids->op_acos,  ids->op_atan,  ids->op_log,   ids->op_exp,
                     ids->op_sqrt,  ids->op_abs,   ids->op_gamma, ids->op_lgamma, ids->op_floor,
                     ids->op_ceil,  ids->op_sign,  ids->id_0,     ids->id_1,     ids->id_2,
                     ids->id_3,     ids->id_4,     ids->id_5,     ids->id_6};
  // 16-bit working rows when every id the rules write fits one (the row's own tokens are checked
  // per row in the kernel, the literal ids per block)
  const int32_t* idv = &ids->op_plus;
  bool narrow = max_id <= INT16_MAX;
  for (size_t i = 0; i < sizeof(ws_simplify_ids) / sizeof(int32_t); ++i)
    narrow = narrow && idv[i] >= INT16_MIN && idv[i] <= INT16_MAX;
  const int n = (int)(L < kMaxFormula ? L : kMaxFormula);
  const size_t smem = narrow ? (size_t)n * kSimpThreads * sizeof(int16_t) : 0;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(simplify_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail_cuda(e, "simplify_batch");
  }
  const int64_t want = (B + kSimpThreads - 1) / kSimpThreads;
  const int64_t cap = (int64_t)device_info().sm_count * 16;
  const int grid = (int)(want < cap ? want : cap);
  simplify_kernel<<<grid, kSimpThreads, smem, static_cast<cudaStream_t>(stream)>>>(
      a, narrow ? 1 : 0);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "simplify_batch");
}
