// ws_compile.cuh -- per-program compiler: uint8 RPN tokens -> accumulator-machine tape.
//
// The reference interprets every token for every row with a 32-slot stack per thread
// (rpn_kernels.cu:245-350).  Here each program is compiled ONCE (one thread per program) into
// a short tape for an accumulator machine, and the evaluator runs that tape over tiles of rows:
//
//   * terminals (x_v, C, literals) emit no instruction: they become operands of the operator
//     that consumes them (vector operand = a variable row of the staged X tile; scalar operand =
//     an immediate or a constant-slot parameter);
//   * the value of the last operator lives in the accumulator ACC (registers, R rows/thread);
//   * subtrees whose leaves are all immediates are folded here with the same device operator
//     code the evaluator runs, so the folded value is bit-identical to per-row evaluation
//     (an operator error while folding makes every row invalid, as it would per row);
//   * binary nodes with two non-terminal children evaluate the subtree with the larger
//     Sethi-Ullman need first and keep the other operand in a shared-memory spill slot; with
//     this order a program of L tokens needs at most floor(log2((L+1)/3)) slots (4 for L=64).
//
// Evaluation order of independent subtrees does not change any value (operators are pure and
// constant slots are resolved in token order here), and any row that errors in the reference
// also errors here, so per-row results and validity match the reference exactly.  The
// reference's push-drop at depth 32 (rpn_kernels.cu:289-293) and constant-slot clamp
// (rpn_kernels.cu:263-271) are applied while parsing.  Programs with a stack underflow, an
// unknown token (rpn_kernels.cu:346) or a final depth != 1 are statically invalid: every row
// of them is invalid, so they are never evaluated.
#pragma once

#include "ws_bounds.cuh"
#include "ws_ops.cuh"

namespace ws {

// ---- tape format -----------------------------------------------------------------------
// ctrl word:
//   [0:7)   case: 0 = NOP, unary class id (16..32), or binary 64 + 4*(cls-T_ADD) + form
//   [7]     SPILL: store ACC into spill slot [8:13) before anything else
//   [13:15) LOADA kind (0 none, 1 X variable, 2 immediate, 3 parameter), index [15:21)
//   [21:23) operand kind (0 none, 1 X variable, 2 spill slot, 3 scalar), [23] scalar is a
//           parameter (else the immediate), index [24:30)
enum : uint32_t {
  CASE_MASK = 0x7Fu,
  F_SPILL = 1u << 7,
  SH_SLOT = 8,
  SH_LA = 13,
  SH_LA_IDX = 15,
  SH_OPK = 21,
  F_OP_PARAM = 1u << 23,
  SH_OP_IDX = 24,
};
enum { LA_NONE = 0, LA_X = 1, LA_IMM = 2, LA_PARAM = 3 };
enum { OK_NONE = 0, OK_X = 1, OK_SLOT = 2, OK_SCALAR = 3 };
// binary forms: AV: ACC = ACC o V, VA: ACC = V o ACC, AS: ACC = ACC o s, SA: ACC = s o ACC
enum { FORM_AV = 0, FORM_VA = 1, FORM_AS = 2, FORM_SA = 3 };
enum { CASE_NOP = 0, CASE_BIN = 64 };
WS_HD uint32_t bin_case(int cls, int form) { return CASE_BIN + 4u * (uint32_t)(cls - T_ADD) + form; }

template <typename T> struct Instr;
template <> struct alignas(8) Instr<float> {
  uint32_t ctrl;
  float imm;
};
template <> struct alignas(16) Instr<double> {
  uint32_t ctrl;
  uint32_t pad;
  double imm;
};

// PROG_UNREPRESENTABLE: an operand offset does not fit the tape word (the host sizes chunks so
// that this cannot happen; the evaluator treats it as an internal error).
enum { PROG_OK = 0, PROG_INVALID = 1, PROG_UNREPRESENTABLE = 2 };
struct alignas(16) ProgHdr {
  int32_t n_instr;  // tape length
  int32_t status;   // PROG_OK / PROG_INVALID
  int32_t n_slots;  // spill slots used
  int32_t n_tok;    // tokens before the first PAD (algorithmic node count)
};

// Spill slots sufficient for any program of L tokens under Sethi-Ullman ordering.
WS_HD int spill_slots_bound(int L) {
  int n = (L + 1) / 3;  // most "need-1" units (unary(leaf) or binary(leaf,leaf)) in L tokens
  int s = 0;
  while ((2 << s) <= n) ++s;  // floor(log2(n)) for n >= 1
  return n >= 1 ? s : 0;
}

// ---- compiler --------------------------------------------------------------------------
enum { N_VAR = 0, N_IMM = 1, N_PARAM = 2, N_OP = 3 };

template <typename T> struct Node {
  T imm;
  int16_t l, r;
  uint8_t kind, cls, idx, need;
};

struct Frame {
  int16_t node;
  uint8_t phase;
  uint8_t spill;  // 1 = first emitted instruction must spill ACC into `slot`
  uint8_t slot;
  uint8_t first_left;
};

// ---- evaluator tape word (the lowering of the logical fields above) ---------------------
//   [0:6)   dense case: 0 = NOP, 1..17 unary (cls - T_SIN + 1), 18..41 binary
//           (18 + 4*(cls-T_ADD) + form); the binary forms AV and VA read a vector operand V
//   [6]     SPILL: store ACC into spill slot [7:10) first
//   [10]    LOADA_X: ACC <- X row at offset [12:21); [11] LOADA_S: ACC <- immediate
//   [21]    SLOW: any of SPILL, LOADA_X, LOADA_S, or V in a deep (global) spill slot -- the
//           evaluator tests this one bit and skips all of them on the common path
//   [22]    V is the spill slot [23:32) (else the X row at offset [23:32))
// Offsets are in units of one pass (32*R rows): variable v of a chunk of RC rows sits at
// v * (RC / pass), spill slot s at s.  Scalar operands are the immediate.  `xmul` = RC / pass
// is fixed by the schedule before compiling.  Spill slots below kSharedSlots live in shared
// memory, deeper ones (0.2% of random 64-token programs) in a per-warp global scratch area.
enum : uint32_t {
  P_CASE_MASK = 0x3Fu,
  P_SPILL = 1u << 6,
  P_SH_SLOT = 7,
  P_LOADA_X = 1u << 10,
  P_LOADA_S = 1u << 11,
  P_SH_LA = 12,
  P_SLOW = 1u << 21,
  P_FETCH_SLOT = 1u << 22,
  P_SH_V = 23,
  P_OFF_MASK = 0x1FFu,
};
enum { PCASE_NOP = 0, PCASE_UNARY0 = 1, PCASE_BIN = 18, PCASE_COUNT = 42 };
constexpr int kSharedSlots = 2;

// True for the cases that read the vector operand V (binary forms AV and VA).
WS_HD bool pcase_fetches(uint32_t cs) {
  return cs >= PCASE_BIN && ((cs - PCASE_BIN) & 3u) <= (uint32_t)FORM_VA;
}

WS_HD uint32_t lower_case(uint32_t logical) {
  const uint32_t c = logical & CASE_MASK;
  if (c == CASE_NOP) return PCASE_NOP;
  if (c < CASE_BIN) return PCASE_UNARY0 + (c - T_SIN);
  return PCASE_BIN + (c - CASE_BIN);
}

template <typename T>
struct Emitter {
  Instr<T>* out;
  int n;
  int xmul;        // RC / pass
  int cap;         // capacity of `out`
  bool ok = true;  // false if an operand is not representable in the tape word
  WS_HD void put(uint32_t c, T imm) { put_at(n++, c, imm); }
  // Encodes logical word c at tape position pos (the same lowering as put).
  WS_HD void put_at(int pos, uint32_t c, T imm) {
    uint32_t w = lower_case(c);
    if (c & F_SPILL) w |= P_SLOW | P_SPILL | (((c >> SH_SLOT) & 7u) << P_SH_SLOT);
    const uint32_t la = (c >> SH_LA) & 3u, lai = (c >> SH_LA_IDX) & 63u;
    if (la == LA_X) {
      const uint32_t off = lai * (uint32_t)xmul;
      ok = ok && off <= P_OFF_MASK;
      w |= P_SLOW | P_LOADA_X | ((off & P_OFF_MASK) << P_SH_LA);
    } else if (la == LA_IMM) {
      w |= P_SLOW | P_LOADA_S;
    } else if (la == LA_PARAM) {
      ok = false;  // parameters are baked into immediates for this tape
    }
    const uint32_t opk = (c >> SH_OPK) & 3u, oi = (c >> SH_OP_IDX) & 63u;
    if (opk == OK_X) {
      const uint32_t off = oi * (uint32_t)xmul;
      ok = ok && off <= P_OFF_MASK;
      w |= (off & P_OFF_MASK) << P_SH_V;
    } else if (opk == OK_SLOT) {
      w |= P_FETCH_SLOT | (oi << P_SH_V);
      if (oi >= (uint32_t)kSharedSlots) w |= P_SLOW;
    } else if (opk == OK_SCALAR && (c & F_OP_PARAM)) {
      ok = false;
    }
    if (pos >= cap) { ok = false; return; }
    Instr<T> ins;
    ins.ctrl = w;
    ins.imm = imm;
    if constexpr (sizeof(Instr<T>) == 16) reinterpret_cast<Instr<double>&>(ins).pad = 0;
    out[pos] = ins;
  }
};

// Tape capacity for programs of L tokens: one word per operator (a single-terminal program
// still needs one).
WS_HD int tape_capacity(int L) { return L > 1 ? L : 1; }

// Loads leaf `nd` into ACC: returns the ctrl bits and sets `imm` for an immediate.
template <typename T>
WS_HD uint32_t loada_bits(const Node<T>& nd, T& imm) {
  if (nd.kind == N_VAR) return ((uint32_t)LA_X << SH_LA) | ((uint32_t)nd.idx << SH_LA_IDX);
  if (nd.kind == N_PARAM) return ((uint32_t)LA_PARAM << SH_LA) | ((uint32_t)nd.idx << SH_LA_IDX);
  imm = nd.imm;
  return (uint32_t)LA_IMM << SH_LA;
}
// Uses leaf `nd` as the second operand.
template <typename T>
WS_HD uint32_t opnd_bits(const Node<T>& nd, T& imm, bool& is_vec) {
  if (nd.kind == N_VAR) {
    is_vec = true;
    return ((uint32_t)OK_X << SH_OPK) | ((uint32_t)nd.idx << SH_OP_IDX);
  }
  is_vec = false;
  if (nd.kind == N_PARAM)
    return ((uint32_t)OK_SCALAR << SH_OPK) | F_OP_PARAM | ((uint32_t)nd.idx << SH_OP_IDX);
  imm = nd.imm;
  return (uint32_t)OK_SCALAR << SH_OPK;
}
WS_HD uint32_t spill_bits(bool spill, int slot) {
  return spill ? (F_SPILL | ((uint32_t)slot << SH_SLOT)) : 0u;
}
// a o b == b o a bit-for-bit for + and *, so the reversed forms are canonicalised away.
WS_HD int canon_form(int cls, int form) {
  if (cls == T_ADD || cls == T_MUL) {
    if (form == FORM_VA) return FORM_AV;
    if (form == FORM_SA) return FORM_AS;
  }
  return form;
}

// Compiles program `prog` (L tokens) into `tape`.  `consts` (K values, may be null when K == 0)
// are baked into immediates when BAKE, otherwise `C` leaves become parameters (slot index).
// `xmul` = rows per chunk / rows per pass of the evaluator schedule (tape offsets are scaled by
// it).  `nodes`/`stk`/`frames` are per-thread scratch of LMAX entries.
template <typename T, bool STRICT, bool BAKE, int LMAX>
__host__ __device__ ProgHdr compile_program(const uint8_t* __restrict__ prog, int L,
                                   const T* __restrict__ consts, int K, const TokenLut& lut,
                                   Instr<T>* __restrict__ tape, int xmul) {
  Node<T> nodes[LMAX];
  int16_t stk[33];
  ProgHdr h;
  h.n_instr = 0;
  h.status = PROG_OK;
  h.n_slots = 0;
  h.n_tok = 0;
  int sp = 0, nn = 0, c_idx = 0;
  const int Lr = L < LMAX ? L : LMAX;

  for (int pc = 0; pc < Lr; ++pc) {
    const int tok = prog[pc];
    const int cls = lut.cls[tok];
    if (cls == T_PAD) break;
    h.n_tok++;
    if (is_leaf(cls)) {
      Node<T> nd;
      nd.l = nd.r = -1;
      nd.need = 0;
      nd.cls = 0;
      nd.idx = 0;
      nd.imm = (T)0;
      if (cls == T_VAR) {
        nd.kind = N_VAR;
        nd.idx = lut.arg[tok];
      } else if (cls == T_CONST) {
        if (K > 0) {
          int slot = c_idx < K ? c_idx : K - 1;
          c_idx++;
          if (BAKE) {
            nd.kind = N_IMM;
            nd.imm = consts[slot];
          } else {
            nd.kind = N_PARAM;
            nd.idx = (uint8_t)slot;
          }
        } else {
          nd.kind = N_IMM;
          nd.imm = (T)1.0;
        }
      } else {
        nd.kind = N_IMM;
        nd.imm = (T)lut.lit[lut.arg[tok]];
      }
      if (sp < 32) {  // a push at depth 32 is dropped (the C slot was still consumed)
        nodes[nn] = nd;
        stk[sp++] = (int16_t)nn++;
      }
      continue;
    }
    if (is_binary(cls)) {
      if (sp < 2) { h.status = PROG_INVALID; break; }
      const int r = stk[--sp], l = stk[--sp];
      Node<T> nd;
      nd.cls = (uint8_t)cls;
      nd.idx = 0;
      if (nodes[l].kind == N_IMM && nodes[r].kind == N_IMM) {
        bool e = false;
        nd.imm = apply_binary<T, STRICT>(cls, nodes[l].imm, nodes[r].imm, e);
        if (e) { h.status = PROG_INVALID; break; }
        nd.kind = N_IMM;
        nd.l = nd.r = -1;
        nd.need = 0;
      } else {
        nd.kind = N_OP;
        nd.l = (int16_t)l;
        nd.r = (int16_t)r;
        nd.imm = (T)0;
        const int a = nodes[l].need, b = nodes[r].need;
        int need;
        if (a == 0 && b == 0) need = 1;
        else if (a == 0) need = b;
        else if (b == 0) need = a;
        else need = (a == b) ? a + 1 : (a > b ? a : b);
        nd.need = (uint8_t)need;
      }
      nodes[nn] = nd;
      stk[sp++] = (int16_t)nn++;
      continue;
    }
    // unary or unknown token
    if (sp < 1) { h.status = PROG_INVALID; break; }
    const int c = stk[--sp];
    if (!is_unary(cls)) { h.status = PROG_INVALID; break; }
    Node<T> nd;
    nd.cls = (uint8_t)cls;
    nd.idx = 0;
    nd.r = -1;
    if (nodes[c].kind == N_IMM) {
      bool e = false;
      nd.imm = apply_unary<T, STRICT>(cls, nodes[c].imm, e);
      if (e) { h.status = PROG_INVALID; break; }
      nd.kind = N_IMM;
      nd.l = -1;
      nd.need = 0;
    } else {
      nd.kind = N_OP;
      nd.l = (int16_t)c;
      nd.imm = (T)0;
      nd.need = (uint8_t)(nodes[c].need > 1 ? nodes[c].need : 1);
    }
    nodes[nn] = nd;
    stk[sp++] = (int16_t)nn++;
  }
  if (h.status == PROG_OK && sp != 1) h.status = PROG_INVALID;
  if (h.status != PROG_OK) return h;

  // ---- emission: post-order walk with Sethi-Ullman child order ---------------------------
  Emitter<T> em{tape, 0, xmul, tape_capacity(Lr)};
  const int root = stk[0];
  if (nodes[root].kind != N_OP) {  // the whole program is one terminal (or folded constant)
    T imm = (T)0;
    uint32_t bits = loada_bits(nodes[root], imm);
    em.put(CASE_NOP | bits, imm);
    h.n_instr = em.n;
    if (!em.ok) h.status = PROG_UNREPRESENTABLE;
    return h;
  }
  Frame fr[LMAX];
  int top = 0, depth = 0, max_depth = 0;
  fr[0] = Frame{(int16_t)root, 0, 0, 0, 0};
  while (top >= 0) {
    Frame& f = fr[top];
    const Node<T>& nd = nodes[f.node];
    if (is_unary(nd.cls)) {
      const Node<T>& ch = nodes[nd.l];
      if (f.phase == 0 && ch.kind != N_OP) {
        T imm = (T)0;
        uint32_t bits = spill_bits(f.spill, f.slot) | loada_bits(ch, imm) | nd.cls;
        em.put(bits, imm);
        --top;
      } else if (f.phase == 0) {
        f.phase = 1;
        fr[top + 1] = Frame{nd.l, 0, f.spill, f.slot, 0};
        ++top;
      } else {
        em.put((uint32_t)nd.cls, (T)0);
        --top;
      }
      continue;
    }
    // binary
    const Node<T>& L_ = nodes[nd.l];
    const Node<T>& R_ = nodes[nd.r];
    const bool lop = L_.kind == N_OP, rop = R_.kind == N_OP;
    if (!lop && !rop) {
      T imm = (T)0;
      uint32_t bits = spill_bits(f.spill, f.slot);
      bool is_vec;
      if (L_.kind == N_VAR) {
        bits |= loada_bits(L_, imm);
        bits |= opnd_bits(R_, imm, is_vec);
        bits |= bin_case(nd.cls, canon_form(nd.cls, is_vec ? FORM_AV : FORM_AS));
      } else if (R_.kind == N_VAR) {
        bits |= loada_bits(R_, imm);
        bits |= opnd_bits(L_, imm, is_vec);  // scalar left operand
        bits |= bin_case(nd.cls, canon_form(nd.cls, FORM_SA));
      } else {  // two scalars that could not be folded (at least one parameter)
        bits |= loada_bits(L_, imm);
        bits |= opnd_bits(R_, imm, is_vec);
        bits |= bin_case(nd.cls, canon_form(nd.cls, FORM_AS));
      }
      em.put(bits, imm);
      --top;
      continue;
    }
    if (lop && !rop) {
      if (f.phase == 0) {
        f.phase = 1;
        fr[top + 1] = Frame{nd.l, 0, f.spill, f.slot, 0};
        ++top;
      } else {
        T imm = (T)0;
        bool is_vec;
        uint32_t bits = opnd_bits(R_, imm, is_vec);
        bits |= bin_case(nd.cls, canon_form(nd.cls, is_vec ? FORM_AV : FORM_AS));
        em.put(bits, imm);
        --top;
      }
      continue;
    }
    if (!lop && rop) {
      if (f.phase == 0) {
        f.phase = 1;
        fr[top + 1] = Frame{nd.r, 0, f.spill, f.slot, 0};
        ++top;
      } else {
        T imm = (T)0;
        bool is_vec;
        uint32_t bits = opnd_bits(L_, imm, is_vec);
        bits |= bin_case(nd.cls, canon_form(nd.cls, is_vec ? FORM_VA : FORM_SA));
        em.put(bits, imm);
        --top;
      }
      continue;
    }
    // both children are operators
    if (f.phase == 0) {
      f.first_left = (L_.need >= R_.need) ? 1 : 0;
      f.phase = 1;
      fr[top + 1] = Frame{f.first_left ? nd.l : nd.r, 0, f.spill, f.slot, 0};
      ++top;
    } else if (f.phase == 1) {
      f.phase = 2;
      const int slot = depth++;
      if (depth > max_depth) max_depth = depth;
      fr[top + 1] = Frame{f.first_left ? nd.r : nd.l, 0, 1, (uint8_t)slot, 0};
      ++top;
    } else {
      const int slot = --depth;
      uint32_t bits = ((uint32_t)OK_SLOT << SH_OPK) | ((uint32_t)slot << SH_OP_IDX);
      // first_left: the left value sits in the slot and ACC holds the right value
      bits |= bin_case(nd.cls, canon_form(nd.cls, f.first_left ? FORM_VA : FORM_AV));
      em.put(bits, (T)0);
      --top;
    }
  }
  h.n_instr = em.n;
  h.n_slots = max_depth;
  if (!em.ok) h.status = PROG_UNREPRESENTABLE;
  return h;
}


// ---- the same compiler with a linear emission -------------------------------------------------
// compile_program_v2 produces the tape of compile_program, word for word, with less divergent
// control flow for a GPU thread per program: the parse keeps the operator-node counts of every
// subtree, and the emission replaces the depth-first walk with two linear passes.  Pass 1 visits
// the nodes from the root down (creation order reversed: a parent is created after its children)
// and gives every operator its tape position, its spill depth and, for the first instruction of
// a subtree that must spill ACC, that spill: for a binary node whose children are both
// operators, the child with the larger Sethi-Ullman need (the left one on a tie) owns the first
// cnt(first) positions of the parent's range, the other child the next cnt(second), the parent
// the last; the second child's first instruction spills ACC into slot depth.  Pass 2 writes every
// operator's word at its position.
enum : uint8_t { ER_ASSIGNED = 1, ER_SPILL = 2, ER_FIRST_LEFT = 4 };
struct EmitRec {
  int16_t pos;    // tape position of the node's own instruction
  uint8_t depth;  // pending spilled values when the node's subtree starts
  uint8_t flags;  // ER_*; with ER_SPILL, slot = bits 3..5
};

template <typename T, bool STRICT, bool BAKE, int LMAX>
__host__ __device__ ProgHdr compile_program_v2(const uint8_t* __restrict__ prog, int L,
                                               const T* __restrict__ consts, int K,
                                               const TokenLut& lut, Instr<T>* __restrict__ tape,
                                               int xmul) {
  Node<T> nodes[LMAX];
  uint8_t cnt[LMAX];  // operator nodes in each node's subtree (< 256: at most L - 1 <= 255)
  EmitRec er[LMAX];
  int16_t stk[33];
  ProgHdr h;
  h.n_instr = 0;
  h.status = PROG_OK;
  h.n_slots = 0;
  h.n_tok = 0;
  int sp = 0, nn = 0, c_idx = 0;
  const int Lr = L < LMAX ? L : LMAX;

  for (int pc = 0; pc < Lr; ++pc) {
    const int tok = prog[pc];
    const int cls = lut.cls[tok];
    if (cls == T_PAD) break;
    h.n_tok++;
    const bool leaf = is_leaf(cls), bin = is_binary(cls), un = is_unary(cls);
    if (!leaf && !bin && !un) { h.status = PROG_INVALID; break; }
    const int ar = bin ? 2 : (un ? 1 : 0);
    if (sp < ar) { h.status = PROG_INVALID; break; }
    Node<T> nd;
    nd.cls = leaf ? 0 : (uint8_t)cls;
    nd.idx = 0;
    nd.need = 0;
    nd.imm = (T)0;
    nd.l = nd.r = -1;
    uint8_t c_ops = 0;
    if (leaf) {
      if (cls == T_VAR) {
        nd.kind = N_VAR;
        nd.idx = lut.arg[tok];
      } else if (cls == T_CONST) {
        nd.kind = N_IMM;
        if (K > 0) {
          const int slot = c_idx < K ? c_idx : K - 1;
          c_idx++;
          if (BAKE) {
            nd.imm = consts[slot];
          } else {
            nd.kind = N_PARAM;
            nd.idx = (uint8_t)slot;
          }
        } else {
          nd.imm = (T)1.0;
        }
      } else {
        nd.kind = N_IMM;
        nd.imm = (T)lut.lit[lut.arg[tok]];
      }
      if (sp >= 32) continue;  // a push at depth 32 is dropped (the C slot was still consumed)
    } else {
      const int r = stk[sp - 1];
      const int l = bin ? stk[sp - 2] : r;  // a unary operator's child is its left
      sp -= ar;
      const Node<T>& L_ = nodes[l];
      const Node<T>& R_ = nodes[r];
      if (L_.kind == N_IMM && R_.kind == N_IMM) {  // fold (for a unary node L_ is R_)
        bool e = false;
        nd.imm = bin ? apply_binary<T, STRICT>(cls, L_.imm, R_.imm, e)
                     : apply_unary<T, STRICT>(cls, L_.imm, e);
        if (e) { h.status = PROG_INVALID; break; }
        nd.kind = N_IMM;
      } else {
        nd.kind = N_OP;
        nd.l = (int16_t)l;
        nd.r = bin ? (int16_t)r : (int16_t)-1;
        const int a = L_.need, b = bin ? R_.need : 0;
        int need;
        if (!bin) need = a > 1 ? a : 1;
        else if (a == 0 && b == 0) need = 1;
        else if (a == 0) need = b;
        else if (b == 0) need = a;
        else need = (a == b) ? a + 1 : (a > b ? a : b);
        nd.need = (uint8_t)need;
        c_ops = (uint8_t)(1 + cnt[l] + (bin ? cnt[r] : 0));
      }
    }
    if (!WS_BC(nn < LMAX, BC_COMPILE_NODES, nn)) {
      h.status = PROG_INVALID;
      break;
    }
    nodes[nn] = nd;
    cnt[nn] = c_ops;
    stk[sp++] = (int16_t)nn++;
  }
  if (h.status == PROG_OK && sp != 1) h.status = PROG_INVALID;
  if (h.status != PROG_OK) return h;

  Emitter<T> em{tape, 0, xmul, tape_capacity(Lr)};
  const int root = stk[0];
  if (nodes[root].kind != N_OP) {  // the whole program is one terminal (or folded constant)
    T imm = (T)0;
    uint32_t bits = loada_bits(nodes[root], imm);
    em.put(CASE_NOP | bits, imm);
    h.n_instr = em.n;
    if (!em.ok) h.status = PROG_UNREPRESENTABLE;
    return h;
  }
  // pass 1: positions, depths, spills (parents before children)
  for (int i = 0; i <= root; ++i) er[i].flags = 0;
  er[root].pos = (int16_t)(cnt[root] - 1);
  er[root].depth = 0;
  er[root].flags = ER_ASSIGNED;
  int max_depth = 0;
  for (int v = root; v >= 0; --v) {
    const uint8_t f = er[v].flags;
    if (!(f & ER_ASSIGNED) || nodes[v].kind != N_OP) continue;
    const Node<T>& nd = nodes[v];
    const int pe = er[v].pos, d = er[v].depth;
    const uint8_t spill = f & (uint8_t)(ER_SPILL | (7u << 3));
    const bool lop = nodes[nd.l].kind == N_OP;
    const bool rop = is_binary(nd.cls) && nodes[nd.r].kind == N_OP;
    if (lop && rop) {
      const bool first_left = nodes[nd.l].need >= nodes[nd.r].need;
      const int F = first_left ? nd.l : nd.r, S = first_left ? nd.r : nd.l;
      er[S].pos = (int16_t)(pe - 1);
      er[S].depth = (uint8_t)(d + 1);
      er[S].flags = (uint8_t)(ER_ASSIGNED | ER_SPILL | ((d & 7) << 3));
      er[F].pos = (int16_t)(pe - 1 - cnt[S]);
      er[F].depth = (uint8_t)d;
      er[F].flags = (uint8_t)(ER_ASSIGNED | spill);
      er[v].flags = (uint8_t)(ER_ASSIGNED | (first_left ? ER_FIRST_LEFT : 0));
      if (d + 1 > max_depth) max_depth = d + 1;
    } else if (lop || rop) {  // the operator child's subtree starts this node's range
      const int c = lop ? nd.l : nd.r;
      er[c].pos = (int16_t)(pe - 1);
      er[c].depth = (uint8_t)d;
      er[c].flags = (uint8_t)(ER_ASSIGNED | spill);
      er[v].flags = ER_ASSIGNED;
    }
    // no operator child: this node's instruction is its subtree's first and keeps the spill
  }
  // pass 2: every operator's word at its position
  for (int v = 0; v <= root; ++v) {
    const uint8_t f = er[v].flags;
    if (!(f & ER_ASSIGNED) || nodes[v].kind != N_OP) continue;
    const Node<T>& nd = nodes[v];
    const uint32_t sb = spill_bits((f & ER_SPILL) != 0, (f >> 3) & 7);
    const Node<T>& L_ = nodes[nd.l];
    T imm = (T)0;
    uint32_t bits;
    if (is_unary(nd.cls)) {
      bits = L_.kind != N_OP ? (sb | loada_bits(L_, imm) | nd.cls) : (uint32_t)nd.cls;
    } else {
      const Node<T>& R_ = nodes[nd.r];
      const bool lop = L_.kind == N_OP, rop = R_.kind == N_OP;
      bool is_vec;
      if (!lop && !rop) {
        bits = sb;
        if (L_.kind == N_VAR) {
          bits |= loada_bits(L_, imm);
          bits |= opnd_bits(R_, imm, is_vec);
          bits |= bin_case(nd.cls, canon_form(nd.cls, is_vec ? FORM_AV : FORM_AS));
        } else if (R_.kind == N_VAR) {
          bits |= loada_bits(R_, imm);
          bits |= opnd_bits(L_, imm, is_vec);
          bits |= bin_case(nd.cls, canon_form(nd.cls, FORM_SA));
        } else {
          bits |= loada_bits(L_, imm);
          bits |= opnd_bits(R_, imm, is_vec);
          bits |= bin_case(nd.cls, canon_form(nd.cls, FORM_AS));
        }
      } else if (lop && !rop) {
        bits = opnd_bits(R_, imm, is_vec);
        bits |= bin_case(nd.cls, canon_form(nd.cls, is_vec ? FORM_AV : FORM_AS));
      } else if (!lop && rop) {
        bits = opnd_bits(L_, imm, is_vec);
        bits |= bin_case(nd.cls, canon_form(nd.cls, is_vec ? FORM_VA : FORM_SA));
      } else {
        bits = ((uint32_t)OK_SLOT << SH_OPK) | ((uint32_t)er[v].depth << SH_OP_IDX);
        bits |= bin_case(nd.cls, canon_form(nd.cls, (f & ER_FIRST_LEFT) ? FORM_VA : FORM_AV));
      }
    }
    em.put_at(er[v].pos, bits, imm);
  }
  h.n_instr = cnt[root];
  h.n_slots = max_depth;
  if (!em.ok) h.status = PROG_UNREPRESENTABLE;
  return h;
}

}  // namespace ws
