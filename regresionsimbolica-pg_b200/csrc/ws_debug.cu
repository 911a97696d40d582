// ws_debug.cu -- host-only introspection entry points (ws_debug_*).
//
// These run the program compiler (ws_compile.cuh) and a scalar interpreter of its tape on the
// HOST, with the C library's math, so the compiler can be verified exactly on a machine
// without a GPU: per-row results of compile+run must equal a direct stack interpretation with
// the same math.  They are not an evaluation path: no fitness entry point calls them.
#include <cstdint>
#include <cstring>
#include <vector>

#include "ws_internal.h"
#include "ws_compile.cuh"

namespace ws {
namespace {

template <typename T, bool STRICT>
int32_t compile_host(const uint8_t* prog, int64_t L, const T* consts, int64_t K,
                     const TokenLut& lut, uint32_t* ctrl_out, double* imm_out, int32_t* hdr_out) {
  const int Lcap = tape_capacity((int)L);
  std::vector<Instr<T>> tape((size_t)Lcap);
  // xmul = 1: tape offsets are plain variable / slot indices
  const ProgHdr h = compile_program_v2<T, STRICT, true, 256>(prog, (int)L, consts, (int)K, lut,
                                                             tape.data(), 1);
  hdr_out[0] = h.n_instr;
  hdr_out[1] = h.status;
  hdr_out[2] = h.n_slots;
  hdr_out[3] = h.n_tok;
  for (int i = 0; i < h.n_instr; ++i) {
    ctrl_out[i] = tape[i].ctrl;
    imm_out[i] = (double)tape[i].imm;
  }
  return h.n_instr;
}

template <typename T, bool STRICT>
void run_host(const uint32_t* ctrl, const double* imm, int n, const T* x, int64_t D,
              T* out_pred, uint8_t* out_err) {
  // xmul = 1: tape offsets of X operands are variable indices
  for (int64_t d = 0; d < D; ++d) {
    T acc = (T)0, slots[32];
    bool err = false;
    for (int i = 0; i < n; ++i) {
      const uint32_t c = ctrl[i];
      const T im = (T)imm[i];
      if (c & P_SPILL) slots[(c >> P_SH_SLOT) & 7u] = acc;
      if (c & P_LOADA_X) acc = x[((c >> P_SH_LA) & P_OFF_MASK) * D + d];
      else if (c & P_LOADA_S) acc = im;
      T v = im;
      const uint32_t cs = c & P_CASE_MASK;
      if (pcase_fetches(cs)) {
        const uint32_t off = c >> P_SH_V;
        v = (c & P_FETCH_SLOT) ? slots[off & 31u] : x[off * D + d];
      }
      bool e = false;
      if (cs == PCASE_NOP) {
      } else if (cs >= PCASE_BIN) {
        const int cls = T_ADD + (int)((cs - PCASE_BIN) >> 2), form = (int)((cs - PCASE_BIN) & 3u);
        const bool acc_left = form == FORM_AV || form == FORM_AS;
        acc = acc_left ? apply_binary<T, STRICT>(cls, acc, v, e)
                       : apply_binary<T, STRICT>(cls, v, acc, e);
      } else {
        acc = apply_unary<T, STRICT>(T_SIN + (int)cs - PCASE_UNARY0, acc, e);
      }
      err = err || e;
    }
    out_pred[d] = acc;
    out_err[d] = err ? 1 : 0;
  }
}

// Compiles each of B programs with the depth-first emitter (compile_program) and the linear one
// (compile_program_v2) and counts the programs whose headers or tape words differ.
template <typename T, bool STRICT>
int64_t compile_agree_host(const uint8_t* progs, int64_t B, int64_t L, const T* consts,
                           int64_t K, const TokenLut& lut, int xmul) {
  const int Lcap = tape_capacity((int)L);
  std::vector<Instr<T>> a((size_t)Lcap), b((size_t)Lcap);
  int64_t bad = 0;
  for (int64_t p = 0; p < B; ++p) {
    const uint8_t* prog = progs + p * L;
    const T* c = K > 0 ? consts + p * K : nullptr;
    std::memset(a.data(), 0, a.size() * sizeof(Instr<T>));
    std::memset(b.data(), 0, b.size() * sizeof(Instr<T>));
    const ProgHdr ha = compile_program<T, STRICT, true, 256>(prog, (int)L, c, (int)K, lut,
                                                             a.data(), xmul);
    const ProgHdr hb = compile_program_v2<T, STRICT, true, 256>(prog, (int)L, c, (int)K, lut,
                                                                b.data(), xmul);
    bool same = ha.status == hb.status && ha.n_tok == hb.n_tok;
    if (same && ha.status == PROG_OK) {
      same = ha.n_instr == hb.n_instr && ha.n_slots == hb.n_slots &&
             std::memcmp(a.data(), b.data(), (size_t)ha.n_instr * sizeof(Instr<T>)) == 0;
    }
    bad += same ? 0 : 1;
  }
  return bad;
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

ws_status ws_debug_token_lut(const ws_token_map* ids, int64_t num_vars, int32_t fused_order,
                             uint8_t* cls_out, uint8_t* arg_out) {
  clear_error();
  if (!ids || !cls_out || !arg_out) return fail("null pointer");
  const TokenLut lut = build_lut(*ids, num_vars, fused_order != 0);
  std::memcpy(cls_out, lut.cls, 256);
  std::memcpy(arg_out, lut.arg, 256);
  return WS_OK;
}

ws_status ws_debug_compile(int32_t dtype, const uint8_t* prog, int64_t L, const void* consts,
                           int64_t K, const ws_token_map* ids, int64_t num_vars,
                           int32_t strict_mode, int32_t fused_order, uint32_t* ctrl_out,
                           double* imm_out, int32_t* hdr_out) {
  clear_error();
  if (!ids || !ctrl_out || !imm_out || !hdr_out) return fail("null pointer");
  if (L < 0 || L > 256) return fail("program length must be in [0, 256]");
  if (K < 0 || (K > 0 && !consts)) return fail("bad constants");
  const TokenLut lut = build_lut(*ids, num_vars, fused_order != 0);
  if (dtype == WS_F32) {
    if (strict_mode) compile_host<float, true>(prog, L, (const float*)consts, K, lut, ctrl_out, imm_out, hdr_out);
    else compile_host<float, false>(prog, L, (const float*)consts, K, lut, ctrl_out, imm_out, hdr_out);
  } else {
    if (strict_mode) compile_host<double, true>(prog, L, (const double*)consts, K, lut, ctrl_out, imm_out, hdr_out);
    else compile_host<double, false>(prog, L, (const double*)consts, K, lut, ctrl_out, imm_out, hdr_out);
  }
  return WS_OK;
}

ws_status ws_debug_compile_agree(int32_t dtype, const uint8_t* progs, int64_t B, int64_t L,
                                 const void* consts, int64_t K, const ws_token_map* ids,
                                 int64_t num_vars, int32_t strict_mode, int32_t fused_order,
                                 int32_t xmul, int64_t* mismatches_out) {
  clear_error();
  if (!ids || !progs || !mismatches_out) return fail("null pointer");
  if (L < 1 || L > 256 || B < 0 || xmul < 1) return fail("bad shape");
  if (K < 0 || (K > 0 && !consts)) return fail("bad constants");
  const TokenLut lut = build_lut(*ids, num_vars, fused_order != 0);
  if (dtype == WS_F32) {
    *mismatches_out = strict_mode
        ? compile_agree_host<float, true>(progs, B, L, (const float*)consts, K, lut, xmul)
        : compile_agree_host<float, false>(progs, B, L, (const float*)consts, K, lut, xmul);
  } else {
    *mismatches_out = strict_mode
        ? compile_agree_host<double, true>(progs, B, L, (const double*)consts, K, lut, xmul)
        : compile_agree_host<double, false>(progs, B, L, (const double*)consts, K, lut, xmul);
  }
  return WS_OK;
}

ws_status ws_debug_run_tape(int32_t dtype, const uint32_t* ctrl, const double* imm, int32_t n,
                            const void* x, int64_t D, int32_t strict_mode, void* out_pred,
                            uint8_t* out_err) {
  clear_error();
  if (!ctrl || !imm || !out_pred || !out_err || n < 0 || D < 0) return fail("bad arguments");
  if (dtype == WS_F32) {
    if (strict_mode) run_host<float, true>(ctrl, imm, n, (const float*)x, D, (float*)out_pred, out_err);
    else run_host<float, false>(ctrl, imm, n, (const float*)x, D, (float*)out_pred, out_err);
  } else {
    if (strict_mode) run_host<double, true>(ctrl, imm, n, (const double*)x, D, (double*)out_pred, out_err);
    else run_host<double, false>(ctrl, imm, n, (const double*)x, D, (double*)out_pred, out_err);
  }
  return WS_OK;
}

}  // extern "C"
