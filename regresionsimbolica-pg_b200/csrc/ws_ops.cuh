// ws_ops.cuh -- RPN token classes and operator semantics shared by every kernel.
//
// The operator definitions reproduce the reference's protected operators
// (src/warpsymbolic/gpu/cuda/rpn_kernels.cu:27-120) and strict operators (:126-199) exactly:
// the same comparisons, constants and libm calls, so that translation units compiled with the
// reference's nvcc flags (-O3 --use_fast_math, src/warpsymbolic/gpu/cuda/setup.py:35) produce
// the same bits per operation.  The interpreter structure around them is new (see ws_compile.cuh
// and ws_fitness.cu); only these scalar definitions must stay alike.
#pragma once

#include <cstdint>
#include <cmath>

#ifndef WS_HD
#define WS_HD __host__ __device__ __forceinline__
#endif

namespace ws {

// Internal token classes.  The host turns the reference's scalar ID arguments into a 256-entry
// lookup table (token byte -> class) once per call, following the reference's precedence
// (PAD, variables, C, literals, binary ops, unary ops; rpn_kernels.cu:249-346).
enum TokenClass : uint8_t {
  T_PAD = 0,
  T_VAR = 1,
  T_CONST = 2,
  T_LIT = 3,
  T_UNKNOWN = 4,
  // binary operators
  T_ADD = 8, T_SUB = 9, T_MUL = 10, T_DIV = 11, T_POW = 12, T_MOD = 13,
  // unary operators
  T_SIN = 16, T_COS, T_TAN, T_LOG, T_EXP, T_SQRT, T_ABS, T_NEG, T_FACT, T_FLOOR, T_CEIL,
  T_SIGN, T_GAMMA, T_LGAMMA, T_ASIN, T_ACOS, T_ATAN,
  T_LAST_UNARY = T_ATAN
};

WS_HD bool is_binary(int c) { return c >= T_ADD && c <= T_MOD; }
WS_HD bool is_unary(int c) { return c >= T_SIN && c <= T_LAST_UNARY; }
WS_HD bool is_leaf(int c) { return c == T_VAR || c == T_CONST || c == T_LIT; }

// Literal slots of the lookup table: 0,1,2,3,4,5,6,10,pi,e.
enum { N_LITERALS = 10 };

struct TokenLut {
  uint8_t cls[256];   // TokenClass per token byte
  uint8_t arg[256];   // variable index (T_VAR) or literal slot (T_LIT)
  double lit[N_LITERALS];
};

// Reference sentinels (rpn_kernels.cu:2320-2323, evaluation.py:23).
template <typename T> struct Limits;
template <> struct Limits<float> {
  static constexpr float invalid = 1e15f;
  static constexpr float max_diff = 4e18f;
  static constexpr float no_value = 1e30f;  // out_preds when sp == 0 (rpn_kernels.cu:243)
};
template <> struct Limits<double> {
  static constexpr double invalid = 1e100;
  static constexpr double max_diff = 1e150;
  static constexpr double no_value = 1e30;
};

// ---- libm wrappers: float calls the f-suffixed functions (mapped to the fast intrinsics when
// the translation unit is built with --use_fast_math, like the reference), double the plain ones.
// The host pass of nvcc resolves the same calls to the C library, which is what the CPU
// verification entry points (ws_debug_*) use.
WS_HD float m_abs(float a) { return fabsf(a); }
WS_HD double m_abs(double a) { return fabs(a); }
WS_HD float m_sin(float a) { return sinf(a); }
WS_HD double m_sin(double a) { return sin(a); }
WS_HD float m_cos(float a) { return cosf(a); }
WS_HD double m_cos(double a) { return cos(a); }
WS_HD float m_tan(float a) { return tanf(a); }
WS_HD double m_tan(double a) { return tan(a); }
WS_HD float m_log(float a) { return logf(a); }
WS_HD double m_log(double a) { return log(a); }
WS_HD float m_exp(float a) { return expf(a); }
WS_HD double m_exp(double a) { return exp(a); }
WS_HD float m_sqrt(float a) { return sqrtf(a); }
WS_HD double m_sqrt(double a) { return sqrt(a); }
WS_HD float m_pow(float a, float b) { return powf(a, b); }
WS_HD double m_pow(double a, double b) { return pow(a, b); }
WS_HD float m_fmod(float a, float b) { return fmodf(a, b); }
WS_HD double m_fmod(double a, double b) { return fmod(a, b); }
WS_HD float m_round(float a) { return roundf(a); }
WS_HD double m_round(double a) { return round(a); }
WS_HD float m_floor(float a) { return floorf(a); }
WS_HD double m_floor(double a) { return floor(a); }
WS_HD float m_ceil(float a) { return ceilf(a); }
WS_HD double m_ceil(double a) { return ceil(a); }
WS_HD float m_tgamma(float a) { return tgammaf(a); }
WS_HD double m_tgamma(double a) { return tgamma(a); }
WS_HD float m_lgamma(float a) { return lgammaf(a); }
WS_HD double m_lgamma(double a) { return lgamma(a); }
WS_HD float m_asin(float a) { return asinf(a); }
WS_HD double m_asin(double a) { return asin(a); }
WS_HD float m_acos(float a) { return acosf(a); }
WS_HD double m_acos(double a) { return acos(a); }
WS_HD float m_atan(float a) { return atanf(a); }
WS_HD double m_atan(double a) { return atan(a); }
template <typename T> WS_HD bool m_isnan(T a) {
#ifdef __CUDA_ARCH__
  return isnan(a);
#else
  return std::isnan(a);
#endif
}
template <typename T> WS_HD bool m_isinf(T a) {
#ifdef __CUDA_ARCH__
  return isinf(a);
#else
  return std::isinf(a);
#endif
}

// ---- binary operators ------------------------------------------------------------------
template <typename T, bool STRICT>
WS_HD T op_div(T a, T b, bool& e) {
  if (STRICT) {  // strict_div, rpn_kernels.cu:127-130
    if (m_abs(b) < (T)1e-9) { e = true; return (T)0.0; }
    return a / b;
  }
  if (m_abs(b) < (T)1e-9) return a;  // safe_div, rpn_kernels.cu:28-33
  return a / b;
}

template <typename T, bool STRICT>
WS_HD T op_mod(T a, T b, bool& e) {
  // safe_mod / strict_mod, rpn_kernels.cu:36-45, 133-138
  if (m_abs(b) < (T)1e-9) {
    if (STRICT) e = true;
    return (T)0.0;
  }
  T r = m_fmod(a, b);
  if ((b > 0 && r < 0) || (b < 0 && r > 0)) r += b;
  return r;
}

template <typename T, bool STRICT>
WS_HD T op_pow(T a, T b, bool& e) {
  // safe_pow / strict_pow, rpn_kernels.cu:66-90, 160-171
  if (a != a || b != b) { e = true; return (T)0.0; }
  if (m_abs(a) < (T)1e-10 && m_abs(b) < (T)1e-10) return (T)1.0;
  if (a < (T)0.0) {
    T ib = m_round(b);
    if (m_abs(b - ib) > (T)1e-3) {
      if (STRICT) { e = true; return (T)0.0; }
      a = m_abs(a);
    } else {
      b = ib;
    }
  }
  if (!STRICT) {
    if (m_abs(a) > (T)1.0 && b > (T)80.0) b = (T)80.0;
    if (m_abs(a) > (T)100.0 && b > (T)10.0) b = (T)10.0;
  }
  T res = m_pow(a, b);
  if (res != res || m_isinf(res)) { e = true; return (T)0.0; }
  return res;
}

template <typename T, bool STRICT>
WS_HD T apply_binary(int cls, T a, T b, bool& e) {
  switch (cls) {
    case T_ADD: return a + b;
    case T_SUB: return a - b;
    case T_MUL: return a * b;
    case T_DIV: return op_div<T, STRICT>(a, b, e);
    case T_POW: return op_pow<T, STRICT>(a, b, e);
    default: return op_mod<T, STRICT>(a, b, e);
  }
}

// ---- unary operators -------------------------------------------------------------------
template <typename T, bool STRICT>
WS_HD T op_log(T a, bool& e) {
  if (STRICT) {  // strict_log, rpn_kernels.cu:141-144
    if (a <= (T)0.0) { e = true; return (T)0.0; }
    return m_log(a);
  }
  return m_log(m_abs(a) + (T)1e-9);  // safe_log, rpn_kernels.cu:48-50
}

template <typename T, bool STRICT>
WS_HD T op_exp(T a, bool& e) {
  if (STRICT) {  // strict_exp, rpn_kernels.cu:147-151
    T res = m_exp(a);
    if (m_isinf(res)) { e = true; return (T)0.0; }
    return res;
  }
  T x = a;  // safe_exp, rpn_kernels.cu:53-58
  if (x < (T)-80.0) x = (T)-80.0;
  if (x > (T)80.0) x = (T)80.0;
  return m_exp(x);
}

template <typename T, bool STRICT>
WS_HD T op_sqrt(T a, bool& e) {
  if (STRICT) {  // strict_sqrt, rpn_kernels.cu:154-157
    if (a < (T)0.0) { e = true; return (T)0.0; }
    return m_sqrt(a);
  }
  return m_sqrt(m_abs(a));  // safe_sqrt, rpn_kernels.cu:61-63
}

template <typename T, bool STRICT>
WS_HD T op_tgamma(T a, bool& e) {
  // safe_tgamma / strict_tgamma, rpn_kernels.cu:107-112, 186-191
  if (a <= (T)0.0 && m_floor(a) == a) {
    if (STRICT) e = true;
    return (T)0.0;
  }
  T res = m_tgamma(a);
  if (res != res || m_isinf(res)) { e = true; return (T)0.0; }
  return res;
}

template <typename T, bool STRICT>
WS_HD T op_lgamma(T a, bool& e) {
  // safe_lgamma / strict_lgamma, rpn_kernels.cu:115-120, 194-199
  if (a <= (T)0.0 && m_floor(a) == a) {
    if (STRICT) e = true;
    return (T)0.0;
  }
  T res = m_lgamma(a);
  if (res != res || m_isinf(res)) { e = true; return (T)0.0; }
  return res;
}

template <typename T, bool STRICT>
WS_HD T op_asin(T a, bool& e) {
  if (STRICT) {  // strict_asin, rpn_kernels.cu:174-177
    if (a < (T)-1.0 || a > (T)1.0) { e = true; return (T)0.0; }
    return m_asin(a);
  }
  if (a < (T)-1.0) a = (T)-1.0;  // safe_asin, rpn_kernels.cu:93-97
  if (a > (T)1.0) a = (T)1.0;
  return m_asin(a);
}

template <typename T, bool STRICT>
WS_HD T op_acos(T a, bool& e) {
  if (STRICT) {  // strict_acos, rpn_kernels.cu:180-183
    if (a < (T)-1.0 || a > (T)1.0) { e = true; return (T)0.0; }
    return m_acos(a);
  }
  if (a < (T)-1.0) a = (T)-1.0;  // safe_acos, rpn_kernels.cu:100-104
  if (a > (T)1.0) a = (T)1.0;
  return m_acos(a);
}

template <typename T>
WS_HD T op_sign(T a) {  // rpn_kernels.cu:341
  return (a > (T)0.0) ? (T)1.0 : ((a < (T)0.0) ? (T)-1.0 : (T)0.0);
}

template <typename T, bool STRICT>
WS_HD T apply_unary(int cls, T a, bool& e) {
  switch (cls) {
    case T_SIN: return m_sin(a);
    case T_COS: return m_cos(a);
    case T_TAN: return m_tan(a);
    case T_LOG: return op_log<T, STRICT>(a, e);
    case T_EXP: return op_exp<T, STRICT>(a, e);
    case T_SQRT: return op_sqrt<T, STRICT>(a, e);
    case T_ABS: return m_abs(a);
    case T_NEG: return -a;
    case T_FACT: return op_tgamma<T, STRICT>(a + (T)1.0, e);
    case T_FLOOR: return m_floor(a);
    case T_CEIL: return m_ceil(a);
    case T_SIGN: return op_sign<T>(a);
    case T_GAMMA: return op_tgamma<T, STRICT>(a, e);
    case T_LGAMMA: return op_lgamma<T, STRICT>(a, e);
    case T_ASIN: return op_asin<T, STRICT>(a, e);
    case T_ACOS: return op_acos<T, STRICT>(a, e);
    case T_ATAN: return m_atan(a);
    default: e = true; return (T)0.0;
  }
}

}  // namespace ws
