// ws_oracle_simplify.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Literal CPU restatement of the reference's simplify_batch_kernel
// (src/warpsymbolic/gpu/cuda/simplify_kernels.cu:100-601), written rule by rule in the
// reference's own order and control flow (each rule ends the position with `continue`; the
// normalisation falls through), independently of the CUDA kernel of this library, which groups
// identical rules.  Folding uses host libm (the reference build uses fast-math intrinsics), so
// results can differ only where a folded value lies within rounding of the 1e-5 acceptance
// boundary.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

constexpr int kMaxLen = 256, kMaxLits = 64;
constexpr int64_t kPad = 0;

struct Ids {
  int op_plus, op_minus, op_mult, op_div, op_neg, op_mod, op_pow;
  int op_sin, op_cos, op_tan, op_asin, op_acos, op_atan;
  int op_log, op_exp, op_sqrt, op_abs, op_gamma, op_lgamma, op_floor, op_ceil, op_sign;
  int id_0, id_1, id_2, id_3, id_4, id_5, id_6;
};

int subtree_start(const int64_t* f, const int32_t* ar, int max_id, int end_idx, int L) {
  if (end_idx < 0 || end_idx >= L) return -1;
  const int64_t tok = f[end_idx];
  if (tok == kPad || tok < 0 || tok >= max_id) return end_idx;
  int balance = 1;
  for (int k = end_idx; k >= 0; k--) {
    const int64_t t = f[k];
    if (t == kPad || t < 0 || t >= max_id) balance -= 1;
    else balance += ar[std::min((int)t, max_id - 1)] - 1;
    if (balance == 0) return k;
  }
  return 0;
}

void compact(int64_t* f, int L) {
  int w = 0;
  for (int r = 0; r < L; r++)
    if (f[r] != kPad) f[w++] = f[r];
  for (int i = w; i < L; i++) f[i] = kPad;
}

bool nearest(float res, const int64_t* ids, const float* vals, int n, int64_t* out) {
  if (std::isnan(res) || std::isinf(res)) return false;
  float best = 1e30f;
  int bi = -1;
  for (int i = 0; i < n; i++) {
    const float d = std::fabs(res - vals[i]);
    if (d < best) {
      best = d;
      bi = i;
    }
  }
  if (bi >= 0 && best < 1e-5f) {
    *out = ids[bi];
    return true;
  }
  return false;
}

void simplify_row(int64_t* row, int L_in, const int32_t* ar, int max_id, const float* vt,
                  const int64_t* lit_ids, const float* lit_vals, int n_lits, int max_passes,
                  const Ids& o) {
  int64_t f[kMaxLen];
  const int L = std::min(L_in, kMaxLen);
  for (int i = 0; i < L; i++) f[i] = row[i];
  for (int i = L; i < kMaxLen; i++) f[i] = kPad;
  const float NaN = std::nanf("");
  for (int pass = 0; pass < max_passes; pass++) {
    bool changed = false;
    for (int j = 1; j < L; j++) {
      const int64_t tok = f[j];
      if (tok == kPad) continue;
      const int64_t prev = f[j - 1];
      if (tok == o.op_neg && prev == o.op_neg) {
        f[j] = kPad;
        f[j - 1] = kPad;
        changed = true;
        continue;
      }
      if (j >= 2 && tok == o.op_sqrt && prev == o.op_pow && f[j - 2] == o.id_2 &&
          o.op_abs != -1) {
        f[j] = o.op_abs;
        f[j - 1] = kPad;
        f[j - 2] = kPad;
        changed = true;
        continue;
      }
      if (tok > 0 && tok < max_id && ar[tok] == 1 && prev != kPad) {
        const bool is0 = prev == o.id_0, is1 = prev == o.id_1, is2 = prev == o.id_2;
        bool zero = false;
        if (is0 && (tok == o.op_sin || tok == o.op_tan || tok == o.op_abs)) zero = true;
        if (is1 && (tok == o.op_log || tok == o.op_lgamma)) zero = true;
        if (is2 && tok == o.op_lgamma) zero = true;
        if (zero && o.id_0 != -1) {
          f[j - 1] = o.id_0;
          f[j] = kPad;
          changed = true;
          continue;
        }
        bool one = false;
        if (is0 && (tok == o.op_cos || tok == o.op_exp)) one = true;
        if ((is1 || is2) && tok == o.op_gamma) one = true;
        if (one && o.id_1 != -1) {
          f[j - 1] = o.id_1;
          f[j] = kPad;
          changed = true;
          continue;
        }
        if (n_lits > 0 && prev > 0 && prev < max_id) {
          const float v = vt[prev];
          if (!std::isnan(v)) {
            float res = NaN;
            if (tok == o.op_sin) res = std::sin(v);
            else if (tok == o.op_cos) res = std::cos(v);
            else if (tok == o.op_tan) res = std::tan(v);
            else if (tok == o.op_log) res = v > 0 ? std::log(v) : NaN;
            else if (tok == o.op_exp) res = v < 80.0f ? std::exp(v) : NaN;
            else if (tok == o.op_sqrt) res = v >= 0 ? std::sqrt(v) : NaN;
            else if (tok == o.op_abs) res = std::fabs(v);
            else if (tok == o.op_neg) res = -v;
            else if (tok == o.op_floor) res = std::floor(v);
            else if (tok == o.op_ceil) res = std::ceil(v);
            else if (tok == o.op_sign) res = v > 0 ? 1.0f : (v < 0 ? -1.0f : 0.0f);
            else if (tok == o.op_asin) res = std::fabs(v) <= 1.0f ? std::asin(v) : NaN;
            else if (tok == o.op_acos) res = std::fabs(v) <= 1.0f ? std::acos(v) : NaN;
            else if (tok == o.op_atan) res = std::atan(v);
            else if (tok == o.op_gamma)
              res = (v > 0 && v < 20.0f) ? std::exp(std::lgamma(v)) : NaN;
            else if (tok == o.op_lgamma) res = v > 0 ? std::lgamma(v) : NaN;
            int64_t lit;
            if (nearest(res, lit_ids, lit_vals, n_lits, &lit)) {
              f[j - 1] = lit;
              f[j] = kPad;
              changed = true;
              continue;
            }
          }
        }
      }
      if (j >= 3 && tok == o.op_plus && f[j - 1] == o.op_neg) {
        const int s_neg_arg = subtree_start(f, ar, max_id, j - 2, L);
        const int e_first = s_neg_arg - 1;
        if (e_first >= 0 && s_neg_arg >= 0) {
          const int s_first = subtree_start(f, ar, max_id, e_first, L);
          if (s_first >= 0) {
            const int len1 = e_first - s_first + 1, len2 = (j - 2) - s_neg_arg + 1;
            if (len1 == len2 && len1 > 0) {
              bool match = true;
              for (int k = 0; k < len1; k++)
                if (f[s_first + k] != f[s_neg_arg + k]) {
                  match = false;
                  break;
                }
              if (match && o.id_0 != -1) {
                f[s_first] = o.id_0;
                for (int k = s_first + 1; k <= j; k++) f[k] = kPad;
                changed = true;
                continue;
              }
            }
          }
        }
      }
    }
    compact(f, L);
    for (int j = 2; j < L; j++) {
      const int64_t op = f[j];
      if (op == kPad) continue;
      if (op < 0 || op >= max_id) continue;
      if (ar[op] != 2) continue;
      const int s2 = subtree_start(f, ar, max_id, j - 1, L);
      const int s1 = subtree_start(f, ar, max_id, s2 - 1, L);
      if (s1 < 0 || s2 < 0) continue;
      const int len1 = s2 - s1, len2 = j - s2;
      const int64_t a2 = (s2 == j - 1) ? f[j - 1] : -999;
      const int64_t a1 = (s1 == s2 - 1) ? f[s2 - 1] : -999;
      const bool a2z = a2 == o.id_0, a2o = a2 == o.id_1, a1z = a1 == o.id_0, a1o = a1 == o.id_1;
      const bool is_pow = op == o.op_pow;
      if ((op == o.op_plus || op == o.op_minus) && a2z) {
        f[j - 1] = kPad;
        f[j] = kPad;
        changed = true;
        continue;
      }
      if ((op == o.op_mult || op == o.op_div || is_pow) && a2o) {
        f[j - 1] = kPad;
        f[j] = kPad;
        changed = true;
        continue;
      }
      if (is_pow && a2z && o.id_1 != -1) {
        for (int k = s1; k <= j; k++) f[k] = kPad;
        f[s1] = o.id_1;
        changed = true;
        continue;
      }
      if (is_pow && a1o && o.id_1 != -1) {
        for (int k = s1; k <= j; k++) f[k] = kPad;
        f[s1] = o.id_1;
        changed = true;
        continue;
      }
      if (op == o.op_plus && a1z) {
        f[s2 - 1] = kPad;
        f[j] = kPad;
        changed = true;
        continue;
      }
      if (op == o.op_mult && a1o) {
        f[s2 - 1] = kPad;
        f[j] = kPad;
        changed = true;
        continue;
      }
      if (op == o.op_mult && (a2z || a1z) && o.id_0 != -1) {
        for (int k = s1; k <= j; k++) f[k] = kPad;
        f[s1] = o.id_0;
        changed = true;
        continue;
      }
      if (op == o.op_minus && a1z && o.op_neg != -1) {
        f[s2 - 1] = kPad;
        f[j] = o.op_neg;
        changed = true;
        continue;
      }
      if (op == o.op_plus || op == o.op_mult) {
        const bool l1 = len1 == 1, l2 = len2 == 1;
        bool c1 = false, c2 = false;
        if (l1 && a1 > 0 && a1 < max_id) c1 = !std::isnan(vt[a1]);
        if (l2 && a2 > 0 && a2 < max_id) c2 = !std::isnan(vt[a2]);
        const int sc1 = c1 ? 0 : (l1 ? 1 : 2), sc2 = c2 ? 0 : (l2 ? 1 : 2);
        bool sw = false;
        if (sc2 < sc1) sw = true;
        if (sc1 == sc2 && sc1 < 2 && a2 != -999 && a1 != -999 && a2 < a1) sw = true;
        if (sc1 == 2 && sc2 == 2 && len2 < len1) sw = true;
        if (sw) {
          if (l1 && l2) {
            f[s2 - 1] = a2;
            f[j - 1] = a1;
          } else {
            std::vector<int64_t> tmp(f + s1, f + s1 + len1);
            for (int k = 0; k < len2; k++) f[s1 + k] = f[s2 + k];
            for (int k = 0; k < len1; k++) f[s1 + len2 + k] = tmp[k];
          }
        }
      }
      if (op == o.op_plus && j >= 6) {
        const int64_t v0 = f[j], v1 = f[j - 1], v2 = f[j - 2], v3 = f[j - 3], v4 = f[j - 4],
                      v5 = f[j - 5], v6 = f[j - 6];
        auto term = [&](int64_t t) { return t >= 0 && t < max_id && ar[t] == 0; };
        if (v0 == o.op_plus && v1 == o.op_mult && v4 == o.op_mult) {
          if (v5 == v2 && v5 != kPad && term(v5) && term(v6) && term(v3)) {
            f[j - 6] = v6;
            f[j - 5] = v3;
            f[j - 4] = o.op_plus;
            f[j - 3] = v5;
            f[j - 2] = o.op_mult;
            f[j - 1] = kPad;
            f[j] = kPad;
            changed = true;
            continue;
          }
          if (v6 == v3 && v6 != kPad && term(v6) && term(v5) && term(v2)) {
            f[j - 6] = v5;
            f[j - 5] = v2;
            f[j - 4] = o.op_plus;
            f[j - 3] = v6;
            f[j - 2] = o.op_mult;
            f[j - 1] = kPad;
            f[j] = kPad;
            changed = true;
            continue;
          }
        }
      }
      if (op == o.op_plus && o.id_2 != -1 && j >= 4 && f[j - 1] == o.op_plus) {
        const int s_ir = subtree_start(f, ar, max_id, j - 2, L);
        if (s_ir >= 1) {
          const int e_il = s_ir - 1;
          const int s_il = subtree_start(f, ar, max_id, e_il, L);
          if (s_il >= 1) {
            const int e_o1 = s_il - 1;
            const int s_o1 = subtree_start(f, ar, max_id, e_o1, L);
            if (s_o1 >= 0) {
              const bool o1s = s_o1 == e_o1, ils = s_il == e_il;
              bool done = false;
              if (o1s && ils && f[s_o1] == f[s_il] && f[s_o1] != kPad) {
                const int y_len = (j - 2) - s_ir + 1;
                if (3 + y_len + 1 <= j - s_o1 + 1) {
                  const int64_t x = f[s_o1];
                  std::vector<int64_t> y(f + s_ir, f + s_ir + y_len);
                  int w = s_o1;
                  f[w++] = o.id_2;
                  f[w++] = x;
                  f[w++] = o.op_mult;
                  for (int k = 0; k < y_len; k++) f[w++] = y[k];
                  f[w++] = o.op_plus;
                  for (int k = w; k <= j; k++) f[k] = kPad;
                  changed = true;
                  done = true;
                }
              }
              if (!done) {
                const int irl = (j - 2) - s_ir + 1;
                if (o1s && irl == 1 && f[s_o1] == f[s_ir] && f[s_o1] != kPad) {
                  const int y_len = e_il - s_il + 1;
                  if (3 + y_len + 1 <= j - s_o1 + 1) {
                    const int64_t x = f[s_o1];
                    std::vector<int64_t> y(f + s_il, f + s_il + y_len);
                    int w = s_o1;
                    f[w++] = o.id_2;
                    f[w++] = x;
                    f[w++] = o.op_mult;
                    for (int k = 0; k < y_len; k++) f[w++] = y[k];
                    f[w++] = o.op_plus;
                    for (int k = w; k <= j; k++) f[k] = kPad;
                    changed = true;
                    done = true;
                  }
                }
              }
              if (done) continue;
            }
          }
        }
      }
      if (n_lits > 0 && a1 != -999 && a2 != -999 && a1 > 0 && a1 < max_id && a2 > 0 &&
          a2 < max_id) {
        const float v1 = vt[a1], v2 = vt[a2];
        if (!std::isnan(v1) && !std::isnan(v2)) {
          float res = NaN;
          if (op == o.op_plus) res = v1 + v2;
          else if (op == o.op_minus) res = v1 - v2;
          else if (op == o.op_mult) res = v1 * v2;
          else if (op == o.op_div && std::fabs(v2) > 1e-9f) res = v1 / v2;
          else if (op == o.op_pow) res = std::pow(v1, v2);
          else if (op == o.op_mod && std::fabs(v2) > 1e-9f) res = std::fmod(v1, v2);
          int64_t lit;
          if (nearest(res, lit_ids, lit_vals, n_lits, &lit)) {
            f[s1] = lit;
            for (int k = s1 + 1; k <= j; k++) f[k] = kPad;
            changed = true;
            continue;
          }
        }
      }
    }
    compact(f, L);
    if (!changed) break;
  }
  for (int i = 0; i < L; i++) row[i] = f[i];
}

}  // namespace

extern "C" void ws_oracle_simplify(int64_t* pop, int64_t B, int64_t L, const int32_t* ar,
                                   int64_t max_id, const float* vt, const int64_t* lit_ids,
                                   const float* lit_vals, int64_t n_lits, int32_t max_passes,
                                   const int32_t* ids29) {
  Ids o;
  int32_t* dst = reinterpret_cast<int32_t*>(&o);
  for (int i = 0; i < 29; ++i) dst[i] = ids29[i];
  const int n = (int)std::min<int64_t>(n_lits, kMaxLits);
  for (int64_t b = 0; b < B; ++b)
    simplify_row(pop + b * L, (int)L, ar, (int)max_id, vt, lit_ids, lit_vals, n, max_passes, o);
}
