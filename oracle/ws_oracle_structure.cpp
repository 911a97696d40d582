// ws_oracle_structure.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Literal CPU restatements of the reference's population-structure routines, used by tests/ as
// the checker of the structure kernels.  Each loop follows the reference's own algorithm (the
// O(L^2) backward scan, the fixed-size subtree-length table, the torch cumulative sums), not the
// faster formulations of the CUDA kernels, so that agreement is evidence of equivalence.  Paths
// are relative to src/warpsymbolic/gpu/ of the reference project.
//
// Pinned against: the reference's torch formulations run on CPU
// (tests/golden/make_structure_golden.py -> structure_torch.npz) and the reference extension's
// own kernels on the same inputs (tests/golden/make_ref_golden.py -> ref_structure.npz).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

int64_t tok_at(const void* pop, int token_bytes, int64_t idx) {
  return token_bytes == 1 ? (int64_t) static_cast<const uint8_t*>(pop)[idx]
                          : static_cast<const int64_t*>(pop)[idx];
}

// validate_rpn_batch_kernel, cuda/rpn_kernels.cu:850-900.
bool validate_kernel_row(const void* pop, int tb, int64_t b, int64_t L, const int32_t* ar,
                         int64_t n_ar, int64_t pad) {
  int64_t stack = 0;
  bool valid = true, pad_seen = false;
  for (int64_t i = 0; i < L; ++i) {
    const int64_t t = tok_at(pop, tb, b * L + i);
    if (t == pad) {
      pad_seen = true;
      continue;
    }
    if (pad_seen) {
      valid = false;
      break;
    }
    int64_t arity = 0;
    if (t >= 0 && t < n_ar) arity = ar[t];
    stack += 1 - arity;
    if (stack < 1) {
      valid = false;
      break;
    }
  }
  if (valid && stack != 1) valid = false;
  return valid;
}

// The torch formulations (operators.py:551-570 and gpu_simplifier.py:513-579): arities looked up
// with the token clamped into the table, deltas 1 - arity with PAD deltas zeroed, then whole-row
// cumulative sums and reductions.
bool validate_torch_row(const void* pop, int tb, int64_t b, int64_t L, const int32_t* ar,
                        int64_t n_ar, int64_t pad, bool simplifier) {
  std::vector<int64_t> cums(L);
  std::vector<bool> is_pad(L);
  int64_t acc = 0;
  for (int64_t i = 0; i < L; ++i) {
    const int64_t t = tok_at(pop, tb, b * L + i);
    const int64_t c = t < 0 ? 0 : (t > n_ar - 1 ? n_ar - 1 : t);
    int64_t delta = 1 - (int64_t)ar[c];
    is_pad[i] = (t == pad);
    if (is_pad[i]) delta = 0;
    acc += delta;
    cums[i] = acc;
  }
  if (L == 0) return false;  // torch: stack_depth[:, -1] of an empty row does not exist
  if (simplifier) {
    const bool cond_final = cums[L - 1] == 1;
    bool has_tokens = false;
    int64_t mn = cums[0];
    for (int64_t i = 0; i < L; ++i) {
      has_tokens = has_tokens || !is_pad[i];
      mn = cums[i] < mn ? cums[i] : mn;
    }
    return cond_final && has_tokens && mn >= 1;
  }
  const bool final_ok = cums[L - 1] == 1;
  bool no_underflow = true, contiguous = true, pad_before = false;
  for (int64_t i = 0; i < L; ++i) {
    if (!is_pad[i] && cums[i] < 1) no_underflow = false;
    if (!is_pad[i] && pad_before) contiguous = false;
    if (is_pad[i]) pad_before = true;
  }
  return final_ok && no_underflow && contiguous;
}

// find_subtree_ranges_kernel, cuda/rpn_kernels.cu:433-504 (one (row, position) at a time).
int64_t subtree_range_at(const uint8_t* row, int64_t tid, const int32_t* ar, int64_t n_ar,
                         int64_t pad) {
  const int64_t token = row[tid];
  if (token == pad) return -1;
  int64_t arity = 0;
  if (token >= 0 && token < n_ar) arity = ar[token];
  if (arity == 0) return tid;
  int64_t needed = arity;
  for (int64_t j = tid - 1; j >= 0; --j) {
    const int64_t t = row[j];
    if (t == pad) break;
    int64_t a = 0;
    if (t >= 0 && t < n_ar) a = ar[t];
    needed -= 1;
    needed += a;
    if (needed == 0) return j;
  }
  return -1;
}

}  // namespace

extern "C" {

void ws_oracle_validate(const void* pop, int32_t token_bytes, int64_t B, int64_t L,
                        const int32_t* ar, int64_t n_ar, int32_t pad, int32_t mode,
                        uint8_t* out) {
  for (int64_t b = 0; b < B; ++b) {
    bool v;
    if (mode == 0) v = validate_kernel_row(pop, token_bytes, b, L, ar, n_ar, pad);
    else v = validate_torch_row(pop, token_bytes, b, L, ar, n_ar, pad, mode == 2);
    out[b] = v ? 1 : 0;
  }
}

// Starts as the reference kernel writes them; out_len = first PAD position, else L (one of the
// values the reference's racing stores can leave; see ws_oracle_subtree_length_candidates).
void ws_oracle_subtree_ranges(const uint8_t* pop, int64_t B, int64_t L, const int32_t* ar,
                              int64_t n_ar, int32_t pad, int64_t* out, int64_t* out_len) {
  for (int64_t b = 0; b < B; ++b) {
    const uint8_t* row = pop + b * L;
    int64_t first_pad = -1;
    for (int64_t i = 0; i < L; ++i) {
      out[b * L + i] = subtree_range_at(row, i, ar, n_ar, pad);
      if (row[i] == pad && first_pad < 0) first_pad = i;
    }
    if (out_len) out_len[b] = first_pad >= 0 ? first_pad : L;
  }
}

// Every value that the reference kernel's out_lengths stores (rpn_kernels.cu:459-467) may leave
// for row b: cand[b * (L + 1) + v] = 1 for each candidate v in [0, L].
void ws_oracle_subtree_length_candidates(const uint8_t* pop, int64_t B, int64_t L, int32_t pad,
                                         uint8_t* cand) {
  for (int64_t b = 0; b < B; ++b) {
    const uint8_t* row = pop + b * L;
    uint8_t* c = cand + b * (L + 1);
    for (int64_t v = 0; v <= L; ++v) c[v] = 0;
    for (int64_t tid = 0; tid < L; ++tid) {
      if (row[tid] == pad) {
        if (tid == 0 || row[tid - 1] != pad) c[tid] = 1;
      } else if (tid == L - 1) {
        c[L] = 1;
      }
    }
  }
}

// precompute_subtree_starts_kernel, cuda/simplify_kernels.cu:612-661 (MAX_FORMULA_LEN 256,
// PAD_ID_CONST 0).
void ws_oracle_subtree_starts(const int64_t* pop, int64_t B, int64_t L, const int32_t* ar,
                              int64_t max_id, int64_t* out) {
  for (int64_t b = 0; b < B; ++b) {
    const int64_t* row = pop + b * L;
    int64_t* out_row = out + b * L;
    const int64_t actual_L = L < 256 ? L : 256;
    int sub_len[256];
    for (int64_t j = 0; j < actual_L; ++j) {
      const int64_t tok = row[j];
      if (tok == 0 || tok < 0 || tok >= max_id) {
        sub_len[j] = 0;
        out_row[j] = -1;
        continue;
      }
      const int ar_j = ar[tok < max_id - 1 ? tok : max_id - 1];
      if (ar_j == 0) {
        sub_len[j] = 1;
      } else if (ar_j == 1 && j >= 1) {
        sub_len[j] = 1 + sub_len[j - 1];
      } else if (ar_j == 2 && j >= 2) {
        const int right_len = sub_len[j - 1];
        const int64_t left_idx = j - 1 - right_len;
        const int left_len = (left_idx >= 0) ? sub_len[left_idx] : 0;
        sub_len[j] = 1 + right_len + left_len;
      } else {
        sub_len[j] = 1;
      }
      out_row[j] = j - sub_len[j] + 1;
    }
    for (int64_t j = actual_L; j < L; ++j) out_row[j] = -1;
  }
}

// tournament_selection_kernel (cuda/rpn_kernels.cu:1535-1601) when rand_off is NULL, else
// tournament_selection_offsets_kernel (:1603-1668).  Plain IEEE float comparisons; the CUDA
// builds flush subnormals (--use_fast_math), so callers keep values out of the subnormal range.
void ws_oracle_tournament(const float* fitness, int64_t B, const float* errors, int64_t n_data,
                          const int64_t* rand_idx, const int32_t* rand_off, int64_t T,
                          const int32_t* rand_cases, const float* lengths, const float* mad_eps,
                          int32_t island_size, int32_t n_islands, int64_t* selected) {
  for (int64_t idx = 0; idx < B; ++idx) {
    int base = 0, span = (int)B;
    if (rand_off && n_islands > 1) {
      span = std::max(1, island_size);
      base = ((int)idx / span) * span;
      span = std::min(span, (int)B - base);
      span = std::max(1, span);
    }
    auto cand = [&](int64_t k) -> int64_t {
      if (!rand_off) return rand_idx[idx * T + k];
      int64_t c = (int64_t)(base + (rand_off[idx * T + k] % span));
      if (c < 0) c = 0;
      if (c >= B) c = B - 1;
      return c;
    };
    const int case_idx = rand_cases ? rand_cases[idx] : -1;
    int64_t best_idx = cand(0);
    float best_val = (case_idx >= 0 && errors) ? errors[best_idx * n_data + case_idx]
                                               : fitness[best_idx];
    float best_len = lengths ? lengths[best_idx] : 1000000.0f;
    for (int64_t k = 1; k < T; ++k) {
      const int64_t c = cand(k);
      const float val = (case_idx >= 0 && errors) ? errors[c * n_data + case_idx] : fitness[c];
      const float len = lengths ? lengths[c] : 1000000.0f;
      bool improve = false;
      if (val < best_val) {
        improve = true;
      } else if (lengths) {
        const float eps = (case_idx >= 0 && mad_eps) ? mad_eps[case_idx]
                                                     : ((case_idx >= 0) ? 1e-3f : 1e-9f);
        if (std::fabs(val - best_val) < eps && len < best_len) improve = true;
      }
      if (improve) {
        best_val = val;
        best_idx = c;
        best_len = len;
      }
    }
    selected[idx] = best_idx;
  }
}

}  // extern "C"
