// ws_decode.cu -- host-side RPN -> infix decoding (no GPU work).
//
// Replaces `decode_rpn(population, constants, vocab, arities, PAD_ID, precision=4)`
// (bindings.cpp:450 -> decoder.cpp:32-152), which renders the final programs of a fit as text:
// constants are printed with `precision` decimals and trailing zeros removed (integral values
// as integers, decoder.cpp:9-29), operators as fn(a) / (a op b) with the reference's aliases,
// tokens outside the vocabulary as "?", and programs that do not leave exactly one value as
// "Invalid".  The output is written as NUL-terminated strings into one caller buffer.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ws_internal.h"

namespace ws {
namespace {

std::string format_const(double val, int precision) {
  if (std::fabs(val - std::round(val)) < 1e-9) return std::to_string((int64_t)std::round(val));
  int n = std::snprintf(nullptr, 0, "%.*f", precision, val);
  std::string s((size_t)(n > 0 ? n : 0), '\0');
  if (n > 0) std::snprintf(&s[0], (size_t)n + 1, "%.*f", precision, val);
  if (s.find('.') != std::string::npos) {
    s.erase(s.find_last_not_of('0') + 1);
    if (!s.empty() && s.back() == '.') s.pop_back();
  }
  return s.empty() ? "0" : s;
}

std::string unary_text(const std::string& tok, const std::string& a) {
  struct Alias { const char* a; const char* b; const char* fn; };
  static const Alias kAliases[] = {
      {"sin", "s", "sin"},     {"cos", "c", "cos"},       {"log", "l", "log"},
      {"exp", "e", "exp"},     {"sqrt", "q", "sqrt"},     {"abs", "a", "abs"},
      {"floor", "_", "floor"}, {"ceil", nullptr, "ceil"}, {"!", "fact", "fact"},
      {"gamma", nullptr, "gamma"}, {"lgamma", "g", "lgamma"}, {"asin", "S", "asin"},
      {"acos", "C", "acos"},   {"atan", "T", "atan"},     {"neg", nullptr, "neg"},
      {"sign", nullptr, "sign"}};
  for (const Alias& al : kAliases)
    if (tok == al.a || (al.b != nullptr && tok == al.b)) return std::string(al.fn) + "(" + a + ")";
  return tok + "(" + a + ")";
}

std::string binary_text(const std::string& tok, const std::string& a, const std::string& b) {
  const char* sym = nullptr;
  if (tok == "+") sym = "+";
  else if (tok == "-") sym = "-";
  else if (tok == "*") sym = "*";
  else if (tok == "/") sym = "/";
  else if (tok == "pow" || tok == "^") sym = "^";
  else if (tok == "%" || tok == "mod") sym = "%";
  return "(" + a + " " + (sym ? std::string(sym) : tok) + " " + b + ")";
}

std::string decode_one(const uint8_t* row, int64_t L, const void* consts, int dtype, int64_t K,
                       const std::vector<std::string>& vocab, const int32_t* ar, int64_t n_ar,
                       int64_t pad, int precision) {
  std::vector<std::string> stack;
  stack.reserve(64);
  int64_t const_idx = 0;
  for (int64_t j = 0; j < L; ++j) {
    const int64_t id = row[j];
    if (id == pad) break;
    if (id < 0 || id >= (int64_t)vocab.size()) {
      stack.push_back("?");
      continue;
    }
    std::string tok = vocab[(size_t)id];
    const int arity = id < n_ar ? ar[id] : 0;
    if (tok == "C") {
      double v = 0.0;
      if (const_idx < K) {
        v = dtype == WS_F32 ? (double)static_cast<const float*>(consts)[const_idx]
                            : static_cast<const double*>(consts)[const_idx];
        const_idx++;
      }
      stack.push_back(format_const(v, precision));
    } else if (arity > 0) {
      if (arity == 1) {
        if (stack.empty()) return "Invalid";
        std::string a = std::move(stack.back());
        stack.pop_back();
        stack.push_back(unary_text(tok, a));
      } else if (arity == 2) {
        if (stack.size() < 2) return "Invalid";
        std::string b = std::move(stack.back());
        stack.pop_back();
        std::string a = std::move(stack.back());
        stack.pop_back();
        stack.push_back(binary_text(tok, a, b));
      }
      // arities above 2 neither pop nor push (decoder.cpp:88-135)
    } else {
      if (tok == "x") tok = "x0";
      stack.push_back(tok);
    }
  }
  return stack.size() == 1 ? stack.back() : std::string("Invalid");
}

}  // namespace
}  // namespace ws

extern "C" ws_status ws_decode_rpn(const uint8_t* population, int64_t B, int64_t L,
                                   const void* constants, int32_t const_dtype, int64_t K,
                                   const char* const* vocab, int64_t n_vocab,
                                   const int32_t* arities, int64_t n_arities, int32_t pad_id,
                                   int32_t precision, char* out, size_t out_bytes,
                                   int64_t* offsets, size_t* needed_bytes) {
  using namespace ws;
  clear_error();
  if (B < 0 || L < 0 || K < 0 || n_vocab < 0 || n_arities < 0)
    return fail("negative dimension");
  if (const_dtype != WS_F32 && const_dtype != WS_F64)
    return fail("constants must be float32 or float64");
  if ((B > 0 && L > 0 && !population) || (K > 0 && B > 0 && !constants) ||
      (n_vocab > 0 && !vocab) || (n_arities > 0 && !arities) || !offsets)
    return fail("null pointer argument");
  if (precision < 0 || precision > 60) return fail("precision must be within 0..60");
  std::vector<std::string> voc((size_t)n_vocab);
  for (int64_t i = 0; i < n_vocab; ++i) voc[(size_t)i] = vocab[i] ? vocab[i] : "";
  const size_t esz = const_dtype == WS_F32 ? sizeof(float) : sizeof(double);
  size_t total = 0;
  std::vector<std::string> res((size_t)B);
  for (int64_t b = 0; b < B; ++b) {
    res[(size_t)b] = decode_one(population + b * L, L,
                                static_cast<const char*>(constants) + (size_t)(b * K) * esz,
                                const_dtype, K, voc, arities, n_arities, pad_id, precision);
    offsets[b] = (int64_t)total;
    total += res[(size_t)b].size() + 1;
  }
  offsets[B] = (int64_t)total;
  if (needed_bytes) *needed_bytes = total;
  if (!out || out_bytes < total) {
    set_error("decode_rpn needs an output buffer of " + std::to_string(total) + " bytes");
    return WS_ERR_WORKSPACE;
  }
  for (int64_t b = 0; b < B; ++b)
    std::memcpy(out + offsets[b], res[(size_t)b].c_str(), res[(size_t)b].size() + 1);
  return WS_OK;
}
