// TEST INFRASTRUCTURE ONLY: CPU restatements of the reference extension's genetic-operator and
// tracker kernels (rpn_kernels.cu:772-813 mutation, :927-1016 splicing; genrand_kernels.cu:70-175
// random programs; best_tracker_kernels.cu:178-231 single-block best update), as checkers.
// The random-program generator divides in IEEE single precision here, where the GPU build
// (fast math) uses an approximate division: streams can part at a category boundary.
#include <algorithm>
#include <cstdint>

extern "C" {

void ws_oracle_mutate(uint8_t* pop, int64_t total, const float* rf, const int64_t* ri,
                      const int32_t* arities, int vocab, const uint8_t* a0, int n0,
                      const uint8_t* a1, int n1, const uint8_t* a2, int n2, float rate, int pad) {
  for (int64_t i = 0; i < total; ++i) {
    const int tok = pop[i];
    if (tok == pad) continue;
    if (rf[i] >= rate) continue;
    int ar = 0;
    if (tok < vocab) ar = arities[tok];
    const uint64_t r = (uint64_t)ri[i];
    int nt = tok;
    if (ar == 0 && n0 > 0) nt = a0[r % n0];
    else if (ar == 1 && n1 > 0) nt = a1[r % n1];
    else if (ar == 2 && n2 > 0) nt = a2[r % n2];
    pop[i] = (uint8_t)nt;
  }
}

static uint8_t piece(const uint8_t* a, const uint8_t* b, int64_t sa, int64_t ea, int64_t sb,
                     int64_t eb, int64_t t, int64_t L, int pad) {
  const int64_t cut = sa + (eb - sb + 1);
  int64_t j;
  const uint8_t* src;
  if (t < sa) { j = t; src = a; }
  else if (t < cut) { j = sb + (t - sa); src = b; }
  else { j = ea + 1 + (t - cut); src = a; }
  return (j >= 0 && j < L) ? src[j] : (uint8_t)pad;
}

void ws_oracle_splice(const uint8_t* p1, const uint8_t* p2, int64_t N, int64_t L,
                      const int64_t* s1, const int64_t* e1, const int64_t* s2, const int64_t* e2,
                      const uint8_t* mask, uint8_t* c1, uint8_t* c2, int pad) {
  for (int64_t n = 0; n < N; ++n)
    for (int64_t t = 0; t < L; ++t) {
      const uint8_t* a = p1 + n * L;
      const uint8_t* b = p2 + n * L;
      if (mask && !mask[n]) {
        c1[n * L + t] = a[t];
        c2[n * L + t] = b[t];
      } else {
        c1[n * L + t] = piece(a, b, s1[n], e1[n], s2[n], e2[n], t, L, pad);
        c2[n * L + t] = piece(b, a, s2[n], e2[n], s1[n], e1[n], t, L, pad);
      }
    }
}

static float xorshift(uint64_t& s) {
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return (float)(s & 0xFFFFFF) / 16777216.0f;
}

void ws_oracle_genrand(uint8_t* pop, int64_t B, int L, const uint8_t* term, int nt,
                       const uint8_t* un, int nu, const uint8_t* bin, int nb, uint64_t seed,
                       float wt, float wu, float wb) {
  for (int64_t b = 0; b < B; ++b) {
    uint64_t s = seed + (uint64_t)b * 6364136223846793005ull + 1442695040888963407ull;
    xorshift(s);
    xorshift(s);
    uint8_t* row = pop + b * L;
    int depth = 0;
    bool done = false;
    for (int j = 0; j < L; ++j) {
      if (done) { row[j] = 0; continue; }
      const int left = L - j - 1;
      bool t_ok = depth + 1 >= 1 && depth + 1 <= 1 + left;
      bool u_ok = nu > 0 && depth >= 1 && depth <= 1 + left;
      bool b_ok = nb > 0 && depth - 1 >= 1 && depth - 1 <= 1 + left;
      if (left == 0) {
        t_ok = t_ok && depth == 0;
        u_ok = u_ok && depth == 1;
        b_ok = b_ok && depth == 2;
      }
      float a = t_ok ? wt : 0.0f, u = u_ok ? wu : 0.0f, c = b_ok ? wb : 0.0f;
      float tot = a + u + c;
      if (tot <= 1e-6f) { a = 1.0f; tot = 1.0f; }
      const float r = xorshift(s);
      const float pa = a / tot, pu = u / tot;
      auto pick = [&](int n) { return std::min((int)(xorshift(s) * n), n - 1); };
      if (r < pa || (r >= pa + pu ? nb == 0 : nu == 0)) { row[j] = term[pick(nt)]; depth += 1; }
      else if (r < pa + pu) { row[j] = un[pick(nu)]; }
      else { row[j] = bin[pick(nb)]; depth -= 1; }
      if (depth == 1 && j > 0) done = true;
    }
    if (depth != 1) {
      row[0] = term[0];
      for (int j = 1; j < L; ++j) row[j] = 0;
    }
  }
}

// best_tracker_kernels.cu:178-231 with 256 threads: per-thread strided first-minimum, then the
// halving tree that keeps the lower thread on ties.
void ws_oracle_batch_best(const uint8_t* pop, int64_t B, int64_t L, const float* consts,
                          int64_t K, const float* fit, uint8_t* brpn, float* bconsts,
                          float* brmse, int32_t* bidx, float tol) {
  float v[256];
  int ix[256];
  for (int t = 0; t < 256; ++t) {
    v[t] = 1e30f;
    ix[t] = -1;
    for (int64_t i = t; i < B; i += 256)
      if (fit[i] < v[t]) { v[t] = fit[i]; ix[t] = (int)i; }
  }
  for (int s = 128; s > 0; s >>= 1)
    for (int t = 0; t < s; ++t)
      if (v[t + s] < v[t]) { v[t] = v[t + s]; ix[t] = ix[t + s]; }
  if (v[0] < brmse[0] - tol && ix[0] >= 0) {
    brmse[0] = v[0];
    bidx[0] = ix[0];
    for (int64_t j = 0; j < L; ++j) brpn[j] = pop[(int64_t)ix[0] * L + j];
    for (int64_t k = 0; k < K; ++k) bconsts[k] = consts[(int64_t)ix[0] * K + k];
  }
}

}  // extern "C"
