// TEST INFRASTRUCTURE ONLY: CPU restatement of one genetic-programming generation as specified
// in regresionsimbolica-pg_b200/csrc/ws_gp.cu (tournament, elitism, subtree crossover, same-arity
// point mutation, constant inheritance and perturbation), with the same SplitMix64 streams, so
// that the GPU step can be checked child by child.  The reference's own generation
// (evolve_generation, rpn_kernels.cu:1810-2237) draws from torch's generator and is pinned only
// statistically; this file pins the B200 step's stated rules.
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Stream {
  uint64_t s;
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    return mix(s);
  }
  float uniform() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
  int randint(int n) { return (int)(((next() >> 32) * (uint64_t)n) >> 32); }
  double normal() {
    const double u1 = ((double)(next() >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(next() >> 11) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct Tables {
  const uint8_t* arity;  // 0 leaf, 1 unary, 2 binary, 3 PAD, 4 other
  const uint8_t* kind;   // 1 variable, 2 C, 3 operator, 4 literal, 0 other
  const uint8_t *vars, *uns, *bins;
  int n_var, n_un, n_bin;
};

int length_of(const Tables& t, const uint8_t* row, int L) {
  int n = 0;
  while (n < L && t.arity[row[n]] != 3) ++n;
  return n;
}

int start_of(const Tables& t, const uint8_t* row, int e) {
  int open = 1;
  for (int j = e; j >= 0; --j) {
    const int a = t.arity[row[j]];
    if (a > 2) return -1;
    open += a - 1;
    if (open == 0) return j;
  }
  return -1;
}

template <typename T>
float score(const T* fit, int64_t i) {
  const float f = (float)fit[i];
  return std::isnan(f) ? INFINITY : f;
}

template <typename T>
int64_t pick(const Tables& t, const uint8_t* pop, const T* fit, int64_t B, int L, Stream& r,
             int size, float eps) {
  int64_t w = r.randint((int)B);
  float fw = score(fit, w);
  for (int k = 1; k < size; ++k) {
    const int64_t i = r.randint((int)B);
    const float f = score(fit, i);
    if (std::fabs(f - fw) < eps) {
      if (length_of(t, pop + i * L, L) < length_of(t, pop + w * L, L)) {
        w = i;
        fw = f;
      }
    } else if (f < fw) {
      w = i;
      fw = f;
    }
  }
  return w;
}

template <typename T>
void step(const uint8_t* pop, int64_t B, int L, const T* consts, int K, const T* fit,
          const Tables& t, uint64_t seed, uint64_t gen, int tsize, int elitism, float cx,
          float mut, float cmut, float csig, float eps, uint8_t* out_pop, T* out_consts) {
  int64_t elite = 0;
  float best = INFINITY;
  for (int64_t i = 0; i < B; ++i) {
    const float f = score(fit, i);
    if (f < best) {
      best = f;
      elite = i;
    }
  }
  for (int64_t c = 0; c < B; ++c) {
    uint8_t* row = out_pop + c * L;
    T* oc = out_consts + c * K;
    if (elitism && c == 0) {
      for (int j = 0; j < L; ++j) row[j] = pop[elite * L + j];
      for (int k = 0; k < K; ++k) oc[k] = consts[elite * K + k];
      continue;
    }
    Stream r{mix(seed + 0x9E3779B97F4A7C15ull * (gen + 1ull)) ^ mix((uint64_t)c + 0x632BE59BD9B4E019ull)};
    const int64_t a = pick(t, pop, fit, B, L, r, tsize, eps);
    const uint8_t* pa = pop + a * L;
    const int la = length_of(t, pa, L);
    int64_t b = a;
    bool spliced = false;
    int sa = 0, ea = 0, sb = 0, eb = 0;
    if (r.uniform() < cx) {
      b = pick(t, pop, fit, B, L, r, tsize, eps);
      const uint8_t* pb = pop + b * L;
      const int lb = length_of(t, pb, L);
      if (la > 0 && lb > 0) {
        const int xa = r.randint(la), xb = r.randint(lb);
        const int s1 = start_of(t, pa, xa), s2 = start_of(t, pb, xb);
        if (s1 >= 0 && s2 >= 0 && la - (xa - s1 + 1) + (xb - s2 + 1) <= L) {
          spliced = true;
          sa = s1; ea = xa; sb = s2; eb = xb;
        }
      }
    }
    // child tokens with, for each C, the (parent, slot) it came from
    std::vector<uint8_t> child;
    std::vector<T> cv;
    auto slot = [&](int64_t p, int idx) { return consts[p * K + (idx < K ? idx : K - 1)]; };
    const uint8_t* pb = pop + b * L;
    int seen_a = 0;
    auto take_a = [&](int j0, int j1) {
      for (int j = j0; j < j1; ++j) {
        if (t.kind[pa[j]] == 2) cv.push_back(slot(a, seen_a));
        if (t.kind[pa[j]] == 2) ++seen_a;
        child.push_back(pa[j]);
      }
    };
    if (!spliced) {
      take_a(0, la);
    } else {
      take_a(0, sa);
      int seen_b = 0;
      for (int j = 0; j < sb; ++j) seen_b += t.kind[pb[j]] == 2;
      for (int j = sb; j <= eb; ++j) {
        if (t.kind[pb[j]] == 2) cv.push_back(slot(b, seen_b++));
        child.push_back(pb[j]);
      }
      for (int j = sa; j <= ea; ++j) seen_a += t.kind[pa[j]] == 2;
      take_a(ea + 1, la);
    }
    for (size_t j = 0; j < child.size(); ++j) {
      if (r.uniform() < mut) {
        const uint8_t tok = child[j];
        if (t.kind[tok] == 3 && t.arity[tok] == 2 && t.n_bin > 0) child[j] = t.bins[r.randint(t.n_bin)];
        else if (t.kind[tok] == 3 && t.arity[tok] == 1 && t.n_un > 0) child[j] = t.uns[r.randint(t.n_un)];
        else if (t.kind[tok] == 1 && t.n_var > 0) child[j] = t.vars[r.randint(t.n_var)];
      }
    }
    for (int j = 0; j < L; ++j) row[j] = j < (int)child.size() ? child[j] : 0;
    for (int k = 0; k < K; ++k) {
      T v = k < (int)cv.size() ? cv[k] : consts[a * K + k];
      if (r.uniform() < cmut) v = (T)((double)v * (1.0 + (double)csig * r.normal()));
      oc[k] = v;
    }
  }
}

}  // namespace

#define WS_ORACLE_GP(SUF, T)                                                                  \
  extern "C" void ws_oracle_gp_step_##SUF(                                                    \
      const uint8_t* pop, int64_t B, int64_t L, const T* consts, int64_t K, const T* fit,     \
      const uint8_t* arity, const uint8_t* kind, const uint8_t* vars, int n_var,              \
      const uint8_t* uns, int n_un, const uint8_t* bins, int n_bin, uint64_t seed,            \
      uint64_t gen, int tsize, int elitism, float cx, float mut, float cmut, float csig,      \
      float eps, uint8_t* out_pop, T* out_consts) {                                           \
    Tables t{arity, kind, vars, uns, bins, n_var, n_un, n_bin};                               \
    step<T>(pop, B, (int)L, consts, (int)K, fit, t, seed, gen, tsize, elitism, cx, mut, cmut, \
            csig, eps, out_pop, out_consts);                                                  \
  }
WS_ORACLE_GP(f32, float)
WS_ORACLE_GP(f64, double)
