// ws_gp.cu -- one genetic-programming generation on the device, for many problems at once.
//
// The reference breeds a generation with a host orchestrator (evolve_generation,
// rpn_kernels.cu:1810-2237): tournament selection (K16), elitism at index 0 (:1905-1907),
// subtree crossover with a length check (K5/K6/K10, :1966-2000), same-arity point mutation
// (K7/K11), constant recombination and perturbation (K12/K13/K15) -- about a dozen launches plus
// torch RNG calls per generation and problem.  Here one child is one thread and the whole
// generation of every problem is three launches (elite argmin, children, copy-back), with a
// counter-based generator (SplitMix64, Steele-Lea-Flood 2014) keyed by (problem seed,
// generation, child), so a problem's offspring do not depend on what else shares the launch and
// the step is graph-capturable (each problem's generation counter lives on the device).
//
// Per child c of a problem with B programs of width L (draws in this order):
//   c == 0 with elitism: the best program (lowest fitness, NaN last, lowest index) unchanged.
//   a = tournament(); child = a.
//   if u < crossover_rate: b = tournament(); e_a = randint(len a), e_b = randint(len b); the
//     subtree of a ending at e_a is replaced by the subtree of b ending at e_b when the child
//     fits in L tokens (and both subtrees are well formed).
//   each child token: if u < mutation_rate, an operator becomes a random operator of the same
//     arity, a variable a random variable; C and literals are kept (constants stay aligned).
//   constants: slot k of the child takes the value of the parent slot its k-th C token came
//     from (slots past the child's C count keep parent a's); then each slot with probability
//     const_mutation_rate is multiplied by (1 + const_sigma * N(0, 1)) (Box-Muller).
// Tournament: `tournament_size` uniform draws, the lowest fitness wins; within parsimony_eps
// the shorter program wins; otherwise the earlier draw.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <string>
#include <vector>

#include "ws_internal.h"

namespace ws {
namespace {

constexpr int kGpMaxList = 64;
constexpr int kGpMaxConsts = 64;

template <typename T>
struct GpDesc {
  uint8_t* pop;
  T* consts;
  const T* fitness;
  int64_t B, child0;
  uint64_t seed;
  int K, n_var, n_un, n_bin;
  uint8_t arity[256];  // 0 leaf, 1 unary, 2 binary, 3 PAD, 4 not an executable token
  uint8_t kind[256];   // 1 variable, 2 C, 3 operator, 4 literal, 0 PAD / unknown
  uint8_t var_ids[kGpMaxList], un_ids[kGpMaxList], bin_ids[kGpMaxList];
};

struct GpParams {
  int L;
  int tournament_size, elitism;
  float crossover_rate, mutation_rate, const_mutation_rate, const_sigma, parsimony_eps;
};

__host__ __device__ __forceinline__ uint64_t sm_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
struct Rng {
  uint64_t s;
  __device__ uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    return sm_mix(s);
  }
  __device__ float uniform() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
  __device__ int randint(int n) { return (int)(((next() >> 32) * (uint64_t)n) >> 32); }
  __device__ double normal() {
    const double u1 = ((double)(next() >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(next() >> 11) * (1.0 / 9007199254740992.0);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};

template <typename T>
__device__ __forceinline__ int prog_len(const GpDesc<T>& d, const uint8_t* row, int L) {
  int n = 0;
  while (n < L && d.arity[row[n]] != 3) ++n;
  return n;
}

// Start of the subtree that ends at e (RPN), or -1 if the tokens before e do not close it.
template <typename T>
__device__ __forceinline__ int subtree_start(const GpDesc<T>& d, const uint8_t* row, int e) {
  int rem = 1;
  for (int j = e; j >= 0; --j) {
    const int a = d.arity[row[j]];
    if (a > 2) return -1;
    rem += a - 1;
    if (rem == 0) return j;
  }
  return -1;
}

template <typename T>
__device__ __forceinline__ float fit_of(const GpDesc<T>& d, int64_t i) {
  const float f = (float)d.fitness[i];
  return f == f ? f : INFINITY;
}

template <typename T>
__device__ int64_t tournament(const GpDesc<T>& d, Rng& r, int size, float eps, int L) {
  int64_t w = r.randint((int)d.B);
  float fw = fit_of(d, w);
  for (int t = 1; t < size; ++t) {
    const int64_t i = r.randint((int)d.B);
    const float f = fit_of(d, i);
    if (fabsf(f - fw) < eps) {
      if (prog_len(d, d.pop + i * L, L) < prog_len(d, d.pop + w * L, L)) { w = i; fw = f; }
    } else if (f < fw) {
      w = i;
      fw = f;
    }
  }
  return w;
}

// Lowest fitness per problem (NaN as +inf, ties to the lowest index): one block per problem.
template <typename T>
__global__ void __launch_bounds__(256) gp_elite_kernel(const GpDesc<T>* __restrict__ desc,
                                                       int64_t* __restrict__ elite) {
  const GpDesc<T>& d = desc[blockIdx.x];
  __shared__ float sv[256];
  __shared__ int64_t si[256];
  float bv = INFINITY;
  int64_t bi = 0x7FFFFFFFFFFFFFFFll;
  for (int64_t i = threadIdx.x; i < d.B; i += blockDim.x) {
    const float f = fit_of(d, i);
    if (f < bv || (f == bv && i < bi)) { bv = f; bi = i; }
  }
  sv[threadIdx.x] = bv;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      const float f = sv[threadIdx.x + o];
      const int64_t i = si[threadIdx.x + o];
      if (f < sv[threadIdx.x] || (f == sv[threadIdx.x] && i < si[threadIdx.x])) {
        sv[threadIdx.x] = f;
        si[threadIdx.x] = i;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) elite[blockIdx.x] = si[0] < d.B ? si[0] : 0;
}

template <typename T>
__device__ __forceinline__ int find_gp_problem(const GpDesc<T>* __restrict__ d, int n, int64_t i) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d[mid].child0 <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One child per thread, written to the scratch generation [sum B, L] / [sum B, Kmax].
template <typename T>
__global__ void __launch_bounds__(128) gp_child_kernel(const GpDesc<T>* __restrict__ desc, int n,
                                                       int64_t total, const int64_t* __restrict__ elite,
                                                       const uint64_t* __restrict__ generation,
                                                       GpParams P, uint8_t* __restrict__ out_pop,
                                                       T* __restrict__ out_consts, int Kmax) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int pi = find_gp_problem(desc, n, g);
  const GpDesc<T>& d = desc[pi];
  const int64_t c = g - d.child0;
  const int L = P.L;
  uint8_t* orow = out_pop + g * (int64_t)L;
  T* oc = out_consts + g * (int64_t)Kmax;
  if (P.elitism && c == 0) {
    const int64_t e = elite[pi];
    for (int j = 0; j < L; ++j) orow[j] = d.pop[e * L + j];
    for (int k = 0; k < d.K; ++k) oc[k] = d.consts[e * d.K + k];
    return;
  }
  Rng r;
  r.s = sm_mix(d.seed + 0x9E3779B97F4A7C15ull * (generation[pi] + 1ull)) ^
        sm_mix((uint64_t)c + 0x632BE59BD9B4E019ull);
  const int64_t a = tournament(d, r, P.tournament_size, P.parsimony_eps, L);
  const uint8_t* ra = d.pop + a * L;
  const int la = prog_len(d, ra, L);
  // child = a[0:sa] + b[sb:eb+1] + a[ea+1:la]; without crossover sa = la (all of a)
  int sa = la, ea = la - 1, sb = 0, eb = -1;
  int64_t b = a;
  if (r.uniform() < P.crossover_rate) {
    b = tournament(d, r, P.tournament_size, P.parsimony_eps, L);
    const uint8_t* rb0 = d.pop + b * L;
    const int lb = prog_len(d, rb0, L);
    if (la > 0 && lb > 0) {
      const int xa = r.randint(la), xb = r.randint(lb);
      const int s1 = subtree_start(d, ra, xa), s2 = subtree_start(d, rb0, xb);
      if (s1 >= 0 && s2 >= 0 && la - (xa - s1 + 1) + (xb - s2 + 1) <= L) {
        sa = s1;
        ea = xa;
        sb = s2;
        eb = xb;
      }
    }
  }
  const uint8_t* rb = d.pop + b * L;
  // assemble in a thread-local row (written out 16 bytes at a time below); the k-th C token of
  // the child takes its constant from (parent, slot)
  uint4 rowbuf[16];  // 256 bytes: the longest program
  uint8_t* crow = reinterpret_cast<uint8_t*>(rowbuf);
  T cval[kGpMaxConsts];
  const int K = d.K;
  int n_out = 0, nc = 0, ca = 0;
  for (int j = 0; j < sa; ++j) {
    const uint8_t t = ra[j];
    if (d.kind[t] == 2) {
      if (nc < K) cval[nc] = d.consts[a * K + (ca < K ? ca : K - 1)];
      ++nc;
      ++ca;
    }
    crow[n_out++] = t;
  }
  if (eb >= sb) {
    int cb = 0;
    for (int j = 0; j < sb; ++j) cb += d.kind[rb[j]] == 2 ? 1 : 0;
    for (int j = sb; j <= eb; ++j) {
      const uint8_t t = rb[j];
      if (d.kind[t] == 2) {
        if (nc < K) cval[nc] = d.consts[b * K + (cb < K ? cb : K - 1)];
        ++nc;
        ++cb;
      }
      crow[n_out++] = t;
    }
    for (int j = sa; j <= ea; ++j) ca += d.kind[ra[j]] == 2 ? 1 : 0;  // skipped part of a
    for (int j = ea + 1; j < la; ++j) {
      const uint8_t t = ra[j];
      if (d.kind[t] == 2) {
        if (nc < K) cval[nc] = d.consts[a * K + (ca < K ? ca : K - 1)];
        ++nc;
        ++ca;
      }
      crow[n_out++] = t;
    }
  }
  for (int j = n_out; j < L; ++j) crow[j] = 0;
  // point mutation: operators within their arity, variables among the variables
  for (int j = 0; j < n_out; ++j) {
    if (r.uniform() < P.mutation_rate) {
      const uint8_t t = crow[j];
      const int kd = d.kind[t], ar = d.arity[t];
      if (kd == 3 && ar == 2 && d.n_bin > 0) crow[j] = d.bin_ids[r.randint(d.n_bin)];
      else if (kd == 3 && ar == 1 && d.n_un > 0) crow[j] = d.un_ids[r.randint(d.n_un)];
      else if (kd == 1 && d.n_var > 0) crow[j] = d.var_ids[r.randint(d.n_var)];
    }
  }
  if (((L & 15) == 0) && ((((uintptr_t)orow) & 15u) == 0)) {
    for (int j = 0; j < L; j += 16) *reinterpret_cast<uint4*>(orow + j) = rowbuf[j >> 4];
  } else {
    for (int j = 0; j < L; ++j) orow[j] = crow[j];
  }
  // constants, then their perturbation
  for (int k = 0; k < K; ++k) {
    T v = k < nc ? cval[k] : d.consts[a * K + k];
    if (r.uniform() < P.const_mutation_rate) v = (T)((double)v * (1.0 + (double)P.const_sigma * r.normal()));
    oc[k] = v;
  }
}

// Next generation back into the problems' own tensors; child 0 of every problem advances its
// problem's counter (the child kernel that read the counters has completed).  Rows are copied
// 16 bytes per load/store when both sides allow it.
template <typename T>
__global__ void __launch_bounds__(128) gp_copyback_kernel(const GpDesc<T>* __restrict__ desc, int n,
                                                          int64_t total, int L, int Kmax,
                                                          const uint8_t* __restrict__ pop_s,
                                                          const T* __restrict__ consts_s,
                                                          uint64_t* __restrict__ generation) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int pi = find_gp_problem(desc, n, g);
  const GpDesc<T>& d = desc[pi];
  const int64_t c = g - d.child0;
  if (c == 0) generation[pi] += 1ull;
  const uint8_t* src = pop_s + g * (int64_t)L;
  uint8_t* dst = d.pop + c * L;
  if (((L & 15) == 0) && ((((uintptr_t)src) | ((uintptr_t)dst)) & 15u) == 0) {
    for (int j = 0; j < L; j += 16)
      *reinterpret_cast<uint4*>(dst + j) = *reinterpret_cast<const uint4*>(src + j);
  } else {
    for (int j = 0; j < L; ++j) dst[j] = src[j];
  }
  for (int k = 0; k < d.K; ++k) d.consts[c * d.K + k] = consts_s[g * (int64_t)Kmax + k];
}

__global__ void gp_set_generation_kernel(uint64_t* generation, int n, uint64_t v) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) generation[i] = v;
}

// Up to kGpUploadChunk descriptors (and starting generations) as one kernel argument, copied
// into the workspace in stream order.
constexpr int kGpUploadChunk = 16;
template <typename T>
struct GpChunk {
  int n, base;
  GpDesc<T> d[kGpUploadChunk];
  uint64_t gen[kGpUploadChunk];
};
template <typename T>
__global__ void __launch_bounds__(128) gp_upload_kernel(const GpChunk<T> c, GpDesc<T>* dst,
                                                        uint64_t* gen_dst) {
  const int nd = c.n * (int)(sizeof(GpDesc<T>) / 4);
  const unsigned* sd = reinterpret_cast<const unsigned*>(c.d);
  unsigned* od = reinterpret_cast<unsigned*>(dst + c.base);
  for (int i = threadIdx.x; i < nd; i += blockDim.x) od[i] = sd[i];
  for (int i = threadIdx.x; i < c.n; i += blockDim.x) gen_dst[c.base + i] = c.gen[i];
}

struct GpLayout {
  size_t desc, elite, gen, pop_s, consts_s, total;
};

GpLayout gp_layout(int n, int64_t total, int64_t L, int Kmax, size_t tsz, size_t desc_sz) {
  GpLayout w;
  size_t off = 0;
  w.desc = off;
  off = align_up(off + (size_t)n * desc_sz, 256);
  w.elite = off;
  off = align_up(off + (size_t)n * sizeof(int64_t), 256);
  w.gen = off;
  off = align_up(off + (size_t)(n > 0 ? n : 1) * sizeof(uint64_t), 256);
  w.pop_s = off;
  off = align_up(off + (size_t)total * L, 256);
  w.consts_s = off;
  off = align_up(off + (size_t)total * (Kmax > 0 ? Kmax : 1) * tsz, 256);
  w.total = off;
  return w;
}

struct GpState {
  int dtype = WS_F32, n = 0, Kmax = 0;
  int64_t L = 0, total = 0;
  GpParams P{};
  GpLayout lay{};
  unsigned char* wsb = nullptr;
};

template <typename T>
ws_status gp_build(GpState& st, const ws_gp_problem* probs, int n,
                   std::vector<GpDesc<T>>& descs) {
  descs.clear();
  int64_t child0 = 0;
  for (int i = 0; i < n; ++i) {
    const ws_gp_problem& q = probs[i];
    GpDesc<T> d;
    std::memset(&d, 0, sizeof(d));
    d.pop = q.population;
    d.consts = static_cast<T*>(q.constants);
    d.fitness = static_cast<const T*>(q.fitness);
    d.B = q.B;
    d.child0 = child0;
    d.seed = q.seed;
    d.K = (int)q.K;
    const TokenLut lut = build_lut(*q.ids, q.num_vars, false);
    for (int t = 0; t < 256; ++t) {
      const int cls = lut.cls[t];
      uint8_t ar = 4, kd = 0;
      if (cls == T_PAD) ar = 3;
      else if (cls == T_VAR) { ar = 0; kd = 1; }
      else if (cls == T_CONST) { ar = 0; kd = 2; }
      else if (cls == T_LIT) { ar = 0; kd = 4; }
      else if (is_binary(cls)) { ar = 2; kd = 3; }
      else if (is_unary(cls)) { ar = 1; kd = 3; }
      d.arity[t] = ar;
      d.kind[t] = kd;
      if (t == 0 && cls != T_PAD) return fail("token 0 must be PAD");
      if (kd == 1 && d.n_var < kGpMaxList) d.var_ids[d.n_var++] = (uint8_t)t;
      if (kd == 3 && ar == 1 && d.n_un < kGpMaxList) d.un_ids[d.n_un++] = (uint8_t)t;
      if (kd == 3 && ar == 2 && d.n_bin < kGpMaxList) d.bin_ids[d.n_bin++] = (uint8_t)t;
    }
    if (q.B > 0) descs.push_back(d);
    child0 += q.B;
  }
  st.total = child0;
  return WS_OK;
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

static ws_status gp_check(int32_t dtype, const ws_gp_problem* problems, int32_t n, int64_t L,
                          int* kmax) {
  if (dtype != WS_F32 && dtype != WS_F64) return fail("fitness and constants must be float32 or float64");
  if (n < 0 || (n > 0 && !problems)) return fail("problem list is null");
  if (L < 1 || L > 256) return fail("program length must be in 1..256");
  int km = 0;
  for (int i = 0; i < n; ++i) {
    const ws_gp_problem& q = problems[i];
    const std::string at = "problem " + std::to_string(i) + ": ";
    if (!q.ids) return fail(at + "token map is required");
    if (q.B < 0 || q.K < 0 || q.num_vars < 0) return fail(at + "negative dimension");
    if (q.B > INT32_MAX) return fail(at + "at most 2^31-1 programs per problem");
    if (q.K > kGpMaxConsts) return fail(at + "at most 64 constants per program");
    if (q.B > 0 && (!q.population || !q.fitness || (q.K > 0 && !q.constants)))
      return fail(at + "null tensor pointer");
    km = (int)q.K > km ? (int)q.K : km;
  }
  *kmax = km;
  return WS_OK;
}

ws_status ws_gp_workspace_bytes(int32_t dtype, const ws_gp_problem* problems, int32_t n_problems,
                                int64_t L, size_t* out_bytes) {
  clear_error();
  if (!out_bytes) return fail("out_bytes is null");
  int km = 0;
  ws_status st = gp_check(dtype, problems, n_problems, L, &km);
  if (st != WS_OK) return st;
  int64_t total = 0;
  for (int i = 0; i < n_problems; ++i) total += problems[i].B;
  const size_t tsz = dtype == WS_F64 ? 8 : 4;
  const size_t dsz = dtype == WS_F64 ? sizeof(GpDesc<double>) : sizeof(GpDesc<float>);
  *out_bytes = gp_layout(n_problems, total, L, km, tsz, dsz).total;
  return WS_OK;
}

ws_status ws_gp_create(int32_t dtype, const ws_gp_problem* problems, int32_t n_problems, int64_t L,
                       const ws_gp_opts* opts, void* workspace, size_t workspace_bytes,
                       void* stream, ws_gp** out) {
  clear_error();
  if (!out || !opts) return fail("options and output handle are required");
  *out = nullptr;
  int km = 0;
  ws_status st = gp_check(dtype, problems, n_problems, L, &km);
  if (st != WS_OK) return st;
  if (opts->tournament_size < 1) return fail("tournament_size must be >= 1");
  GpState* gs = new GpState();
  gs->dtype = dtype;
  gs->L = L;
  gs->Kmax = km;
  gs->P = GpParams{(int)L, opts->tournament_size, opts->elitism ? 1 : 0, opts->crossover_rate,
                   opts->mutation_rate, opts->const_mutation_rate, opts->const_sigma,
                   opts->parsimony_eps};
  gs->wsb = static_cast<unsigned char*>(workspace);
  auto upload = [&](auto tag) -> ws_status {
    using T = decltype(tag);
    std::vector<GpDesc<T>> descs;
    std::vector<uint64_t> gens;  // each problem's starting generation, in descriptor order
    for (int i = 0; i < n_problems; ++i)
      if (problems[i].B > 0) gens.push_back(problems[i].generation);
    ws_status s2 = gp_build<T>(*gs, problems, n_problems, descs);
    if (s2 != WS_OK) return s2;
    gs->n = (int)descs.size();
    gs->lay = gp_layout(n_problems, gs->total, L, km, sizeof(T), sizeof(GpDesc<T>));
    if (!workspace || workspace_bytes < gs->lay.total || ((uintptr_t)workspace & 255u)) {
      set_error("workspace of " + std::to_string(gs->lay.total) +
                " bytes (256-byte aligned) required (got " + std::to_string(workspace_bytes) + ")");
      return WS_ERR_WORKSPACE;
    }
    for (size_t b0 = 0; b0 < descs.size(); b0 += kGpUploadChunk) {
      GpChunk<T> ch;
      std::memset(&ch, 0, sizeof(ch));
      ch.base = (int)b0;
      ch.n = (int)std::min(descs.size() - b0, (size_t)kGpUploadChunk);
      for (int j = 0; j < ch.n; ++j) {
        ch.d[j] = descs[b0 + j];
        ch.gen[j] = gens[b0 + j];
      }
      gp_upload_kernel<T><<<1, 128, 0, (cudaStream_t)stream>>>(
          ch, reinterpret_cast<GpDesc<T>*>(gs->wsb + gs->lay.desc),
          reinterpret_cast<uint64_t*>(gs->wsb + gs->lay.gen));
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return fail_cuda(e, "GP descriptor upload");
    }
    return WS_OK;
  };
  st = dtype == WS_F64 ? upload(double()) : upload(float());
  if (st != WS_OK) {
    delete gs;
    return st;
  }
  *out = reinterpret_cast<ws_gp*>(gs);
  return WS_OK;
}

ws_status ws_gp_step(ws_gp* handle, void* stream) {
  clear_error();
  NvtxRange nvtx("ws_gp_step");
  if (!handle) return fail("handle is null");
  GpState* gs = reinterpret_cast<GpState*>(handle);
  if (gs->total == 0) return WS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  auto run = [&](auto tag) -> ws_status {
    using T = decltype(tag);
    const GpDesc<T>* desc = reinterpret_cast<const GpDesc<T>*>(gs->wsb + gs->lay.desc);
    int64_t* elite = reinterpret_cast<int64_t*>(gs->wsb + gs->lay.elite);
    uint64_t* gen = reinterpret_cast<uint64_t*>(gs->wsb + gs->lay.gen);
    uint8_t* pop_s = gs->wsb + gs->lay.pop_s;
    T* consts_s = reinterpret_cast<T*>(gs->wsb + gs->lay.consts_s);
    const int Kstride = gs->Kmax > 0 ? gs->Kmax : 1;
    gp_elite_kernel<T><<<gs->n, 256, 0, s>>>(desc, elite);
    const unsigned grid = (unsigned)((gs->total + 127) / 128);
    gp_child_kernel<T><<<grid, 128, 0, s>>>(desc, gs->n, gs->total, elite, gen, gs->P, pop_s,
                                            consts_s, Kstride);
    gp_copyback_kernel<T><<<grid, 128, 0, s>>>(desc, gs->n, gs->total, (int)gs->L, Kstride, pop_s,
                                               consts_s, gen);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "GP step launch");
    return WS_OK;
  };
  return gs->dtype == WS_F64 ? run(double()) : run(float());
}

ws_status ws_gp_set_generation(ws_gp* handle, uint64_t generation, void* stream) {
  clear_error();
  if (!handle) return fail("handle is null");
  GpState* gs = reinterpret_cast<GpState*>(handle);
  if (gs->n == 0) return WS_OK;
  gp_set_generation_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(
      reinterpret_cast<uint64_t*>(gs->wsb + gs->lay.gen), gs->n, generation);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "generation write");
}

void ws_gp_destroy(ws_gp* handle) { delete reinterpret_cast<GpState*>(handle); }

}  // extern "C"
