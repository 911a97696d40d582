// ws_pso.cu -- particle-swarm constant fitting.
//
//   ws_pso_update        velocity / position step        (pso_kernels.cu:29-70)
//   ws_pso_update_bests  personal + swarm bests          (pso_kernels.cu:74-233)
//   ws_fused_pso         whole PSO loop in one launch    (fused_pso_kernels.cu:35-515)
//
// Results are the reference's bit for bit: the update arithmetic is written as the same
// expressions (so the compiler contracts them into the same fused multiply-adds under the same
// flags), the swarm-best tie rules are the reference's, and the fused loop draws the same
// curand XORWOW streams (seed + b * P + p) in the same order.
//
// B200 layout of the fused loop: a particle per lane, instead of one P-thread block per program
// (20-thread blocks leave 12 lanes of every warp idle and cap residency at 32 blocks per SM).
// A swarm owns a block of four or eight warps that split its rows (one warp per row group up to
// 32 particles, two above); row group 0 adds the row errors in row order and runs the swarm's
// update.  The program and its constants live in shared memory; the token dispatch is a table
// lookup instead of a ~40-way comparison chain; each lane carries 16 rows through one pass over
// the program (one decode per token for 16 rows), and the rows' squared errors are added one at
// a time in row order, so every RMSE keeps the reference's bits.
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <cstdint>
#include <string>

#include "ws_internal.h"

namespace ws {
namespace {

// ------------------------------------------------------------------------------------------
// pso_update: V = w V + c1 r1 (pbest - X) + c2 r2 (gbest - X); X += V
template <typename T>
__global__ void __launch_bounds__(256)
    pso_update_kernel(T* __restrict__ pos, T* __restrict__ vel, const T* __restrict__ pbest,
                      const T* __restrict__ gbest, const T* __restrict__ r1,
                      const T* __restrict__ r2, float w, float c1, float c2, int64_t B, int64_t P,
                      int64_t K) {
  const int64_t total = B * P * K;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx % K;
    const int64_t b = (idx / K) / P;
    const T my_pos = pos[idx];
    const T my_vel = vel[idx];
    const T my_pbest = pbest[idx];
    const T my_gbest = gbest[b * K + k];
    const T my_r1 = r1[idx];
    const T my_r2 = r2[idx];
    const T new_vel =
        w * my_vel + c1 * my_r1 * (my_pbest - my_pos) + c2 * my_r2 * (my_gbest - my_pos);
    vel[idx] = new_vel;
    pos[idx] = my_pos + new_vel;
  }
}

// ------------------------------------------------------------------------------------------
// pso_update_bests: one warp per swarm.  Lanes first move improved particles into their
// personal bests (the reference's first kernel), then reduce the personal-best errors with the
// reference's rule (lane-strided strict minimum, then a shuffle-down tree in which a lane takes
// its partner's value only when strictly smaller) and replace the swarm best when strictly
// better (its second kernel).
template <typename T>
__global__ void __launch_bounds__(256)
    pso_bests_kernel(const T* __restrict__ cur_err, T* __restrict__ pb_err,
                     T* __restrict__ pb_pos, const T* __restrict__ cur_pos,
                     T* __restrict__ gb_err, T* __restrict__ gb_pos, int64_t B, int64_t P,
                     int64_t K) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t b = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); b < B;
       b += warps) {
    for (int64_t p = lane; p < P; p += 32) {
      const int64_t i = b * P + p;
      const T curr = cur_err[i];
      if (curr < pb_err[i]) {
        pb_err[i] = curr;
        for (int64_t k = 0; k < K; ++k) pb_pos[i * K + k] = cur_pos[i * K + k];
      }
    }
    __syncwarp();
    T best = (T)1e30;
    int bp = -1;
    for (int64_t p = lane; p < P; p += 32) {
      const T e = pb_err[b * P + p];
      if (e < best) {
        best = e;
        bp = (int)p;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const T oe = __shfl_down_sync(0xffffffffu, best, off);
      const int op = __shfl_down_sync(0xffffffffu, bp, off);
      if (oe < best) {
        best = oe;
        bp = op;
      }
    }
    if (lane == 0 && bp >= 0 && best < gb_err[b]) {
      gb_err[b] = best;
      for (int64_t k = 0; k < K; ++k) gb_pos[b * K + k] = pb_pos[(b * P + bp) * K + k];
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------------------------------
// Fused PSO (float only, as the reference).
constexpr int kPsoMaxL = 256, kPsoMaxK = 16, kPsoMaxD = 1024, kPsoMaxP = 64, kPsoStack = 32;
constexpr float kPsoInf = 1e30f;
constexpr int kPsoRows = 16;  // rows a lane evaluates per program decode

// Token classes of eval_rpn_single's precedence (fused_pso_kernels.cu:81-183): PAD, variables,
// literals 0..6, 10, pi, e, then C, then the binary operators, then the unary operators in the
// order sin cos tan abs neg sqrt log exp floor ceil sign asin acos atan fact gamma lgamma;
// any other token pops one value and pushes 0 (T_UNKNOWN).
struct PsoLut {
  uint8_t cls[256];
  uint8_t arg[256];
};

__device__ __forceinline__ float safe_pow_pso(float a, float b) {
  if (a != a || b != b) return kPsoInf;
  const bool is_int = (floorf(b) == b);
  if (a < 0.0f && !is_int) {
    if (fabsf(b - roundf(b)) < 1e-4f) b = roundf(b);
    else return kPsoInf;
  }
  if (a == 0.0f && b < 0.0f) return kPsoInf;
  const float res = powf(a, b);
  if (res != res || isinf(res)) return kPsoInf;
  if (fabsf(res) > 1e18f) return kPsoInf;
  return res;
}

// R consecutive rows of eval_rpn_single (fused_pso_kernels.cu:57-197) at once; constants are this
// lane's column of the shared [K][G] position table.  The control flow of eval_rpn_single depends
// on the tokens only (pushes, pops, the push-drop at depth 32, stack underflow), so the R rows
// share it; where one row would stop with an error (a domain check, a non-finite result) it is
// flagged instead and its later values are ignored.  One decode of a token serves R rows and the
// stack moves R values per access.  Each row's result is the reference's for that row.
template <int R>
struct __align__(16) PsoV {
  float v[R];
};

template <int R>
__device__ __forceinline__ void pso_eval_rows(const uint8_t* s_prog, int L, const uint8_t* s_cls,
                                              const uint8_t* s_arg, const float* s_lit,
                                              const float* __restrict__ x, int64_t D, int d0,
                                              int nrows, const float* pos, int G, int K,
                                              float (&out)[R]) {
  using PsoV4 = PsoV<R>;
  PsoV4 stack[kPsoStack];
  int sp = 0;
  int c_idx = 0;
  bool bad[R];
#define WS_R4 _Pragma("unroll") for (int r = 0; r < R; ++r)
  WS_R4 bad[r] = false;
  for (int pc = 0; pc < L; ++pc) {
    const int tok = s_prog[pc];
    const int cls = s_cls[tok];
    if (cls == T_PAD) break;
    if (cls == T_VAR || cls == T_LIT || cls == T_CONST) {
      PsoV4 val;
      if (cls == T_VAR) {
        const float* xr = x + (int64_t)s_arg[tok] * D + d0;
        WS_R4 val.v[r] = r < nrows ? __ldg(xr + r) : 0.0f;
      } else {
        float c;
        if (cls == T_LIT) {
          c = s_lit[s_arg[tok]];
        } else {
          const int rr = c_idx < K ? c_idx : K - 1;
          c = rr >= 0 ? pos[rr * G] : 1.0f;
          c_idx++;
        }
        WS_R4 val.v[r] = c;
      }
      if (sp < kPsoStack) stack[sp++] = val;
      continue;
    }
    if (cls >= T_ADD && cls <= T_MOD) {
      if (sp < 2) {
        WS_R4 out[r] = kPsoInf;
        return;
      }
      const PsoV4 b = stack[--sp];
      const PsoV4 a = stack[--sp];
      PsoV4 res;
      switch (cls) {
        case T_ADD: WS_R4 res.v[r] = a.v[r] + b.v[r]; break;
        case T_SUB: WS_R4 res.v[r] = a.v[r] - b.v[r]; break;
        case T_MUL: WS_R4 res.v[r] = a.v[r] * b.v[r]; break;
        case T_DIV:
          WS_R4 {
            if (fabsf(b.v[r]) < 1e-12f) {
              bad[r] = true;
              res.v[r] = 0.0f;
            } else {
              res.v[r] = a.v[r] / b.v[r];
            }
          }
          break;
        case T_POW:
          WS_R4 {
            res.v[r] = safe_pow_pso(a.v[r], b.v[r]);
            if (res.v[r] >= 1e29f) bad[r] = true;
          }
          break;
        default:
          WS_R4 {
            if (fabsf(b.v[r]) < 1e-12f) {
              bad[r] = true;
              res.v[r] = 0.0f;
            } else {
              res.v[r] = fmodf(a.v[r], b.v[r]);
            }
          }
          break;
      }
      stack[sp++] = res;
      continue;
    }
    if (sp < 1) {
      WS_R4 out[r] = kPsoInf;
      return;
    }
    const PsoV4 a = stack[--sp];
    PsoV4 res;
    switch (cls) {
      case T_SIN: WS_R4 res.v[r] = sinf(a.v[r]); break;
      case T_COS: WS_R4 res.v[r] = cosf(a.v[r]); break;
      case T_TAN: WS_R4 res.v[r] = tanf(a.v[r]); break;
      case T_ABS: WS_R4 res.v[r] = fabsf(a.v[r]); break;
      case T_NEG: WS_R4 res.v[r] = -a.v[r]; break;
      case T_SQRT:
        WS_R4 {
          if (a.v[r] < 0.0f) bad[r] = true;
          res.v[r] = a.v[r] < 0.0f ? 0.0f : sqrtf(a.v[r]);
        }
        break;
      case T_LOG:
        WS_R4 {
          if (a.v[r] <= 1e-12f) bad[r] = true;
          res.v[r] = a.v[r] <= 1e-12f ? 0.0f : logf(a.v[r]);
        }
        break;
      case T_EXP:
        WS_R4 {
          if (a.v[r] > 80.0f) {
            bad[r] = true;
            res.v[r] = 0.0f;
          } else if (a.v[r] < -80.0f) {
            res.v[r] = 0.0f;
          } else {
            res.v[r] = expf(a.v[r]);
          }
        }
        break;
      case T_FLOOR: WS_R4 res.v[r] = floorf(a.v[r]); break;
      case T_CEIL: WS_R4 res.v[r] = ceilf(a.v[r]); break;
      case T_SIGN:
        WS_R4 res.v[r] = (a.v[r] > 0.0f) ? 1.0f : ((a.v[r] < 0.0f) ? -1.0f : 0.0f);
        break;
      case T_ASIN:
        WS_R4 {
          const bool out_of = a.v[r] < -1.0f || a.v[r] > 1.0f;
          if (out_of) bad[r] = true;
          res.v[r] = out_of ? 0.0f : asinf(a.v[r]);
        }
        break;
      case T_ACOS:
        WS_R4 {
          const bool out_of = a.v[r] < -1.0f || a.v[r] > 1.0f;
          if (out_of) bad[r] = true;
          res.v[r] = out_of ? 0.0f : acosf(a.v[r]);
        }
        break;
      case T_ATAN: WS_R4 res.v[r] = atanf(a.v[r]); break;
      case T_FACT:
        WS_R4 {
          const float v = a.v[r];
          if ((v <= -1.0f && floorf(v + 1.0f) == (v + 1.0f)) || v > 50.0f) {
            bad[r] = true;
            res.v[r] = 0.0f;
          } else {
            res.v[r] = tgammaf(v + 1.0f);
          }
        }
        break;
      case T_GAMMA:
        WS_R4 {
          const float v = a.v[r];
          if ((v <= 0.0f && floorf(v) == v) || v > 50.0f) {
            bad[r] = true;
            res.v[r] = 0.0f;
          } else {
            res.v[r] = tgammaf(v);
          }
        }
        break;
      case T_LGAMMA:
        WS_R4 {
          const float v = a.v[r];
          if (v <= 0.0f && floorf(v) == v) {
            bad[r] = true;
            res.v[r] = 0.0f;
          } else {
            res.v[r] = lgammaf(v);
          }
        }
        break;
      default: WS_R4 res.v[r] = 0.0f; break;  // tokens without a rule push 0
    }
    WS_R4 if (res.v[r] != res.v[r] || isinf(res.v[r])) bad[r] = true;
    stack[sp++] = res;
  }
  if (sp != 1) {
    WS_R4 out[r] = kPsoInf;
    return;
  }
  WS_R4 {
    const float v = stack[0].v[r];
    out[r] = (bad[r] || v != v || isinf(v)) ? kPsoInf : v;
  }
#undef WS_R4
}

struct FusedPsoArgs {
  const uint8_t* pop;
  const float* init;
  const float* x;
  const float* y;
  float* out_pos;
  float* out_err;
  int64_t B;
  int L, K, P, steps, G;  // G = particles of a row group: 32, or 64 above 32 particles
  int64_t D;
  float w, c1, c2, cmin, cmax;
  uint64_t seed;
  int pad_id, id_C;
};

// Per-swarm shared state: program bytes, the particles' positions [K][G] (constants are read by
// slot), the swarm best, and the per-particle personal-best errors for the swarm reduction.
struct SwarmSmem {
  uint8_t prog[kPsoMaxL];
  float pos[kPsoMaxK * kPsoMaxP];
  float gbest_pos[kPsoMaxK];
  float perr[kPsoMaxP];
  float gbest_err;
  int best_particle;
  int n_active;
};

// Row-split form: one swarm per block of W warps.  The swarm's G = 32 * H particles (H = 1 up
// to 32 particles, 2 up to 64) take H warps, lane l of the h-th being particle 32 h + l; the
// block's W / H such row groups split the rows.  Each step walks the rows in chunks of
// (W / H) * kSplitWarpRows; row group g evaluates rows [g * kSplitWarpRows, (g + 1) *
// kSplitWarpRows) of the chunk for all particles and leaves each row's difference to the target
// in shared memory; row group 0 then adds the chunk's squared differences one row at a time in
// row order (the reference's summation, so every RMSE keeps its bits) and alone holds the curand
// streams, velocities and personal bests.  A particle whose row fails is flagged and no warp
// evaluates its later chunks (its RMSE is the error value whatever the other rows give).
constexpr int kSplitMaxWarps = 8, kSplitWarpRows = 32;

// dynamic shared memory of a W-warp block: the chunk's row differences, [W / H * 32 rows][G]
constexpr size_t split_smem(int W) { return (size_t)W * kSplitWarpRows * 32 * sizeof(float); }

template <int H>
__global__ void __launch_bounds__(kSplitMaxWarps * 32)
    fused_pso_rows_kernel(FusedPsoArgs a, PsoLut lut, float pi_val, float e_val) {
  constexpr int R = kPsoRows;
  constexpr int G = 32 * H;
  __shared__ uint8_t s_cls[256], s_arg[256];
  __shared__ float s_lit[N_LITERALS];
  __shared__ SwarmSmem sw;
  extern __shared__ float s_diff[];  // [chunk rows][G]
  __shared__ int s_bad[G];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    s_cls[t] = lut.cls[t];
    s_arg[t] = lut.arg[t];
  }
  if (threadIdx.x < N_LITERALS) {
    const float lits[N_LITERALS] = {0.f, 1.f, 2.f, 3.f, 4.f, 5.f, 6.f, 10.f, pi_val, e_val};
    s_lit[threadIdx.x] = lits[threadIdx.x];
  }
  const int warp = threadIdx.x >> 5;
  const int grp = warp / H;                           // row group
  const int p = (warp % H) * 32 + (threadIdx.x & 31);  // particle
  const bool lead = grp == 0;                          // row group 0 owns the swarm's state
  const int chunk = (int)(blockDim.x >> 5) / H * kSplitWarpRows;
  const int K = a.K;
  const int D = (int)a.D;
  const bool active = p < a.P;
  float* my_pos = sw.pos + p;  // slot k at my_pos[k * G]

  for (int64_t b = blockIdx.x; b < a.B; b += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < a.L; i += blockDim.x) sw.prog[i] = a.pop[b * a.L + i];
    __syncthreads();
    if (threadIdx.x == 0) {
      int count = 0;
      for (int i = 0; i < a.L; ++i) {
        if (sw.prog[i] == a.pad_id) break;
        if (sw.prog[i] == a.id_C && count < K) count++;
      }
      sw.n_active = count > 0 ? count : 1;
    }
    __syncthreads();
    const int n_active = sw.n_active;

    curandState rng;
    float vel[kPsoMaxK], pbest_pos[kPsoMaxK];
    float pbest_err = kPsoInf;
    if (lead && active) {
      curand_init(a.seed + (uint64_t)b * a.P + p, 0, 0, &rng);
      const float range = (float)(a.cmax - a.cmin);
      const float jitter_sigma = range * 0.15f;
      const float vel_sigma = range * 0.02f;
      const float* init = a.init + b * K;
#pragma unroll
      for (int k = 0; k < kPsoMaxK; ++k) {
        if (k < K) {
          float pk = init[k];
          if (p > 0 && k < n_active) {
            pk += curand_normal(&rng) * jitter_sigma;
            if (pk < a.cmin) pk = a.cmin;
            if (pk > a.cmax) pk = a.cmax;
          }
          vel[k] = curand_normal(&rng) * vel_sigma;
          pbest_pos[k] = pk;
          my_pos[k * G] = pk;
        }
      }
    }
    if (threadIdx.x == 0) {
      sw.gbest_err = kPsoInf;
      for (int k = 0; k < K; ++k) sw.gbest_pos[k] = a.init[b * K + k];
    }

    for (int step = 0; step < a.steps; ++step) {
      if (lead) s_bad[p] = 0;
      __syncthreads();
      // 1. evaluate every particle over every row, a chunk at a time
      float mse_sum = 0.0f;
      for (int c = 0; c < D; c += chunk) {
        const int lo = c + grp * kSplitWarpRows;
        const int hi = lo + kSplitWarpRows < D ? lo + kSplitWarpRows : D;
        if (active && !s_bad[p]) {
          for (int d = lo; d < hi; d += R) {
            const int nr = hi - d < R ? hi - d : R;
            float pr[R];
            pso_eval_rows<R>(sw.prog, a.L, s_cls, s_arg, s_lit, a.x, a.D, d, nr, my_pos, G, K,
                             pr);
            bool bad = false;
#pragma unroll
            for (int r = 0; r < R; ++r) {
              if (r < nr) {
                if (pr[r] >= 1e29f) bad = true;
                s_diff[(d - c + r) * G + p] = pr[r] - a.y[d + r];
              }
            }
            if (bad) {
              s_bad[p] = 1;
              break;
            }
          }
        }
        __syncthreads();
        if (lead && active && !s_bad[p]) {
          const int n = D - c < chunk ? D - c : chunk;
          for (int r = 0; r < n; ++r) {
            const float diff = s_diff[r * G + p];
            mse_sum += diff * diff;
          }
        }
        __syncthreads();
      }
      // 2. personal best
      if (lead && active) {
        const float rmse = s_bad[p] ? kPsoInf : sqrtf(mse_sum / (float)a.D);
        if (rmse < pbest_err) {
          pbest_err = rmse;
#pragma unroll
          for (int k = 0; k < kPsoMaxK; ++k)
            if (k < K) pbest_pos[k] = my_pos[k * G];
        }
        sw.perr[p] = pbest_err;
      }
      __syncthreads();
      // 3. swarm best: serial scan in particle order, strict improvement
      if (threadIdx.x == 0) {
        int bp = -1;
        float be = sw.gbest_err;
        for (int pp = 0; pp < a.P; ++pp)
          if (sw.perr[pp] < be) {
            be = sw.perr[pp];
            bp = pp;
          }
        sw.best_particle = bp;
        if (bp >= 0) sw.gbest_err = be;
      }
      __syncthreads();
      if (lead && active && sw.best_particle == p) {
#pragma unroll
        for (int k = 0; k < kPsoMaxK; ++k)
          if (k < K) sw.gbest_pos[k] = pbest_pos[k];
      }
      __syncthreads();
      // 4. inertia decays linearly from w to 0.4; velocity / position update of active slots
      if (lead && active) {
        const float w_curr =
            a.w - (a.w - 0.4f) * (float)step / (float)(a.steps > 1 ? a.steps - 1 : 1);
#pragma unroll
        for (int k = 0; k < kPsoMaxK; ++k) {
          if (k < n_active) {
            const float r1 = curand_uniform(&rng);
            const float r2 = curand_uniform(&rng);
            float pk = my_pos[k * G];
            vel[k] = w_curr * vel[k] + a.c1 * r1 * (pbest_pos[k] - pk) +
                     a.c2 * r2 * (sw.gbest_pos[k] - pk);
            pk += vel[k];
            if (pk < a.cmin) pk = a.cmin;
            if (pk > a.cmax) pk = a.cmax;
            my_pos[k * G] = pk;
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      a.out_err[b] = sw.gbest_err;
      for (int k = 0; k < K; ++k) a.out_pos[b * K + k] = sw.gbest_pos[k];
    }
  }
}

PsoLut build_pso_lut(const ws_token_map& m, int64_t num_vars) {
  PsoLut lut;
  const int lit_ids[N_LITERALS] = {m.id_0, m.id_1, m.id_2, m.id_3, m.id_4,
                                   m.id_5, m.id_6, m.id_10, m.id_pi, m.id_e};
  const int bin_ids[6] = {m.op_add, m.op_sub, m.op_mul, m.op_div, m.op_pow, m.op_mod};
  const uint8_t bin_cls[6] = {T_ADD, T_SUB, T_MUL, T_DIV, T_POW, T_MOD};
  const int un_ids[17] = {m.op_sin,   m.op_cos,  m.op_tan,  m.op_abs,   m.op_neg,  m.op_sqrt,
                          m.op_log,   m.op_exp,  m.op_floor, m.op_ceil, m.op_sign, m.op_asin,
                          m.op_acos,  m.op_atan, m.op_fact, m.op_gamma, m.op_lgamma};
  const uint8_t un_cls[17] = {T_SIN,   T_COS,  T_TAN,   T_ABS,  T_NEG,  T_SQRT,
                              T_LOG,   T_EXP,  T_FLOOR, T_CEIL, T_SIGN, T_ASIN,
                              T_ACOS,  T_ATAN, T_FACT,  T_GAMMA, T_LGAMMA};
  for (int t = 0; t < 256; ++t) {
    uint8_t cls = T_UNKNOWN, arg = 0;
    bool done = false;
    if (t == m.pad_id) {
      cls = T_PAD;
      done = true;
    } else if ((int64_t)t >= (int64_t)m.id_x_start &&
               (int64_t)t < (int64_t)m.id_x_start + num_vars) {
      cls = T_VAR;
      arg = (uint8_t)(t - m.id_x_start);
      done = true;
    }
    for (int i = 0; i < N_LITERALS && !done; ++i)
      if (t == lit_ids[i]) {
        cls = T_LIT;
        arg = (uint8_t)i;
        done = true;
      }
    if (!done && t == m.id_C) {
      cls = T_CONST;
      done = true;
    }
    for (int i = 0; i < 6 && !done; ++i)
      if (t == bin_ids[i]) {
        cls = bin_cls[i];
        done = true;
      }
    for (int i = 0; i < 17 && !done; ++i)
      if (t == un_ids[i]) {
        cls = un_cls[i];
        done = true;
      }
    lut.cls[t] = cls;
    lut.arg[t] = arg;
  }
  return lut;
}

}  // namespace
}  // namespace ws

extern "C" ws_status ws_pso_update(int32_t dtype, void* pos, void* vel, const void* pbest,
                                   const void* gbest, const void* r1, const void* r2, float w,
                                   float c1, float c2, int64_t B, int64_t P, int64_t K,
                                   void* stream) {
  using namespace ws;
  clear_error();
  if (dtype != WS_F32 && dtype != WS_F64) return fail("pos must be float32 or float64");
  if (B < 0 || P < 0 || K < 0) return fail("negative dimension");
  const int64_t total = B * P * K;
  if (total == 0) return WS_OK;
  if (!pos || !vel || !pbest || !gbest || !r1 || !r2) return fail("null tensor pointer");
  const int64_t want = (total + 255) / 256;
  const int64_t cap = (int64_t)device_info().sm_count * 8;
  const int grid = (int)(want < cap ? want : cap);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == WS_F32)
    pso_update_kernel<float><<<grid, 256, 0, s>>>(
        (float*)pos, (float*)vel, (const float*)pbest, (const float*)gbest, (const float*)r1,
        (const float*)r2, w, c1, c2, B, P, K);
  else
    pso_update_kernel<double><<<grid, 256, 0, s>>>(
        (double*)pos, (double*)vel, (const double*)pbest, (const double*)gbest,
        (const double*)r1, (const double*)r2, w, c1, c2, B, P, K);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "pso_update");
}

extern "C" ws_status ws_pso_update_bests(int32_t dtype, const void* current_err, void* pbest_err,
                                         void* pbest_pos, const void* current_pos,
                                         void* gbest_err, void* gbest_pos, int64_t B, int64_t P,
                                         int64_t K, void* stream) {
  using namespace ws;
  clear_error();
  if (dtype != WS_F32 && dtype != WS_F64) return fail("errors must be float32 or float64");
  if (B < 0 || P < 0 || K < 0) return fail("negative dimension");
  if (B == 0 || P == 0) return WS_OK;
  if (!current_err || !pbest_err || !gbest_err || (K > 0 && (!pbest_pos || !current_pos ||
                                                             !gbest_pos)))
    return fail("null tensor pointer");
  const int64_t want = (B + 7) / 8;  // 8 warps per block, a warp per swarm
  const int64_t cap = (int64_t)device_info().sm_count * 8;
  const int grid = (int)(want < cap ? want : cap);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == WS_F32)
    pso_bests_kernel<float><<<grid, 256, 0, s>>>(
        (const float*)current_err, (float*)pbest_err, (float*)pbest_pos,
        (const float*)current_pos, (float*)gbest_err, (float*)gbest_pos, B, P, K);
  else
    pso_bests_kernel<double><<<grid, 256, 0, s>>>(
        (const double*)current_err, (double*)pbest_err, (double*)pbest_pos,
        (const double*)current_pos, (double*)gbest_err, (double*)gbest_pos, B, P, K);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "pso_update_bests");
}

extern "C" ws_status ws_fused_pso(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                                  const void* init_consts, int64_t K, const void* x,
                                  int64_t num_vars, int64_t D, const void* y_target,
                                  void* out_gbest_pos, void* out_gbest_err,
                                  int32_t num_particles, int32_t num_steps, float w, float c1,
                                  float c2, float const_min, float const_max,
                                  const ws_token_map* ids, uint64_t rng_seed, void* stream) {
  using namespace ws;
  clear_error();
  NvtxRange nvtx("ws_fused_pso");
  if (!ids) return fail("token map is required");
  // launch_fused_pso's checks, in its order (fused_pso_kernels.cu:466-476)
  if (L > kPsoMaxL) return fail("Formula length exceeds PSO_MAX_L");
  if (K > kPsoMaxK) return fail("Constants exceed PSO_MAX_K");
  if (D > kPsoMaxD) return fail("Data samples exceed PSO_MAX_D");
  if (num_particles > kPsoMaxP) return fail("Particles exceed PSO_MAX_PARTICLES");
  if (dtype != WS_F32)
    return fail("fused_pso currently supports float32 only; use the multi-kernel fallback for "
                "float64");
  if (B < 0 || L < 0 || K < 0 || D < 0 || num_vars < 0 || num_steps < 0)
    return fail("negative dimension");
  if (num_particles < 1) return fail("num_particles must be at least 1");
  if (num_vars > 255) return fail("at most 255 variables are addressable by uint8 tokens");
  if (B == 0) return WS_OK;
  if (!population || (K > 0 && !init_consts) || (num_vars > 0 && D > 0 && !x) ||
      (D > 0 && !y_target) || (K > 0 && !out_gbest_pos) || !out_gbest_err)
    return fail("null tensor pointer");
  FusedPsoArgs a;
  a.pop = population;
  a.init = static_cast<const float*>(init_consts);
  a.x = static_cast<const float*>(x);
  a.y = static_cast<const float*>(y_target);
  a.out_pos = static_cast<float*>(out_gbest_pos);
  a.out_err = static_cast<float*>(out_gbest_err);
  a.B = B;
  a.L = (int)L;
  a.K = (int)K;
  a.P = num_particles;
  a.steps = num_steps;
  a.G = num_particles > 32 ? 64 : 32;
  a.D = D;
  a.w = w;
  a.c1 = c1;
  a.c2 = c2;
  a.cmin = const_min;
  a.cmax = const_max;
  a.seed = rng_seed;
  a.pad_id = ids->pad_id;
  a.id_C = ids->id_C;
  const PsoLut lut = build_pso_lut(*ids, num_vars);
  const int sms = device_info().sm_count;
  // Row-split form, a block per swarm: the block scheduler hands the next swarm to whichever
  // SM frees a slot first, which balances programs of different lengths (a persistent grid
  // striding over the swarms left the SMs idle half of the time on 1,024 swarms).  Eight warps
  // per swarm, four beyond seven waves of 8-warp blocks, where row group 0's serial row sum and
  // the barriers weigh more than the spread (measured on B200 with 20-32 particles and
  // 100-1,024 rows: 100-2,048 swarms favour eight, 4,000 and 8,192 four).  Above 32 particles a
  // row group is two warps.
  const bool two = a.G == 64;
  int per_sm8 = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm8, two ? fused_pso_rows_kernel<2> : fused_pso_rows_kernel<1>, 8 * 32,
      split_smem(8));
  if (e != cudaSuccess) return fail_cuda(e, "fused_pso");
  const int64_t cap8 = (int64_t)sms * (per_sm8 > 0 ? per_sm8 : 1);
  const int W = B > 7 * cap8 ? 4 : 8;
  const int grid = (int)(B < 0x7fffffff ? B : 0x7fffffff);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (two)
    fused_pso_rows_kernel<2><<<grid, W * 32, split_smem(W), st>>>(a, lut, (float)ids->pi_val,
                                                                 (float)ids->e_val);
  else
    fused_pso_rows_kernel<1><<<grid, W * 32, split_smem(W), st>>>(a, lut, (float)ids->pi_val,
                                                                 (float)ids->e_val);
  e = cudaGetLastError();
  return e == cudaSuccess ? WS_OK : fail_cuda(e, "fused_pso");
}
