// ws_lbfgs_batch.cu -- per-program L-BFGS over the adjoint gradient, for populations of any size.
//
// The reference fits constants at scale with torch.optim.LBFGS (strong-Wolfe line search) over
// RPNBackwardFunction (optimization.py:281-343): one joint problem whose loss is the sum of every
// program's mean squared error, with [B, D] predictions, stack depths and errors written to HBM
// by the classic evaluator and re-read by torch.  Here every program runs its own L-BFGS with
// the algorithm of torch.optim.LBFGS.step and its _strong_wolfe / _cubic_interpolate line search
// (torch/optim/lbfgs.py; Nocedal & Wright, Numerical Optimization, algorithms 3.5, 3.6 and 7.4),
// restated as a resumable state machine, one thread per program:
//
//   round:  loss_grad launch (ws_backward.cu, loss mode: loss and adjoint gradient of every
//           active program at its trial constants, no per-row tensors)
//        -> state launch (consume the evaluation, advance the line search / iteration, emit the
//           next trial constants or finish the program).
//
// For one program the sequence of trial points is the one torch.optim.LBFGS produces with the
// same loss and gradients (the reference's closure clamps gradients to [-1e4, 1e4]; so does
// `grad_clip`).  Differences: dot products, norms and the two-loop recursion run in FP64 (torch
// uses the parameter dtype); a non-finite loss or gradient at a trial point counts as an infinite
// loss, and an interpolation that meets one returns the bracket midpoint (torch propagates NaN);
// a program whose initial loss is not finite is left as it is.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "ws_internal.h"

namespace ws {
namespace {

constexpr int kLbbMaxK = 32;
constexpr int kLbbMaxHistory = 32;
constexpr double kC1 = 1e-4, kC2 = 0.9, kLsTolChange = 1e-9;  // _strong_wolfe defaults

enum : int32_t { PH_INIT = 0, PH_BRACKET = 1, PH_ZOOM = 2, PH_DONE = 3 };

struct LbState {
  double f, prev_loss, t, gtd, d_norm;
  double t_prev, f_prev, gtd_prev;
  double h_diag;
  double bt[2], bf[2], bgtd[2];
  int32_t phase, n_iter, evals, ls_iter, ls_evals, num_old, head, low, insuf, done_ls, nb, pad;
};

// Vectors of one program, K values each: x (current constants), d (direction), g (gradient at x),
// prev_g (gradient at the previous iterate), g_prev (line search: gradient at t_prev), bg0 / bg1
// (gradients at the bracket ends), then `history` curvature differences y and `history` steps s.
enum : int { V_X = 0, V_D, V_G, V_PREVG, V_GPREV, V_BG0, V_BG1, V_HIST };

template <typename T>
struct LbbArgs {
  int64_t B, K, D, n_splits;
  int m;  // history
  int max_iter, max_eval, max_ls;
  double lr, tol_grad, tol_change, clip;
  LbState* st;
  double* ro;       // [B, m]
  T* vec;           // [B, V_HIST + 2m, K]
  T* trial;         // [B, K] constants evaluated next
  int32_t* active;  // [B]
  int32_t* count;   // active programs after this launch
  const double* part_loss;
  const double* part_grad;
  T* consts;        // caller's constants (read at init, written at finish)
  double* out_loss;
  int32_t* out_evals;
};

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

// _cubic_interpolate: minimiser of the cubic through (x1, f1, g1), (x2, f2, g2), clamped to the
// bounds; the bounds' midpoint when the cubic has no real minimiser (or an input is not finite).
__device__ double cubic_interpolate(double x1, double f1, double g1, double x2, double f2,
                                    double g2, bool has_bounds, double lo, double hi) {
  double xmin_b, xmax_b;
  if (has_bounds) {
    xmin_b = lo;
    xmax_b = hi;
  } else if (x1 <= x2) {
    xmin_b = x1;
    xmax_b = x2;
  } else {
    xmin_b = x2;
    xmax_b = x1;
  }
  if (!(finite_d(f1) && finite_d(f2) && finite_d(g1) && finite_d(g2)))
    return (xmin_b + xmax_b) / 2.0;
  const double d1 = g1 + g2 - 3.0 * (f1 - f2) / (x1 - x2);
  const double d2_square = d1 * d1 - g1 * g2;
  if (d2_square >= 0.0) {
    const double d2 = sqrt(d2_square);
    double min_pos;
    if (x1 <= x2) min_pos = x2 - (x2 - x1) * ((g2 + d2 - d1) / (g2 - g1 + 2.0 * d2));
    else min_pos = x1 - (x1 - x2) * ((g1 + d2 - d1) / (g1 - g2 + 2.0 * d2));
    if (!finite_d(min_pos)) return (xmin_b + xmax_b) / 2.0;
    return fmin(fmax(min_pos, xmin_b), xmax_b);
  }
  return (xmin_b + xmax_b) / 2.0;
}

template <typename T>
__device__ __forceinline__ double dot(const T* a, const T* b, int K) {
  double s = 0.0;
  for (int k = 0; k < K; ++k) s += (double)a[k] * (double)b[k];
  return s;
}
template <typename T>
__device__ __forceinline__ double max_abs(const T* a, int K) {
  double s = 0.0;
  for (int k = 0; k < K; ++k) s = fmax(s, fabs((double)a[k]));
  return s;
}
template <typename T>
__device__ __forceinline__ void copy(T* dst, const T* src, int K) {
  for (int k = 0; k < K; ++k) dst[k] = src[k];
}

template <typename T>
__global__ void __launch_bounds__(128) lbfgs_state_kernel(LbbArgs<T> a, int mode) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool act = false;
  if (b < a.B) {
    const int K = (int)a.K, m = a.m;
    LbState s = a.st[b];
    T* V = a.vec + b * (int64_t)(V_HIST + 2 * m) * K;
    T* x = V + V_X * K;
    T* dv = V + V_D * K;
    T* g = V + V_G * K;
    T* prev_g = V + V_PREVG * K;
    T* g_prev = V + V_GPREV * K;
    T* bg[2] = {V + V_BG0 * K, V + V_BG1 * K};
    T* dirs = V + V_HIST * K;
    T* stps = dirs + (int64_t)m * K;
    double* ro = a.ro + b * m;
    T* trial = a.trial + b * K;

    if (mode == 0) {  // start: evaluate at the caller's constants
      for (int k = 0; k < K; ++k) x[k] = a.consts[b * K + k];
      copy(trial, x, K);
      s = LbState{};
      s.phase = PH_INIT;
      act = true;
    } else if (mode == 2) {  // finish: write back
      for (int k = 0; k < K; ++k) a.consts[b * K + k] = x[k];
      if (a.out_loss) a.out_loss[b] = s.f;
      if (a.out_evals) a.out_evals[b] = s.evals;
    } else if (s.phase != PH_DONE) {
      // ---- consume the evaluation at `trial` -------------------------------------------------
      T gn[kLbbMaxK];
      double f_new = 0.0;
      for (int64_t q = 0; q < a.n_splits; ++q) f_new += a.part_loss[b * a.n_splits + q];
      f_new /= (double)a.D;
      bool ok = finite_d(f_new);
      for (int k = 0; k < K; ++k) {
        double gs = 0.0;
        for (int64_t q = 0; q < a.n_splits; ++q) gs += a.part_grad[(b * a.n_splits + q) * K + k];
        T gk = (T)gs;
        if (a.clip > 0.0) gk = (T)fmin(fmax((double)gk, -a.clip), a.clip);
        ok = ok && finite_d((double)gk);
        gn[k] = gk;
      }
      if (!ok) {
        f_new = __longlong_as_double(0x7ff0000000000000ll);
        for (int k = 0; k < K; ++k) gn[k] = (T)0;
      }
      const double gtd_new = dot(gn, dv, K);

      // stage: 0 start a new iteration, 1 bracketing checks, 2 zoom loop, 3 line search done,
      // 4 emit, 5 finished
      int stage = 5;
      if (s.phase == PH_INIT) {
        s.f = f_new;
        copy(g, gn, K);
        s.evals = 1;
        if (!ok || max_abs(g, K) <= a.tol_grad) stage = 5;
        else stage = 0;
      } else if (s.phase == PH_BRACKET) {
        s.ls_evals += 1;
        s.ls_iter += 1;
        if (s.ls_iter >= a.max_ls) {  // bracketing ran out: bracket [0, t]
          s.nb = 2;
          s.bt[0] = 0.0; s.bf[0] = s.f; copy(bg[0], g, K);
          s.bt[1] = s.t; s.bf[1] = f_new; copy(bg[1], gn, K);
          s.low = s.bf[0] <= s.bf[1] ? 0 : 1;
          stage = 3;
        } else {
          // torch's order: sufficient decrease fails (or no progress) -> bracket; strong Wolfe
          // holds -> done; slope turned non-negative -> bracket; else extrapolate
          const bool armijo_fails =
              f_new > s.f + kC1 * s.t * s.gtd || (s.ls_iter > 1 && f_new >= s.f_prev);
          const bool wolfe = !armijo_fails && fabs(gtd_new) <= -kC2 * s.gtd;
          const bool bracket = armijo_fails || (!wolfe && gtd_new >= 0.0);
          if (bracket) {
            s.nb = 2;
            s.bt[0] = s.t_prev; s.bf[0] = s.f_prev; copy(bg[0], g_prev, K);
            s.bgtd[0] = s.gtd_prev;
            s.bt[1] = s.t; s.bf[1] = f_new; copy(bg[1], gn, K); s.bgtd[1] = gtd_new;
            s.low = s.bf[0] <= s.bf[1] ? 0 : 1;
            s.insuf = 0;
            stage = 2;
          } else if (wolfe) {
            s.nb = 1;
            s.bt[0] = s.t; s.bf[0] = f_new; copy(bg[0], gn, K);
            s.low = 0;
            s.done_ls = 1;
            stage = 3;
          }
        }
        if (stage == 5 && s.phase == PH_BRACKET) {  // extrapolate
          const double min_step = s.t + 0.01 * (s.t - s.t_prev);
          const double max_step = s.t * 10.0;
          const double tmp = s.t;
          s.t = cubic_interpolate(s.t_prev, s.f_prev, s.gtd_prev, s.t, f_new, gtd_new, true,
                                  min_step, max_step);
          s.t_prev = tmp;
          s.f_prev = f_new;
          copy(g_prev, gn, K);
          s.gtd_prev = gtd_new;
          stage = 4;
        }
      } else {  // PH_ZOOM: the evaluation at the zoom trial s.t
        s.ls_evals += 1;
        s.ls_iter += 1;
        const int lo = s.low, hi = 1 - s.low;
        if (f_new > s.f + kC1 * s.t * s.gtd || f_new >= s.bf[lo]) {
          s.bt[hi] = s.t; s.bf[hi] = f_new; copy(bg[hi], gn, K); s.bgtd[hi] = gtd_new;
          s.low = s.bf[0] <= s.bf[1] ? 0 : 1;
        } else {
          if (fabs(gtd_new) <= -kC2 * s.gtd) {
            s.done_ls = 1;
          } else if (gtd_new * (s.bt[hi] - s.bt[lo]) >= 0.0) {
            s.bt[hi] = s.bt[lo]; s.bf[hi] = s.bf[lo]; copy(bg[hi], bg[lo], K);
            s.bgtd[hi] = s.bgtd[lo];
          }
          s.bt[lo] = s.t; s.bf[lo] = f_new; copy(bg[lo], gn, K); s.bgtd[lo] = gtd_new;
        }
        stage = 2;
      }

      // ---- advance until an evaluation is needed or the program is finished ------------------
      for (int guard = 0; guard < 4 && stage != 4 && stage != 5; ++guard) {
        if (stage == 2) {  // zoom loop head
          if (s.done_ls || s.ls_iter >= a.max_ls ||
              fabs(s.bt[1] - s.bt[0]) * s.d_norm < kLsTolChange) {
            stage = 3;
            continue;
          }
          double t = cubic_interpolate(s.bt[0], s.bf[0], s.bgtd[0], s.bt[1], s.bf[1], s.bgtd[1],
                                       false, 0.0, 0.0);
          const double bmax = fmax(s.bt[0], s.bt[1]), bmin = fmin(s.bt[0], s.bt[1]);
          const double eps = 0.1 * (bmax - bmin);
          if (fmin(bmax - t, t - bmin) < eps) {
            if (s.insuf || t >= bmax || t <= bmin) {
              t = fabs(t - bmax) < fabs(t - bmin) ? bmax - eps : bmin + eps;
              s.insuf = 0;
            } else {
              s.insuf = 1;
            }
          } else {
            s.insuf = 0;
          }
          s.t = t;
          s.phase = PH_ZOOM;
          stage = 4;
        } else if (stage == 3) {  // line search result: step to the bracket's low end
          const int lo = s.low;
          const double t = s.bt[lo];
          const double f_ls = s.bf[lo];
          copy(g, bg[lo], K);
          for (int k = 0; k < K; ++k) x[k] = fma((T)t, dv[k], x[k]);
          s.t = t;
          s.f = f_ls;
          s.evals += s.ls_evals;
          double step_max = 0.0;
          for (int k = 0; k < K; ++k) step_max = fmax(step_max, fabs((double)dv[k] * t));
          if (s.n_iter >= a.max_iter || s.evals >= a.max_eval || max_abs(g, K) <= a.tol_grad ||
              step_max <= a.tol_change || fabs(s.f - s.prev_loss) < a.tol_change)
            stage = 5;
          else
            stage = 0;
        } else if (stage == 0) {  // new iteration: direction, initial step, line search start
          s.n_iter += 1;
          if (s.n_iter == 1) {
            for (int k = 0; k < K; ++k) dv[k] = -g[k];
            s.num_old = 0;
            s.head = 0;
            s.h_diag = 1.0;
          } else {
            // curvature pair from the last step: y = g - prev_g, s = d * t
            T yv[kLbbMaxK], sv[kLbbMaxK];
            for (int k = 0; k < K; ++k) {
              yv[k] = g[k] - prev_g[k];
              sv[k] = dv[k] * (T)s.t;
            }
            const double ys = dot(yv, sv, K);
            if (ys > 1e-10) {
              int slot;
              if (s.num_old == m) {
                slot = s.head;
                s.head = (s.head + 1) % m;
              } else {
                slot = (s.head + s.num_old) % m;
                s.num_old += 1;
              }
              copy(dirs + (int64_t)slot * K, yv, K);
              copy(stps + (int64_t)slot * K, sv, K);
              ro[slot] = 1.0 / ys;
              s.h_diag = ys / dot(yv, yv, K);
            }
            // two-loop recursion in FP64
            double q[kLbbMaxK], al[kLbbMaxHistory];
            for (int k = 0; k < K; ++k) q[k] = -(double)g[k];
            for (int i = s.num_old - 1; i >= 0; --i) {
              const int j = (s.head + i) % m;
              const T* sj = stps + (int64_t)j * K;
              const T* yj = dirs + (int64_t)j * K;
              double sq = 0.0;
              for (int k = 0; k < K; ++k) sq += (double)sj[k] * q[k];
              al[i] = sq * ro[j];
              for (int k = 0; k < K; ++k) q[k] -= al[i] * (double)yj[k];
            }
            for (int k = 0; k < K; ++k) q[k] *= s.h_diag;
            for (int i = 0; i < s.num_old; ++i) {
              const int j = (s.head + i) % m;
              const T* sj = stps + (int64_t)j * K;
              const T* yj = dirs + (int64_t)j * K;
              double yr = 0.0;
              for (int k = 0; k < K; ++k) yr += (double)yj[k] * q[k];
              const double be = yr * ro[j];
              for (int k = 0; k < K; ++k) q[k] += (al[i] - be) * (double)sj[k];
            }
            for (int k = 0; k < K; ++k) dv[k] = (T)q[k];
          }
          copy(prev_g, g, K);
          s.prev_loss = s.f;
          if (s.n_iter == 1) {
            double gsum = 0.0;
            for (int k = 0; k < K; ++k) gsum += fabs((double)g[k]);
            s.t = fmin(1.0, 1.0 / gsum) * a.lr;
          } else {
            s.t = a.lr;
          }
          s.gtd = dot(g, dv, K);
          if (!(s.gtd <= -a.tol_change)) {
            stage = 5;
            continue;
          }
          s.d_norm = max_abs(dv, K);
          copy(g_prev, g, K);
          s.t_prev = 0.0;
          s.f_prev = s.f;
          s.gtd_prev = s.gtd;
          s.ls_iter = -1;
          s.ls_evals = 0;
          s.done_ls = 0;
          s.nb = 0;
          s.phase = PH_BRACKET;
          stage = 4;
        }
      }
      if (stage == 4) {
        for (int k = 0; k < K; ++k) trial[k] = fma((T)s.t, dv[k], x[k]);
        act = true;
      } else {
        s.phase = PH_DONE;
      }
    }
    if (mode != 2) {
      a.st[b] = s;
      a.active[b] = act ? 1 : 0;
    }
  }
  const unsigned ballot = __ballot_sync(0xffffffffu, act);
  if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(a.count, __popc(ballot));
}

struct LbbLayout {
  size_t state, ro, vec, trial, active, count, part_loss, part_grad, buckets, total;
};

size_t al256(size_t v) { return (v + 255) / 256 * 256; }

LbbLayout lbb_layout(int64_t B, int64_t K, int m, int64_t n_splits, size_t tsize) {
  LbbLayout l;
  size_t o = 0;
  l.state = o; o = al256(o + (size_t)B * sizeof(LbState));
  l.ro = o; o = al256(o + (size_t)B * m * sizeof(double));
  l.vec = o; o = al256(o + (size_t)B * (V_HIST + 2 * m) * K * tsize);
  l.trial = o; o = al256(o + (size_t)B * K * tsize);
  l.active = o; o = al256(o + (size_t)B * sizeof(int32_t));
  l.count = o; o = al256(o + 16);
  l.part_loss = o; o = al256(o + (size_t)B * n_splits * sizeof(double));
  l.part_grad = o; o = al256(o + (size_t)B * n_splits * K * sizeof(double));
  l.buckets = o; o = al256(o + loss_grad_bucket_bytes(B));
  l.total = o;
  return l;
}

template <typename T>
ws_status lbfgs_batch_typed(const uint8_t* pop, int64_t B, int64_t L, const void* x,
                            int64_t num_vars, int64_t D, void* consts, int64_t K, const void* y,
                            const ws_lbfgs_opts& o, double* out_loss, int32_t* out_evals,
                            const ws_token_map& ids, void* workspace, size_t workspace_bytes,
                            cudaStream_t stream) {
  int64_t n_splits = 1;
  ws_status st = launch_loss_grad<T>(nullptr, B, L, nullptr, D, nullptr, K, nullptr, nullptr,
                                     ids, num_vars, nullptr, nullptr, nullptr, nullptr, nullptr,
                                     &n_splits, nullptr);
  if (st != WS_OK) return st;
  const LbbLayout lay = lbb_layout(B, K, o.history, n_splits, sizeof(T));
  if (workspace_bytes < lay.total) return fail("lbfgs workspace too small");
  unsigned char* w = static_cast<unsigned char*>(workspace);
  LbbArgs<T> a;
  a.B = B;
  a.K = K;
  a.D = D;
  a.n_splits = n_splits;
  a.m = o.history;
  a.max_iter = o.max_iter;
  a.max_eval = o.max_eval;
  a.max_ls = o.max_ls;
  a.lr = o.lr;
  a.tol_grad = o.tolerance_grad;
  a.tol_change = o.tolerance_change;
  a.clip = o.grad_clip;
  a.st = reinterpret_cast<LbState*>(w + lay.state);
  a.ro = reinterpret_cast<double*>(w + lay.ro);
  a.vec = reinterpret_cast<T*>(w + lay.vec);
  a.trial = reinterpret_cast<T*>(w + lay.trial);
  a.active = reinterpret_cast<int32_t*>(w + lay.active);
  a.count = reinterpret_cast<int32_t*>(w + lay.count);
  a.part_loss = reinterpret_cast<double*>(w + lay.part_loss);
  a.part_grad = reinterpret_cast<double*>(w + lay.part_grad);
  a.consts = static_cast<T*>(consts);
  a.out_loss = out_loss;
  a.out_evals = out_evals;
  double* part_loss = reinterpret_cast<double*>(w + lay.part_loss);
  double* part_grad = reinterpret_cast<double*>(w + lay.part_grad);
  const unsigned blocks = (unsigned)((B + 127) / 128);

  auto state = [&](int mode) -> ws_status {
    cudaError_t e = cudaMemsetAsync(a.count, 0, sizeof(int32_t), stream);
    if (e != cudaSuccess) return fail_cuda(e, "lbfgs");
    lbfgs_state_kernel<T><<<blocks, 128, 0, stream>>>(a, mode);
    e = cudaGetLastError();
    return e == cudaSuccess ? WS_OK : fail_cuda(e, "lbfgs");
  };
  // every program evaluates at most (max_eval - 1) + (max_ls + 1) times, and at most
  // 1 + max_iter * (max_ls + 1) times
  int64_t rounds = 1 + (int64_t)o.max_iter * (o.max_ls + 1);
  const int64_t by_eval = (int64_t)o.max_eval + o.max_ls;
  if (by_eval < rounds) rounds = by_eval;
  if ((st = state(0)) != WS_OK) return st;
  for (int64_t r = 0; r < rounds; ++r) {
    st = launch_loss_grad<T>(pop, B, L, x, D, a.trial, K, y, a.active, ids, num_vars, part_loss,
                             part_grad, nullptr, nullptr,
                             reinterpret_cast<int32_t*>(w + lay.buckets), nullptr, stream);
    if (st != WS_OK) return st;
    if ((st = state(1)) != WS_OK) return st;
    if (o.sync_every > 0 && (r + 1) % o.sync_every == 0) {
      int32_t n_active = 0;
      cudaError_t e = cudaMemcpyAsync(&n_active, a.count, sizeof(int32_t),
                                      cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) return fail_cuda(e, "lbfgs");
      if (n_active == 0) break;
    }
  }
  return state(2);
}

}  // namespace
}  // namespace ws

extern "C" ws_status ws_lbfgs_adjoint_workspace_bytes(int32_t dtype, int64_t B, int64_t L,
                                                      int64_t num_vars, int64_t D, int64_t K,
                                                      int32_t history, size_t* bytes) {
  using namespace ws;
  clear_error();
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (!bytes) return fail("null output pointer");
  if (B < 0 || L < 0 || D < 0 || K < 0) return fail("negative dimension");
  if (num_vars < 0 || num_vars > 255) return fail("num_vars must be in [0, 255]");
  if (K > kLbbMaxK) return fail("lbfgs supports at most 32 constants per program");
  if (history < 1 || history > kLbbMaxHistory) return fail("history must be in [1, 32]");
  *bytes = 0;
  if (B == 0) return WS_OK;
  if (D == 0 || L == 0) return fail("lbfgs needs at least one row and one token");
  int64_t n_splits = 1;
  ws_token_map none{};
  ws_status st = dtype == WS_F32
                     ? launch_loss_grad<float>(nullptr, B, L, nullptr, D, nullptr, K, nullptr,
                                               nullptr, none, num_vars, nullptr, nullptr,
                                               nullptr, nullptr, nullptr, &n_splits, nullptr)
                     : launch_loss_grad<double>(nullptr, B, L, nullptr, D, nullptr, K, nullptr,
                                                nullptr, none, num_vars, nullptr, nullptr,
                                                nullptr, nullptr, nullptr, &n_splits, nullptr);
  if (st != WS_OK) return st;
  *bytes = lbb_layout(B, K, history, n_splits, dtype == WS_F32 ? 4 : 8).total;
  return WS_OK;
}

extern "C" ws_status ws_lbfgs_adjoint(int32_t dtype, const uint8_t* population, int64_t B,
                                      int64_t L, const void* x, int64_t num_vars, int64_t D,
                                      void* constants, int64_t K, const void* y,
                                      const ws_lbfgs_opts* opts, double* out_loss,
                                      int32_t* out_evals, const ws_token_map* ids,
                                      void* workspace, size_t workspace_bytes, void* stream) {
  using namespace ws;
  clear_error();
  NvtxRange nvtx("ws_lbfgs_adjoint");
  if (!opts || !ids) return fail("options and token map are required");
  const ws_lbfgs_opts& o = *opts;
  if (o.max_iter < 1 || o.max_eval < 1 || o.max_ls < 1) return fail("iteration limits must be positive");
  if (!(o.lr > 0.0)) return fail("lr must be positive");
  size_t need = 0;
  ws_status st = ws_lbfgs_adjoint_workspace_bytes(dtype, B, L, num_vars, D, K, o.history, &need);
  if (st != WS_OK) return st;
  if (B == 0) return WS_OK;
  if (!population || !y || (K > 0 && !constants) || (num_vars > 0 && !x) || !workspace)
    return fail("null tensor pointer");
  if (workspace_bytes < need) return fail("lbfgs workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == WS_F32)
    return lbfgs_batch_typed<float>(population, B, L, x, num_vars, D, constants, K, y, o,
                                    out_loss, out_evals, *ids, workspace, workspace_bytes, s);
  return lbfgs_batch_typed<double>(population, B, L, x, num_vars, D, constants, K, y, o, out_loss,
                                   out_evals, *ids, workspace, workspace_bytes, s);
}
