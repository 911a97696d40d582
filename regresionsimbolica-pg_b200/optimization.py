"""Constant fitting: mirror of GPUOptimizer (src/warpsymbolic/gpu/optimization.py:90-566) on top
of libwarpsym.

  nano_pso / nano_pso_adaptive   fused single-launch PSO inside the reference's envelope
                                 (_can_use_fused_pso, optimization.py:163-191), else the
                                 multi-kernel PSO (:418-566) whose evaluation step is one
                                 fitness launch over the particle-expanded population (no
                                 [B*P, D] predictions) and whose bests / update steps are the
                                 pso_update_bests / pso_update kernels;
  lbfgs_optimize_top_k           the L-BFGS kernel for <= 64 programs and <= 1024 rows, else the
                                 torch L-BFGS (strong Wolfe) over RPNBackwardFunction, accepting
                                 only improvements (:193-343); with per_program=True, one L-BFGS
                                 per program over the one-launch loss and adjoint gradient
                                 (constfit.lbfgs).

The random draws of the multi-kernel path are torch's, in the reference's order; the fused path
draws the kernel's curand streams from the same seed formula.  As in the reference, the native
calls receive pi and e as math.pi / math.e.
"""
from __future__ import annotations

import math
from typing import Tuple

import torch

from . import rpn_cuda_native as _rcn
from .autograd import evaluate_with_gradients

CONSTANT_MIN_VALUE = -25.0   # GpuGlobals.CONSTANT_MIN_VALUE (config.py:111)
CONSTANT_MAX_VALUE = 25.0    # GpuGlobals.CONSTANT_MAX_VALUE (config.py:112)


class GPUOptimizer:
    def __init__(self, evaluator, device, dtype=torch.float64,
                 const_min: float = CONSTANT_MIN_VALUE, const_max: float = CONSTANT_MAX_VALUE):
        self.evaluator = evaluator
        self.device = torch.device(device)
        self.dtype = dtype
        self.const_min = float(const_min)
        self.const_max = float(const_max)
        self._pso_call_counter = 0

    @property
    def _ids(self):
        return self.evaluator.vm.ids

    # ---- PSO ---------------------------------------------------------------------------------
    def nano_pso(self, population, constants, x, y, steps: int = 20, num_particles: int = 20,
                 w: float = 0.5, c1: float = 1.5, c2: float = 1.5) -> Tuple[torch.Tensor, torch.Tensor]:
        if self._can_use_fused_pso(population, constants, x, y, num_particles):
            return self._fused_nano_pso(population, constants, x, y, steps, num_particles, w, c1,
                                        c2)
        return self._multi_kernel_nano_pso(population, constants, x, y, steps, num_particles, w,
                                           c1, c2)

    def nano_pso_adaptive(self, population, constants, x, y, steps: int = 20,
                          num_particles: int = 20, w_max: float = 0.9, w_min: float = 0.4,
                          c1: float = 1.5, c2: float = 1.5):
        if self._can_use_fused_pso(population, constants, x, y, num_particles):
            return self._fused_nano_pso(population, constants, x, y, steps, num_particles, w_max,
                                        c1, c2)
        w_avg = (w_max + w_min) / 2.0
        return self._multi_kernel_nano_pso(population, constants, x, y, steps, num_particles,
                                           w_avg, c1, c2)

    def _can_use_fused_pso(self, population, constants, x, y, num_particles) -> bool:
        return (population.ndim == 2 and constants.ndim == 2 and y.numel() <= 1024
                and population.shape[1] <= 63 and constants.shape[1] <= 16
                and num_particles <= 64 and population.is_cuda and constants.is_cuda
                and x.is_cuda and y.is_cuda and constants.dtype == torch.float32
                and x.dtype == torch.float32 and y.dtype == torch.float32)

    @staticmethod
    def _vars_major(x, D):
        if x.ndim == 2 and x.shape[0] == D and x.shape[1] != D:
            return x.T.contiguous()
        return x.contiguous()

    def _fused_nano_pso(self, population, constants, x, y, steps, num_particles, w, c1, c2):
        B, K = constants.shape
        x = self._vars_major(x, y.numel())
        gbest_pos = torch.empty((B, K), device=self.device, dtype=constants.dtype)
        gbest_err = torch.empty((B,), device=self.device, dtype=constants.dtype)
        rng_seed = (int(torch.initial_seed()) + self._pso_call_counter * 0x9E3779B1) \
            & 0x7FFFFFFFFFFFFFFF
        self._pso_call_counter += 1
        _rcn.fused_pso(population.contiguous(), constants.contiguous(), x, y.contiguous(),
                       gbest_pos, gbest_err, num_particles, steps, w, c1, c2, self.const_min,
                       self.const_max, *self._ids, math.pi, math.e, rng_seed)
        return gbest_pos.to(self.dtype), gbest_err.to(self.dtype)

    def _multi_kernel_nano_pso(self, population, constants, x, y, steps=20, num_particles=20,
                               w=0.5, c1=1.5, c2=1.5):
        B, K = constants.shape
        P = num_particles
        dt = self.dtype
        pop_expanded = population.repeat_interleave(P, dim=0)
        pos = constants.to(dt).unsqueeze(1).repeat(1, P, 1)
        const_range = self.const_max - self.const_min
        noise = torch.randn(B, P - 1, K, device=self.device, dtype=dt) * (const_range * 0.15)
        pos[:, 1:, :] += noise
        pos.clamp_(self.const_min, self.const_max)
        vel = (torch.randn_like(pos) * (const_range * 0.02)).reshape(-1, K).contiguous()
        flat_pos = pos.reshape(-1, K).contiguous()
        pbest_pos = flat_pos.clone()
        pbest_err = torch.full((B * P,), float("inf"), device=self.device, dtype=dt)
        gbest_pos = constants.to(dt).clone().contiguous()
        gbest_err = torch.full((B,), float("inf"), device=self.device, dtype=dt)
        for step in range(steps):
            w_curr = w - (w - 0.4) * (step / (steps - 1 if steps > 1 else 1))
            errors = self.evaluator.evaluate_batch(pop_expanded, x, y, flat_pos).to(dt)
            _rcn.pso_update_bests(errors.view(B, P).contiguous(), pbest_err.view(B, P),
                                  pbest_pos.view(B, P, K), flat_pos.view(B, P, K), gbest_err,
                                  gbest_pos)
            r1 = torch.rand(B, P, K, device=self.device, dtype=dt)
            r2 = torch.rand(B, P, K, device=self.device, dtype=dt)
            _rcn.pso_update(flat_pos.view(B, P, K), vel.view(B, P, K), pbest_pos.view(B, P, K),
                            gbest_pos, r1, r2, w_curr, c1, c2)
            flat_pos.clamp_(self.const_min, self.const_max)
        return gbest_pos, gbest_err

    # ---- L-BFGS ------------------------------------------------------------------------------
    def lbfgs_optimize_top_k(self, population, constants, x, y_target, top_k: int = 50,
                             max_iter: int = 30, per_program: bool = False,
                             history_size: int = 10):
        """per_program=False (default): the reference's dispatch.  per_program=True: one L-BFGS
        per program over the adjoint gradient (constfit.lbfgs) with the reference fallback's
        options (strong Wolfe, max_eval = 2 * max_iter, gradients clamped to 1e4), then the same
        clamp, re-evaluation and improvement-only acceptance."""
        B, K = constants.shape
        if K == 0 or top_k <= 0 or B == 0:
            return constants, torch.full((B,), float("inf"), device=self.device, dtype=self.dtype)
        actual_k = min(top_k, B)
        pop_k = population[:actual_k].contiguous()
        c = constants[:actual_k].clone().to(self.dtype)
        best_errs_k = self.evaluator.evaluate_batch(pop_k, x, y_target, c).to(self.dtype)
        best_c_k = c.clone()
        if per_program:
            return self._lbfgs_per_program(pop_k, c, x, y_target, best_errs_k, best_c_k,
                                           constants, max_iter, history_size)
        if actual_k <= 64 and y_target.numel() <= 1024:
            c_final, final_errs_k = self._lbfgs_cuda(pop_k, c, x, y_target, max_iter)
            improved = torch.isfinite(final_errs_k) & (final_errs_k < best_errs_k)
            best_c_k[improved] = c_final[improved]
            best_errs_k[improved] = final_errs_k[improved]
            result = constants.clone()
            result[:actual_k] = best_c_k.to(constants.dtype)
            full = torch.full((B,), float("inf"), device=self.device, dtype=self.dtype)
            full[:actual_k] = best_errs_k
            return result, full
        return self._lbfgs_pytorch_fallback(pop_k, c, x, y_target, best_errs_k, best_c_k,
                                            constants, max_iter)

    def _lbfgs_cuda(self, population, constants, x, y_target, max_iter):
        B = population.shape[0]
        x_cuda = self._vars_major(x, y_target.numel()).to(constants.dtype)
        y = y_target.to(constants.dtype).contiguous()
        out_rmse = torch.empty(B, device=self.device, dtype=constants.dtype)
        c = constants.contiguous()
        _rcn.lbfgs_optimize(population.contiguous(), c, x_cuda, y, out_rmse, max_iter, 10, 1e-7,
                            self.const_min, self.const_max, *self._ids, math.pi, math.e)
        return c, out_rmse

    def _lbfgs_per_program(self, pop_k, c, x, y_target, best_errs_k, best_c_k, constants,
                           max_iter, history_size):
        from .constfit import lbfgs
        x_v = self._vars_major(x, y_target.numel()).to(c.dtype)
        y = y_target.to(c.dtype).contiguous()
        c_fit, _, evals = lbfgs(pop_k, x_v, c.contiguous(), y, self._ids, max_iter=max_iter,
                                max_eval=max_iter * 2, history_size=history_size,
                                tolerance_grad=1e-7, tolerance_change=1e-9, grad_clip=1e4)
        self.last_lbfgs_evals = evals  # loss evaluations per program (device tensor)
        return self._accept(pop_k, c_fit, x, y_target, best_errs_k, best_c_k, constants)

    def _accept(self, pop_k, c_fit, x, y_target, best_errs_k, best_c_k, constants):
        actual_k = pop_k.shape[0]
        c_final = c_fit.detach().clamp(self.const_min, self.const_max)
        final_errs_k = self.evaluator.evaluate_batch(pop_k, x, y_target, c_final).to(self.dtype)
        improved = torch.isfinite(final_errs_k) & (final_errs_k < best_errs_k)
        best_c_k[improved] = c_final[improved]
        best_errs_k[improved] = final_errs_k[improved]
        result = constants.clone()
        result[:actual_k] = best_c_k.to(constants.dtype)
        full = torch.full((constants.shape[0],), float("inf"), device=self.device,
                          dtype=self.dtype)
        full[:actual_k] = best_errs_k
        return result, full

    def _lbfgs_pytorch_fallback(self, pop_k, c, x, y_target, best_errs_k, best_c_k, constants,
                                max_iter):
        actual_k = pop_k.shape[0]
        c.requires_grad_(True)
        optimizer = torch.optim.LBFGS([c], lr=1.0, max_iter=max_iter, max_eval=max_iter * 2,
                                      tolerance_grad=1e-7, tolerance_change=1e-9,
                                      history_size=10, line_search_fn="strong_wolfe")
        vm = self.evaluator.vm
        x_v = self._vars_major(x, y_target.numel()).to(c.dtype)
        y = y_target.to(c.dtype)

        def closure():
            optimizer.zero_grad()
            loss, _ = evaluate_with_gradients(pop_k, c, x_v, y, vm)
            if loss.requires_grad:
                loss.backward()
            if c.grad is not None:
                c.grad.data.clamp_(-1e4, 1e4)
            return loss

        try:
            optimizer.step(closure)
        except RuntimeError:
            pass
        return self._accept(pop_k, c, x, y_target, best_errs_k, best_c_k, constants)
