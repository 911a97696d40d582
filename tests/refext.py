"""Loader of the reference extension built from its own sources by oracle/build_ref.sh
(test infrastructure: a parity checker on GPU boxes; absent => the dependent tests skip)."""
from __future__ import annotations

import glob
import importlib.util
import os

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_cache = {}


def path(variant: str = "fastmath"):
    hits = glob.glob(os.path.join(REPO, "oracle", "_ref", variant, "rpn_cuda_native*.so"))
    return hits[0] if hits else None


def load(variant: str = "fastmath"):
    """The reference module (same name as the original: rpn_cuda_native), or None."""
    if variant in _cache:
        return _cache[variant]
    p = path(variant)
    if p is None:
        return None
    import torch  # noqa: F401  (the extension links libtorch)
    spec = importlib.util.spec_from_file_location("rpn_cuda_native", p)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    _cache[variant] = mod
    return mod


def classic_rmse(ref, ids, pop, x, consts, y, strict, inf_val):
    """The reference's classic evaluate_batch path (evaluation.py:140-192) with its own
    eval_rpn kernel: validity masks, torch mean over rows, sqrt and the INF sentinels."""
    import torch
    B = pop.shape[0]
    D = x.shape[1]
    out = torch.full((B,), inf_val, device=x.device, dtype=x.dtype)
    inf_t = torch.tensor(inf_val, device=x.device, dtype=x.dtype)
    step = max(1, min(B, (2**31 - 1) // D))
    for i in range(0, B, step):
        j = min(B, i + step)
        preds = torch.empty((j - i, D), dtype=x.dtype, device=x.device)
        sp = torch.empty((j - i, D), dtype=torch.int32, device=x.device)
        err = torch.empty((j - i, D), dtype=torch.uint8, device=x.device)
        ref.eval_rpn(pop[i:j].contiguous(), x, consts[i:j].contiguous(), preds, sp, err, *ids,
                     3.14159265359, 2.718281828, strict)
        valid = (sp == 1) & (err == 0) & ~torch.isnan(preds) & ~torch.isinf(preds)
        p = torch.where(valid, preds, torch.zeros_like(preds))
        ind = valid.all(dim=1)
        mse = torch.mean((p - y.reshape(1, -1)) ** 2, dim=1)
        score = torch.sqrt(torch.where(torch.isnan(mse) | torch.isinf(mse), inf_t, mse))
        out[i:j] = torch.where(ind, score, inf_t)
    return out
