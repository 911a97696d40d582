"""ws_eval_fitness_static: fitness evaluation for callers that cannot allocate device memory.

Some callers have no device allocator at hand when they need a fitness evaluation -- a host
runtime that reaches this library through a plain C FFI with only device pointers from another
framework, or a loop that must not call cudaMalloc because it synchronises the device.  For them
ws_eval_fitness_static takes no workspace: its scratch is a static array inside the library.

This file is named to be collected last, so a run that stops at the first failure has run every
other test before it; it also passes when run alone in a fresh process.  Results must equal those
of ws_eval_fitness (the same pipeline on a caller-provided workspace), on two calls in a row,
since every call reuses the same static scratch.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import ws_testlib as tl

pytestmark = pytest.mark.gpu


def _static_call(g, pop, X, consts, y, policy, loss, strict=0, invalid=1e15):
    lib = tl.N.lib()
    B, L = pop.shape
    V, D = X.shape
    K = consts.shape[1]
    out = torch.empty(B, dtype=torch.float64 if loss == "sse" else X.dtype, device=X.device)
    ninv = torch.empty(B, dtype=torch.int32, device=X.device)
    pol = {"fused": tl.N.WS_POLICY_FUSED, "classic": tl.N.WS_POLICY_CLASSIC}[policy]
    lk = {"rmse": 0, "mse": 1, "r2": 2, "sse": 3}[loss]
    opts = tl.N.FitnessOpts(strict, pol, lk, 0, invalid, 0, 0)
    m = tl.token_map(g)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = tl.N.WS_F32 if X.dtype == torch.float32 else tl.N.WS_F64
    tl.N.check(lib.ws_eval_fitness_static(code, C.c_void_p(pop.data_ptr()), B, L,
                                          C.c_void_p(X.data_ptr()), V, D,
                                          C.c_void_p(consts.data_ptr()), K,
                                          C.c_void_p(y.data_ptr()), C.c_void_p(out.data_ptr()),
                                          C.c_void_p(ninv.data_ptr()), C.byref(m), C.byref(opts),
                                          stream))
    return out, ninv


@pytest.mark.parametrize("case", ["c1_like", "scale_like", "f64_strict"])
def test_static_scratch_matches_workspace_entry_point(case):
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(77)
    if case == "c1_like":
        g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
        pop, consts = tl.random_population(g, 1024, 30, 4, rng, valid_only=False)
        X = rng.uniform(-3, 3, size=(2, 1024)).astype(np.float32)
        policy, loss, strict, dt = "fused", "rmse", 0, np.float32
    elif case == "scale_like":
        g = tl.GPUGrammar(num_variables=5, operators=tl.C1_OPERATORS)
        pop, consts = tl.random_population(g, 20000, 64, 8, rng, valid_only=True)
        X = rng.uniform(-3, 3, size=(5, 20000)).astype(np.float32)
        policy, loss, strict, dt = "classic", "mse", 0, np.float32
    else:
        g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
        pop, consts = tl.random_population(g, 3000, 48, 6, rng, valid_only=False)
        X = rng.uniform(-3, 3, size=(3, 777))
        policy, loss, strict, dt = "classic", "rmse", 1, np.float64
    y = rng.standard_normal(X.shape[1]).astype(dt)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    pop_t, X_t, c_t, y_t = T(pop), T(X.astype(dt)), T(consts.astype(dt)), T(y)
    inv = 1e15 if dt == np.float32 else 1e100
    vm = CudaRPNVM(g, dev)
    ninv_ref = torch.empty(len(pop), dtype=torch.int32, device=dev)
    want = vm.eval_fitness(pop_t, X_t, c_t, y_t, strict_mode=strict, policy=policy, loss=loss,
                           invalid_value=inv, out_ninvalid=ninv_ref).cpu().numpy()
    for _ in range(2):  # the second call reuses the scratch left by the first
        got, ninv = _static_call(g, pop_t, X_t, c_t, y_t, policy, loss, strict, inv)
        torch.cuda.synchronize()
        tl.assert_fitness_close(got.cpu().numpy(), want, rtol=1e-5, atol=1e-7, iv=inv, min_frac=1.0)
        assert np.array_equal(ninv.cpu().numpy(), ninv_ref.cpu().numpy())


def test_static_scratch_rejects_requests_beyond_its_size():
    lib = tl.N.lib()
    cap = lib.ws_static_scratch_bytes()
    B = 1 << 20  # 1,048,576 programs of 64 tokens need far more than the static scratch
    assert lib.ws_fitness_workspace_bytes(B, 64, tl.N.WS_F32) > cap
    g = tl.GPUGrammar(num_variables=2)
    m = tl.token_map(g)
    opts = tl.N.FitnessOpts(0, 1, 1, 0, 1e15, 0, 0)
    dummy = C.c_void_p(256)
    st = lib.ws_eval_fitness_static(0, dummy, B, 64, dummy, 2, 100, dummy, 4, dummy, dummy, None,
                                    C.byref(m), C.byref(opts), None)
    assert st != 0
    assert "static scratch" in lib.ws_last_error().decode()


def test_static_scratch_largest_request_and_no_device_allocation():
    """The largest population of 64-token FP32 programs that fits the static scratch (found by
    bisection on ws_fitness_workspace_bytes) evaluates like the workspace entry point, one more
    program is rejected, and the calls take no device memory (free device memory is unchanged
    across them once the library's module is loaded)."""
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    lib = tl.N.lib()
    cap = lib.ws_static_scratch_bytes()
    L = 64
    lo, hi = 1, 1 << 22
    assert lib.ws_fitness_workspace_bytes(lo, L, tl.N.WS_F32) <= cap
    assert lib.ws_fitness_workspace_bytes(hi, L, tl.N.WS_F32) > cap
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if lib.ws_fitness_workspace_bytes(mid, L, tl.N.WS_F32) <= cap:
            lo = mid
        else:
            hi = mid
    Bmax = lo
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(91)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    pop = tl.synthetic.random_programs(g, Bmax + 1, 3, L, L, rng, max_consts=6)
    consts = rng.uniform(-2, 2, size=(Bmax + 1, 6)).astype(np.float32)
    X = rng.uniform(-3, 3, size=(3, 300)).astype(np.float32)
    y = rng.standard_normal(300).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    pop_t, c_t, X_t, y_t = T(pop), T(consts), T(X), T(y)
    want = CudaRPNVM(g, dev).eval_fitness(pop_t[:Bmax], X_t, c_t[:Bmax], y_t, policy="classic",
                                          loss="mse").cpu().numpy()
    got, _ = _static_call(g, pop_t[:Bmax], X_t, c_t[:Bmax], y_t, "classic", "mse")
    torch.cuda.synchronize()
    tl.assert_fitness_close(got.cpu().numpy(), want, rtol=1e-5, atol=1e-7, min_frac=1.0)
    with pytest.raises(RuntimeError, match="static scratch"):
        _static_call(g, pop_t, X_t, c_t, y_t, "classic", "mse")
    # no device allocation by the calls: outputs are allocated first, then free memory is read
    # before and after each call (the first call above already loaded the module)
    for _ in range(2):
        out = torch.empty(Bmax, dtype=torch.float32, device=dev)
        ninv = torch.empty(Bmax, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(dev)
        lk = tl.N.WS_LOSS_MSE
        opts = tl.N.FitnessOpts(0, tl.N.WS_POLICY_CLASSIC, lk, 0, 1e15, 0, 0)
        m = tl.token_map(g)
        tl.N.check(lib.ws_eval_fitness_static(
            tl.N.WS_F32, C.c_void_p(pop_t.data_ptr()), Bmax, L, C.c_void_p(X_t.data_ptr()), 3,
            300, C.c_void_p(c_t.data_ptr()), 6, C.c_void_p(y_t.data_ptr()),
            C.c_void_p(out.data_ptr()), C.c_void_p(ninv.data_ptr()), C.byref(m), C.byref(opts),
            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(dev)
        assert free1 == free0, (free0, free1)
        tl.assert_fitness_close(out.cpu().numpy(), want, rtol=1e-5, atol=1e-7, min_frac=1.0)
