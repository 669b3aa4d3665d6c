"""calaman_expm_* and calaman_expm_vjp_* replay a captured CUDA graph of their
launches (everything after the 1-norm readback) when a call repeats the
previous call's size, plan, pointers and stream: the replayed results match
the directly launched ones, a replay reads the buffers' current contents, a
new plan leaves the graph, and the oracle agrees throughout."""
import ctypes

import numpy as np
import pytest

from helpers import Runner, _dev, colmajor_buffer, from_buffer, gaussian_scaled, gue_skew, rel_frob, vp

pytestmark = pytest.mark.gpu

BAR = {"s": 1e-5, "c": 1e-5, "d": 1e-12, "z": 1e-12}


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.lib.calamanSetExpmGraphs(r.h, 1)
    r.close()


def matrix(suf, n, target, seed):
    if suf in "cz":
        return gue_skew(n, target, seed)
    return gaussian_scaled(n, target, seed)


@pytest.mark.parametrize("suf", ["d", "z", "s", "c"])
def test_replay_matches_direct_and_rereads_inputs(run, oracle, suf):
    import torch

    n, target = 300, 20.0  # several panels (look-ahead stream) and squarings
    a0, a1 = matrix(suf, n, target, 900), matrix(suf, n, target, 901)
    lib = run.lib
    dA = _dev(colmajor_buffer(a0, n, suf))
    dE = torch.empty(n * n, dtype=dA.dtype, device="cuda")
    b = ctypes.c_size_t()
    assert getattr(lib, f"calaman_expm_bufferSize_{suf}")(run.h, n, ctypes.byref(b)).ok
    w = run.workspace(b.value)
    info = torch.full((2,), -99, dtype=torch.int32, device="cuda")
    side = torch.cuda.Stream()  # a capturable (non-default) stream
    fn = getattr(lib, f"calaman_expm_{suf}")

    def call():
        plan = run.capi.ExpmPlan()
        st = fn(run.h, run.h, ctypes.c_void_p(side.cuda_stream), n, vp(dA), n, vp(dE), n, vp(w), b.value,
                ctypes.cast(info.data_ptr(), run.capi.c_int_p), ctypes.byref(plan))
        torch.cuda.synchronize()
        assert st.ok, st
        assert list(info.cpu().numpy()) == [0, 0]
        return (plan.m, plan.s), from_buffer(dE.cpu().numpy(), n, n)

    en, cached = ctypes.c_int(-1), ctypes.c_int(-1)
    assert lib.calamanSetExpmGraphs(run.h, 0).ok
    plan0, direct0 = call()
    dA.copy_(torch.from_numpy(colmajor_buffer(a1, n, suf)))
    plan1, direct1 = call()
    assert plan0 == plan1 and plan0[1] > 0
    assert lib.calamanSetExpmGraphs(run.h, 1).ok
    try:
        dA.copy_(torch.from_numpy(colmajor_buffer(a0, n, suf)))
        for k in range(4):  # direct, capture, replay, replay
            before = lib.calamanGetLaunchCount()
            plan, got = call()
            assert plan == plan0
            assert lib.calamanGetLaunchCount() - before > 0
            assert rel_frob(got, direct0) <= 1e-13 * (1e7 if suf in "sc" else 1)
            assert lib.calamanGetExpmGraphs(run.h, ctypes.byref(en), ctypes.byref(cached)).ok
            assert en.value == 1 and (k == 0 or cached.value >= 1)
        # the same configuration, new contents: the replay reads them
        dA.copy_(torch.from_numpy(colmajor_buffer(a1, n, suf)))
        plan, got = call()
        assert plan == plan1
        assert rel_frob(got, direct1) <= 1e-13 * (1e7 if suf in "sc" else 1)
        ref, oplan, _ = oracle.expm(a1.astype(np.complex128 if suf in "cz" else np.float64))
        assert rel_frob(got, ref) <= BAR[suf]
        # a smaller norm: another plan, so the call runs directly again
        dA.copy_(torch.from_numpy(colmajor_buffer(a0 / 64, n, suf)))
        plan, got = call()
        assert plan[1] < plan0[1]
        ref, _, _ = oracle.expm((a0 / 64).astype(np.complex128 if suf in "cz" else np.float64))
        assert rel_frob(got, ref) <= BAR[suf]
    finally:
        lib.calamanSetExpmGraphs(run.h, 1)


@pytest.mark.parametrize("suf", ["d", "s"])
def test_adjoint_replay_matches_direct(run, suf):
    """calaman_expm_vjp_* replays its launches the same way: the gradient and
    the exponential of a replayed call equal the directly launched ones, also
    after the inputs' contents change."""
    import torch

    n, target = 200, 12.0
    a0, a1 = gaussian_scaled(n, target, 950), gaussian_scaled(n, target, 951)
    g0 = np.random.default_rng(952).standard_normal((n, n))
    lib = run.lib
    dA = _dev(colmajor_buffer(a0, n, suf))
    dG = _dev(colmajor_buffer(g0, n, suf))
    dD = torch.empty(n * n, dtype=dA.dtype, device="cuda")
    dE = torch.empty(n * n, dtype=dA.dtype, device="cuda")
    b = ctypes.c_size_t()
    assert getattr(lib, f"calaman_expm_vjp_bufferSize_{suf}")(run.h, n, ctypes.byref(b)).ok
    w = run.workspace(b.value)
    info = torch.full((2,), -99, dtype=torch.int32, device="cuda")
    side = torch.cuda.Stream()
    fn = getattr(lib, f"calaman_expm_vjp_{suf}")
    tol = 1e-13 if suf == "d" else 1e-6

    def call():
        plan = run.capi.ExpmPlan()
        st = fn(run.h, run.h, ctypes.c_void_p(side.cuda_stream), n, vp(dA), n, vp(dG), n, vp(dD), n, vp(dE), n,
                vp(w), b.value, ctypes.cast(info.data_ptr(), run.capi.c_int_p), ctypes.byref(plan))
        torch.cuda.synchronize()
        assert st.ok, st
        assert list(info.cpu().numpy()) == [0, 0]
        return (plan.m, plan.s), from_buffer(dD.cpu().numpy(), n, n), from_buffer(dE.cpu().numpy(), n, n)

    en, cached = ctypes.c_int(-1), ctypes.c_int(-1)
    assert lib.calamanSetExpmGraphs(run.h, 0).ok
    plan0, grad0, exp0 = call()
    dA.copy_(torch.from_numpy(colmajor_buffer(a1, n, suf)))
    plan1, grad1, exp1 = call()
    assert plan0 == plan1 and plan0[1] > 0
    assert lib.calamanSetExpmGraphs(run.h, 1).ok
    try:
        dA.copy_(torch.from_numpy(colmajor_buffer(a0, n, suf)))
        for k in range(4):  # direct, capture, replay, replay
            plan, grad, ex = call()
            assert plan == plan0
            assert rel_frob(grad, grad0) <= tol and rel_frob(ex, exp0) <= tol
        assert lib.calamanGetExpmGraphs(run.h, ctypes.byref(en), ctypes.byref(cached)).ok
        assert en.value == 1 and cached.value >= 1
        dA.copy_(torch.from_numpy(colmajor_buffer(a1, n, suf)))
        plan, grad, ex = call()
        assert plan == plan1
        assert rel_frob(grad, grad1) <= tol and rel_frob(ex, exp1) <= tol
    finally:
        lib.calamanSetExpmGraphs(run.h, 1)
