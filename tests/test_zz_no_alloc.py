"""calaman_expm_noalloc_d: the expm entry point for callers that cannot call
cudaMalloc (their workspace lives in a static device array of the library).
Checked through the C ABI against calaman_expm_d, which takes a caller
workspace, on two calls in a row; collected last so that a failure here leaves
every other test already run."""
import ctypes

import numpy as np
import pytest

from helpers import Runner, colmajor_buffer, from_buffer, gaussian_scaled, rel_frob

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64-tier tolerance of the other expm tests


def noalloc(run, a):
    import torch

    n = a.shape[0]
    dA = torch.from_numpy(colmajor_buffer(a, n, "d")).cuda()
    dE = torch.full((n * n,), -5.0, dtype=torch.float64, device="cuda")
    info = torch.full((2,), -9, dtype=torch.int32, device="cuda")
    plan = run.capi.ExpmPlan()
    st = run.lib.calaman_expm_noalloc_d(
        run.h, ctypes.c_void_p(run.stream), n, ctypes.c_void_p(dA.data_ptr()), n,
        ctypes.c_void_p(dE.data_ptr()), n, ctypes.cast(info.data_ptr(), run.capi.c_int_p),
        ctypes.byref(plan))
    torch.cuda.synchronize()
    return st, plan, from_buffer(dE.cpu().numpy(), n, n), info.cpu().tolist()


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def test_matches_expm_on_two_calls_in_a_row(run, oracle):
    cases = [gaussian_scaled(200, 5.0, 11), gaussian_scaled(256, 40.0, 12)]  # m=13 s=0; s=3
    for a in cases:
        st, plan, got, info = noalloc(run, a)
        st2, plan2, want, _, info2 = run.expm(a, "d")
        assert st.ok and st2.ok, (st, st2)
        assert (plan.m, plan.s) == (plan2.m, plan2.s)
        assert info == [0, 0] and list(info2) == [0, 0]
        assert rel_frob(got, want) <= TOL
        ref, oplan, _ = oracle.expm(a)  # and the FP64 oracle itself
        assert (plan.m, plan.s) == (oplan.m, oplan.s)
        assert rel_frob(got, ref) <= TOL


def test_rejects_sizes_beyond_the_static_workspace(run):
    a = gaussian_scaled(257, 1.0, 13)
    st, _, _, _ = noalloc(run, a)
    assert st.code == 15  # CALAMAN_STATUS_NOT_SUPPORTED
