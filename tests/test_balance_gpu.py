"""GPU parity of the scaling half of gebal and of the balanced expm, through
the C ABI: FP64 / complex128 scale factors and balanced matrices bit-identical
to the oracle's restatement (same summation order), the reference's spec
checks for every element type, and the balanced expm against the oracle."""
import ctypes

import numpy as np
import pytest

from helpers import NP_DTYPE, REAL, Runner, _dev, colmajor_buffer, from_buffer, rel_frob

pytestmark = pytest.mark.gpu

JOB_SCALE, JOB_PERMUTE = 2, 1


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def badly_scaled(n, seed, spread=12, cplx=False):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    if cplx:
        a = a + 1j * rng.standard_normal((n, n))
    d = 2.0 ** rng.integers(-spread, spread + 1, n)
    return (a * d[:, None]) / d[None, :]


def gebal(run, a, suf, job=JOB_SCALE, ld=None):
    n = a.shape[0]
    ld = ld or max(n, 1)
    dA = _dev(colmajor_buffer(a, ld, suf))
    ds = _dev(np.zeros(max(n, 1), dtype=REAL[suf]))
    lw = ctypes.c_int()
    assert run.lib.calaman_gebal_bufferSize(n, ctypes.byref(lw)).ok
    dw = run.torch.zeros(max(lw.value, 1), dtype=run.torch.int32, device="cuda")
    ilo, ihi, sweeps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = getattr(run.lib, f"calaman_gebal_{suf}")(
        ctypes.c_void_p(run.stream), job, n, ctypes.c_void_p(dA.data_ptr()), ld, ctypes.byref(ilo),
        ctypes.byref(ihi), ctypes.c_void_p(ds.data_ptr()), ctypes.c_void_p(dw.data_ptr()), 0,
        ctypes.byref(sweeps))
    run.torch.cuda.synchronize()
    b = from_buffer(dA.cpu().numpy(), n, ld) if n else np.zeros((0, 0))
    return st, b, ds.cpu().numpy()[:n], (ilo.value, ihi.value, sweeps.value)


@pytest.mark.parametrize("suf,n", [("d", 1), ("d", 9), ("d", 200), ("d", 700), ("z", 33), ("z", 300)])
def test_bit_identical_to_oracle(run, oracle, suf, n):
    a = badly_scaled(n, 100 + n, cplx=suf == "z")
    st, b, d, (ilo, ihi, sweeps) = gebal(run, a, suf)
    ob, od, osweeps = oracle.gebal_scale(a)
    assert st.ok and (ilo, ihi) == (1, n) and sweeps == osweeps
    assert np.array_equal(d, od)
    assert np.array_equal(b, ob)


@pytest.mark.parametrize("suf", ["s", "d", "c", "z"])
def test_spec_analytic_reproduce_stationary(run, suf):
    st, b, d, _ = gebal(run, np.array([[1.0, 2.0 ** 10], [2.0 ** -10, 1.0]]), suf)
    assert st.ok and np.array_equal(b, np.ones((2, 2))) and np.array_equal(d, [2.0 ** 10, 1.0])
    a = badly_scaled(64, 7, spread=8, cplx=suf in "cz").astype(NP_DTYPE[suf])
    st, b, d, _ = gebal(run, a, suf)
    assert st.ok
    assert np.array_equal((b * d[:, None] / d[None, :]).astype(NP_DTYPE[suf]), a)
    st, b2, d2, (_, _, sweeps) = gebal(run, b, suf)
    assert st.ok and np.array_equal(b2, b) and np.all(d2 == 1) and sweeps == 1


def test_job_none_permute_and_padding(run):
    a = badly_scaled(10, 3)
    st, b, d, _ = gebal(run, a, "d", job=0)
    assert st.ok and np.array_equal(b, a) and np.all(d == 1)
    st, *_ = gebal(run, a, "d", job=JOB_PERMUTE)
    assert st.code == run.capi.NOT_SUPPORTED
    st, b, d, _ = gebal(run, a, "d", ld=13)
    ob, od, _ = gebal(run, a, "d")[1:3] + (None,)
    assert st.ok and np.array_equal(b, ob)


def expm_balanced(run, a, suf):
    n = a.shape[0]
    dA = _dev(colmajor_buffer(a, n, suf))
    dE = _dev(np.zeros(n * n, dtype=NP_DTYPE[suf]))
    nb = ctypes.c_size_t()
    assert getattr(run.lib, f"calaman_expm_balanced_bufferSize_{suf}")(run.h, n, ctypes.byref(nb)).ok
    w = run.workspace(nb.value)
    info = run.torch.zeros(2, dtype=run.torch.int32, device="cuda")
    plan = run.capi.ExpmPlan()
    st = getattr(run.lib, f"calaman_expm_balanced_{suf}")(
        run.h, run.h, ctypes.c_void_p(run.stream), n, ctypes.c_void_p(dA.data_ptr()), n,
        ctypes.c_void_p(dE.data_ptr()), n, ctypes.c_void_p(w.data_ptr()), nb.value,
        ctypes.cast(info.data_ptr(), run.capi.c_int_p), ctypes.byref(plan))
    run.torch.cuda.synchronize()
    return st, plan, from_buffer(dE.cpu().numpy(), n, n)


@pytest.mark.parametrize("suf,n", [("d", 40), ("d", 257), ("z", 64)])
def test_balanced_expm_matches_oracle(run, oracle, suf, n):
    a = badly_scaled(n, 200 + n, cplx=suf == "z")
    a *= 4.0 / np.abs(a).sum(axis=0).max() * 50  # large 1-norm before balancing
    st, plan, e = expm_balanced(run, a, suf)
    ref, oplan = oracle.expm_balanced(a)
    _, plain, _ = oracle.expm(a)
    assert st.ok and (plan.m, plan.s) == (oplan.m, oplan.s) and plan.s < plain.s
    assert rel_frob(e, ref) <= 1e-12


def test_balanced_expm_single_tier(run, oracle):
    a = badly_scaled(96, 300, spread=6).astype(np.float32)
    st, plan, e = expm_balanced(run, a, "s")
    # the FP32 sweep sums in FP32, so its factors may differ from the FP64
    # oracle's by a radix step on a borderline index; exp(A) may not
    ref, _ = oracle.expm_balanced(a.astype(np.float64), single=True)
    assert st.ok
    assert rel_frob(e, ref) <= 2e-5
