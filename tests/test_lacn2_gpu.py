"""GPU parity of lacn2 (the reverse-communication 1-norm estimator) through the
C ABI, against the oracle's xLACN2 restatement (itself pinned to LAPACK's own
routine by tests/test_oracle_lacn2.py).

The caller's products are made two ways: on the host, with the same ordered
sums the oracle's driver uses (so the two runs see identical vectors and must
take identical branches: same kase sequence and isave states, estimate and v
to the order of the sums), and on the GPU with torch for matrix-free operators
of n up to 200,000 (the multi-block reduction path), where the estimate is
exact by Hager's theorem (diagonal, nonnegative rank one) or checked against
the true 1-norm."""
import ctypes
import os
import sys

import numpy as np
import pytest

from helpers import Runner

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from lacn2_cases import CASES, make_matrix, operators  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def drive(run, n, apply, apply_t, single, max_calls=64, work_bytes=None):
    """Run the estimator to completion; apply / apply_t map a device vector to
    A x / A^T x (device tensors of the working dtype)."""
    torch = run.torch
    dt = torch.float32 if single else torch.float64
    suf = "s" if single else "d"
    ct = ctypes.c_float if single else ctypes.c_double
    lib = run.lib
    nbytes = getattr(lib, f"calaman_lacn2_bufferSize_{suf}")(n)
    work = run.workspace(nbytes)
    v = torch.zeros(n, dtype=dt, device="cuda")
    x = torch.zeros(n, dtype=dt, device="cuda")
    est, kase = ct(0), ctypes.c_int(0)
    isave = (ctypes.c_int * 3)()
    fn = getattr(lib, f"calaman_lacn2_{suf}")
    kases, isaves = [], []
    for _ in range(max_calls):
        st = fn(run.h, n, ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                ctypes.c_void_p(work.data_ptr()), nbytes if work_bytes is None else work_bytes,
                ctypes.byref(est), ctypes.byref(kase), isave)
        assert st.ok, st
        kases.append(kase.value)
        isaves.append(list(isave))
        if kase.value == 0:
            torch.cuda.synchronize()
            return kases, isaves, float(est.value), v.cpu().numpy()
        y = apply(x) if kase.value == 1 else apply_t(x)
        x.copy_(y)
    raise AssertionError("lacn2 did not finish")


def host_ops(run, a, single):
    """The ordered host sums of lacn2_cases.operators, wrapped for device vectors."""
    torch = run.torch
    dt = torch.float32 if single else torch.float64
    f, ft = operators(a)

    def wrap(g):
        return lambda x: torch.from_numpy(
            g(x.cpu().numpy().astype(np.float64)).astype(np.float32 if single else np.float64)
        ).to("cuda", dt)

    return wrap(f), wrap(ft)


def _rel(x, y):
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    return np.abs(x - y).max(initial=0.0) / max(np.abs(y).max(initial=0.0), 1e-300)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_matches_oracle_trace(run, oracle, case):
    name, kind, n, seed, single = case
    a = make_matrix(kind, n, seed)
    if single:
        a = a.astype(np.float32).astype(np.float64)
    kases, isaves, est, v = drive(run, n, *host_ops(run, a, single), single)
    ref = oracle.lacn2(*operators(a), n, single=single)
    assert kases == ref.kases
    assert isaves == [list(s) for s in ref.isaves]
    if kind == "nan":
        assert np.isnan(est) and np.isnan(ref.est)
        return
    rel = 1e-6 if single else 1e-13
    assert abs(est - ref.est) <= rel * max(abs(ref.est), 1e-300)
    assert _rel(v, ref.v) <= rel


@pytest.mark.parametrize("n", [8192, 8193, 50_000, 200_000])
def test_matrix_free_diagonal_exact(run, n):
    """A = diag(d): Hager's estimate is exact, est = max |d_j|, v = A e_j."""
    torch = run.torch
    g = torch.Generator(device="cuda").manual_seed(n)
    d = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    kases, _, est, v = drive(run, n, lambda x: d * x, lambda x: d * x, False)
    assert kases[0] == 1 and kases[-1] == 0
    dmax = float(d.abs().max())
    assert est == dmax
    assert np.count_nonzero(v) == 1 and float(np.abs(v).max()) == dmax


@pytest.mark.parametrize("single", [False, True])
def test_matrix_free_rank_one_nonnegative(run, single):
    """A = u w^T with u, w > 0: ||A||_1 = max_j w_j sum_i u_i, attained."""
    torch = run.torch
    n = 120_000
    dt = torch.float32 if single else torch.float64
    g = torch.Generator(device="cuda").manual_seed(7)
    u = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) + 0.5
    w = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) + 0.5
    true = float(w.max() * u.sum())
    kases, _, est, _ = drive(run, n, lambda x: (u * torch.dot(w, x.double())).to(dt),
                             lambda x: (w * torch.dot(u, x.double())).to(dt), single)
    assert kases[-1] == 0
    assert abs(est - true) <= (2e-6 if single else 1e-12) * true


def test_dense_gpu_products_bound(run):
    """Dense 3000 x 3000 with GPU products: est <= ||A||_1 and within the
    underestimate Hager's method shows on Gaussian matrices (a factor of 3)."""
    torch = run.torch
    n = 3000
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
    _, _, est, v = drive(run, n, lambda x: A @ x, lambda x: A.T @ x, False)
    true = float(A.abs().sum(0).max())
    assert true / 3 <= est <= true * (1 + 1e-13)


def test_workspace_reuse_and_restart(run, oracle):
    """Two runs on the same workspace: the second starts from kase 0 and
    repeats the first exactly (ISGN is rewritten before it is read)."""
    a = make_matrix("gauss", 77, 5)
    first = drive(run, 77, *host_ops(run, a, False), False)
    second = drive(run, 77, *host_ops(run, a, False), False)
    assert first[0] == second[0] and first[2] == second[2]
    assert np.array_equal(first[3], second[3])


def test_python_wrapper(cuda):
    import torch

    import calaman_g_b200 as cm

    n = 500
    g = torch.Generator(device="cuda").manual_seed(9)
    A = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64).abs()
    est, v = cm.lacn2_estimate(lambda x: A @ x, lambda x: A.T @ x, n)
    true = float(A.sum(0).max())
    assert abs(est - true) <= 1e-13 * true  # nonnegative: exact
    assert abs(float(v.abs().sum()) - est) <= 1e-13 * true
