"""GPU parity of paterson_stockmeyer and horner (restates
test/paterson_stockmeyer/paterson_stockmeyer_tests.cpp and
test/horner/horner_tests.cpp) against the power-series oracle, with the
reference's bound poly_tol = 64 eps n sum |c_k| ||A||_F^k."""
import json
import os

import numpy as np
import pytest

from helpers import NP_DTYPE, Runner, eps

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def poly_reference(a, c):
    n = a.shape[0]
    res = c[0] * np.eye(n)
    p = np.eye(n)
    for k in range(1, len(c)):
        p = p @ a
        res = res + c[k] * p
    return res


def poly_tol(a, c, suf):
    an = np.linalg.norm(a)
    return 64 * eps(suf) * sum(abs(ck) * an ** k for k, ck in enumerate(c)) * a.shape[0]


def inputs(n, degree, seed, suf):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-0.5, 0.5, (n, n)).astype(NP_DTYPE[suf]).astype(np.float64)
    c = (rng.uniform(-0.5, 0.5, degree + 1) * 2).astype(NP_DTYPE[suf]).astype(np.float64)
    return a, c


CASES = [(5, 0, 1), (6, 1, 4), (5, 2, 5), (4, 4, 10), (6, 8, 11), (4, 6, 20), (6, 10, 21),
         (16, 12, 30), (16, 16, 31), (64, 9, 32), (200, 7, 33)]


@pytest.mark.parametrize("kind", ["ps", "horner"])
@pytest.mark.parametrize("suf", ["s", "d"])
@pytest.mark.parametrize("n,degree,seed", CASES)
def test_matches_power_series(run, kind, suf, n, degree, seed):
    a, c = inputs(n, degree, seed, suf)
    st, got, _ = run.poly(kind, a, c, suf)
    assert st.ok, st
    ref = poly_reference(a, c)
    assert np.abs(got - ref).max() <= poly_tol(a, c, suf)


def test_all_block_sizes_agree(run):
    n, degree = 5, 7
    a, c = inputs(n, degree, 77, "d")
    ref = poly_reference(a, c)
    for s in range(1, degree + 2):
        st, got, _ = run.poly("ps", a, c, "d", s_requested=s)
        assert st.ok
        assert np.abs(got - ref).max() <= poly_tol(a, c, "d"), s


def test_ps_matches_horner(run):
    for degree in (3, 6, 9):
        a, c = inputs(8, degree, 90 + degree, "d")
        _, ps, _ = run.poly("ps", a, c, "d")
        _, hn, _ = run.poly("horner", a, c, "d")
        assert np.abs(ps - hn).max() <= poly_tol(a, c, "d")


@pytest.mark.parametrize("kind", ["ps", "horner"])
def test_zero_polynomial_is_exact(run, kind):
    a, _ = inputs(6, 8, 40, "d")
    st, got, _ = run.poly(kind, a, np.zeros(9), "d", out_fill=7.0)
    assert st.ok and np.all(got == 0.0)


@pytest.mark.parametrize("kind", ["ps", "horner"])
def test_nilpotent_series_terminates(run, kind):
    n, degree = 5, 9
    a = np.zeros((n, n))
    for j in range(n):
        for i in range(j):
            a[i, j] = 0.3 * (i + j + 1)
    c = np.random.default_rng(50).uniform(-1, 1, degree + 1)
    st, got, _ = run.poly(kind, a, c, "d")
    assert st.ok
    assert np.abs(got - poly_reference(a, c)).max() <= poly_tol(a, c, "d")


@pytest.mark.parametrize("kind", ["ps", "horner"])
@pytest.mark.parametrize("degree", [7, 8])
def test_padding_rows_untouched(run, kind, degree):
    n, ldp = 5, 8
    a, c = inputs(n, degree, 60 + degree, "d")
    st, got, full = run.poly(kind, a, c, "d", ldp=ldp, out_fill=-123.5)
    assert st.ok
    assert np.all(full.reshape(n, ldp)[:, n:] == -123.5)
    assert np.abs(got - poly_reference(a, c)).max() <= poly_tol(a, c, "d")


def test_golden_rational_polynomials(run):
    with open(os.path.join(os.path.dirname(__file__), "golden", "poly_rational.json")) as f:
        cases = json.load(f)["cases"]
    for case in cases:
        a, c, want = np.array(case["a"]), np.array(case["c"]), np.array(case["p"])
        for kind in ("ps", "horner"):
            st, got, _ = run.poly(kind, a, c, "d")
            assert st.ok
            assert np.abs(got - want).max() <= 1e-14 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("kind", ["ps", "horner"])
@pytest.mark.parametrize("n,degree,seed", [(64, 9, 40), (200, 7, 41), (256, 12, 42)])
def test_float_products_on_the_tensor_cores_with_a_handle_workspace(run, kind, n, degree, seed):
    """horner_s / paterson_stockmeyer_s with a workspace attached to the handle:
    the products take the split-BF16 tensor-core path (three launches per
    product: two operand splits and the GEMM) and stay within poly_tol."""
    import ctypes

    a, c = inputs(n, degree, seed, "s")
    base = run.lib.calamanGetLaunchCount()
    st0, got0, _ = run.poly(kind, a, c, "s")
    simt_launches = run.lib.calamanGetLaunchCount() - base
    nb = run.lib.calaman_poly_tensor_workspace_s(n)
    w = run.workspace(nb)
    assert run.lib.calamanSetWorkspace(run.h, ctypes.c_void_p(w.data_ptr()), nb).ok
    try:
        base = run.lib.calamanGetLaunchCount()
        st1, got1, _ = run.poly(kind, a, c, "s")
        tc_launches = run.lib.calamanGetLaunchCount() - base
    finally:
        assert run.lib.calamanSetWorkspace(run.h, None, 0).ok
    assert st0.ok and st1.ok
    ref = poly_reference(a, c)
    tol = poly_tol(a, c, "s")
    assert np.abs(got0 - ref).max() <= tol
    assert np.abs(got1 - ref).max() <= tol
    assert tc_launches > simt_launches  # the split kernels ran


def test_handle_workspace_arguments(run):
    import ctypes

    w = run.workspace(4096)
    assert run.lib.calamanSetWorkspace(run.h, None, 16).code == 7
    assert run.lib.calamanSetWorkspace(run.h, ctypes.c_void_p(w.data_ptr() + 8), 1024).code == 7
    assert run.lib.calamanSetWorkspace(None, ctypes.c_void_p(w.data_ptr()), 1024).code == 1
    assert run.lib.calamanSetWorkspace(run.h, None, 0).ok
