"""GPU parity of expm / pade / matrix_norm1 against the FP64 oracle, through
the C ABI. Restates test/expm/expm_tests.cpp (closed forms, identities, degree
ladder, padding, pointer mode, argument checks) and adds the oracle parity
bars: FP64 tiers within 1e-12 relative Frobenius of the oracle, single tiers
within the stated bound below."""
import ctypes

import numpy as np
import pytest

from helpers import (Runner, elem_tol, gaussian_scaled, gue_skew, rel_frob, scaled_random)

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12       # FP64 tiers vs the FP64 oracle (relative Frobenius)
SINGLE_REL = 2e-5      # single tiers (FP32 storage) vs the FP64 oracle


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def cplx_of(suf):
    return suf in "cz"


# ---- closed forms -----------------------------------------------------------
@pytest.mark.parametrize("suf,n", [("s", 5), ("d", 6), ("c", 4), ("z", 4)])
def test_zero_is_identity(run, suf, n):
    a = np.zeros((n, n), dtype=complex if cplx_of(suf) else float)
    st, plan, e, _, info = run.expm(a, suf, out_fill=-7.0)
    assert st.ok, st
    assert np.abs(e - np.eye(n)).max() <= elem_tol(np.eye(n), n, 64, suf)
    assert plan.m == 3 and plan.s == 0 and list(info) == [0, 0]


@pytest.mark.parametrize("suf,n,seed", [("s", 5, 1), ("d", 6, 2), ("z", 5, 3)])
def test_diagonal(run, suf, n, seed):
    rng = np.random.default_rng(seed)
    d = rng.uniform(-1, 1, n) + (1j * rng.uniform(-1, 1, n) if cplx_of(suf) else 0)
    st, _, e, _, _ = run.expm(np.diag(d), suf)
    want = np.diag(np.exp(d))
    assert st.ok
    assert np.abs(e - want).max() <= elem_tol(want, n, 128, suf)


@pytest.mark.parametrize("suf,n,seed", [("d", 5, 10), ("c", 4, 11)])
def test_nilpotent(run, suf, n, seed):
    rng = np.random.default_rng(seed)
    N = np.triu(rng.uniform(-0.5, 0.5, (n, n)), 1)
    if cplx_of(suf):
        N = N + 1j * np.triu(rng.uniform(-0.5, 0.5, (n, n)), 1)
    want, P, f = np.eye(n, dtype=N.dtype), np.eye(n, dtype=N.dtype), 1.0
    for k in range(1, n):
        P = P @ N
        f *= k
        want = want + P / f
    st, _, e, _, _ = run.expm(N, suf)
    assert st.ok
    assert np.abs(e - want).max() <= elem_tol(want, n, 128, suf)


# ---- identities ---------------------------------------------------------------
@pytest.mark.parametrize("suf,n,target,seed", [("s", 5, 0.7, 20), ("d", 6, 1.5, 21),
                                               ("z", 5, 1.2, 22)])
def test_inverse_identity(run, suf, n, target, seed):
    a = scaled_random(n, target, seed, cplx_of(suf))
    st1, _, e1, _, _ = run.expm(a, suf)
    st2, _, e2, _, _ = run.expm(-a, suf)
    assert st1.ok and st2.ok
    prod = e1.astype(np.complex128) @ e2.astype(np.complex128)
    assert np.abs(prod - np.eye(n)).max() <= elem_tol(np.eye(n), n, 256, suf)


@pytest.mark.parametrize("suf,n,target,seed", [("d", 6, 3.0, 30), ("c", 4, 2.0, 31)])
def test_half_squared(run, suf, n, target, seed):
    a = scaled_random(n, target, seed, cplx_of(suf))
    _, _, ea, _, _ = run.expm(a, suf)
    _, _, eh, _, _ = run.expm(a / 2, suf)
    sq = eh.astype(np.complex128) @ eh.astype(np.complex128)
    assert np.abs(ea - sq).max() <= elem_tol(sq, n, 256, suf)


@pytest.mark.parametrize("suf,n", [("d", 5), ("s", 5), ("z", 4)])
def test_degree_ladder_against_r13(run, suf, n):
    single = suf in "sc"
    prev, seed = 0.0, 100
    for m in (3, 5, 7, 9, 13):
        th = run.lib.calaman_pade_theta_s(m) if single else run.lib.calaman_pade_theta_d(m)
        a = scaled_random(n, 0.5 * (prev + th), seed, cplx_of(suf))
        prev, seed = th, seed + 1
        st, plan, e, _, _ = run.expm(a, suf)
        assert st.ok and plan.s == 0 and plan.m <= m
        st, r13, info = run.pade(a, 13, suf)
        assert st.ok and list(info) == [0, 0]
        assert np.abs(e - r13).max() <= elem_tol(r13, n, 256, suf)


# ---- padding, pointer mode, argument/NaN handling --------------------------------
def test_padded_output_leading_dimension(run):
    n, lde = 5, 8
    a = scaled_random(n, 1.5, 60)
    st, _, e, full, _ = run.expm(a, "d", lde=lde, out_fill=-123.5)
    assert st.ok
    pad = full.reshape(n, lde)[:, n:]
    assert np.all(pad == -123.5)
    assert np.linalg.norm(e) > 0


def test_padded_input_leading_dimension(run, oracle):
    n, lda = 37, 41
    a = gaussian_scaled(n, 7.0, 61)
    st, plan, e, _, _ = run.expm(a, "d", lda=lda, lde=n + 2)
    ref, oplan, _ = oracle.expm(a)
    assert st.ok and (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(e, ref) <= FP64_REL


def test_restores_device_pointer_mode(run):
    assert run.lib.calamanSetPointerMode(run.h, 1).ok
    st, _, _, _, _ = run.expm(scaled_random(4, 1.0, 70), "d")
    assert st.ok
    mode = ctypes.c_int(-1)
    assert run.lib.calamanGetPointerMode(run.h, ctypes.byref(mode)).ok
    assert mode.value == 1
    run.lib.calamanSetPointerMode(run.h, 0)


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_non_finite_norm_is_rejected(run, bad):
    a = scaled_random(6, 1.0, 5)
    a[3, 2] = bad
    st, _, _, _, _ = run.expm(a, "d")
    assert st.code == 7  # INVALID_VALUE


def test_short_workspace_is_rejected(run):
    st, _, _, _, _ = run.expm(scaled_random(6, 1.0, 5), "d", lwork=1024)
    assert st.code == 3  # ALLOC_FAILED


@pytest.mark.parametrize("suf", ["s", "d", "c", "z"])
def test_matrix_norm1(run, oracle, suf):
    a = scaled_random(70, 3.25, 9, cplx_of(suf))
    got = run.norm1(a, suf)
    want = oracle.norm1(a.astype(np.complex64 if suf == "c" else (np.float32 if suf == "s" else a.dtype)))
    assert got == pytest.approx(want, rel=1e-6 if suf in "sc" else 1e-14)
    b = a.copy()
    b[5, 7] = np.nan
    assert np.isnan(run.norm1(b, suf))


# ---- oracle parity --------------------------------------------------------------
@pytest.mark.parametrize("n,target", [(1, 0.3), (2, 1.0), (5, 4.0), (17, 0.01), (33, 0.2),
                                      (64, 0.9), (100, 2.0), (129, 5.0), (256, 4.0),
                                      (200, 30.0), (300, 80.0)])
def test_fp64_parity(run, oracle, n, target):
    a = gaussian_scaled(n, target, 1000 + n)
    st, plan, e, _, info = run.expm(a, "d")
    ref, oplan, oinfo = oracle.expm(a)
    assert st.ok and list(info) == [0, 0]
    assert (plan.m, plan.s, plan.num_gemms) == (oplan.m, oplan.s, oplan.num_gemms)
    assert rel_frob(e, ref) <= FP64_REL


@pytest.mark.parametrize("n,target", [(3, 0.5), (64, 50.0), (129, 12.0), (256, 50.0)])
def test_complex128_parity(run, oracle, n, target):
    a = gue_skew(n, target, 2000 + n)
    st, plan, e, _, info = run.expm(a, "z")
    ref, oplan, _ = oracle.expm(a)
    assert st.ok and list(info) == [0, 0]
    assert (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(e, ref) <= FP64_REL
    assert np.linalg.norm(e.conj().T @ e - np.eye(n)) <= 1e-12 * n  # unitary


@pytest.mark.parametrize("suf,n,target", [("s", 64, 4.0), ("s", 256, 8.0), ("s", 130, 40.0),
                                          ("c", 96, 20.0)])
def test_single_parity(run, oracle, suf, n, target):
    a = gue_skew(n, target, 3000 + n) if suf == "c" else gaussian_scaled(n, target, 3000 + n)
    a = a.astype(np.complex64 if suf == "c" else np.float32)
    st, plan, e, _, _ = run.expm(a, suf)
    ref_same_plan, oplan, _ = oracle.expm(a, single=True)
    assert st.ok and (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(e, ref_same_plan) <= SINGLE_REL


def test_golden_rational_cases(run):
    import json
    import os

    with open(os.path.join(os.path.dirname(__file__), "golden", "expm_rational.json")) as f:
        cases = json.load(f)["cases"]
    for c in cases:
        a, want = np.array(c["a"]), np.array(c["expm"])
        for suf in ("d", "z"):
            st, plan, e, _, _ = run.expm(a.astype(complex) if suf == "z" else a, suf)
            assert st.ok and (plan.m, plan.s) == (c["m"], c["s"])
            assert rel_frob(e, want) <= 1e-13


@pytest.mark.parametrize("m", [3, 5, 7, 9, 13])
@pytest.mark.parametrize("suf", ["d", "z"])
def test_pade_parity(run, oracle, m, suf):
    n = 90
    a = scaled_random(n, 0.8 * oracle.pade_theta(m), 40 + m, cplx_of(suf))
    st, r, info = run.pade(a, m, suf)
    ref, _ = oracle.pade(a, m)
    assert st.ok and list(info) == [0, 0]
    assert rel_frob(r, ref) <= FP64_REL


def test_lu_pivoting_path_large_panel(run, oracle):
    """n > one panel cluster's rows: several panels, several CTAs per cluster."""
    n = 700
    a = gaussian_scaled(n, 60.0, 77)
    st, plan, e, _, info = run.expm(a, "d")
    ref, oplan, _ = oracle.expm(a)
    assert st.ok and list(info) == [0, 0] and plan.s == oplan.s
    assert rel_frob(e, ref) <= FP64_REL
