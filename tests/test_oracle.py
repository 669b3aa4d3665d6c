"""Pin the CPU oracle to the reference's known answers (CPU only).

Each check cites the calaman_G test or table it restates; the golden fixtures
under tests/golden/ come from exact-arithmetic derivations (make_golden.py).
"""
import json
import os
from decimal import Decimal
from fractions import Fraction

import numpy as np
import pytest
import scipy.linalg

from helpers import elem_tol, gue_skew, scaled_random

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DEGREES = (3, 5, 7, 9, 13)


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


# ---- tables ---------------------------------------------------------------
def test_pade_coefficients_match_factorial_formula(oracle):
    """b_j = (2m-j)! m! / ((2m)! j! (m-j)!) (src/expm/expm_bridge.h:58-91)."""
    g = load("theta.json")["pade_b"]
    for m in DEGREES:
        got = oracle.pade_coeffs(m)
        want = [float(Fraction(s)) for s in g[str(m)]]
        assert got == want, m
    assert oracle.pade_coeffs(4) is None and oracle.pade_coeffs(11) is None


def test_theta_table_matches_exact_rederivation(oracle):
    """theta_m re-derived from the backward-error series at 60 digits."""
    g = load("theta.json")["theta"]
    for m in DEGREES:
        d = float(Decimal(g[str(m)]["double"]))
        s = float(np.float32(float(Decimal(g[str(m)]["single"]))))
        assert oracle.pade_theta(m) == pytest.approx(d, rel=2e-16), m
        assert oracle.pade_theta(m, single=True) == s, m


def test_theta_off_ladder_and_monotone(oracle):
    """test/expm/expm_tests.cpp:423-435"""
    assert oracle.pade_theta(4) == 0.0 and oracle.pade_theta(0) == 0.0
    assert oracle.pade_theta(11, single=True) == 0.0
    th = [oracle.pade_theta(m) for m in DEGREES]
    assert th == sorted(th) and len(set(th)) == 5


@pytest.mark.parametrize("single", [False, True])
def test_plan_ladder(oracle, single):
    """check_plan_ladder, test/expm/expm_tests.cpp:389-421"""
    want = {3: 2, 5: 3, 7: 4, 9: 5, 13: 6}
    for m in DEGREES:
        p = oracle.expm_plan(oracle.pade_theta(m, single) * 0.99, single)
        assert p.s == 0 and p.m <= m and p.num_gemms == want[p.m]
    assert oracle.expm_plan(oracle.pade_theta(13, single), single).s == 0
    big = oracle.expm_plan(oracle.pade_theta(13, single) * 40, single)
    assert big.m == 13 and big.s > 0 and big.num_gemms == 6 + big.s
    assert [oracle.pade_num_gemms(m) for m in DEGREES] == [2, 3, 4, 5, 6]
    assert [oracle.pade_num_powers(m) for m in DEGREES] == [1, 2, 3, 4, 3]


# ---- Paterson-Stockmeyer plan (test/paterson_stockmeyer/paterson_stockmeyer_tests.cpp:235-291)
def test_ps_cost_table(oracle):
    assert [oracle.ps_plan(d).num_gemms for d in (4, 8, 16, 30)] == [3, 4, 7, 10]
    p12 = oracle.ps_plan(12)
    assert (p12.s, p12.num_gemms, p12.num_blocks) == (3, 6, 3)


def test_ps_edges(oracle):
    p0, p1, p2 = oracle.ps_plan(0), oracle.ps_plan(1), oracle.ps_plan(2)
    assert (p0.num_gemms, p0.num_blocks) == (0, 0)
    assert (p1.s, p1.num_gemms, p1.num_blocks) == (2, 0, 0)
    assert (p2.s, p2.num_gemms) == (3, 1)


def test_ps_argmin_through_32(oracle):
    for d in range(1, 33):
        best = oracle.ps_plan(d).num_gemms
        assert best <= d
        assert all(best <= oracle.ps_cost(d, s) for s in range(1, d + 2))
        assert best == oracle.ps_cost(d, oracle.ps_plan(d).s)


def test_ps_override_clamp(oracle):
    assert oracle.ps_plan(10, 1).num_gemms == 10
    assert oracle.ps_plan(5, 999).s == 6
    assert oracle.ps_plan(9, 4).s == 4


# ---- golden: the reference algorithm in exact arithmetic ------------------
def test_expm_matches_exact_rational_evaluation(oracle):
    for case in load("expm_rational.json")["cases"]:
        a = np.array(case["a"])
        want = np.array(case["expm"])
        got, plan, info = oracle.expm(a)
        assert (plan.m, plan.s) == (case["m"], case["s"])
        assert info == 0
        assert np.linalg.norm(got - want) <= 1e-14 * np.linalg.norm(want) * max(1, case["s"] * 4)


def test_poly_matches_exact_rational_evaluation(oracle):
    for case in load("poly_rational.json")["cases"]:
        a, c, want = np.array(case["a"]), np.array(case["c"]), np.array(case["p"])
        tol = 1e-14 * max(1.0, np.abs(want).max())
        assert np.abs(oracle.paterson_stockmeyer(a, c) - want).max() <= tol
        assert np.abs(oracle.horner(a, c) - want).max() <= tol


# ---- closed forms and identities (test/expm/expm_tests.cpp:471-698) --------
def test_exp_zero_is_identity(oracle):
    for cplx in (False, True):
        a = np.zeros((6, 6), dtype=complex if cplx else float)
        e, plan, _ = oracle.expm(a)
        assert np.array_equal(e, np.eye(6))


def test_exp_diagonal(oracle):
    rng = np.random.default_rng(2)
    for cplx in (False, True):
        d = rng.uniform(-1, 1, 6) + (1j * rng.uniform(-1, 1, 6) if cplx else 0)
        e, _, _ = oracle.expm(np.diag(d))
        want = np.diag(np.exp(d))
        assert np.abs(e - want).max() <= elem_tol(want, 6, 128, "d")


def test_exp_nilpotent(oracle):
    rng = np.random.default_rng(10)
    n = 5
    N = np.triu(rng.uniform(-0.5, 0.5, (n, n)), 1)
    want = np.eye(n)
    P = np.eye(n)
    f = 1.0
    for k in range(1, n):
        P = P @ N
        f *= k
        want = want + P / f
    e, _, _ = oracle.expm(N)
    assert np.abs(e - want).max() <= elem_tol(want, n, 128, "d")


@pytest.mark.parametrize("cplx", [False, True])
def test_inverse_identity(oracle, cplx):
    a = scaled_random(6, 1.5, 21, cplx)
    e1, _, _ = oracle.expm(a)
    e2, _, _ = oracle.expm(-a)
    assert np.abs(e1 @ e2 - np.eye(6)).max() <= elem_tol(np.eye(6), 6, 256, "d")


def test_half_squared(oracle):
    a = scaled_random(6, 3.0, 30)
    ea, _, _ = oracle.expm(a)
    eh, _, _ = oracle.expm(a / 2)
    sq = eh @ eh
    assert np.abs(ea - sq).max() <= elem_tol(sq, 6, 256, "d")


@pytest.mark.parametrize("cplx", [False, True])
def test_degree_ladder_against_r13(oracle, cplx):
    prev = 0.0
    seed = 100
    for m in DEGREES:
        th = oracle.pade_theta(m)
        a = scaled_random(5, 0.5 * (prev + th), seed, cplx)
        prev = th
        seed += 1
        e, plan, _ = oracle.expm(a)
        assert plan.s == 0 and plan.m <= m
        r13, _ = oracle.pade(a, 13)
        assert np.abs(e - r13).max() <= elem_tol(r13, 5, 256, "d")


def test_norm1_is_true_modulus_and_nan_sticky(oracle):
    a = np.array([[3 + 4j, 0], [0, 1]])
    assert oracle.norm1(a) == 5.0
    b = np.ones((4, 4))
    b[2, 1] = np.nan
    assert np.isnan(oracle.norm1(b))
    with pytest.raises(FloatingPointError):
        oracle.expm(b)


# ---- an independent algorithm as a sanity check ---------------------------
@pytest.mark.parametrize("n,target,cplx", [(32, 4.0, False), (48, 50.0, True), (20, 0.05, False),
                                           (64, 9.0, False)])
def test_against_scipy(oracle, n, target, cplx):
    """scipy.linalg.expm (Al-Mohy & Higham 2009) is a different method; the two
    agree to a few ulps on well-conditioned inputs."""
    a = gue_skew(n, target, 7) if cplx else scaled_random(n, target, 8)
    e, _, _ = oracle.expm(a)
    ref = scipy.linalg.expm(a)
    assert np.linalg.norm(e - ref) <= 1e-13 * np.linalg.norm(ref)


def test_lu_matches_scipy_factorization(oracle):
    rng = np.random.default_rng(4)
    for n in (1, 7, 64, 130):
        a = rng.standard_normal((n, n))
        lu, piv, info = oracle.getrf(a)
        ref_lu, ref_piv = scipy.linalg.lu_factor(a)
        assert info == 0
        assert np.array_equal(piv, ref_piv)
        assert np.abs(lu - ref_lu).max() <= 1e-12 * max(1, np.abs(ref_lu).max())


def test_thread_count_does_not_change_results(oracle):
    a = gue_skew(96, 30.0, 3)
    oracle.set_threads(1)
    e1, _, _ = oracle.expm(a)
    oracle.set_threads(4)
    e4, _, _ = oracle.expm(a)
    oracle.set_threads(1)
    assert np.array_equal(e1, e4)


def test_ps_all_block_sizes_and_horner(oracle):
    rng = np.random.default_rng(77)
    n, degree = 5, 7
    a = rng.uniform(-0.5, 0.5, (n, n))
    c = rng.uniform(-1, 1, degree + 1)
    series = sum(c[k] * np.linalg.matrix_power(a, k) for k in range(degree + 1))
    for s in range(1, degree + 2):
        assert np.abs(oracle.paterson_stockmeyer(a, c, s) - series).max() < 1e-14
    assert np.abs(oracle.horner(a, c) - series).max() < 1e-14
