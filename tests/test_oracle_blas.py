"""The timing restatement of the CPU baseline (CPU only).

oracle.expm_blas runs the reference's scaling and squaring with its products
on numpy's BLAS and its solve on LAPACK xGESV: the form the reference's own
CPU path takes (GEMM through BLAS, LU through LAPACK). It must pick the same
(m, s) as the oracle and agree with it to rounding, and it must reproduce the
exact rational evaluations of the golden fixture like the oracle does.
"""
import json
import os

import numpy as np
import pytest

from helpers import scaled_random

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("n,target", [(1, 0.5), (6, 0.01), (6, 2.0), (40, 5.0), (40, 60.0), (150, 400.0)])
def test_same_plan_and_result_as_oracle(oracle, n, target, cplx, single):
    a = scaled_random(n, target, 9000 + n, cplx)
    e, plan, _ = oracle.expm(a, single)
    f, plan_b = oracle.expm_blas(a, single)
    assert (plan_b.m, plan_b.s) == (plan.m, plan.s)
    assert np.linalg.norm(f - e) <= 1e-13 * max(1, plan.s) * np.linalg.norm(e)


def test_exact_rational_evaluation():
    from oracle import oracle as O

    with open(os.path.join(GOLDEN, "expm_rational.json")) as fh:
        cases = json.load(fh)["cases"]
    for case in cases:
        a = np.array(case["a"])
        want = np.array(case["expm"])
        got, plan = O.expm_blas(a)
        assert (plan.m, plan.s) == (case["m"], case["s"])
        assert np.linalg.norm(got - want) <= 1e-14 * np.linalg.norm(want) * max(1, case["s"] * 4)


def test_balanced_and_geodesic_variants(oracle):
    rng = np.random.default_rng(5)
    n = 24
    d = 2.0 ** rng.integers(-12, 12, n)
    a = (rng.standard_normal((n, n)) * d[:, None] / d[None, :])
    e, plan = oracle.expm_balanced(a)
    f, plan_b = oracle.expm_balanced(a, blas=True)
    assert (plan.m, plan.s) == (plan_b.m, plan_b.s)
    assert np.linalg.norm(f - e) <= 1e-12 * np.linalg.norm(e)
    h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = (h - h.conj().T) / 2  # skew-Hermitian: exp(step h) is unitary
    w = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0]
    ref = oracle.geodesic_points(w, h, 0.3, 5)
    got = oracle.geodesic_points(w, h, 0.3, 5, blas=True)
    assert len(got) == len(ref) == 4
    for g, r in zip(got, ref):
        assert np.linalg.norm(g - r) <= 1e-13 * np.linalg.norm(r)
