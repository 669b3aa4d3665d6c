"""The oracle's adjoint of expm, pinned without a GPU: its forward-mode
Frechet restatement against the exact derivative (Mathias' block formula
through the oracle expm), against central finite differences of the oracle
expm, and against the closed form for diagonal matrices."""
import numpy as np
import pytest

from helpers import gaussian_scaled, gue_skew, rel_frob


@pytest.mark.parametrize("target,m,s", [(0.01, 3, 0), (0.2, 5, 0), (0.9, 7, 0), (2.0, 9, 0),
                                        (4.0, 13, 0), (6.0, 13, 1), (40.0, 13, 3)])
@pytest.mark.parametrize("cplx", [False, True])
def test_frechet_restatement_equals_block(oracle, target, m, s, cplx):
    n = 12
    a = gue_skew(n, target, 11) if cplx else gaussian_scaled(n, target, 11)
    rng = np.random.default_rng(12)
    g = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    d, e, plan = oracle.expm_vjp_frechet(a, g)
    assert (plan.m, plan.s) == (m, s)
    assert rel_frob(d, oracle.expm_vjp_block(a, g)) <= 1e-13
    assert rel_frob(e, oracle.expm(a)[0]) <= 1e-13


@pytest.mark.parametrize("cplx", [False, True])
def test_block_matches_central_difference(oracle, cplx):
    n, h = 10, 1e-6
    a = gue_skew(n, 6.0, 21) if cplx else gaussian_scaled(n, 6.0, 21)
    rng = np.random.default_rng(22)
    g = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    v = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)

    def loss(x):
        return float(np.real(np.vdot(g, oracle.expm(x)[0])))

    fd = (loss(a + h * v) - loss(a - h * v)) / (2 * h)
    ad = float(np.real(np.vdot(oracle.expm_vjp_block(a, g), v)))
    assert abs(fd - ad) <= 1e-7 * abs(ad)


def test_diagonal_closed_form(oracle):
    lam = np.array([-1.5, -0.25, 0.0, 0.75, 1.25, 2.0])
    g = np.arange(36, dtype=float).reshape(6, 6) - 17.0
    li, lj = np.meshgrid(lam, lam, indexing="ij")
    same = li == lj
    dd = np.where(same, np.exp(li), (np.exp(li) - np.exp(lj)) / np.where(same, 1.0, li - lj))
    d, _, _ = oracle.expm_vjp_frechet(np.diag(lam), g)
    assert rel_frob(d, g * dd) <= 1e-14
