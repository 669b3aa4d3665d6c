"""The oracle's expm_herm (eigendecomposition route) against the reference's
own specification for it (test/expm/expm_tests.cpp:769-900, as the reference's
expm README summarises, src/expm/README.md:286-291): the general scaling-and-
squaring expm is the independent oracle on a self-adjoint matrix, plus the
closed forms exp(0) = I and exp(diag) = diag(exp), both triangles."""
import numpy as np
import pytest

from helpers import rel_frob


def self_adjoint(n, target, seed, cplx):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n))
    if cplx:
        x = x + 1j * rng.standard_normal((n, n))
    h = (x + x.conj().T) / 2
    return h * (target / np.abs(h).sum(axis=0).max())


@pytest.mark.parametrize("n,target,cplx,upper", [(6, 1.5, False, True), (6, 2.5, False, False),
                                                 (5, 1.5, True, True), (4, 1.0, True, False),
                                                 (64, 20.0, True, False), (200, 8.0, False, True)])
def test_vs_general_expm(oracle, n, target, cplx, upper):
    a = self_adjoint(n, target, 200 + n, cplx)
    e, _, _ = oracle.expm(a)
    assert rel_frob(oracle.expm_herm(a, upper), e) <= 1e-12


def test_reads_one_triangle(oracle):
    a = self_adjoint(9, 3.0, 7, True)
    junk_lower = np.triu(a) + np.tril(np.full((9, 9), 99.0 + 7j), -1)
    junk_upper = np.tril(a) + np.triu(np.full((9, 9), -55.0), 1)
    ref = oracle.expm_herm(a)
    assert rel_frob(oracle.expm_herm(junk_lower, upper=True), ref) <= 1e-14
    assert rel_frob(oracle.expm_herm(junk_upper, upper=False), ref) <= 1e-14


def test_closed_forms(oracle):
    assert np.allclose(oracle.expm_herm(np.zeros((5, 5))), np.eye(5), atol=0, rtol=0)
    d = np.random.default_rng(210).uniform(-1, 1, 6)
    e = oracle.expm_herm(np.diag(d))
    assert np.allclose(e, np.diag(np.exp(d)), rtol=1e-15, atol=1e-15)
