"""The oracle's scaling half of gebal against the reference's own specification
(test/gebal/gebal_tests.cpp, as the reference's gebal README lists it): the
analytic 2x2, exact reproduction of A from (B, D), and stationarity of a second
pass; and the balanced expm against the plain one."""
import numpy as np

from helpers import rel_frob


def badly_scaled(n, seed, spread=12, cplx=False):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    if cplx:
        a = a + 1j * rng.standard_normal((n, n))
    d = 2.0 ** rng.integers(-spread, spread + 1, n)
    return (a * d[:, None]) / d[None, :]


def test_analytic_2x2(oracle):
    b, d, _ = oracle.gebal_scale(np.array([[1.0, 2.0 ** 10], [2.0 ** -10, 1.0]]))
    assert np.array_equal(b, np.ones((2, 2)))
    assert np.array_equal(d, [2.0 ** 10, 1.0])


def test_exact_reproduce_and_stationarity(oracle):
    for n, cplx in ((1, False), (7, False), (40, True), (130, False)):
        a = badly_scaled(n, 5 + n, cplx=cplx)
        b, d, _ = oracle.gebal_scale(a)
        assert np.array_equal(b * d[:, None] / d[None, :], a)  # powers of two: exact
        assert np.all(np.log2(d) == np.round(np.log2(d)))
        b2, d2, sweeps = oracle.gebal_scale(b)
        assert np.array_equal(b2, b) and np.all(d2 == 1.0) and sweeps == 1


def test_balanced_expm_removes_squarings(oracle):
    a = badly_scaled(40, 9)
    e_bal, plan_bal = oracle.expm_balanced(a)
    e, plan, _ = oracle.expm(a)
    assert plan_bal.s < plan.s
    # balancing is a similarity: same exponential up to the accuracy of the
    # unbalanced evaluation (many more squarings)
    assert rel_frob(e_bal, e) <= 1e-3
