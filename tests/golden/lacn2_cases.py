"""Seeded operators for the 1-norm estimator (xLACN2) fixtures and tests.

Each case is (name, kind, n, seed, single). ``make_matrix`` builds the dense
matrix the reverse-communication loop multiplies by; the estimator itself
never sees it. The classes follow the reference's lacn2 suite
(src/lapack/lacn2/README.md:40-47): n = 1, diagonal, nonnegative and
one-dominant-column matrices (where Hager's method is exact), general
Gaussian matrices (where it may underestimate), and edge cases (zero matrix,
rows summing to zero so A e = 0 and the sign test meets +0, a NaN entry).
"""
from __future__ import annotations

import numpy as np

CASES = [
    ("n1", "gauss", 1, 11, False),
    ("n2", "gauss", 2, 12, False),
    ("gauss5", "gauss", 5, 1, False),
    ("gauss50", "gauss", 50, 13, False),
    ("gauss333", "gauss", 333, 14, False),
    ("gauss1000", "gauss", 1000, 15, False),
    ("diag40", "diag", 40, 16, False),
    ("nonneg60", "nonneg", 60, 17, False),
    ("dominant45", "dominant", 45, 18, False),
    ("zero7", "zero", 7, 19, False),
    ("rowsum0_30", "rowsum0", 30, 20, False),
    ("nan12", "nan", 12, 21, False),
    ("lowrank80", "lowrank", 80, 22, False),
    ("s_gauss64", "gauss", 64, 31, True),
    ("s_gauss500", "gauss", 500, 32, True),
    ("s_nonneg33", "nonneg", 33, 33, True),
] + [(f"gauss30_{k}", "gauss", 30, 100 + k, False) for k in range(12)]


def make_matrix(kind: str, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if kind == "gauss":
        return rng.standard_normal((n, n))
    if kind == "diag":
        return np.diag(rng.standard_normal(n))
    if kind == "nonneg":
        return np.abs(rng.standard_normal((n, n)))
    if kind == "dominant":
        a = 0.01 * rng.standard_normal((n, n))
        a[:, n // 3] += 10.0 * rng.standard_normal(n)
        return a
    if kind == "zero":
        return np.zeros((n, n))
    if kind == "rowsum0":
        a = rng.standard_normal((n, n))
        a[:, -1] = -a[:, :-1].sum(axis=1)
        # A e is zero only up to rounding; make it exactly zero row by row
        a[:, -1] = -np.array([np.sum(a[i, :-1]) for i in range(n)])
        return a
    if kind == "nan":
        a = rng.standard_normal((n, n))
        a[3, 5] = np.nan
        return a
    if kind == "lowrank":
        u = rng.standard_normal((n, 2))
        w = rng.standard_normal((2, n))
        return u @ w
    raise ValueError(kind)


def operators(a: np.ndarray):
    """A x and A^T x in float64, summed in index order (so every caller,
    CPU or GPU test, hands the estimator the same vectors)."""
    def apply(x):
        return np.array([float(np.sum(a[i, :] * x)) for i in range(a.shape[0])])

    def apply_t(x):
        return np.array([float(np.sum(a[:, j] * x)) for j in range(a.shape[1])])

    return apply, apply_t
