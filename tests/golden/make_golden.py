"""Generate the golden fixtures the oracle (and, through it, the GPU path) is
pinned to. Run: ``python tests/golden/make_golden.py`` (pure Python, ~1 min).

calaman_G ships no fixture files and cannot be built here, so every fixture is
derived from first principles by exact arithmetic, independently of the oracle:

* ``theta.json`` -- the backward-error thresholds theta_m for u = 2^-53 and
  u = 2^-24, re-derived the way the reference documents them
  (src/expm/README.md:84-98, src/expm/plan.cppm:43-48): the Taylor series of
  h(x) = log(exp(-x) r_m(x)) in exact rationals (log p from L' = p'/p),
  truncated at k = 200, and bisection for the root of
  sum_{k>=2m+1} |h_k| x^(k-1) = u at 60 significant digits. Also the Pade
  coefficients b_j = (2m-j)! m! / ((2m)! j! (m-j)!) as exact fractions.
* ``expm_rational.json`` -- small matrices with dyadic entries pushed through
  the reference algorithm (1-norm -> (m, s) -> scale by 2^-s -> r_m by the
  even/odd split and the degree-13 nested form -> exact Gaussian elimination
  -> s squarings) entirely in exact rational arithmetic, then rounded once.
  An FP64 restatement of the same algorithm must agree to rounding.
* ``poly_rational.json`` -- p(A) = sum c_k A^k in exact arithmetic for the
  Paterson-Stockmeyer / Horner checks.
"""
from __future__ import annotations

import json
import os
import random
from decimal import Decimal, getcontext
from fractions import Fraction
from math import factorial

HERE = os.path.dirname(os.path.abspath(__file__))
DEGREES = (3, 5, 7, 9, 13)
getcontext().prec = 60


def pade_b(m: int) -> list[Fraction]:
    return [Fraction(factorial(2 * m - j) * factorial(m),
                     factorial(2 * m) * factorial(j) * factorial(m - j)) for j in range(m + 1)]


def log_series(p: list[Fraction], order: int) -> list[Fraction]:
    """Coefficients of log p(x) (p(0) = 1) up to x^order, via L' = p'/p."""
    dp = [i * p[i] for i in range(1, len(p))] + [Fraction(0)] * order
    q = [Fraction(0)] * order  # q = p'/p, power series division
    for k in range(order):
        acc = dp[k] if k < len(dp) else Fraction(0)
        for i in range(1, min(k, len(p) - 1) + 1):
            acc -= p[i] * q[k - i]
        q[k] = acc  # p[0] == 1
    return [Fraction(0)] + [q[k - 1] / k for k in range(1, order + 1)]


def theta(m: int, u: Fraction, kmax: int = 200) -> Decimal:
    L = log_series(pade_b(m), kmax)
    # h(x) = -x + log p(x) - log p(-x): odd part doubled, minus x
    h = [Fraction(0)] * (kmax + 1)
    for k in range(1, kmax + 1):
        h[k] = (L[k] - (-1) ** k * L[k]) - (1 if k == 1 else 0)
    tail = [(k, abs(h[k])) for k in range(2 * m + 1, kmax + 1) if h[k] != 0]
    tail_d = [(k, Decimal(c.numerator) / Decimal(c.denominator)) for k, c in tail]
    ud = Decimal(u.numerator) / Decimal(u.denominator)

    def f(x: Decimal) -> Decimal:
        return sum((c * x ** (k - 1) for k, c in tail_d), Decimal(0)) - ud

    lo, hi = Decimal(0), Decimal(1)
    while f(hi) < 0:
        hi *= 2
    for _ in range(200):
        mid = (lo + hi) / 2
        if f(mid) <= 0:
            lo = mid
        else:
            hi = mid
    return lo


# ---- exact evaluation of the reference algorithm ---------------------------
def mat_mul(a, b):
    n = len(a)
    return [[sum(a[i][l] * b[l][j] for l in range(n)) for j in range(n)] for i in range(n)]


def mat_add(a, b, s=1):
    return [[a[i][j] + s * b[i][j] for j in range(len(a))] for i in range(len(a))]


def eye(n):
    return [[Fraction(int(i == j)) for j in range(n)] for i in range(n)]


def scal(c, a):
    return [[c * x for x in row] for row in a]


def solve(q, p):
    """q^-1 p by Gaussian elimination in exact arithmetic."""
    n = len(q)
    aug = [q[i][:] + p[i][:] for i in range(n)]
    for c in range(n):
        piv = next(r for r in range(c, n) if aug[r][c] != 0)
        aug[c], aug[piv] = aug[piv], aug[c]
        inv = 1 / aug[c][c]
        aug[c] = [x * inv for x in aug[c]]
        for r in range(n):
            if r != c and aug[r][c] != 0:
                f = aug[r][c]
                aug[r] = [x - f * y for x, y in zip(aug[r], aug[c])]
    return [row[n:] for row in aug]


def pade_exact(a, m):
    b = pade_b(m)
    n = len(a)
    I = eye(n)
    a2 = mat_mul(a, a)
    if m != 13:
        pw = [I, a2]
        for _ in range(2, (m - 1) // 2 + 1):
            pw.append(mat_mul(pw[-1], a2))
        V = [[Fraction(0)] * n for _ in range(n)]
        W = [[Fraction(0)] * n for _ in range(n)]
        for i, P in enumerate(pw):
            V = mat_add(V, scal(b[2 * i], P))
            W = mat_add(W, scal(b[2 * i + 1], P))
    else:
        a4 = mat_mul(a2, a2)
        a6 = mat_mul(a4, a2)
        X = mat_add(mat_add(scal(b[9], a2), scal(b[11], a4)), scal(b[13], a6))
        W = mat_add(mat_add(mat_add(scal(b[1], I), scal(b[3], a2)), scal(b[5], a4)), scal(b[7], a6))
        W = mat_add(W, mat_mul(a6, X))
        X = mat_add(mat_add(scal(b[8], a2), scal(b[10], a4)), scal(b[12], a6))
        V = mat_add(mat_add(mat_add(scal(b[0], I), scal(b[2], a2)), scal(b[4], a4)), scal(b[6], a6))
        V = mat_add(V, mat_mul(a6, X))
    U = mat_mul(a, W)
    return solve(mat_add(V, U, -1), mat_add(V, U))


def plan(norm: Fraction, thetas: dict[int, float]):
    for m in DEGREES:
        if norm <= Fraction(thetas[m]):
            return m, 0
    s = 0
    while norm / 2 ** s > Fraction(thetas[13]):
        s += 1
    return 13, s


def expm_exact(a, thetas):
    n = len(a)
    norm = max(sum(abs(a[i][j]) for i in range(n)) for j in range(n))
    m, s = plan(norm, thetas)
    As = scal(Fraction(1, 2 ** s), a)
    X = pade_exact(As, m)
    for _ in range(s):
        X = mat_mul(X, X)
    return X, m, s


def dyadic_matrix(rng, n, target, bits=10):
    """Entries k/2^bits scaled by a power of two so the 1-norm is near target."""
    a = [[Fraction(rng.randint(-(2 ** bits), 2 ** bits), 2 ** bits) for _ in range(n)]
         for _ in range(n)]
    norm = max(sum(abs(a[i][j]) for i in range(n)) for j in range(n))
    e = 0
    while norm * Fraction(2) ** e > target * 1.5:
        e -= 1
    while norm * Fraction(2) ** e < target / 1.5:
        e += 1
    return scal(Fraction(2) ** e, a)


def main() -> None:
    out = {"u_double": "2^-53", "u_single": "2^-24", "kmax": 200, "digits": 60, "theta": {},
           "pade_b": {}}
    for m in DEGREES:
        out["theta"][str(m)] = {"double": str(theta(m, Fraction(1, 2 ** 53))),
                                "single": str(theta(m, Fraction(1, 2 ** 24)))}
        out["pade_b"][str(m)] = [f"{x.numerator}/{x.denominator}" for x in pade_b(m)]
    with open(os.path.join(HERE, "theta.json"), "w") as f:
        json.dump(out, f, indent=1)
    thetas_d = {m: float(Decimal(out["theta"][str(m)]["double"])) for m in DEGREES}

    rng = random.Random(20261203)
    cases = []
    # one case per rung (no scaling), and a few past theta_13 (scaled)
    targets = [0.01, 0.2, 0.8, 1.8, 4.5, 9.0, 20.0, 45.0]
    for i, tgt in enumerate(targets):
        n = 4 if tgt < 20 else 3
        a = dyadic_matrix(rng, n, tgt)
        X, m, s = expm_exact(a, thetas_d)
        cases.append({"n": n, "a": [[float(x) for x in row] for row in a],
                      "m": m, "s": s, "expm": [[float(x) for x in row] for row in X]})
    with open(os.path.join(HERE, "expm_rational.json"), "w") as f:
        json.dump({"column_major": False, "note": "row lists; a[i][j] is row i, column j",
                   "cases": cases}, f, indent=1)

    poly = []
    for n, degree in ((4, 4), (5, 7), (3, 9), (4, 0), (4, 1)):
        a = [[Fraction(rng.randint(-32, 32), 64) for _ in range(n)] for _ in range(n)]
        c = [Fraction(rng.randint(-64, 64), 64) for _ in range(degree + 1)]
        P = scal(c[0], eye(n))
        Ak = eye(n)
        for k in range(1, degree + 1):
            Ak = mat_mul(Ak, a)
            P = mat_add(P, scal(c[k], Ak))
        poly.append({"n": n, "degree": degree, "a": [[float(x) for x in r] for r in a],
                     "c": [float(x) for x in c], "p": [[float(x) for x in r] for r in P]})
    with open(os.path.join(HERE, "poly_rational.json"), "w") as f:
        json.dump({"cases": poly}, f, indent=1)


if __name__ == "__main__":
    main()
