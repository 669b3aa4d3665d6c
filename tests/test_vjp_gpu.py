"""GPU parity of expm_vjp (the adjoint of expm) through the C ABI.

Checks, per tier:
- against the oracle's numpy restatement of the same forward-mode Frechet
  evaluation (same (m, s), same product order): FP64 tiers within 1e-12
  relative Frobenius, single tiers within the single-tier bound;
- against the exact derivative, the upper-right block of the oracle's
  expm([[A^H, G], [0, A^H]]) (2n x 2n): FP64 within 1e-12;
- against a central finite difference (h = 1e-6, FP64) of <G, expm(A)> taken
  with the library's own expm, at the n = 2048 benchmark size;
- closed form: for diagonal A the derivative is G times the divided
  differences of exp;
- the expm(A) it returns equals expm's, argument checks, aliasing, padding.
"""
import ctypes

import numpy as np
import pytest

from helpers import Runner, gaussian_scaled, gue_skew, rel_frob

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
SINGLE_REL = 5e-5


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def _pair(n, target, seed, cplx):
    rng = np.random.default_rng(seed)
    a = gue_skew(n, target, seed) if cplx else gaussian_scaled(n, target, seed)
    g = rng.standard_normal((n, n))
    if cplx:
        g = g + 1j * rng.standard_normal((n, n))
    return a, g


# targets put ||A||_1 on every rung of the degree ladder (m = 3, 5, 7, 9, 13)
# and into scaling (s > 0)
LADDER = [(0.01, 3), (0.2, 5), (0.9, 7), (2.0, 9), (4.0, 13), (6.0, 13), (40.0, 13)]


@pytest.mark.parametrize("n", [1, 7, 64, 130])
@pytest.mark.parametrize("target,m", LADDER)
def test_fp64_matches_frechet_restatement(run, oracle, n, target, m):
    a, g = _pair(n, target, 4000 + n, False)
    st, plan, d, e, _, info = run.vjp(a, g, "d")
    ref, eref, oplan = oracle.expm_vjp_frechet(a, g)
    assert st.ok and list(info) == [0, 0]
    assert (plan.m, plan.s) == (oplan.m, oplan.s) and plan.m == m
    assert rel_frob(d, ref) <= FP64_REL
    assert rel_frob(e, eref) <= FP64_REL


@pytest.mark.parametrize("n,target", [(5, 0.3), (48, 6.0), (96, 50.0)])
def test_complex128_matches_frechet_and_block(run, oracle, n, target):
    a, g = _pair(n, target, 4100 + n, True)
    st, plan, d, e, _, info = run.vjp(a, g, "z")
    ref, _, oplan = oracle.expm_vjp_frechet(a, g)
    assert st.ok and list(info) == [0, 0] and (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(d, ref) <= FP64_REL
    assert rel_frob(d, oracle.expm_vjp_block(a, g)) <= FP64_REL


@pytest.mark.parametrize("n,target", [(16, 0.5), (64, 6.0), (128, 6.0), (200, 20.0)])
def test_fp64_matches_block_exact_derivative(run, oracle, n, target):
    a, g = _pair(n, target, 4200 + n, False)
    st, _, d, _, _, _ = run.vjp(a, g, "d")
    assert st.ok
    assert rel_frob(d, oracle.expm_vjp_block(a, g)) <= FP64_REL


@pytest.mark.parametrize("suf,n,target", [("s", 128, 6.0), ("s", 64, 0.5), ("s", 100, 30.0),
                                          ("c", 64, 6.0)])
def test_single_tiers(run, oracle, suf, n, target):
    a, g = _pair(n, target, 4300 + n, suf == "c")
    dt = np.complex64 if suf == "c" else np.float32
    a, g = a.astype(dt), g.astype(dt)
    st, plan, d, e, _, _ = run.vjp(a, g, suf)
    ref, eref, oplan = oracle.expm_vjp_frechet(a, g, single=True)
    assert st.ok and (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(d, ref) <= SINGLE_REL
    assert rel_frob(e, eref) <= SINGLE_REL


@pytest.mark.parametrize("suf", ["d", "z"])
def test_diagonal_divided_differences(run, suf):
    n = 24
    rng = np.random.default_rng(77)
    lam = rng.uniform(-2.0, 2.0, n)
    if suf == "z":
        lam = lam + 1j * rng.uniform(-2.0, 2.0, n)
    a = np.diag(lam)
    g = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if suf == "z" else 0)
    st, _, d, _, _, _ = run.vjp(a, g, suf)
    assert st.ok
    mu = lam.conj()  # the derivative is taken at A^H
    li, lj = np.meshgrid(mu, mu, indexing="ij")
    same = np.isclose(li, lj)
    dd = np.where(same, np.exp(li), (np.exp(li) - np.exp(lj)) / np.where(same, 1.0, li - lj))
    assert rel_frob(d, g * dd) <= 1e-13


def test_expm_output_equals_expm(run):
    a, g = _pair(96, 20.0, 4400, True)
    st, _, _, e, _, _ = run.vjp(a, g, "z")
    st2, _, e2, _, _ = run.expm(a, "z")
    assert st.ok and st2.ok
    assert rel_frob(e, e2) <= 1e-13


def test_fd_directional_derivative_2048(run):
    """The benchmark's FP64 2048 x 2048 case, ||A||_1 = 6 (m = 13, s = 1):
    <dL/dA, V> against (L(A + hV) - L(A - hV)) / 2h with L = <G, expm(A)>."""
    n, h = 2048, 1e-6
    a, g = _pair(n, 6.0, 4500, False)
    # unit-variance entries: h V moves each entry by ~1e-6 against entries of
    # ~4e-3, so the O(h^2) term stays far below the tolerance while the
    # difference stays far above the rounding of the two sums
    v = np.random.default_rng(4501).standard_normal((n, n))
    st, plan, d, _, _, _ = run.vjp(a, g, "d", want_expm=False)
    assert st.ok and (plan.m, plan.s) == (13, 1)
    lp = float(np.sum(g * run.expm(a + h * v, "d")[2]))
    lm = float(np.sum(g * run.expm(a - h * v, "d")[2]))
    fd = (lp - lm) / (2 * h)
    ad = float(np.sum(d * v))
    assert abs(fd - ad) <= 1e-6 * abs(ad)


def test_gradient_may_overwrite_g_and_padding_kept(run, oracle):
    n, ld = 40, 45
    a, g = _pair(n, 3.0, 4600, False)
    ref, _, _ = oracle.expm_vjp_frechet(a, g)
    st, _, d, _, full, _ = run.vjp(a, g, "d", ld=ld, alias_g=True)
    assert st.ok and rel_frob(d, ref) <= FP64_REL
    st, _, d, _, full, _ = run.vjp(a, g, "d", ld=ld)
    pad = full.reshape(n, ld)[:, n:]
    assert st.ok and np.all(pad == -123.5)


def test_argument_checks(run):
    a, g = _pair(8, 1.0, 4700, False)
    st, *_ = run.vjp(a, g, "d", lwork=1024)
    assert st.code == run.capi.ALLOC_FAILED
    bad = a.copy()
    bad[2, 3] = np.nan
    st, *_ = run.vjp(bad, g, "d")
    assert st.code == run.capi.INVALID_VALUE
    lib = run.lib
    st = lib.calaman_expm_vjp_d(run.h, run.h, ctypes.c_void_p(run.stream), 0, None, 1, None, 1,
                                None, 1, None, 1, None, 0, None, None)
    assert st.code == run.capi.INVALID_VALUE


def test_autograd_function_matches_torch(cuda):
    import torch

    import calaman_g_b200 as cm

    a, g = _pair(64, 5.0, 4800, True)
    x = torch.from_numpy(a).to(cuda).requires_grad_(True)
    gt = torch.from_numpy(g).to(cuda)
    (cm.expm_ad(x) * gt.conj()).real.sum().backward()
    ours = x.grad.detach().cpu().numpy()
    y = torch.from_numpy(a).to(cuda).requires_grad_(True)
    (torch.linalg.matrix_exp(y) * gt.conj()).real.sum().backward()
    assert rel_frob(ours, y.grad.detach().cpu().numpy()) <= 1e-11
