"""GPU parity of expm_vjp_batched through the C ABI: every pair of a batch of
mixed sizes and norms against the oracle's restatement of the adjoint (FP64
within 1e-12, FP32 tier within the single-tier bound) and against the
one-pair entry point; padding, optional expm outputs, argument checks."""
import numpy as np
import pytest

from helpers import Runner, gaussian_scaled, rel_frob, run_vjp_batched

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
SINGLE_REL = 5e-5


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def pairs_of(cases, seed):
    out = []
    for i, (n, t) in enumerate(cases):
        a = gaussian_scaled(n, t, seed + i)
        g = np.random.default_rng(seed + 1000 + i).standard_normal((n, n))
        out.append((a, g))
    return out


CASES = [(1, 0.3), (3, 0.01), (16, 0.2), (31, 0.9), (40, 2.0), (64, 5.0), (65, 6.0),
         (100, 30.0), (128, 6.0), (200, 1.5), (256, 12.0)]


def test_fp64_batch_matches_oracle(run, oracle):
    pairs = pairs_of(CASES, 500)
    st, plans, grads, exps, _, info = run_vjp_batched(run, pairs, "d")
    assert st.ok, st
    assert (info == 0).all()
    for (a, g), d, e, p in zip(pairs, grads, exps, plans):
        ref, eref, op = oracle.expm_vjp_frechet(a, g)
        assert (p.m, p.s) == (op.m, op.s)
        assert rel_frob(d, ref) <= FP64_REL, (a.shape[0], p.m, p.s)
        assert rel_frob(e, eref) <= FP64_REL


def test_fp64_batch_matches_single_pair_entry(run):
    pairs = pairs_of(CASES[:6], 600)
    st, _, grads, _, _, _ = run_vjp_batched(run, pairs, "d", want_expm=False)
    assert st.ok
    for (a, g), d in zip(pairs, grads):
        st1, _, d1, _, _, _ = run.vjp(a, g, "d", want_expm=False)
        assert st1.ok and rel_frob(d, d1) <= 1e-13


def test_fp32_batch_matches_oracle(run, oracle):
    pairs = [(a.astype(np.float32), g.astype(np.float32)) for a, g in pairs_of(CASES, 700)]
    st, plans, grads, exps, _, _ = run_vjp_batched(run, pairs, "s")
    assert st.ok
    for (a, g), d, e, p in zip(pairs, grads, exps, plans):
        ref, eref, op = oracle.expm_vjp_frechet(a, g, single=True)
        assert (p.m, p.s) == (op.m, op.s)
        assert rel_frob(d, ref) <= SINGLE_REL, (a.shape[0], p.m, p.s)
        assert rel_frob(e, eref) <= SINGLE_REL


def test_padding_and_argument_checks(run):
    pairs = pairs_of([(7, 1.0), (40, 3.0)], 800)
    st, _, _, _, fulls, _ = run_vjp_batched(run, pairs, "d", lds=[9, 44])
    assert st.ok
    for (a, _), f, ld in zip(pairs, fulls, [9, 44]):
        n = a.shape[0]
        assert np.all(f.reshape(n, ld)[:, n:] == -123.5)
    st, *_ = run_vjp_batched(run, pairs_of([(257, 1.0)], 900), "d")
    assert st.code == run.capi.NOT_SUPPORTED
    bad = pairs_of([(8, 1.0), (9, 1.0)], 910)
    bad[1][0][2, 2] = np.nan
    st, _, grads, _, _, _ = run_vjp_batched(run, bad, "d")
    assert st.code == run.capi.INVALID_VALUE
    assert all(np.all(d == -123.5) for d in grads)
    st, *_ = run_vjp_batched(run, pairs, "d", lwork=256)
    assert st.code == run.capi.ALLOC_FAILED
