"""GPU parity of expm_herm and of the eigensolver behind it (calaman_heevd_*)
through the C ABI.

expm_herm is checked the way the reference checks it (test/expm/expm_tests.cpp:
769-900): against the general scaling-and-squaring expm on the same
self-adjoint matrix (here the oracle's), the closed forms exp(0) = I and
exp(diag) = diag(exp), both triangles, a padded output leading dimension and
host-side argument rejection -- and, beyond that, against the oracle's
eigendecomposition route (LAPACK xHEEVD through numpy) at the sizes of the
benchmark, including the complex128 1024 x 1024 GUE case. The eigensolver is
checked on its own: eigenvalues against LAPACK's, the residual ||A U - U W||
and the orthogonality ||U^H U - I||, on inputs that exercise every deflation
path (repeated eigenvalues, a zero matrix, a diagonal, clusters) and the range
scaling (entries of 1e-200 and 1e+200).
"""
import numpy as np
import pytest

from helpers import Runner, rel_frob

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
SINGLE_REL = 2e-6


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def self_adjoint(n, target, seed, cplx):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n))
    if cplx:
        x = x + 1j * rng.standard_normal((n, n))
    h = (x + x.conj().T) / 2
    return h * (target / np.abs(h).sum(axis=0).max())


def _dt(suf):
    return {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}[suf]


@pytest.mark.parametrize("suf,n,target,upper", [("d", 6, 1.5, True), ("d", 6, 2.5, False),
                                                ("s", 5, 1.0, True), ("z", 5, 1.5, True),
                                                ("c", 4, 1.0, False)])
def test_vs_general_expm_small(run, oracle, suf, n, target, upper):
    a = self_adjoint(n, target, 200 + n, suf in "cz").astype(_dt(suf))
    st, e, _, info = run.expm_herm(a, suf, upper=upper)
    assert st.ok and info == 0
    ref, _, _ = oracle.expm(a.astype(np.complex128 if suf in "cz" else np.float64))
    assert rel_frob(e, ref) <= (FP64_REL if suf in "dz" else SINGLE_REL)


@pytest.mark.parametrize("suf", ["d", "z"])
@pytest.mark.parametrize("n", [1, 2, 3, 17, 64, 65, 129, 256, 300, 513])
def test_matches_eigen_route(run, oracle, suf, n):
    a = self_adjoint(n, 10.0, 300 + n, suf == "z")
    st, e, _, info = run.expm_herm(a, suf)
    assert st.ok and info == 0
    assert rel_frob(e, oracle.expm_herm(a)) <= FP64_REL


@pytest.mark.parametrize("suf", ["s", "c"])
def test_single_tiers(run, oracle, suf):
    a = self_adjoint(200, 10.0, 77, suf == "c").astype(_dt(suf))
    st, e, _, info = run.expm_herm(a, suf, upper=True)
    assert st.ok and info == 0
    ref = oracle.expm_herm(a.astype(np.complex128 if suf == "c" else np.float64), upper=True)
    assert rel_frob(e, ref) <= SINGLE_REL


def test_gue_1024_benchmark_shape(run, oracle):
    """complex128 1024 x 1024 GUE Hermitian, ||H||_1 = 50 (the headline shape)."""
    a = self_adjoint(1024, 50.0, 2024, True)
    st, e, _, info = run.expm_herm(a, "z")
    assert st.ok and info == 0
    ref = oracle.expm_herm(a)
    assert rel_frob(e, ref) <= FP64_REL


@pytest.mark.parametrize("suf", ["d", "z"])
def test_reads_only_its_triangle(run, suf):
    a = self_adjoint(40, 4.0, 41, suf == "z")
    junk = np.full((40, 40), 1e3 + (3e2j if suf == "z" else 0))
    st, lower, _, _ = run.expm_herm(np.tril(a) + np.triu(junk, 1), suf, upper=False)
    st2, upper, _, _ = run.expm_herm(np.triu(a) + np.tril(junk, -1), suf, upper=True)
    assert st.ok and st2.ok
    assert rel_frob(lower, upper) <= 1e-13


@pytest.mark.parametrize("suf", ["d", "z"])
def test_closed_forms(run, suf):
    st, e, _, info = run.expm_herm(np.zeros((5, 5), dtype=_dt(suf)), suf)
    assert st.ok and info == 0 and np.abs(e - np.eye(5)).max() <= 64 * 2.2e-16
    d = np.random.default_rng(210).uniform(-1, 1, 6)
    st, e, _, _ = run.expm_herm(np.diag(d).astype(_dt(suf)), suf, upper=False)
    assert st.ok and np.abs(e - np.diag(np.exp(d))).max() <= 128 * 2.2e-16


def test_padded_output_leading_dimension(run, oracle):
    a = self_adjoint(5, 1.5, 220, False)
    st, e, full, _ = run.expm_herm(a, "d", lde=8)
    assert st.ok and rel_frob(e, oracle.expm_herm(a)) <= FP64_REL
    assert np.all(full.reshape(5, 8)[:, 5:] == -123.5)


def test_argument_checks(run):
    import ctypes

    lib, h, cap = run.lib, run.h, run.capi
    b = ctypes.c_size_t()
    assert lib.calaman_expm_herm_bufferSize_d(h, cap.FILL_LOWER, 0, ctypes.byref(b)).code == cap.INVALID_VALUE
    assert lib.calaman_expm_herm_bufferSize_d(h, 7, 4, ctypes.byref(b)).code == cap.INVALID_VALUE
    buf = ctypes.c_void_p(1 << 20)  # never dereferenced: every call below returns before device work
    f = lib.calaman_expm_herm_d
    s = ctypes.c_void_p(run.stream)
    assert f(h, h, s, cap.FILL_UPPER, 0, buf, 4, buf, 4, buf, 1 << 20, None).code == cap.INVALID_VALUE
    assert f(h, h, s, cap.FILL_UPPER, 4, buf, 3, buf, 4, buf, 1 << 20, ctypes.cast(buf, cap.c_int_p)).code == cap.INVALID_VALUE
    assert f(h, h, s, cap.FILL_UPPER, 4, buf, 4, buf, 3, buf, 1 << 20, ctypes.cast(buf, cap.c_int_p)).code == cap.INVALID_VALUE
    assert f(h, h, s, cap.FILL_UPPER, 4, buf, 4, buf, 4, None, 1 << 20, ctypes.cast(buf, cap.c_int_p)).code == cap.INVALID_VALUE
    assert f(h, h, s, cap.FILL_UPPER, 4, buf, 4, buf, 4, buf, 16, ctypes.cast(buf, cap.c_int_p)).code == cap.ALLOC_FAILED


def _check_eig(a, w, u, wref, tol_w, tol_r):
    n = a.shape[0]
    h = a
    scale = max(np.abs(wref).max(), 1e-300)
    assert np.abs(w - wref).max() <= tol_w * scale
    # residual of the scaled problem (entries of 1e+200 would overflow the norm)
    assert np.linalg.norm((h / scale) @ u - u * (w / scale)) <= tol_r * n
    assert np.linalg.norm(u.conj().T @ u - np.eye(n)) <= tol_r * n


@pytest.mark.parametrize("suf", ["d", "z"])
@pytest.mark.parametrize("n", [1, 5, 31, 100, 257, 1000])
def test_heevd_random(run, oracle, suf, n):
    a = self_adjoint(n, 5.0, 500 + n, suf == "z")
    st, w, u, info = run.heevd(a, suf, upper=(n % 2 == 0))
    assert st.ok and info == 0
    h = oracle.hermitian_from_triangle(a, n % 2 == 0)
    wref, _ = oracle.heevd(a, n % 2 == 0)
    _check_eig(h, w, u, wref, 1e-13, 1e-15)


@pytest.mark.parametrize("case", ["zero", "identity", "diag", "repeated", "clusters", "tiny", "huge"])
def test_heevd_structured(run, oracle, case):
    rng = np.random.default_rng(7)
    n = 96
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    if case == "zero":
        a = np.zeros((n, n))
    elif case == "identity":
        a = np.eye(n)
    elif case == "diag":
        a = np.diag(rng.standard_normal(n))
    elif case == "repeated":
        a = q @ np.diag(np.repeat([1.0, -2.0, 3.0], n // 3)) @ q.T
    elif case == "clusters":
        a = q @ np.diag(np.concatenate([1 + 1e-12 * rng.standard_normal(n // 2),
                                        rng.standard_normal(n - n // 2)])) @ q.T
    elif case == "tiny":
        a = 1e-200 * self_adjoint(n, 5.0, 9, False)
    else:
        a = 1e200 * self_adjoint(n, 5.0, 9, False)
    a = (a + a.T) / 2
    st, w, u, info = run.heevd(a, "d")
    assert st.ok and info == 0
    wref, _ = oracle.heevd(a)
    _check_eig(a, w, u, wref, 1e-13, 1e-15)


@pytest.mark.parametrize("suf,n", [("z", 1300), ("d", 2100)])
def test_heevd_columns_in_l2(run, oracle, suf, n):
    """Sizes whose own columns no longer fit in shared memory: the reduction
    keeps them in L2 and its vectors in a per-CTA global scratch."""
    a = self_adjoint(n, 5.0, 600 + n, suf == "z")
    st, w, u, info = run.heevd(a, suf)
    assert st.ok and info == 0
    h = oracle.hermitian_from_triangle(a, False)
    wref, _ = oracle.heevd(a, False)
    _check_eig(h, w, u, wref, 1e-13, 1e-15)


def test_expm_herm_columns_in_l2(run, oracle):
    a = self_adjoint(1536, 20.0, 1536, True)
    st, e, _, info = run.expm_herm(a, "z", upper=True)
    assert st.ok and info == 0
    assert rel_frob(e, oracle.expm_herm(a, upper=True)) <= FP64_REL


@pytest.mark.parametrize("suf", ["d", "z"])
def test_nan_input_completes(run, suf):
    """A NaN entry propagates (no fault, no hang): the divide-and-conquer merge
    order it scrambles never turns into an out-of-range index."""
    a = self_adjoint(70, 3.0, 70, suf == "z")
    a[5, 3] = np.nan
    a[3, 5] = np.nan
    st, w, u, info = run.heevd(a, suf)
    assert st.ok and info == 0
    assert np.isnan(w).any() or np.isnan(u).any()
    st, e, _, info = run.expm_herm(a, suf)
    assert st.ok and np.isnan(e).any()


def test_grid_barrier_wait_runs_out_and_the_context_survives(run):
    """The tridiagonal reduction's grid barrier is bounded: with one CTA that
    never arrives, the waiting CTA gives up after its (short) limit, sets the
    failure flag and returns; the context then still runs expm_herm."""
    import ctypes

    w = run.workspace(256)
    code = ctypes.c_int(-1)
    st = run.lib.calaman_grid_barrier_wait_check(None, 1 << 12, ctypes.c_void_p(w.data_ptr()), 256,
                                                 ctypes.byref(code))
    assert st.ok, st
    assert code.value == 1
    rng = np.random.default_rng(5)
    x = rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64))
    h = (x + x.conj().T) / 2
    st, e, _, info = run.expm_herm(h, "z")
    wv, v = np.linalg.eigh(h)
    want = (v * np.exp(wv)) @ v.conj().T
    assert st.ok and np.linalg.norm(e - want) <= 1e-12 * np.linalg.norm(want)
