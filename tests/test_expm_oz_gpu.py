"""expm / pade / expm_vjp with their FP64 and complex128 products emulated on
the INT8 tensor cores (Ozaki scheme), against the FP64 oracle at the FP64
tier's bar (1e-12 relative Frobenius), through the C ABI: by default (n >=
1536) and forced with calamanSetDoubleEmulation at the benchmark workloads."""
import ctypes

import numpy as np
import pytest

import bench
from helpers import Runner, gaussian_scaled, gue_skew, rel_frob

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.lib.calamanSetDoubleEmulation(r.h, -1)
    r.close()


@pytest.fixture(scope="module")
def orc(oracle):
    import os

    oracle.set_threads(os.cpu_count() or 1)
    yield oracle
    oracle.set_threads(1)


def set_digits(run, d):
    assert run.lib.calamanSetDoubleEmulation(run.h, d).ok
    got = ctypes.c_int(99)
    assert run.lib.calamanGetDoubleEmulation(run.h, ctypes.byref(got)).ok
    assert got.value == d


def test_setting_is_checked_and_sizes_the_workspace(run):
    for bad in (-2, 1, 9):
        assert run.lib.calamanSetDoubleEmulation(run.h, bad).code == 7
    sizes = {}
    for d in (0, 7):
        set_digits(run, d)
        b = ctypes.c_size_t()
        assert run.lib.calaman_expm_bufferSize_d(run.h, 512, ctypes.byref(b)).ok
        sizes[d] = b.value
    assert sizes[7] > sizes[0]  # the digit planes
    set_digits(run, -1)
    b = ctypes.c_size_t()
    assert run.lib.calaman_expm_bufferSize_d(run.h, 512, ctypes.byref(b)).ok
    assert b.value == sizes[0]  # below the size threshold: FP64 tensor cores


def test_default_float64_2048_uses_and_matches(run, orc):
    """The float64 2048 x 2048, ||A||_1 = 6 workload on the default setting
    (emulated products, 7 digits)."""
    set_digits(run, -1)
    cfg = bench.CONFIGS["expm_f64_2048"]
    a = bench.make_matrix(cfg)
    st, plan, e, _, info = run.expm(a, "d")
    ref, oplan, _ = orc.expm(a)
    assert st.ok and list(info) == [0, 0]
    assert (plan.m, plan.s) == (oplan.m, oplan.s) == (13, 1)
    assert rel_frob(e, ref) <= FP64_REL


@pytest.mark.parametrize("digits", [7, 8])
def test_forced_complex128_1024_gue_norm50(run, orc, digits):
    set_digits(run, digits)
    cfg = bench.CONFIGS["expm_c128_1024"]
    a = bench.make_matrix(cfg)
    st, plan, e, _, info = run.expm(a, "z")
    set_digits(run, -1)
    ref, oplan, _ = orc.expm(a)
    assert st.ok and list(info) == [0, 0] and (plan.m, plan.s) == (13, 4)
    assert rel_frob(e, ref) <= FP64_REL
    n = a.shape[0]
    assert np.linalg.norm(e.conj().T @ e - np.eye(n)) <= 1e-12 * n


@pytest.mark.parametrize("n,target", [(129, 5.0), (256, 4.0), (300, 80.0), (700, 60.0)])
def test_forced_float64_parity(run, orc, n, target):
    set_digits(run, 7)
    a = gaussian_scaled(n, target, 5000 + n)
    st, plan, e, _, info = run.expm(a, "d")
    set_digits(run, -1)
    ref, oplan, _ = orc.expm(a)
    assert st.ok and list(info) == [0, 0] and (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(e, ref) <= FP64_REL


@pytest.mark.parametrize("n,target", [(200, 20.0), (256, 50.0)])
def test_forced_complex128_parity(run, orc, n, target):
    set_digits(run, 7)
    a = gue_skew(n, target, 6000 + n)
    st, plan, e, _, _ = run.expm(a, "z")
    set_digits(run, -1)
    ref, oplan, _ = orc.expm(a)
    assert st.ok and (plan.m, plan.s) == (oplan.m, oplan.s)
    assert rel_frob(e, ref) <= FP64_REL


@pytest.mark.parametrize("m", [5, 13])
def test_forced_pade(run, orc, m):
    set_digits(run, 7)
    a = gaussian_scaled(256, 0.8 * orc.pade_theta(m), 70 + m)
    st, r, info = run.pade(a, m, "d")
    set_digits(run, -1)
    ref, _ = orc.pade(a, m)
    assert st.ok and list(info) == [0, 0]
    assert rel_frob(r, ref) <= FP64_REL


def test_forced_vjp_matches_the_fp64_tensor_core_path(run):
    a = gaussian_scaled(256, 6.0, 81)
    g = np.random.default_rng(82).standard_normal((256, 256))
    set_digits(run, 0)
    st0, _, ga0, e0, _, _ = run.vjp(a, g, "d")
    set_digits(run, 7)
    st1, _, ga1, e1, _, _ = run.vjp(a, g, "d")
    set_digits(run, -1)
    assert st0.ok and st1.ok
    assert rel_frob(ga1, ga0) <= FP64_REL and rel_frob(e1, e0) <= FP64_REL
