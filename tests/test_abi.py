"""The C ABI on the CPU: the library loads, exports every declared symbol, and
every host-only entry (plans, thresholds, buffer sizes, argument rejection)
matches the reference's contracts -- no device work is needed for any of these,
exactly as in the reference's host-only suites (`ctest -LE gpu`)."""
import ctypes

import numpy as np
import pytest

from calaman_g_b200 import capi


@pytest.fixture(scope="module")
def lib():
    return capi.load()


def test_exports_every_declared_symbol(lib):
    import subprocess

    declared = capi.declared_symbols()
    assert len(declared) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        getattr(lib, s)  # resolvable through the loader too
    assert set(capi.SIGNATURES) <= set(declared)


def test_version(lib):
    assert b"sm_100a" in lib.calamanGetVersion()


@pytest.mark.parametrize("suf,single", [("s", True), ("d", False)])
def test_plan_and_theta_match_oracle(lib, oracle, suf, single):
    theta = getattr(lib, f"calaman_pade_theta_{suf}")
    plan = getattr(lib, f"calaman_expm_plan_{suf}")
    for m in (3, 5, 7, 9, 13):
        assert theta(m) == pytest.approx(oracle.pade_theta(m, single), rel=1e-15 if not single else 0)
    assert theta(4) == 0 and theta(0) == 0
    for x in np.geomspace(1e-4, 1e4, 400):
        p = plan(float(x))
        o = oracle.expm_plan(float(np.float32(x)) if single else float(x), single)
        assert (p.m, p.s, p.num_gemms) == (o.m, o.s, o.num_gemms), x
    assert [lib.calaman_pade_num_gemms(m) for m in (3, 5, 7, 9, 13)] == [2, 3, 4, 5, 6]
    assert lib.calaman_pade_num_gemms(6) == 0


def test_ps_plan_matches_oracle(lib, oracle):
    for d in range(0, 40):
        for s in (0, 1, 2, 3, 5, 50):
            p, o = lib.calaman_paterson_stockmeyer_plan(d, s), oracle.ps_plan(d, s)
            assert (p.s, p.r, p.num_powers, p.num_blocks, p.num_gemms) == (
                o.s, o.r, o.num_powers, o.num_blocks, o.num_gemms)
        assert lib.calaman_paterson_stockmeyer_block_size(d) == oracle.ps_block_size(d)
        for s in range(1, d + 2):
            assert lib.calaman_paterson_stockmeyer_cost(d, s) == oracle.ps_cost(d, s)


def test_ps_buffer_size(lib):
    """test/paterson_stockmeyer/paterson_stockmeyer_tests.cpp:297-331"""
    for n in (1, 2, 5, 7, 16):
        for degree in (2, 4, 8, 16):
            plan = lib.calaman_paterson_stockmeyer_plan(degree, 0)
            block = ((n * n * 8 + 255) // 256) * 256
            b = lib.calaman_paterson_stockmeyer_bufferSize_d(n, degree, 0)
            assert b == plan.num_blocks * block and b % 256 == 0
    want = lib.calaman_paterson_stockmeyer_plan(10, 1).num_blocks * (((8 * 8 * 4) + 255) // 256) * 256
    assert lib.calaman_paterson_stockmeyer_bufferSize_s(8, 10, 1) == want
    assert lib.calaman_paterson_stockmeyer_bufferSize_d(10, 0, 0) == 0
    assert lib.calaman_paterson_stockmeyer_bufferSize_d(10, 1, 0) == 0
    assert lib.calaman_paterson_stockmeyer_bufferSize_s(10, 1, 0) == 0
    assert lib.calaman_paterson_stockmeyer_power_stride_d(5) == 256 // 8
    assert lib.calaman_paterson_stockmeyer_power_stride_s(1) == 256 // 4


def test_horner_buffer_size(lib):
    """test/horner/horner_tests.cpp:199-221"""
    for n in (1, 2, 5, 7, 16, 33):
        floor = n * n * 8
        b = lib.calaman_horner_bufferSize_d(n)
        assert floor <= b < floor + 256 and b % 256 == 0
    assert lib.calaman_horner_bufferSize_s(10) >= 400
    assert lib.calaman_horner_bufferSize_d(0) >= 8


def _status(st):
    return st.code


def test_expm_rejects_bad_arguments_before_device_work(lib):
    """test/expm/expm_tests.cpp:441-465 -- null handles, host pointers."""
    n = 4
    a = np.ones(n * n)
    e = np.zeros(n * n)
    work = np.zeros(64)
    info = (ctypes.c_int * 2)()
    ap = a.ctypes.data_as(ctypes.c_void_p)
    ep = e.ctypes.data_as(ctypes.c_void_p)
    wp = work.ctypes.data_as(ctypes.c_void_p)

    def call(nn, lda, lde, w, lw=work.nbytes):
        return lib.calaman_expm_d(None, None, None, nn, ap, lda, ep, lde, w, lw, info, None).code

    assert call(0, n, n, wp) == capi.INVALID_VALUE
    assert call(n, n - 1, n, wp) == capi.INVALID_VALUE
    assert call(n, n, n - 1, wp) == capi.INVALID_VALUE
    assert call(n, n, n, None) == capi.INVALID_VALUE
    assert call(46341, 46341, 46341, wp) == capi.INVALID_VALUE
    assert call(n, n, n, wp, 16) == capi.ALLOC_FAILED  # undersized workspace
    b = ctypes.c_size_t()
    assert lib.calaman_expm_bufferSize_d(None, 0, ctypes.byref(b)).code == capi.INVALID_VALUE
    assert lib.calaman_pade_bufferSize_d(None, 4, 0, ctypes.byref(b)).code == capi.INVALID_VALUE
    assert lib.calaman_pade_bufferSize_d(None, 6, 4, ctypes.byref(b)).code == capi.INVALID_VALUE
    for suf in "sdcz":
        assert getattr(lib, f"calaman_expm_bufferSize_{suf}")(None, 8, ctypes.byref(b)).ok
        assert b.value % 256 == 0 and b.value > 0
        for m in (3, 5, 7, 9, 13):
            assert getattr(lib, f"calaman_pade_bufferSize_{suf}")(None, m, 8, ctypes.byref(b)).ok


def test_pade_rejects_bad_arguments(lib):
    n = 4
    a = np.ones(n * n)
    r = np.zeros(n * n)
    work = np.zeros(64)
    info = (ctypes.c_int * 2)()
    ap, rp, wp = (x.ctypes.data_as(ctypes.c_void_p) for x in (a, r, work))
    for m, nn, lda, ldr, w in ((6, n, n, n, wp), (13, 0, n, n, wp), (13, n, n - 1, n, wp),
                               (13, n, n, n - 1, wp), (13, n, n, n, None)):
        st = lib.calaman_pade_d(None, None, None, m, nn, ap, lda, rp, ldr, w, work.nbytes, info)
        assert st.code == capi.INVALID_VALUE
    st = lib.calaman_pade_d(None, None, None, 13, n, ap, n, rp, n, wp, 8, info)
    assert st.code == capi.ALLOC_FAILED


def test_pade_buffer_size_grows_with_degree(lib):
    b = {}
    for m in (3, 9, 13):
        x = ctypes.c_size_t()
        assert lib.calaman_pade_bufferSize_d(None, m, 64, ctypes.byref(x)).ok
        b[m] = x.value
    block = 64 * 64 * 8
    assert b[3] < b[9] and b[9] == b[13]
    assert b[13] - b[3] == 3 * block  # 3 blocks at m = 3, 6 at m = 9 and 13
    e = ctypes.c_size_t()
    assert lib.calaman_expm_bufferSize_d(None, 64, ctypes.byref(e)).ok
    assert e.value >= b[13] + block


def test_ps_rejects_bad_arguments(lib):
    """test/paterson_stockmeyer/paterson_stockmeyer_tests.cpp:336-383"""
    n, degree = 4, 4
    c = np.ones(degree + 1)
    a = np.ones(n * n)
    p = np.zeros(n * n)
    wbytes = lib.calaman_paterson_stockmeyer_bufferSize_d(n, degree, 0)
    assert wbytes > 0
    work = np.zeros(wbytes // 8)
    C, A, P, W = (x.ctypes.data_as(ctypes.c_void_p) for x in (c, a, p, work))

    def call(nn, deg, dc, da, lda, dp, ldp, dw, wb, s):
        return lib.calaman_paterson_stockmeyer_d(None, nn, dc, deg, da, lda, dp, ldp, dw, wb, s).code

    NI = capi.NOT_INITIALIZED
    assert call(0, degree, C, A, n, P, n, W, wbytes, 0) == NI
    assert call(n, -1, C, A, n, P, n, W, wbytes, 0) == NI
    assert call(n, degree, C, A, n - 1, P, n, W, wbytes, 0) == NI
    assert call(n, degree, C, A, n, P, n - 1, W, wbytes, 0) == NI
    assert call(n, degree, C, A, n, P, n, W, wbytes, -1) == NI
    assert call(n, degree, None, A, n, P, n, W, wbytes, 0) == NI
    assert call(n, degree, C, None, n, P, n, W, wbytes, 0) == NI
    assert call(n, degree, C, A, n, None, n, W, wbytes, 0) == NI
    assert call(n, degree, C, A, n, P, n, None, wbytes, 0) == NI
    assert call(n, degree, C, A, n, P, n, W, wbytes - 1, 0) == NI


def test_horner_rejects_bad_arguments(lib):
    """test/horner/horner_tests.cpp:223-271"""
    n, degree = 4, 3
    c = np.ones(degree + 1)
    a = np.ones(n * n)
    p = np.zeros(n * n)
    wbytes = lib.calaman_horner_bufferSize_d(n)
    work = np.zeros(wbytes // 8)
    C, A, P, W = (x.ctypes.data_as(ctypes.c_void_p) for x in (c, a, p, work))

    def call(nn, deg, dc, da, lda, dp, ldp, dw, wb):
        return lib.calaman_horner_d(None, nn, dc, deg, da, lda, dp, ldp, dw, wb).code

    NI = capi.NOT_INITIALIZED
    assert call(0, degree, C, A, n, P, n, W, wbytes) == NI
    assert call(n, -1, C, A, n, P, n, W, wbytes) == NI
    assert call(n, degree, C, A, n - 1, P, n, W, wbytes) == NI
    assert call(n, degree, C, A, n, P, n - 1, W, wbytes) == NI
    assert call(n, degree, None, A, n, P, n, W, wbytes) == NI
    assert call(n, degree, C, None, n, P, n, W, wbytes) == NI
    assert call(n, degree, C, A, n, None, n, W, wbytes) == NI
    assert call(n, degree, C, A, n, P, n, None, wbytes) == NI
    assert call(n, degree, C, A, n, P, n, W, wbytes - 1) == NI


def test_handle_calls_reject_null(lib):
    assert lib.calamanDestroy(None).code == capi.NOT_INITIALIZED
    assert lib.calamanSetStream(None, None).code == capi.NOT_INITIALIZED
    mode = ctypes.c_int()
    assert lib.calamanGetPointerMode(None, ctypes.byref(mode)).code == capi.NOT_INITIALIZED
    assert lib.calamanCreate(None).code == capi.INVALID_VALUE


def test_norm1_rejects_bad_arguments(lib):
    assert np.isnan(lib.calaman_matrix_norm1_d(None, 0, None, 1, None))
    assert np.isnan(lib.calaman_matrix_norm1_s(None, 4, None, 4, None))


def test_lacn2_size_and_rejections(lib):
    """calaman::lacn2's argument contract (src/lapack/lacn2/interface.cppm:119-126):
    INVALID_VALUE for n < 1, null vectors or workspace, a state outside 1..5
    with kase != 0, and a short workspace -- all before device work."""
    for suf, ct in (("s", ctypes.c_float), ("d", ctypes.c_double)):
        size = getattr(lib, f"calaman_lacn2_bufferSize_{suf}")
        assert size(1000) >= 1000 * 4 and size(1000) % 256 == 0
        fn = getattr(lib, f"calaman_lacn2_{suf}")
        est, kase = ct(0), ctypes.c_int(0)
        isave = (ctypes.c_int * 3)()
        buf = ctypes.c_void_p(1 << 20)  # never dereferenced: every call below is rejected
        iv = capi.INVALID_VALUE

        def call(n, v, x, w, nbytes, k=0, s0=0):
            kase.value, isave[0] = k, s0
            return fn(None, n, v, x, w, nbytes, ctypes.byref(est), ctypes.byref(kase), isave).code

        assert call(0, buf, buf, buf, size(4)) == iv
        assert call(4, None, buf, buf, size(4)) == iv
        assert call(4, buf, None, buf, size(4)) == iv
        assert call(4, buf, buf, None, size(4)) == iv
        assert call(4, buf, buf, buf, size(4) - 1) == iv
        assert call(4, buf, buf, buf, size(4), k=1, s0=0) == iv
        assert call(4, buf, buf, buf, size(4), k=2, s0=6) == iv
