"""The Ozaki-scheme INT8 tensor-core GEMM (the FP64 tiers' emulated dense
products) against the FP64 product of the same inputs (numpy's BLAS), through
the C ABI. The scheme's error is about 2^(-7 digits) relative to |A| |B| row
by column; the bounds below are normwise, relative to ||A||_F ||B||_F."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bound(digits):
    return 32.0 * 2.0 ** (-7 * digits)


@pytest.fixture(scope="module")
def lib(cuda):
    from calaman_g_b200 import capi

    return capi.load()


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def colmajor(x, ld):
    rows, cols = x.shape
    buf = np.zeros((cols, ld), dtype=x.dtype)
    buf[:, :rows] = x.T
    return buf.reshape(-1)


def run_oz(lib, a, b, c0, alpha, beta, digits, lda=None, ldc=None):
    import torch

    cplx = np.iscomplexobj(a)
    dt = np.complex128 if cplx else np.float64
    m, k = a.shape
    n = b.shape[1]
    lda = lda or m
    ldc = ldc or m
    dA = torch.from_numpy(colmajor(a.astype(dt), lda)).cuda()
    dB = torch.from_numpy(colmajor(b.astype(dt), k)).cuda()
    dC = torch.from_numpy(colmajor(c0.astype(dt), ldc)).cuda()
    nb = ctypes.c_size_t()
    assert lib.calaman_gemm_ozaki_bufferSize(m, n, k, int(cplx), digits, ctypes.byref(nb)).ok
    w = torch.zeros(nb.value, dtype=torch.uint8, device="cuda")
    fn = lib.calaman_gemm_ozaki_z if cplx else lib.calaman_gemm_ozaki_d
    st = fn(None, m, n, k, alpha, vp(dA), lda, vp(dB), k, beta, vp(dC), ldc, digits, vp(w), nb.value)
    torch.cuda.synchronize()
    assert st.ok, st
    err_word = int(w[:4].view(torch.int32).item())
    assert err_word == 0, err_word
    full = dC.cpu().numpy().reshape(n, ldc)
    return full[:, :m].T, full


def rand(shape, seed, cplx=False):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(shape)
    if cplx:
        x = x + 1j * rng.standard_normal(shape)
    return x


def rel(c, want, a, b):
    return np.linalg.norm(c - want) / (np.linalg.norm(a) * np.linalg.norm(b))


@pytest.mark.parametrize("m,n,k", [(128, 128, 128), (100, 70, 33), (300, 520, 129), (1024, 1024, 1024),
                                   (2048, 2048, 2048)])
def test_real_product_digits7(lib, m, n, k):
    a, b = rand((m, k), m + k), rand((k, n), n + 3 * k)
    c, _ = run_oz(lib, a, b, np.zeros((m, n)), 1.0, 0.0, 7)
    assert rel(c, a @ b, a, b) <= bound(7)


@pytest.mark.parametrize("m,n,k", [(128, 128, 128), (300, 200, 77), (1024, 1024, 1024)])
def test_complex_product_digits7(lib, m, n, k):
    a, b = rand((m, k), m + k, True), rand((k, n), n + 3 * k, True)
    c, _ = run_oz(lib, a, b, np.zeros((m, n), dtype=complex), 1.0, 0.0, 7)
    assert rel(c, a @ b, a, b) <= bound(7)


@pytest.mark.parametrize("digits", [2, 3, 4, 5, 6, 8])
def test_error_follows_the_digit_count(lib, digits):
    a, b = rand((256, 256), 1), rand((256, 256), 2)
    c, _ = run_oz(lib, a, b, np.zeros((256, 256)), 1.0, 0.0, digits)
    e = rel(c, a @ b, a, b)
    assert e <= bound(digits)
    if digits <= 5:  # above FP64 rounding the truncation error is visible
        assert e >= bound(digits) / 1e5


def test_alpha_beta_padding_and_badly_scaled_rows(lib):
    m, n, k = 200, 150, 190
    a, b = rand((m, k), 5), rand((k, n), 6)
    a[::7] *= 2.0 ** 40   # rows of very different magnitude: row scaling keeps each exact
    b[:, ::5] *= 2.0 ** -30
    c0 = rand((m, n), 7)
    c, full = run_oz(lib, a, b, c0, -0.5, 2.0, 7, lda=m + 3, ldc=m + 5)
    want = -0.5 * (a @ b) + 2.0 * c0
    # per-row, per-column scale: the error is relative to |A||B| entry by entry
    scale = np.abs(a) @ np.abs(b) + np.abs(c0)
    assert np.max(np.abs(c - want) / scale) <= 64 * 2.0 ** -49 * k
    pad = full.reshape(n, m + 5)[:, m:]
    assert np.all(pad == 0.0)  # padding rows of C untouched


def test_complex_conjugate_structure(lib):
    """exp(-iH)-like operands: unitary U times U^H is the identity."""
    rng = np.random.default_rng(9)
    q, _ = np.linalg.qr(rng.standard_normal((256, 256)) + 1j * rng.standard_normal((256, 256)))
    c, _ = run_oz(lib, q, q.conj().T, np.zeros((256, 256), dtype=complex), 1.0, 0.0, 7)
    assert rel(c, np.eye(256), q, q) <= bound(7)
    assert np.linalg.norm(c - np.eye(256)) <= 1e-12 * 256  # the unitarity bar of the expm tests


def test_bounded_waits_run_out_and_the_context_survives(lib):
    """The kernel's producer issues no copy: every wait must give up after its
    (short) limit, record a code and unwind; the GPU context stays usable."""
    import torch

    w = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    code = ctypes.c_int(-1)
    st = lib.calaman_gemm_ozaki_wait_check(None, 1 << 12, vp(w), w.numel(), ctypes.byref(code))
    assert st.ok, st
    assert code.value in (1, 2, 3, 4), code.value
    a, b = rand((128, 128), 11), rand((128, 128), 12)
    c, _ = run_oz(lib, a, b, np.zeros((128, 128)), 1.0, 0.0, 7)
    assert rel(c, a @ b, a, b) <= bound(7)


@pytest.mark.parametrize("cplx", [False, True])
def test_square_products_split_off_the_diagonal(lib, cplx):
    """I-dominated square operands (the shape of W and of the quotient before
    its squarings): the diagonals are taken out of the digits and added back
    exactly, so the small off-diagonal part keeps the full digit precision."""
    n = 512
    g1, g2 = rand((n, n), 21, cplx), rand((n, n), 22, cplx)
    x = 3.0 * np.eye(n) + 1e-3 * g1
    z = -2.0 * np.eye(n) + 1e-3 * g2
    c, _ = run_oz(lib, x, z, np.zeros((n, n), dtype=x.dtype), 1.0, 0.0, 7)
    want = x @ z
    off = ~np.eye(n, dtype=bool)
    assert np.linalg.norm((c - want)[off]) / np.linalg.norm(want[off]) <= 1e-13
    assert np.linalg.norm(c - want) / np.linalg.norm(want) <= 1e-14
