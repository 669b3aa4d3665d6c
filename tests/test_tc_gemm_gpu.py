"""The split-BF16 tcgen05 GEMM (the FP32 tier's dense products) against an
FP64 product of the same FP32 inputs. Bounds are normwise relative to
||A||_F ||B||_F: the x6 split keeps ~24 operand bits (FP32-like), x3 ~16."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUND = {3: 2e-5, 6: 2e-6}


@pytest.fixture(scope="module")
def lib(cuda):
    from calaman_g_b200 import capi

    return capi.load()


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def run_tc(lib, a, b, c0, alpha, beta, terms, lda=None):
    import torch

    m, k = a.shape
    n = b.shape[1]
    lda = lda or m
    abuf = np.zeros((k, lda), dtype=np.float32)
    abuf[:, :m] = a.T
    dA = torch.from_numpy(abuf.reshape(-1)).cuda()
    dB = torch.from_numpy(np.asfortranarray(b, dtype=np.float32).reshape(-1, order="F")).cuda()
    dC = torch.from_numpy(np.asfortranarray(c0, dtype=np.float32).reshape(-1, order="F")).cuda()
    nb = ctypes.c_size_t()
    assert lib.calaman_gemm_bf16x_bufferSize(m, n, k, terms, ctypes.byref(nb)).ok
    w = torch.zeros(nb.value, dtype=torch.uint8, device="cuda")
    st = lib.calaman_gemm_bf16x_s(None, m, n, k, alpha, vp(dA), lda, vp(dB), k, beta, vp(dC), m,
                                  terms, vp(w), nb.value)
    torch.cuda.synchronize()
    assert st.ok, st
    err_word = int(w[:4].view(torch.int32).item())
    assert err_word == 0, f"kernel reported wait timeout code {err_word}"
    return dC.cpu().numpy().reshape(n, m).T


@pytest.mark.parametrize("terms", [6, 3])
@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (100, 70, 33), (300, 520, 129), (1024, 1024, 1024)])
def test_split_gemm_matches_fp64(lib, terms, m, n, k):
    rng = np.random.default_rng(m * 7 + n + k)
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    got = run_tc(lib, a, b, np.zeros((m, n), np.float32), 1.0, 0.0, terms)
    ref = a.astype(np.float64) @ b.astype(np.float64)
    rel = np.linalg.norm(got - ref) / (np.linalg.norm(a) * np.linalg.norm(b))
    assert rel <= BOUND[terms], rel


def test_split_gemm_alpha_beta_and_padded_lda(lib):
    rng = np.random.default_rng(5)
    m, n, k = 200, 300, 150
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    c = rng.standard_normal((m, n)).astype(np.float32)
    got = run_tc(lib, a, b, c, -1.0, 1.0, 6, lda=m + 7)
    ref = c.astype(np.float64) - a.astype(np.float64) @ b.astype(np.float64)
    rel = np.linalg.norm(got - ref) / (np.linalg.norm(a) * np.linalg.norm(b) + np.linalg.norm(c))
    assert rel <= 2e-6, rel


def test_x6_is_fp32_accurate(lib):
    """x6 is as accurate as an FP32-accumulating SGEMM (the host BLAS here)."""
    rng = np.random.default_rng(9)
    m = n = k = 512
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    ref = a.astype(np.float64) @ b.astype(np.float64)
    got = run_tc(lib, a, b, np.zeros((m, n), np.float32), 1.0, 0.0, 6)
    sgemm = (a @ b).astype(np.float64)
    assert np.linalg.norm(got - ref) <= 4 * np.linalg.norm(sgemm - ref)


def run_tc_c(lib, a, b, c0, alpha, beta, terms, lda=None):
    import torch

    m, k = a.shape
    n = b.shape[1]
    lda = lda or m
    abuf = np.zeros((k, lda), dtype=np.complex64)
    abuf[:, :m] = a.T
    dA = torch.from_numpy(abuf.reshape(-1)).cuda()
    dB = torch.from_numpy(np.asfortranarray(b, dtype=np.complex64).reshape(-1, order="F")).cuda()
    dC = torch.from_numpy(np.asfortranarray(c0, dtype=np.complex64).reshape(-1, order="F")).cuda()
    nb = ctypes.c_size_t()
    assert lib.calaman_gemm_bf16x_bufferSize_c(m, n, k, terms, ctypes.byref(nb)).ok
    w = torch.zeros(nb.value, dtype=torch.uint8, device="cuda")
    st = lib.calaman_gemm_bf16x_c(None, m, n, k, alpha, vp(dA), lda, vp(dB), k, beta, vp(dC), m,
                                  terms, vp(w), nb.value)
    torch.cuda.synchronize()
    assert st.ok, st
    assert int(w[:4].view(torch.int32).item()) == 0
    return dC.cpu().numpy().reshape(n, m).T


@pytest.mark.parametrize("terms", [6, 3])
@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (100, 70, 33), (300, 260, 129), (512, 512, 512)])
def test_complex64_split_gemm_matches_fp64(lib, terms, m, n, k):
    """complex64 as one real product of the block form [[Ar, -Ai]; [Ai, Ar]] [Br; Bi]"""
    rng = np.random.default_rng(m + 3 * n + 7 * k)
    a = (rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))).astype(np.complex64)
    b = (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))).astype(np.complex64)
    got = run_tc_c(lib, a, b, np.zeros((m, n), np.complex64), 1.0, 0.0, terms)
    ref = a.astype(np.complex128) @ b.astype(np.complex128)
    rel = np.linalg.norm(got - ref) / (np.linalg.norm(a) * np.linalg.norm(b))
    assert rel <= BOUND[terms], rel


def test_complex64_alpha_beta_and_padded_lda(lib):
    rng = np.random.default_rng(6)
    m, n, k = 150, 90, 200
    a = (rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))).astype(np.complex64)
    b = (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))).astype(np.complex64)
    c = (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64)
    got = run_tc_c(lib, a, b, c, 0.5, -2.0, 6, lda=m + 5)
    ref = 0.5 * (a.astype(np.complex128) @ b.astype(np.complex128)) - 2.0 * c.astype(np.complex128)
    rel = np.linalg.norm(got - ref) / (np.linalg.norm(a) * np.linalg.norm(b) + np.linalg.norm(c))
    assert rel <= 2e-6, rel
