"""GPU LU with partial pivoting and the n-RHS solve (the getrf/getrs pade()
runs on q_m(A)), against the oracle's xGETRF restatement: identical pivot
sequences and factors (FP64 tiers), backward-stable solves (all tiers), and
LAPACK's info code on singular input. Inputs are dense Gaussian matrices, so
every column pivots -- unlike the Pade denominators of well-scaled matrices,
which are close to diagonally dominant."""
import ctypes

import numpy as np
import pytest

from helpers import NP_DTYPE, colmajor_buffer, eps, from_buffer

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(cuda):
    from calaman_g_b200 import capi

    return capi.load()


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def gaussian(n, suf, seed, m=None):
    rng = np.random.default_rng(seed)
    m = m or n
    a = rng.standard_normal((n, m))
    if suf in "cz":
        a = a + 1j * rng.standard_normal((n, m))
    return a.astype(NP_DTYPE[suf])


def run_getrf(lib, a, suf, lda=None):
    import torch

    n = a.shape[0]
    lda = lda or n
    dA = torch.from_numpy(colmajor_buffer(a, lda, suf)).cuda()
    b = ctypes.c_size_t()
    assert lib.calaman_getrf_bufferSize(n, ctypes.byref(b)).ok
    scratch = torch.zeros(b.value, dtype=torch.uint8, device="cuda")
    info = torch.full((1,), -5, dtype=torch.int32, device="cuda")
    st = getattr(lib, f"calaman_getrf_{suf}")(None, n, vp(dA), lda, vp(scratch),
                                             ctypes.cast(info.data_ptr(), ctypes.POINTER(ctypes.c_int)))
    torch.cuda.synchronize()
    assert st.ok, st
    ipiv = scratch[: 4 * n].view(torch.int32).cpu().numpy()
    return dA, scratch, from_buffer(dA.cpu().numpy(), n, lda), ipiv, int(info.item())


@pytest.mark.parametrize("suf", ["d", "z"])
@pytest.mark.parametrize("n", [1, 2, 7, 63, 64, 65, 100, 300, 513, 1024])
def test_getrf_matches_oracle_exactly_in_pivots(lib, oracle, suf, n):
    a = gaussian(n, suf, 500 + n)
    _, _, lu, ipiv, info = run_getrf(lib, a, suf)
    olu, opiv, oinfo = oracle.getrf(a)
    assert info == 0 and oinfo == 0
    assert np.array_equal(ipiv, opiv)
    assert np.abs(lu - olu).max() <= 1e-12 * max(1.0, np.abs(olu).max()) * np.sqrt(n)


@pytest.mark.parametrize("suf", ["s", "c"])
@pytest.mark.parametrize("n", [5, 64, 200, 700, 3001])  # 3001: the tallest one-CTA panel class
def test_getrf_single_backward_error(lib, suf, n):
    a = gaussian(n, suf, 600 + n)
    _, _, lu, ipiv, info = run_getrf(lib, a, suf)
    assert info == 0
    L = np.tril(lu, -1) + np.eye(n)
    U = np.triu(lu)
    pa = a.astype(np.complex128).copy()
    for j, p in enumerate(ipiv):  # replay the row swaps
        pa[[j, p]] = pa[[p, j]]
    res = np.abs(pa - L.astype(np.complex128) @ U.astype(np.complex128)).max()
    assert res <= 64 * eps(suf) * n * np.abs(a).max()
    # partial pivoting on |Re|+|Im| bounds |l_ij| by 1 (real) and sqrt(2) (complex)
    bound = np.sqrt(2.0) if suf in "cz" else 1.0
    assert np.all(np.abs(np.tril(lu, -1)) <= bound * (1 + 1e-6))


@pytest.mark.parametrize("suf", ["s", "d", "c", "z"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (9, 3), (64, 64), (130, 7), (400, 400), (1500, 77)])
def test_getrs_solves(lib, suf, n, nrhs):
    import torch

    a = gaussian(n, suf, 700 + n)
    b = gaussian(n, suf, 800 + n, nrhs)
    dA, scratch, _, _, info = run_getrf(lib, a, suf)
    assert info == 0
    dB = torch.from_numpy(np.asfortranarray(b).reshape(-1, order="F")).cuda()
    dX = torch.empty_like(dB)
    dinfo = torch.full((1,), -5, dtype=torch.int32, device="cuda")
    st = getattr(lib, f"calaman_getrs_{suf}")(None, n, nrhs, vp(dA), n, vp(scratch), vp(dB), n,
                                             vp(dX), n,
                                             ctypes.cast(dinfo.data_ptr(), ctypes.POINTER(ctypes.c_int)))
    torch.cuda.synchronize()
    assert st.ok and int(dinfo.item()) == 0
    x = dX.cpu().numpy().reshape(nrhs, n).T.astype(np.complex128)
    a64, b64 = a.astype(np.complex128), b.astype(np.complex128)
    res = np.linalg.norm(a64 @ x - b64) / (np.linalg.norm(a64) * np.linalg.norm(x) + np.linalg.norm(b64))
    assert res <= 32 * eps(suf) * np.sqrt(n)


@pytest.mark.parametrize("suf", ["d", "z"])
def test_getrf_singular_info(lib, oracle, suf):
    n = 70
    a = gaussian(n, suf, 900)
    a[:, 5] = 0.0  # column 5 exactly zero -> U(5,5) = 0
    _, _, _, _, info = run_getrf(lib, a, suf)
    _, _, oinfo = oracle.getrf(a)
    assert info == oinfo == 6


def test_getrf_padded_leading_dimension(lib, oracle):
    n, lda = 90, 97
    a = gaussian(n, "d", 901)
    _, _, lu, ipiv, info = run_getrf(lib, a, "d", lda=lda)
    olu, opiv, _ = oracle.getrf(a)
    assert info == 0 and np.array_equal(ipiv, opiv)
    assert np.abs(lu - olu).max() <= 1e-12 * np.abs(olu).max()


@pytest.mark.parametrize("suf,m,target", [("d", 13, 30.0), ("z", 13, 25.0), ("d", 3, 4.0),
                                          ("s", 9, 20.0), ("c", 13, 20.0)])
def test_pade_large_norm_pivoting(oracle, suf, m, target, cuda):
    """pade() does not scale: a large norm makes q_m(A) far from diagonally
    dominant, so the LU inside pivots on most columns."""
    from helpers import Runner, rel_frob, scaled_random

    run = Runner()
    a = scaled_random(120, target, 31 + m, suf in "cz")
    a = a.astype(NP_DTYPE[suf])
    st, r, info = run.pade(a, m, suf)
    ref, _ = oracle.pade(a, m)
    run.close()
    assert st.ok and list(info) == [0, 0]
    assert rel_frob(r, ref) <= (1e-11 if suf in "dz" else 1e-3)
