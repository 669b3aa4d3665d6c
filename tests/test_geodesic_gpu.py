"""GPU parity of the geodesic trial points of the cg_unitary line searches
(calaman_geodesic_points_*): W_j = exp(j step H) W, j = 1..N-1, against the
oracle's restatement in the reference's order (R_1 = expm(step H) by the general
expm, R_j = R_{j-1} R_1, W_j = R_j W; src/cg_unitary/geodesic_search.cppm:354-410).
Also: unitary (orthogonal) trial points stay unitary, only H's lower triangle is
read, N = 1 writes nothing, the sample counts of both searches (P + 1 = 6 for
Table 1, 31 for Table 2), and host-side argument rejection."""
import ctypes

import numpy as np
import pytest

from helpers import Runner, _dev, colmajor_buffer, rel_frob, vp

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
SINGLE_REL = 2e-5
DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def point_and_direction(n, cplx, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    w, _ = np.linalg.qr(x)
    y = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    h = (y - y.conj().T) / 2
    nrm = np.linalg.norm(h, 2)
    h = h * (scale / nrm) if nrm > 0 else h  # a 1 x 1 real skew-symmetric H is 0
    return w, h


def geodesic(run, w, h, step, num, suf, ldw=None, ldh=None, out_fill=-7.25):
    n = w.shape[0]
    ldw, ldh = ldw or n, ldh or n
    dW = _dev(colmajor_buffer(w, ldw, suf))
    dH = _dev(colmajor_buffer(h, ldh, suf))
    nout = max(num - 1, 1) * n * n
    dO = _dev(np.full(nout, out_fill, dtype=DT[suf]))
    b = ctypes.c_size_t()
    assert getattr(run.lib, f"calaman_geodesic_points_bufferSize_{suf}")(run.h, n, num, ctypes.byref(b)).ok
    work = run.workspace(b.value)
    info = run.torch.full((1,), -99, dtype=run.torch.int32, device="cuda")
    st = getattr(run.lib, f"calaman_geodesic_points_{suf}")(
        run.h, run.h, ctypes.c_void_p(run.stream), n, vp(dW), ldw, vp(dH), ldh, float(step), num, vp(dO),
        vp(work), b.value, ctypes.cast(info.data_ptr(), run.capi.c_int_p))
    run.torch.cuda.synchronize()
    flat = dO.cpu().numpy()
    blocks = [flat[j * n * n:(j + 1) * n * n].reshape(n, n).T for j in range(max(num - 1, 0))]
    return st, blocks, flat, int(info.cpu()[0])


@pytest.mark.parametrize("suf", ["z", "d"])
@pytest.mark.parametrize("n,num,scale", [(1, 2, 1.0), (2, 6, 3.0), (7, 6, 0.5), (64, 6, 8.0), (64, 31, 2.0),
                                         (257, 6, 4.0)])
def test_matches_reference_order(run, oracle, suf, n, num, scale):
    w, h = point_and_direction(n, suf == "z", 900 + n + num, scale)
    step = 0.3
    st, blocks, _, info = geodesic(run, w, h, step, num, suf)
    assert st.ok and info == 0
    ref = oracle.geodesic_points(w, h, step, num)
    for got, want in zip(blocks, ref):
        assert rel_frob(got, want) <= FP64_REL
        assert np.linalg.norm(got.conj().T @ got - np.eye(n)) <= 1e-12 * n


@pytest.mark.parametrize("suf", ["c", "s"])
def test_single_tiers(run, oracle, suf):
    w, h = point_and_direction(96, suf == "c", 77, 4.0)
    w, h = w.astype(DT[suf]), h.astype(DT[suf])
    st, blocks, _, info = geodesic(run, w, h, 0.25, 6, suf)
    assert st.ok and info == 0
    ref = oracle.geodesic_points(w, h, 0.25, 6)
    for got, want in zip(blocks, ref):
        assert rel_frob(got, want) <= SINGLE_REL


def test_benchmark_shape_1024(run, oracle):
    """complex128 1024 x 1024, the Table 1 sample count (P + 1 = 6)."""
    w, h = point_and_direction(1024, True, 1024, 10.0)
    st, blocks, _, info = geodesic(run, w, h, 0.1, 6, "z")
    assert st.ok and info == 0
    ref = oracle.geodesic_points(w, h, 0.1, 6)
    for got, want in zip(blocks, ref):
        assert rel_frob(got, want) <= FP64_REL


def test_reads_lower_triangle_and_padding(run):
    w, h = point_and_direction(40, True, 5, 2.0)
    junk = np.tril(h) + np.triu(np.full((40, 40), 9.0 + 4j), 1)
    st, a, _, _ = geodesic(run, w, h, 0.5, 4, "z")
    st2, b, _, _ = geodesic(run, w, junk, 0.5, 4, "z", ldw=43, ldh=41)
    assert st.ok and st2.ok
    for x, y in zip(a, b):
        assert rel_frob(x, y) <= 1e-13


def test_one_sample_writes_nothing(run):
    w, h = point_and_direction(8, True, 6)
    st, blocks, flat, info = geodesic(run, w, h, 0.5, 1, "z")
    assert st.ok and info == 0 and blocks == [] and np.all(flat == -7.25)


def test_argument_checks(run):
    lib, hdl, cap = run.lib, run.h, run.capi
    b = ctypes.c_size_t()
    assert lib.calaman_geodesic_points_bufferSize_z(hdl, 8, 0, ctypes.byref(b)).code == cap.INVALID_VALUE
    assert lib.calaman_geodesic_points_bufferSize_z(hdl, 8, 65, ctypes.byref(b)).code == cap.INVALID_VALUE
    buf = ctypes.c_void_p(1 << 20)  # never dereferenced: every call below returns before device work
    ip = ctypes.cast(buf, cap.c_int_p)
    s = ctypes.c_void_p(run.stream)
    f = lib.calaman_geodesic_points_z
    assert f(hdl, hdl, s, 0, buf, 1, buf, 1, 0.1, 2, buf, buf, 1 << 30, ip).code == cap.INVALID_VALUE
    assert f(hdl, hdl, s, 8, buf, 7, buf, 8, 0.1, 2, buf, buf, 1 << 30, ip).code == cap.INVALID_VALUE
    assert f(hdl, hdl, s, 8, buf, 8, buf, 8, float("nan"), 2, buf, buf, 1 << 30, ip).code == cap.INVALID_VALUE
    assert f(hdl, hdl, s, 8, buf, 8, buf, 8, 0.1, 2, buf, buf, 64, ip).code == cap.ALLOC_FAILED
