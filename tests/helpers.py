"""Shared test helpers: seeded inputs in the reference's test shapes, the
reference's tolerance formulas, and thin runners that call the C ABI directly
(column-major buffers, explicit leading dimensions) through ctypes."""
from __future__ import annotations

import ctypes

import numpy as np

NP_DTYPE = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
REAL = {"s": np.float32, "d": np.float64, "c": np.float32, "z": np.float64}


def eps(suf: str) -> float:
    return float(np.finfo(REAL[suf]).eps)


def norm1(a: np.ndarray) -> float:
    return float(np.abs(a).sum(axis=0).max())


def scaled_random(n: int, target: float, seed: int, cplx: bool = False) -> np.ndarray:
    """U(-1,1) entries rescaled to 1-norm `target` (test/expm/expm_tests.cpp:316-336)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1.0, 1.0, (n, n))
    if cplx:
        a = a + 1j * rng.uniform(-1.0, 1.0, (n, n))
    nrm = norm1(a)
    return a * (target / nrm) if nrm > 0 else a


def gaussian_scaled(n: int, target: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    return a * (target / norm1(a))


def gue_skew(n: int, target: float, seed: int) -> np.ndarray:
    """A = -i H, H = (X + X^H)/2, X complex N(0,1); rescaled to 1-norm target."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = (x + x.conj().T) / 2
    a = -1j * h
    return a * (target / norm1(a))


def elem_tol(oracle: np.ndarray, n: int, factor: float, suf: str) -> float:
    """factor * eps * max(1, ||oracle||_F) * n (test/expm/expm_tests.cpp:206-217)."""
    return factor * eps(suf) * max(1.0, float(np.linalg.norm(oracle))) * n


def rel_frob(got: np.ndarray, ref: np.ndarray) -> float:
    return float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300))


# ---------------------------------------------------------------------------
# device runners (torch provides the memory and the stream)
# ---------------------------------------------------------------------------
def _dev(x: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def colmajor_buffer(a: np.ndarray, ld: int, suf: str, fill=-123.5) -> np.ndarray:
    """Flat column-major buffer of an n x n matrix with leading dimension ld;
    padding rows carry the sentinel `fill`."""
    n = a.shape[0]
    buf = np.full((n, ld), fill, dtype=NP_DTYPE[suf])
    buf[:, :n] = a.T.astype(NP_DTYPE[suf])
    return buf.reshape(-1)


def from_buffer(buf: np.ndarray, n: int, ld: int) -> np.ndarray:
    return buf.reshape(n, ld)[:, :n].T.copy()


def vp(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


class Runner:
    """Calls the C ABI with a fresh handle bound to torch's current stream."""

    def __init__(self):
        import torch

        from calaman_g_b200 import capi

        self.torch = torch
        self.capi = capi
        self.lib = capi.load()
        h = ctypes.c_void_p()
        st = self.lib.calamanCreate(ctypes.byref(h))
        assert st.ok, st
        self.h = h
        self.stream = torch.cuda.current_stream().cuda_stream
        assert self.lib.calamanSetStream(h, ctypes.c_void_p(self.stream)).ok

    def close(self):
        self.lib.calamanDestroy(self.h)

    def workspace(self, nbytes: int):
        return self.torch.empty(max(nbytes, 256), dtype=self.torch.uint8, device="cuda")

    def expm_herm(self, a: np.ndarray, suf: str, upper: bool = False, lda: int | None = None,
                  lde: int | None = None, out_fill=-123.5, lwork: int | None = None):
        """calaman_expm_herm_<suf>: returns (status, E (n x n), full E buffer, info)."""
        n = a.shape[0]
        lda = lda or n
        lde = lde or n
        dA = _dev(colmajor_buffer(a, lda, suf))
        dE = _dev(np.full(n * lde, out_fill, dtype=NP_DTYPE[suf]))
        b = ctypes.c_size_t()
        uplo = self.capi.FILL_UPPER if upper else self.capi.FILL_LOWER
        assert getattr(self.lib, f"calaman_expm_herm_bufferSize_{suf}")(self.h, uplo, n, ctypes.byref(b)).ok
        w = self.workspace(b.value)
        info = self.torch.full((1,), -99, dtype=self.torch.int32, device="cuda")
        st = getattr(self.lib, f"calaman_expm_herm_{suf}")(
            self.h, self.h, ctypes.c_void_p(self.stream), uplo, n, vp(dA), lda, vp(dE), lde, vp(w),
            b.value if lwork is None else lwork, ctypes.cast(info.data_ptr(), self.capi.c_int_p))
        self.torch.cuda.synchronize()
        full = dE.cpu().numpy()
        e = full.reshape(n, lde)[:, :n].T
        return st, e, full, int(info.cpu()[0])

    def heevd(self, a: np.ndarray, suf: str, upper: bool = False, lda: int | None = None):
        """calaman_heevd_<suf>: returns (status, w, U (n x n), info)."""
        n = a.shape[0]
        lda = lda or n
        dA = _dev(colmajor_buffer(a, lda, suf))
        real = self.torch.float32 if suf in ("s", "c") else self.torch.float64
        dw = self.torch.full((n,), float("nan"), dtype=real, device="cuda")
        b = ctypes.c_size_t()
        uplo = self.capi.FILL_UPPER if upper else self.capi.FILL_LOWER
        assert getattr(self.lib, f"calaman_heevd_bufferSize_{suf}")(uplo, n, ctypes.byref(b)).ok
        w = self.workspace(b.value)
        info = self.torch.full((1,), -99, dtype=self.torch.int32, device="cuda")
        st = getattr(self.lib, f"calaman_heevd_{suf}")(
            ctypes.c_void_p(self.stream), uplo, n, vp(dA), lda, vp(dw), vp(w), b.value,
            ctypes.cast(info.data_ptr(), self.capi.c_int_p))
        self.torch.cuda.synchronize()
        u = dA.cpu().numpy().reshape(n, lda)[:, :n].T
        return st, dw.cpu().numpy(), u, int(info.cpu()[0])

    def expm(self, a: np.ndarray, suf: str, lda: int | None = None, lde: int | None = None,
             out_fill=-123.5, lwork: int | None = None):
        n = a.shape[0]
        lda = lda or n
        lde = lde or n
        dA = _dev(colmajor_buffer(a, lda, suf))
        dE = _dev(np.full(n * lde, out_fill, dtype=NP_DTYPE[suf]))
        b = ctypes.c_size_t()
        assert getattr(self.lib, f"calaman_expm_bufferSize_{suf}")(self.h, n, ctypes.byref(b)).ok
        w = self.workspace(b.value)
        info = self.torch.full((2,), -99, dtype=self.torch.int32, device="cuda")
        plan = self.capi.ExpmPlan()
        st = getattr(self.lib, f"calaman_expm_{suf}")(
            self.h, self.h, ctypes.c_void_p(self.stream), n, vp(dA), lda, vp(dE), lde, vp(w),
            b.value if lwork is None else lwork, ctypes.cast(info.data_ptr(), self.capi.c_int_p),
            ctypes.byref(plan))
        self.torch.cuda.synchronize()
        full = dE.cpu().numpy()
        return st, plan, from_buffer(full, n, lde), full, info.cpu().numpy()

    def pade(self, a: np.ndarray, m: int, suf: str):
        n = a.shape[0]
        dA = _dev(colmajor_buffer(a, n, suf))
        dR = _dev(np.zeros(n * n, dtype=NP_DTYPE[suf]))
        b = ctypes.c_size_t()
        assert getattr(self.lib, f"calaman_pade_bufferSize_{suf}")(self.h, m, n, ctypes.byref(b)).ok
        w = self.workspace(b.value)
        info = self.torch.full((2,), -99, dtype=self.torch.int32, device="cuda")
        st = getattr(self.lib, f"calaman_pade_{suf}")(
            self.h, self.h, ctypes.c_void_p(self.stream), m, n, vp(dA), n, vp(dR), n, vp(w),
            b.value, ctypes.cast(info.data_ptr(), self.capi.c_int_p))
        self.torch.cuda.synchronize()
        return st, from_buffer(dR.cpu().numpy(), n, n), info.cpu().numpy()

    def norm1(self, a: np.ndarray, suf: str) -> float:
        n = a.shape[0]
        dA = _dev(colmajor_buffer(a, n, suf))
        cs = self.torch.empty(n, dtype=self.torch.float32 if suf in "sc" else self.torch.float64,
                              device="cuda")
        return getattr(self.lib, f"calaman_matrix_norm1_{suf}")(
            ctypes.c_void_p(self.stream), n, vp(dA), n, vp(cs))

    def poly(self, kind: str, a: np.ndarray, c: np.ndarray, suf: str, s_requested: int = 0,
             ldp: int | None = None, out_fill=0.0):
        n = a.shape[0]
        ldp = ldp or n
        degree = len(c) - 1
        dA = _dev(colmajor_buffer(a, n, suf))
        dc = _dev(np.asarray(c, dtype=NP_DTYPE[suf]))
        dP = _dev(np.full(n * ldp, out_fill, dtype=NP_DTYPE[suf]))
        if kind == "horner":
            nb = getattr(self.lib, f"calaman_horner_bufferSize_{suf}")(n) if degree > 0 else 0
            w = self.workspace(nb) if nb else None
            st = getattr(self.lib, f"calaman_horner_{suf}")(
                self.h, n, vp(dc), degree, vp(dA), n, vp(dP), ldp,
                vp(w) if w is not None else None, nb)
        else:
            nb = getattr(self.lib, f"calaman_paterson_stockmeyer_bufferSize_{suf}")(
                n, degree, s_requested)
            w = self.workspace(nb) if nb else None
            st = getattr(self.lib, f"calaman_paterson_stockmeyer_{suf}")(
                self.h, n, vp(dc), degree, vp(dA), n, vp(dP), ldp,
                vp(w) if w is not None else None, nb, s_requested)
        self.torch.cuda.synchronize()
        full = dP.cpu().numpy()
        return st, from_buffer(full, n, ldp), full

    def vjp(self, a: np.ndarray, g: np.ndarray, suf: str, ld: int | None = None,
            want_expm: bool = True, out_fill=-123.5, lwork: int | None = None,
            alias_g: bool = False):
        """calaman_expm_vjp_<suf>: returns (status, plan, gradA, expA or None,
        flat gradA buffer, info). ``alias_g`` writes the gradient over G."""
        n = a.shape[0]
        ld = ld or n
        dA = _dev(colmajor_buffer(a, ld, suf))
        dG = _dev(colmajor_buffer(g, ld, suf))
        dD = dG if alias_g else _dev(np.full(n * ld, out_fill, dtype=NP_DTYPE[suf]))
        dE = _dev(np.full(n * ld, out_fill, dtype=NP_DTYPE[suf])) if want_expm else None
        b = ctypes.c_size_t()
        assert getattr(self.lib, f"calaman_expm_vjp_bufferSize_{suf}")(self.h, n, ctypes.byref(b)).ok
        w = self.workspace(b.value)
        info = self.torch.full((2,), -99, dtype=self.torch.int32, device="cuda")
        plan = self.capi.ExpmPlan()
        st = getattr(self.lib, f"calaman_expm_vjp_{suf}")(
            self.h, self.h, ctypes.c_void_p(self.stream), n, vp(dA), ld, vp(dG), ld, vp(dD), ld,
            vp(dE) if dE is not None else None, ld, vp(w), b.value if lwork is None else lwork,
            ctypes.cast(info.data_ptr(), self.capi.c_int_p), ctypes.byref(plan))
        self.torch.cuda.synchronize()
        full = dD.cpu().numpy()
        e = from_buffer(dE.cpu().numpy(), n, ld) if dE is not None else None
        return st, plan, from_buffer(full, n, ld), e, full, info.cpu().numpy()

    def batched(self, mats, suf: str, lds=None, ldes=None, out_fill=-123.5, lwork=None):
        """calaman_expm_batched_<suf> over a list of square matrices. Returns
        (status, plans, outputs, flat output buffers, info[batch, 2])."""
        torch = self.torch
        b = len(mats)
        ns = [m.shape[0] for m in mats]
        lds = lds or ns
        ldes = ldes or ns
        dt = NP_DTYPE[suf]
        a_host = [colmajor_buffer(m, ld, suf) for m, ld in zip(mats, lds)]
        e_host = [np.full(n * ld, out_fill, dtype=dt) for n, ld in zip(ns, ldes)]
        dA = [_dev(x) for x in a_host]
        dE = [_dev(x) for x in e_host]
        IntArr = ctypes.c_int * max(b, 1)
        PtrArr = ctypes.c_void_p * max(b, 1)
        h_n, h_lda, h_lde = IntArr(*ns), IntArr(*lds), IntArr(*ldes)
        h_A = PtrArr(*[t.data_ptr() for t in dA])
        h_E = PtrArr(*[t.data_ptr() for t in dE])
        nb = ctypes.c_size_t()
        st = getattr(self.lib, f"calaman_expm_batched_bufferSize_{suf}")(
            self.h, b, ctypes.cast(h_n, self.capi.c_int_p), ctypes.byref(nb))
        if not st.ok:
            return st, None, None, None, None
        w = self.workspace(nb.value)
        info = torch.full((max(2 * b, 2),), -99, dtype=torch.int32, device="cuda")
        plans = (self.capi.ExpmPlan * max(b, 1))()
        st = getattr(self.lib, f"calaman_expm_batched_{suf}")(
            self.h, self.h, ctypes.c_void_p(self.stream), b, ctypes.cast(h_n, self.capi.c_int_p),
            ctypes.cast(h_A, ctypes.POINTER(ctypes.c_void_p)), ctypes.cast(h_lda, self.capi.c_int_p),
            ctypes.cast(h_E, ctypes.POINTER(ctypes.c_void_p)), ctypes.cast(h_lde, self.capi.c_int_p),
            vp(w), nb.value if lwork is None else lwork,
            ctypes.cast(info.data_ptr(), self.capi.c_int_p), plans)
        torch.cuda.synchronize()
        fulls = [t.cpu().numpy() for t in dE]
        outs = [from_buffer(f, n, ld) for f, n, ld in zip(fulls, ns, ldes)]
        return st, list(plans)[:b], outs, fulls, info.cpu().numpy()[: 2 * b].reshape(-1, 2)


def c4_batch(count: int, seed: int, nmax: int = 256):
    """The batched workload: n uniform on {16, 32, ..., nmax}, N(0,1) entries
    rescaled to a 1-norm log-uniform in [0.1, 100]."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, nmax // 16 + 1, count) * 16
    norms = np.exp(rng.uniform(np.log(0.1), np.log(100.0), count))
    mats = []
    for n, t in zip(sizes, norms):
        a = rng.standard_normal((n, n))
        mats.append(a * (t / norm1(a)))
    return mats


def run_vjp_batched(runner, pairs, suf: str, want_expm: bool = True, lds=None, out_fill=-123.5,
                    lwork=None):
    """calaman_expm_vjp_batched_<suf> over a list of (A, G) pairs. Returns
    (status, plans, gradients, expms or None, flat gradient buffers, info[batch, 2])."""
    torch = runner.torch
    b = len(pairs)
    ns = [a.shape[0] for a, _ in pairs]
    lds = lds or ns
    dt = NP_DTYPE[suf]
    dA = [_dev(colmajor_buffer(a, ld, suf)) for (a, _), ld in zip(pairs, lds)]
    dG = [_dev(colmajor_buffer(g, ld, suf)) for (_, g), ld in zip(pairs, lds)]
    dD = [_dev(np.full(n * ld, out_fill, dtype=dt)) for n, ld in zip(ns, lds)]
    dE = [_dev(np.full(n * ld, out_fill, dtype=dt)) for n, ld in zip(ns, lds)] if want_expm else None
    IntArr = ctypes.c_int * max(b, 1)
    PtrArr = ctypes.c_void_p * max(b, 1)
    h_n, h_ld = IntArr(*ns), IntArr(*lds)
    PP = ctypes.POINTER(ctypes.c_void_p)
    h_A = PtrArr(*[t.data_ptr() for t in dA])
    h_G = PtrArr(*[t.data_ptr() for t in dG])
    h_D = PtrArr(*[t.data_ptr() for t in dD])
    h_E = PtrArr(*[t.data_ptr() for t in dE]) if dE is not None else None
    ip = ctypes.cast(h_n, runner.capi.c_int_p)
    ldp = ctypes.cast(h_ld, runner.capi.c_int_p)
    nb = ctypes.c_size_t()
    st = getattr(runner.lib, f"calaman_expm_vjp_batched_bufferSize_{suf}")(runner.h, b, ip, ctypes.byref(nb))
    if not st.ok:
        return st, None, None, None, None, None
    w = runner.workspace(nb.value)
    info = torch.full((max(2 * b, 2),), -99, dtype=torch.int32, device="cuda")
    plans = (runner.capi.ExpmPlan * max(b, 1))()
    st = getattr(runner.lib, f"calaman_expm_vjp_batched_{suf}")(
        runner.h, runner.h, ctypes.c_void_p(runner.stream), b, ip, ctypes.cast(h_A, PP), ldp,
        ctypes.cast(h_G, PP), ldp, ctypes.cast(h_D, PP), ldp,
        ctypes.cast(h_E, PP) if h_E is not None else None, ldp, vp(w),
        nb.value if lwork is None else lwork, ctypes.cast(info.data_ptr(), runner.capi.c_int_p), plans)
    torch.cuda.synchronize()
    fulls = [t.cpu().numpy() for t in dD]
    grads = [from_buffer(f, n, ld) for f, n, ld in zip(fulls, ns, lds)]
    exps = [from_buffer(t.cpu().numpy(), n, ld) for t, n, ld in zip(dE, ns, lds)] if dE is not None else None
    return st, list(plans)[:b], grads, exps, fulls, info.cpu().numpy()[: 2 * b].reshape(-1, 2)
