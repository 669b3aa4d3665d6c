"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is a C restatement of calaman_G's expm / pade / matrix_norm1 /
paterson_stockmeyer / horner path, computed in FP64 (see oracle.h for the
per-function citations). Only tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; the product library never
does.

Matrices are numpy arrays; they are passed column-major (Fortran order), the
layout the reference uses.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc only; seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _ExpmPlan(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("s", ctypes.c_int), ("num_gemms", ctypes.c_int)]


class _PsPlan(ctypes.Structure):
    _fields_ = [
        ("s", ctypes.c_int),
        ("r", ctypes.c_int),
        ("num_powers", ctypes.c_int),
        ("num_blocks", ctypes.c_int),
        ("num_gemms", ctypes.c_int),
    ]


@dataclass(frozen=True)
class ExpmPlan:
    m: int
    s: int
    num_gemms: int


@dataclass(frozen=True)
class PsPlan:
    s: int
    r: int
    num_powers: int
    num_blocks: int
    num_gemms: int


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.oracle_set_threads.argtypes = [c_int]
        L.oracle_get_threads.restype = c_int
        L.oracle_pade_theta.argtypes = [c_int, c_int]
        L.oracle_pade_theta.restype = c_double
        L.oracle_expm_plan.argtypes = [c_double, c_int]
        L.oracle_expm_plan.restype = _ExpmPlan
        L.oracle_pade_coeffs.argtypes = [c_int]
        L.oracle_pade_coeffs.restype = dp
        L.oracle_pade_num_powers.argtypes = [c_int]
        L.oracle_pade_num_gemms.argtypes = [c_int]
        L.oracle_ps_cost.argtypes = [c_int, c_int]
        L.oracle_ps_block_size.argtypes = [c_int]
        L.oracle_ps_plan.argtypes = [c_int, c_int]
        L.oracle_ps_plan.restype = _PsPlan
        for suf in ("d", "z"):
            getattr(L, f"oracle_norm1_{suf}").argtypes = [c_int, dp, c_int]
            getattr(L, f"oracle_norm1_{suf}").restype = c_double
            getattr(L, f"oracle_pade_{suf}").argtypes = [c_int, c_int, dp, c_int, dp, c_int, ip]
            getattr(L, f"oracle_expm_{suf}").argtypes = [
                c_int, dp, c_int, dp, c_int, c_int, ctypes.POINTER(_ExpmPlan), ip]
            getattr(L, f"oracle_getrf_{suf}").argtypes = [c_int, dp, c_int, ip]
            getattr(L, f"oracle_getrs_{suf}").argtypes = [c_int, c_int, dp, c_int, ip, dp, c_int]
            getattr(L, f"oracle_gebal_scale_{suf}").argtypes = [c_int, dp, c_int, dp, c_int, ip]
        L.oracle_gemm_d.argtypes = [c_int, c_int, c_int, c_double, dp, c_int, dp, c_int,
                                    c_double, dp, c_int]
        L.oracle_gemm_z.argtypes = [c_int, c_int, c_int, dp, dp, c_int, dp, c_int, dp, dp, c_int]
        L.oracle_paterson_stockmeyer_d.argtypes = [c_int, dp, c_int, dp, c_int, dp, c_int, c_int]
        L.oracle_horner_d.argtypes = [c_int, dp, c_int, dp, c_int, dp, c_int]
        for suf, ct in (("s", ctypes.c_float), ("d", c_double)):
            rp = ctypes.POINTER(ct)
            getattr(L, f"oracle_lacn2_{suf}").argtypes = [c_int, rp, rp, ip, rp, ip, ip]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _suffix(a: np.ndarray) -> str:
    return "z" if np.iscomplexobj(a) else "d"


def _as_f64(a) -> np.ndarray:
    a = np.asarray(a)
    dt = np.complex128 if np.iscomplexobj(a) else np.float64
    return np.asfortranarray(a, dtype=dt)


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def pade_theta(m: int, single: bool = False) -> float:
    return lib().oracle_pade_theta(m, int(single))


def expm_plan(norm1: float, single: bool = False) -> ExpmPlan:
    p = lib().oracle_expm_plan(float(norm1), int(single))
    return ExpmPlan(p.m, p.s, p.num_gemms)


def pade_coeffs(m: int):
    p = lib().oracle_pade_coeffs(m)
    if not p:
        return None
    return [p[i] for i in range(m + 1)]


def pade_num_powers(m: int) -> int:
    return lib().oracle_pade_num_powers(m)


def pade_num_gemms(m: int) -> int:
    return lib().oracle_pade_num_gemms(m)


def ps_cost(degree: int, s: int) -> int:
    return lib().oracle_ps_cost(degree, s)


def ps_block_size(degree: int) -> int:
    return lib().oracle_ps_block_size(degree)


def ps_plan(degree: int, s_requested: int = 0) -> PsPlan:
    p = lib().oracle_ps_plan(degree, s_requested)
    return PsPlan(p.s, p.r, p.num_powers, p.num_blocks, p.num_gemms)


def norm1(a) -> float:
    a = _as_f64(a)
    n = a.shape[0]
    return getattr(lib(), f"oracle_norm1_{_suffix(a)}")(n, _dp(a), max(n, 1))


def gemm(a, b, c=None, alpha=1.0, beta=0.0) -> np.ndarray:
    a, b = _as_f64(a), _as_f64(b)
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b) or (c is not None and np.iscomplexobj(c))
    dt = np.complex128 if cplx else np.float64
    a, b = np.asfortranarray(a, dtype=dt), np.asfortranarray(b, dtype=dt)
    m, k = a.shape
    n = b.shape[1]
    out = np.zeros((m, n), dtype=dt, order="F") if c is None else np.array(c, dtype=dt, order="F")
    if cplx:
        al = np.array([complex(alpha).real, complex(alpha).imag])
        be = np.array([complex(beta).real, complex(beta).imag])
        lib().oracle_gemm_z(m, n, k, _dp(al), _dp(a), max(m, 1), _dp(b), max(k, 1), _dp(be),
                            _dp(out), max(m, 1))
    else:
        lib().oracle_gemm_d(m, n, k, float(alpha), _dp(a), max(m, 1), _dp(b), max(k, 1),
                            float(beta), _dp(out), max(m, 1))
    return out


def getrf(a):
    """LU with partial pivoting; returns (LU, ipiv 0-based, info)."""
    a = np.array(_as_f64(a), order="F")
    n = a.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    info = getattr(lib(), f"oracle_getrf_{_suffix(a)}")(n, _dp(a), n, _ip(ipiv))
    return a, ipiv, info


def pade(a, m: int):
    """Unscaled r_m(A). Returns (R, getrf_info)."""
    a = _as_f64(a)
    n = a.shape[0]
    r = np.zeros_like(a, order="F")
    info = ctypes.c_int(0)
    rc = getattr(lib(), f"oracle_pade_{_suffix(a)}")(m, n, _dp(a), n, _dp(r), n,
                                                      ctypes.byref(info))
    if rc != 0:
        raise ValueError(f"oracle pade rejected its arguments (rc={rc})")
    return r, info.value


def expm(a, single: bool = False):
    """exp(A) by the reference's scaling and squaring, in FP64.

    ``single`` selects the single-precision theta ladder, i.e. the (m, s) the
    float / complex-float path picks. Returns (E, ExpmPlan, getrf_info).
    """
    a = _as_f64(a)
    n = a.shape[0]
    e = np.zeros_like(a, order="F")
    plan = _ExpmPlan()
    info = ctypes.c_int(0)
    rc = getattr(lib(), f"oracle_expm_{_suffix(a)}")(n, _dp(a), n, _dp(e), n, int(single),
                                                      ctypes.byref(plan), ctypes.byref(info))
    if rc == -2:
        raise FloatingPointError("1-norm is not finite")
    if rc != 0:
        raise ValueError(f"oracle expm rejected its arguments (rc={rc})")
    return e, ExpmPlan(plan.m, plan.s, plan.num_gemms), info.value


def expm_blas(a, single: bool = False):
    """Timing restatement of expm(): the same plan, Pade degree, scaling and
    product order (src/expm/expm.cppm:121-171, src/expm/pade.cppm:127-188:
    A2, A4 = A2 A2, A6 = A4 A2, A8 = A4 A4, degree 13 nested), with every
    product on numpy's BLAS and the solve on LAPACK xGESV (xGETRF + xGETRS),
    the reference's own CPU form of the path (GEMM through BLAS, LU through
    LAPACK; here the bundled OpenBLAS, threaded). FP64. Not bit-identical to
    expm() (the BLAS sums in its own order); expm() stays the checker.
    Returns (E, ExpmPlan)."""
    a = _as_f64(a)
    n = a.shape[0]
    plan = expm_plan(norm1(a), single)
    m, s = plan.m, plan.s
    b = pade_coeffs(m)
    x = np.asfortranarray(a * (2.0 ** (-s)))
    eye = np.eye(n, dtype=x.dtype)
    p = [x @ x]
    npw = pade_num_powers(m)
    if npw >= 2:
        p.append(p[0] @ p[0])
    if npw >= 3:
        p.append(p[1] @ p[0])
    if npw >= 4:
        p.append(p[1] @ p[1])
    if m != 13:
        v = b[0] * eye + sum(b[2 * (k + 1)] * p[k] for k in range(npw))
        w = b[1] * eye + sum(b[2 * (k + 1) + 1] * p[k] for k in range(npw))
    else:
        w = b[1] * eye + b[3] * p[0] + b[5] * p[1] + b[7] * p[2] + p[2] @ (b[9] * p[0] + b[11] * p[1] + b[13] * p[2])
        v = b[0] * eye + b[2] * p[0] + b[4] * p[1] + b[6] * p[2] + p[2] @ (b[8] * p[0] + b[10] * p[1] + b[12] * p[2])
    u = x @ w
    r = np.linalg.solve(v - u, v + u)
    for _ in range(s):
        r = r @ r
    return np.asfortranarray(r), plan


def paterson_stockmeyer(a, coeffs, s_requested: int = 0) -> np.ndarray:
    a = np.asfortranarray(a, dtype=np.float64)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    n = a.shape[0]
    p = np.zeros((n, n), order="F")
    rc = lib().oracle_paterson_stockmeyer_d(n, _dp(c), len(c) - 1, _dp(a), n, _dp(p), n,
                                            int(s_requested))
    if rc != 0:
        raise ValueError("oracle paterson_stockmeyer rejected its arguments")
    return p


def horner(a, coeffs) -> np.ndarray:
    a = np.asfortranarray(a, dtype=np.float64)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    n = a.shape[0]
    p = np.zeros((n, n), order="F")
    rc = lib().oracle_horner_d(n, _dp(c), len(c) - 1, _dp(a), n, _dp(p), n)
    if rc != 0:
        raise ValueError("oracle horner rejected its arguments")
    return p


def expm_vjp_block(a, g) -> np.ndarray:
    """dL/dA = L(A^H, G) for L = Re<G, expm(A)>, as the upper-right n x n block
    of expm([[A^H, G], [0, A^H]]) (Mathias' block formula; the form of
    torch.matrix_exp's backward), evaluated by the oracle's expm in FP64.
    This is the exact derivative up to the oracle expm's own accuracy; it does
    not depend on the (m, s) that expm picks for A."""
    a = _as_f64(a)
    g = _as_f64(g)
    n = a.shape[0]
    ah = a.conj().T
    blk = np.zeros((2 * n, 2 * n), dtype=a.dtype, order="F")
    blk[:n, :n] = ah
    blk[n:, n:] = ah
    blk[:n, n:] = g
    e, _, _ = expm(blk)
    return np.asfortranarray(e[:n, n:])


def expm_vjp_frechet(a, g, single: bool = False):
    """The adjoint the library computes, restated in numpy FP64: the forward-mode
    Frechet derivative (Al-Mohy and Higham 2009, Algorithm 6.4) at A^H in
    direction G of r_m(X / 2^s)^(2^s), (m, s) = expm_plan(||A||_1) (``single``:
    the single-precision theta ladder). Products in the library's order
    (A4 = A2 A2, A6 = A4 A2, A8 = A4 A4; degree 13 in the nested form of the
    oracle's pade). Returns (dL/dA, expm(A), ExpmPlan)."""
    a = _as_f64(a)
    g = _as_f64(g)
    n = a.shape[0]
    plan = expm_plan(norm1(a), single)
    m, s = plan.m, plan.s
    b = pade_coeffs(m)
    f = 2.0 ** (-s)
    x = f * a.conj().T
    d = f * g
    eye = np.eye(n, dtype=a.dtype)
    p = [x @ x]
    dm = [x @ d + d @ x]
    np_ = pade_num_powers(m)
    if np_ >= 2:
        p.append(p[0] @ p[0])
        dm.append(p[0] @ dm[0] + dm[0] @ p[0])
    if np_ >= 3:
        p.append(p[1] @ p[0])
        dm.append(dm[1] @ p[0] + p[1] @ dm[0])
    if np_ >= 4:
        p.append(p[1] @ p[1])
        dm.append(p[1] @ dm[1] + dm[1] @ p[1])
    if m != 13:
        v = b[0] * eye + sum(b[2 * (k + 1)] * p[k] for k in range(np_))
        w = b[1] * eye + sum(b[2 * (k + 1) + 1] * p[k] for k in range(np_))
        lv = sum(b[2 * (k + 1)] * dm[k] for k in range(np_))
        lw = sum(b[2 * (k + 1) + 1] * dm[k] for k in range(np_))
    else:
        w1 = b[9] * p[0] + b[11] * p[1] + b[13] * p[2]
        lw1 = b[9] * dm[0] + b[11] * dm[1] + b[13] * dm[2]
        w = b[1] * eye + b[3] * p[0] + b[5] * p[1] + b[7] * p[2] + p[2] @ w1
        lw = b[3] * dm[0] + b[5] * dm[1] + b[7] * dm[2] + p[2] @ lw1 + dm[2] @ w1
        z1 = b[8] * p[0] + b[10] * p[1] + b[12] * p[2]
        lz1 = b[8] * dm[0] + b[10] * dm[1] + b[12] * dm[2]
        v = b[0] * eye + b[2] * p[0] + b[4] * p[1] + b[6] * p[2] + p[2] @ z1
        lv = b[2] * dm[0] + b[4] * dm[1] + b[6] * dm[2] + p[2] @ lz1 + dm[2] @ z1
    u = x @ w
    lu = x @ lw + d @ w
    num, den = v + u, v - u
    dnum, dden = lv + lu, lv - lu
    r = np.linalg.solve(den, num)
    dr = np.linalg.solve(den, dnum - dden @ r)
    for _ in range(s):
        dr = r @ dr + dr @ r
        r = r @ r
    return np.asfortranarray(dr), np.asfortranarray(r.conj().T), plan


def gebal_scale(a, max_sweeps: int = 1000):
    """The scaling half of ?gebal (Parlett-Reinsch, powers of two): returns
    (B = D^-1 A D, diag(D), sweeps). The norms are summed in the library's
    sweep order, so FP64 results are bit-identical to it."""
    b = np.array(_as_f64(a), order="F")
    n = b.shape[0]
    d = np.ones(n)
    sweeps = ctypes.c_int(0)
    getattr(lib(), f"oracle_gebal_scale_{_suffix(b)}")(n, _dp(b), max(n, 1), _dp(d), max_sweeps,
                                                       ctypes.byref(sweeps))
    return b, d, sweeps.value


def expm_balanced(a, single: bool = False, blas: bool = False):
    """D exp(D^-1 A D) D^-1 with D from gebal_scale; returns (E, ExpmPlan of B).
    blas: the inner expm is the timing restatement expm_blas()."""
    b, d, _ = gebal_scale(a)
    e, plan = expm_blas(b, single) if blas else expm(b, single)[:2]
    return np.asfortranarray(e * d[:, None] / d[None, :]), plan


class Lacn2Trace:
    """One run of the 1-norm estimator: the kase returned by every call, the
    isave state after it, the final estimate and v (= A w)."""

    def __init__(self, kases, isaves, est, v):
        self.kases, self.isaves, self.est, self.v = kases, isaves, est, v


def lacn2(apply, apply_t, n: int, single: bool = False, max_calls: int = 64) -> Lacn2Trace:
    """Drive the reverse-communication estimator (xLACN2, oracle_lacn2_{s,d})
    to completion. ``apply(x)`` / ``apply_t(x)`` return A x / A^T x as numpy
    vectors; they are evaluated in float64 and rounded to the working
    precision."""
    dt = np.float32 if single else np.float64
    ct = ctypes.c_float if single else ctypes.c_double
    fn = getattr(lib(), "oracle_lacn2_" + ("s" if single else "d"))
    v = np.zeros(n, dtype=dt)
    x = np.zeros(n, dtype=dt)
    isgn = np.zeros(max(n, 1), dtype=np.int32)
    est, kase = ct(0), ctypes.c_int(0)
    isave = (ctypes.c_int * 3)()
    rp = ctypes.POINTER(ct)
    kases, isaves = [], []
    for _ in range(max_calls):
        rc = fn(n, v.ctypes.data_as(rp), x.ctypes.data_as(rp), _ip(isgn), ctypes.byref(est),
                ctypes.byref(kase), isave)
        if rc != 0:
            raise ValueError("oracle_lacn2: invalid argument or state")
        kases.append(kase.value)
        isaves.append(tuple(isave))
        if kase.value == 0:
            return Lacn2Trace(kases, isaves, float(est.value), v.copy())
        y = apply(x.astype(np.float64)) if kase.value == 1 else apply_t(x.astype(np.float64))
        x[:] = np.asarray(y, dtype=np.float64).astype(dt)
    raise RuntimeError("oracle_lacn2 did not finish")


def hermitian_from_triangle(a, upper: bool) -> np.ndarray:
    """The symmetric / Hermitian matrix whose `upper` (else lower) triangle is
    a's, diagonal real: what an eigensolver reading one triangle sees."""
    a = _as_f64(a)
    t = np.triu(a) if upper else np.tril(a)
    h = t + (np.triu(a, 1) if upper else np.tril(a, -1)).conj().T
    np.fill_diagonal(h, np.real(np.diag(a)))
    return np.asfortranarray(h)


def heevd(a, upper: bool = False):
    """Eigenvalues (ascending) and eigenvectors of the Hermitian matrix read
    from one triangle: LAPACK xSYEVD / xHEEVD through numpy.linalg.eigh (the
    routine the reference reaches through WarpWraps as the vendor's syevd /
    heevd, src/expm/expm_herm.cppm:176-182)."""
    h = hermitian_from_triangle(a, upper)
    w, u = np.linalg.eigh(h)
    return w, np.asfortranarray(u)


def expm_herm(a, upper: bool = False) -> np.ndarray:
    """exp(A) = U diag(exp(w)) U^H for symmetric / Hermitian A read from one
    triangle (calaman::expm_herm, src/expm/expm_herm.cppm:163-196: eigensolve,
    column scale by exp(w_j), one product with U^H)."""
    w, u = heevd(a, upper)
    return np.asfortranarray((u * np.exp(w)[None, :]) @ u.conj().T)


def geodesic_points(w, h, step: float, num_samples: int, blas: bool = False):
    """The rotation half of the cg_unitary sampling sweep in the reference's
    order (src/cg_unitary/geodesic_search.cppm:354-410): R_1 = expm(step H)
    with the general expm, R_j = R_{j-1} R_1, W_j = R_j W, j = 1..N-1.
    blas: R_1 by the timing restatement expm_blas()."""
    w = _as_f64(w)
    h = _as_f64(h)
    r1 = expm_blas(step * h)[0] if blas else expm(step * h)[0]
    out, r = [], None
    for j in range(1, num_samples):
        r = r1 if j == 1 else r @ r1
        out.append(np.asfortranarray(r @ w))
    return out
