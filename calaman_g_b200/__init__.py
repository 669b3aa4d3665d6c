"""B200-native matrix exponential: calaman_G's expm / pade / matrix_norm1 /
horner / paterson_stockmeyer path on sm_100a kernels.

The product is the C ABI in ``include/calaman_b200.h`` (``lib/libcalaman_b200.so``).
This module is the Python host mirror of the reference interface: the same
function names, argument meaning and status codes, operating on torch CUDA
tensors (torch supplies device memory and streams, nothing else). Every call
goes through the C ABI; there is no CPU fallback.

Matrices are square 2-D tensors. They are handed to the library column-major,
as the reference stores them, so the 1-norm (and with it the Pade degree and
scaling) is the maximum absolute COLUMN sum of the matrix as written.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import capi
from .capi import ExpmPlan, PsPlan, Status

__all__ = [
    "Handle", "Status", "ExpmPlan", "PsPlan", "CalamanError", "expm", "pade", "matrix_norm1",
    "expm_plan", "pade_theta", "expm_bufferSize", "pade_bufferSize", "expm_vjp",
    "expm_vjp_bufferSize", "expm_ad", "horner",
    "horner_bufferSize", "paterson_stockmeyer", "paterson_stockmeyer_plan",
    "paterson_stockmeyer_bufferSize", "paterson_stockmeyer_cost",
    "paterson_stockmeyer_block_size", "to_colmajor", "from_colmajor", "lib",
    "lacn2_bufferSize", "lacn2_estimate",
]


def lib() -> ctypes.CDLL:
    return capi.load()


class CalamanError(RuntimeError):
    def __init__(self, what: str, status: Status):
        super().__init__(f"{what} failed: {status!r}")
        self.status = status


def _check(what: str, st: Status) -> None:
    if not st.ok:
        raise CalamanError(what, st)


def _torch():
    import torch

    return torch


_SUFFIX = None


def _suffix(dtype) -> str:
    global _SUFFIX
    if _SUFFIX is None:
        torch = _torch()
        _SUFFIX = {torch.float32: "s", torch.float64: "d", torch.complex64: "c",
                   torch.complex128: "z"}
    try:
        return _SUFFIX[dtype]
    except KeyError as e:
        raise TypeError(f"unsupported dtype {dtype}: float32/float64/complex64/complex128") from e


class Handle:
    """calamanHandle_t: the device, stream and pointer mode of a call."""

    def __init__(self, stream=None):
        h = ctypes.c_void_p()
        _check("calamanCreate", lib().calamanCreate(ctypes.byref(h)))
        self.ptr = h
        self.set_stream(stream)

    def set_stream(self, stream=None) -> None:
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream()
        raw = s.cuda_stream if hasattr(s, "cuda_stream") else int(s)
        _check("calamanSetStream", lib().calamanSetStream(self.ptr, ctypes.c_void_p(raw)))
        self.stream = raw

    def close(self) -> None:
        if self.ptr:
            lib().calamanDestroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: Handle | None = None


def default_handle() -> Handle:
    global _default
    if _default is None:
        _default = Handle()
    _default.set_stream()
    return _default


def to_colmajor(a):
    """A square tensor -> a contiguous buffer holding it column-major."""
    return a.transpose(0, 1).contiguous()


def from_colmajor(buf, n: int):
    """A column-major n x n buffer -> the matrix as an (n, n) tensor view."""
    return buf.reshape(n, n).transpose(0, 1)


def _vp(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def pade_theta(m: int, single: bool = False) -> float:
    return lib().calaman_pade_theta_s(m) if single else lib().calaman_pade_theta_d(m)


def expm_plan(norm1: float, single: bool = False) -> ExpmPlan:
    return lib().calaman_expm_plan_s(norm1) if single else lib().calaman_expm_plan_d(norm1)


def expm_bufferSize(n: int, dtype) -> int:
    b = ctypes.c_size_t()
    _check("expm_bufferSize",
           getattr(lib(), f"calaman_expm_bufferSize_{_suffix(dtype)}")(None, n, ctypes.byref(b)))
    return b.value


def pade_bufferSize(m: int, n: int, dtype) -> int:
    b = ctypes.c_size_t()
    _check("pade_bufferSize",
           getattr(lib(), f"calaman_pade_bufferSize_{_suffix(dtype)}")(None, m, n, ctypes.byref(b)))
    return b.value


@dataclass
class _Buffers:
    work: object
    info: object


def _buffers(nbytes: int, device):
    torch = _torch()
    return _Buffers(torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device),
                    torch.zeros(2, dtype=torch.int32, device=device))


def expm(a, handle: Handle | None = None, out=None, return_plan: bool = False):
    """exp(A) for a square CUDA tensor (float32/float64/complex64/complex128).

    Scaling and squaring with the diagonal Pade degree chosen from the 1-norm
    (src/expm/expm.cppm:87-174). Synchronises the stream once.
    """
    torch = _torch()
    n = a.shape[0]
    h = handle or default_handle()
    A = to_colmajor(a)
    E = torch.empty_like(A) if out is None else out
    bufs = _buffers(expm_bufferSize(n, a.dtype), a.device)
    plan = ExpmPlan()
    st = getattr(lib(), f"calaman_expm_{_suffix(a.dtype)}")(
        h.ptr, h.ptr, ctypes.c_void_p(h.stream), n, _vp(A), n, _vp(E), n, _vp(bufs.work),
        bufs.work.numel(), ctypes.cast(bufs.info.data_ptr(), capi.c_int_p), ctypes.byref(plan))
    _check("expm", st)
    res = from_colmajor(E, n)
    return (res, plan) if return_plan else res


def expm_vjp_bufferSize(n: int, dtype) -> int:
    b = ctypes.c_size_t()
    _check("expm_vjp_bufferSize",
           getattr(lib(), f"calaman_expm_vjp_bufferSize_{_suffix(dtype)}")(None, n, ctypes.byref(b)))
    return b.value


def expm_vjp(a, g, handle: Handle | None = None, return_expm: bool = False,
             return_plan: bool = False):
    """dL/dA for a real loss L of E = expm(A), given G = dL/dE.

    L(A^H, G): the Frechet derivative at A^H (A^T for real dtypes), in
    direction G, of the Pade-based function expm evaluates for A -- the
    convention of torch.matrix_exp's backward. With return_expm, also returns
    expm(A) from the same evaluation. Synchronises the stream once.
    """
    torch = _torch()
    n = a.shape[0]
    if g.shape != a.shape or g.dtype != a.dtype:
        raise ValueError("expm_vjp: G must match A in shape and dtype")
    h = handle or default_handle()
    A = to_colmajor(a)
    G = to_colmajor(g)
    D = torch.empty_like(A)
    E = torch.empty_like(A) if return_expm else None
    bufs = _buffers(expm_vjp_bufferSize(n, a.dtype), a.device)
    plan = ExpmPlan()
    st = getattr(lib(), f"calaman_expm_vjp_{_suffix(a.dtype)}")(
        h.ptr, h.ptr, ctypes.c_void_p(h.stream), n, _vp(A), n, _vp(G), n, _vp(D), n,
        _vp(E) if E is not None else None, n, _vp(bufs.work), bufs.work.numel(),
        ctypes.cast(bufs.info.data_ptr(), capi.c_int_p), ctypes.byref(plan))
    _check("expm_vjp", st)
    out = [from_colmajor(D, n)]
    if return_expm:
        out.append(from_colmajor(E, n))
    if return_plan:
        out.append(plan)
    return out[0] if len(out) == 1 else tuple(out)


_ExpmFn = None


def expm_ad(a):
    """expm(A) as a differentiable torch op: forward through calaman expm,
    backward through calaman expm_vjp."""
    global _ExpmFn
    torch = _torch()
    if _ExpmFn is None:
        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, x):
                ctx.save_for_backward(x)
                return expm(x)

            @staticmethod
            def backward(ctx, grad):
                (x,) = ctx.saved_tensors
                return expm_vjp(x, grad.contiguous())

        _ExpmFn = _Fn
    return _ExpmFn.apply(a)


def pade(a, m: int, handle: Handle | None = None):
    """Unscaled r_m(A) (src/expm/pade.cppm:77-191); never synchronises."""
    torch = _torch()
    n = a.shape[0]
    h = handle or default_handle()
    A = to_colmajor(a)
    R = torch.empty_like(A)
    bufs = _buffers(pade_bufferSize(m, n, a.dtype), a.device)
    st = getattr(lib(), f"calaman_pade_{_suffix(a.dtype)}")(
        h.ptr, h.ptr, ctypes.c_void_p(h.stream), m, n, _vp(A), n, _vp(R), n, _vp(bufs.work),
        bufs.work.numel(), ctypes.cast(bufs.info.data_ptr(), capi.c_int_p))
    _check("pade", st)
    return from_colmajor(R, n)


def matrix_norm1(a, handle: Handle | None = None) -> float:
    """Maximum absolute column sum (true modulus); synchronises."""
    torch = _torch()
    n = a.shape[0]
    h = handle or default_handle()
    A = to_colmajor(a)
    real = torch.float32 if a.dtype in (torch.float32, torch.complex64) else torch.float64
    cs = torch.empty(n, dtype=real, device=a.device)
    return getattr(lib(), f"calaman_matrix_norm1_{_suffix(a.dtype)}")(
        ctypes.c_void_p(h.stream), n, _vp(A), n, _vp(cs))


def lacn2_bufferSize(n: int, dtype) -> int:
    return getattr(lib(), f"calaman_lacn2_bufferSize_{_suffix(dtype)}")(n)


def lacn2_estimate(apply, apply_t, n: int, dtype=None, handle: Handle | None = None,
                   device=None):
    """Estimate ||A||_1 of an operator given only its products, by driving the
    reverse-communication estimator (calaman_lacn2_*, LAPACK xLACN2) to
    completion. ``apply(x)`` / ``apply_t(x)`` return A x / A^T x for a CUDA
    vector x of ``dtype`` (float32 or float64), on the handle's stream.
    Returns (est, v) with est <= ||A||_1 and v = A w, est = ||v||_1 / ||w||_1."""
    torch = _torch()
    dtype = dtype or torch.float64
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("lacn2 is real only (float32 or float64)")
    suf = _suffix(dtype)
    ct = ctypes.c_float if dtype == torch.float32 else ctypes.c_double
    h = handle or default_handle()
    dev = device or torch.device("cuda", torch.cuda.current_device())
    nbytes = lacn2_bufferSize(n, dtype)
    work = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
    v = torch.zeros(n, dtype=dtype, device=dev)
    x = torch.zeros(n, dtype=dtype, device=dev)
    est, kase = ct(0), ctypes.c_int(0)
    isave = (ctypes.c_int * 3)()
    fn = getattr(lib(), f"calaman_lacn2_{suf}")
    while True:
        _check("lacn2", fn(h.ptr, n, _vp(v), _vp(x), _vp(work), nbytes, ctypes.byref(est),
                           ctypes.byref(kase), isave))
        if kase.value == 0:
            return float(est.value), v
        x.copy_(apply(x) if kase.value == 1 else apply_t(x))


def horner_bufferSize(n: int, dtype) -> int:
    return getattr(lib(), f"calaman_horner_bufferSize_{_suffix(dtype)}")(n)


def horner(a, coeffs, handle: Handle | None = None):
    """p(A) = sum c_k A^k by Horner's rule; coefficients ascending."""
    torch = _torch()
    n = a.shape[0]
    h = handle or default_handle()
    A = to_colmajor(a)
    c = torch.as_tensor(coeffs, dtype=a.dtype, device=a.device).contiguous()
    P = torch.empty_like(A)
    degree = c.numel() - 1
    w = torch.empty(max(horner_bufferSize(n, a.dtype), 256), dtype=torch.uint8, device=a.device)
    st = getattr(lib(), f"calaman_horner_{_suffix(a.dtype)}")(
        h.ptr, n, _vp(c), degree, _vp(A), n, _vp(P), n, _vp(w), w.numel())
    _check("horner", st)
    return from_colmajor(P, n)


def paterson_stockmeyer_cost(degree: int, s: int) -> int:
    return lib().calaman_paterson_stockmeyer_cost(degree, s)


def paterson_stockmeyer_block_size(degree: int) -> int:
    return lib().calaman_paterson_stockmeyer_block_size(degree)


def paterson_stockmeyer_plan(degree: int, s_requested: int = 0) -> PsPlan:
    return lib().calaman_paterson_stockmeyer_plan(degree, s_requested)


def paterson_stockmeyer_bufferSize(n: int, degree: int, dtype, s_requested: int = 0) -> int:
    return getattr(lib(), f"calaman_paterson_stockmeyer_bufferSize_{_suffix(dtype)}")(
        n, degree, s_requested)


def paterson_stockmeyer(a, coeffs, s_requested: int = 0, handle: Handle | None = None):
    """p(A) = sum c_k A^k by Paterson-Stockmeyer; coefficients ascending."""
    torch = _torch()
    n = a.shape[0]
    h = handle or default_handle()
    A = to_colmajor(a)
    c = torch.as_tensor(coeffs, dtype=a.dtype, device=a.device).contiguous()
    P = torch.empty_like(A)
    degree = c.numel() - 1
    nb = paterson_stockmeyer_bufferSize(n, degree, a.dtype, s_requested)
    w = torch.empty(max(nb, 256), dtype=torch.uint8, device=a.device)
    st = getattr(lib(), f"calaman_paterson_stockmeyer_{_suffix(a.dtype)}")(
        h.ptr, n, _vp(c), degree, _vp(A), n, _vp(P), n, _vp(w), w.numel(), s_requested)
    _check("paterson_stockmeyer", st)
    return from_colmajor(P, n)
