"""ctypes binding of the C ABI declared in ``include/calaman_b200.h``.

This is the reference-side binding a Python caller would write: plain
pointers and sizes, no torch types. Loading fails loudly when the CUDA
library has not been built -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcalaman_b200.so")

c_int, c_float, c_double, c_size_t, c_void_p = (
    ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_size_t_p = ctypes.POINTER(ctypes.c_size_t)

# numerical status codes (include/calaman_b200.h)
SUCCESS = 0
NOT_INITIALIZED = 1
ALLOC_FAILED = 3
INVALID_VALUE = 7
NOT_SUPPORTED = 15
DOMAIN_BLAS, DOMAIN_SOLVER, DOMAIN_RUNTIME = 0, 1, 2
POINTER_MODE_HOST, POINTER_MODE_DEVICE = 0, 1
FILL_LOWER, FILL_UPPER = 0, 1

_NAMES = {0: "SUCCESS", 1: "NOT_INITIALIZED", 3: "ALLOC_FAILED", 7: "INVALID_VALUE",
          8: "ARCH_MISMATCH", 13: "EXECUTION_FAILED", 14: "INTERNAL_ERROR", 15: "NOT_SUPPORTED"}


class Status(ctypes.Structure):
    """calamanStatus_t: {domain, code}; every success compares equal."""

    _fields_ = [("domain", ctypes.c_int32), ("code", ctypes.c_int32)]

    @property
    def ok(self) -> bool:
        return self.code == 0

    def name(self) -> str:
        if self.domain == DOMAIN_RUNTIME:
            return f"cudaError({self.code})"
        return _NAMES.get(self.code, f"status({self.code})")

    def __eq__(self, other) -> bool:  # outcome equality, as the reference's Status
        if isinstance(other, int):
            return self.code == other if other != 0 else self.ok
        if isinstance(other, Status):
            if self.ok or other.ok:
                return self.ok and other.ok
            return (self.domain, self.code) == (other.domain, other.code)
        return NotImplemented

    def __repr__(self) -> str:
        dom = {0: "blas", 1: "solver", 2: "runtime"}.get(self.domain, "?")
        return f"Status({dom}, {self.name()})"


class ExpmPlan(ctypes.Structure):
    _fields_ = [("m", c_int), ("s", c_int), ("num_gemms", c_int)]

    def __repr__(self) -> str:
        return f"ExpmPlan(m={self.m}, s={self.s}, num_gemms={self.num_gemms})"


class PsPlan(ctypes.Structure):
    _fields_ = [("s", c_int), ("r", c_int), ("num_powers", c_int), ("num_blocks", c_int),
                ("num_gemms", c_int)]


class KernelTiming(ctypes.Structure):
    _fields_ = [("gemm_launches", ctypes.c_longlong), ("gemm_ms", c_double),
                ("gemm_flops", c_double)]


# symbol -> (restype, argtypes); the list mirrors include/calaman_b200.h
_H = c_void_p  # calamanHandle_t
_EXPM = [_H, _H, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_size_t, c_int_p,
         ctypes.POINTER(ExpmPlan)]
_PADE = [_H, _H, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_size_t,
         c_int_p]
# expm_vjp: blas, solver, stream, n, A, lda, G, ldg, gradA, ldga, expA, lde, work, bytes, info, plan
_VJP = [_H, _H, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int,
        c_void_p, c_size_t, c_int_p, ctypes.POINTER(ExpmPlan)]
_HORNER = [_H, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_size_t]
_PS = _HORNER + [c_int]

SIGNATURES = {
    "calamanCreate": (Status, [ctypes.POINTER(c_void_p)]),
    "calamanDestroy": (Status, [_H]),
    "calamanSetStream": (Status, [_H, c_void_p]),
    "calamanGetStream": (Status, [_H, ctypes.POINTER(c_void_p)]),
    "calamanSetPointerMode": (Status, [_H, c_int]),
    "calamanGetPointerMode": (Status, [_H, c_int_p]),
    "calamanGetVersion": (ctypes.c_char_p, []),
    "calaman_pade_theta_s": (c_float, [c_int]),
    "calaman_pade_theta_d": (c_double, [c_int]),
    "calaman_expm_plan_s": (ExpmPlan, [c_float]),
    "calaman_expm_plan_d": (ExpmPlan, [c_double]),
    "calaman_pade_num_powers": (c_int, [c_int]),
    "calaman_pade_num_gemms": (c_int, [c_int]),
    "calaman_horner_bufferSize_s": (c_size_t, [c_int]),
    "calaman_horner_bufferSize_d": (c_size_t, [c_int]),
    "calaman_horner_s": (Status, _HORNER),
    "calaman_horner_d": (Status, _HORNER),
    "calaman_paterson_stockmeyer_cost": (c_int, [c_int, c_int]),
    "calaman_paterson_stockmeyer_block_size": (c_int, [c_int]),
    "calaman_paterson_stockmeyer_plan": (PsPlan, [c_int, c_int]),
    "calaman_paterson_stockmeyer_power_stride_s": (c_size_t, [c_int]),
    "calaman_paterson_stockmeyer_power_stride_d": (c_size_t, [c_int]),
    "calaman_paterson_stockmeyer_bufferSize_s": (c_size_t, [c_int, c_int, c_int]),
    "calaman_paterson_stockmeyer_bufferSize_d": (c_size_t, [c_int, c_int, c_int]),
    "calaman_paterson_stockmeyer_s": (Status, _PS),
    "calaman_paterson_stockmeyer_d": (Status, _PS),
    "calamanGetLaunchCount": (ctypes.c_ulonglong, []),
    "calamanSetKernelTiming": (Status, [_H, c_int]),
    "calamanGetKernelTiming": (Status, [_H, ctypes.POINTER(KernelTiming)]),
}
_GEMM = [c_void_p, c_int, c_int, c_int, c_double, c_void_p, c_int, c_void_p, c_int, c_double,
         c_void_p, c_int]
for _suf, _real in (("s", c_float), ("d", c_double), ("c", c_float), ("z", c_double)):
    SIGNATURES[f"calaman_expm_bufferSize_{_suf}"] = (Status, [_H, c_int, c_size_t_p])
    SIGNATURES[f"calaman_pade_bufferSize_{_suf}"] = (Status, [_H, c_int, c_int, c_size_t_p])
    SIGNATURES[f"calaman_expm_{_suf}"] = (Status, _EXPM)
    SIGNATURES[f"calaman_expm_vjp_bufferSize_{_suf}"] = (Status, [_H, c_int, c_size_t_p])
    SIGNATURES[f"calaman_expm_vjp_{_suf}"] = (Status, _VJP)
    SIGNATURES[f"calaman_pade_{_suf}"] = (Status, _PADE)
    SIGNATURES[f"calaman_matrix_norm1_{_suf}"] = (_real, [c_void_p, c_int, c_void_p, c_int, c_void_p])
    SIGNATURES[f"calaman_gemm_{_suf}"] = (Status, _GEMM)
    SIGNATURES[f"calaman_getrf_{_suf}"] = (Status, [c_void_p, c_int, c_void_p, c_int, c_void_p,
                                                   c_int_p])
    SIGNATURES[f"calaman_getrs_{_suf}"] = (Status, [c_void_p, c_int, c_int, c_void_p, c_int,
                                                   c_void_p, c_void_p, c_int, c_void_p, c_int,
                                                   c_int_p])
SIGNATURES["calaman_getrf_bufferSize"] = (Status, [c_int, c_size_t_p])
SIGNATURES["calaman_gemm_bf16x_bufferSize"] = (Status, [c_int, c_int, c_int, c_int, c_size_t_p])
SIGNATURES["calaman_gemm_bf16x_s"] = (Status, _GEMM + [c_int, c_void_p, c_size_t])
SIGNATURES["calaman_gemm_bf16x_bufferSize_c"] = (Status, [c_int, c_int, c_int, c_int, c_size_t_p])
SIGNATURES["calaman_gemm_bf16x_c"] = (Status, _GEMM + [c_int, c_void_p, c_size_t])
SIGNATURES["calamanSetWorkspace"] = (Status, [_H, c_void_p, c_size_t])
SIGNATURES["calaman_poly_tensor_workspace_s"] = (c_size_t, [c_int])
SIGNATURES["calaman_grid_barrier_wait_check"] = (Status, [c_void_p, ctypes.c_uint, c_void_p, c_size_t, c_int_p])
SIGNATURES["calamanSetBatchedGraphs"] = (Status, [_H, c_int])
SIGNATURES["calamanGetBatchedGraphs"] = (Status, [_H, c_int_p, c_int_p])
SIGNATURES["calamanSetExpmGraphs"] = (Status, [_H, c_int])
SIGNATURES["calamanGetExpmGraphs"] = (Status, [_H, c_int_p, c_int_p])
SIGNATURES["calamanSetBatchedTuning"] = (Status, [_H, c_int_p, c_int])
SIGNATURES["calamanGetBatchedTuning"] = (Status, [_H, c_int_p, c_int_p])
SIGNATURES["calamanTuneBatched_bufferSize"] = (c_size_t, [c_int])
SIGNATURES["calamanTuneBatched"] = (Status, [_H, c_int, c_void_p, c_size_t, c_int_p, c_int_p])
SIGNATURES["calamanSetDoubleEmulation"] = (Status, [_H, c_int])
SIGNATURES["calamanGetDoubleEmulation"] = (Status, [_H, c_int_p])
SIGNATURES["calaman_gemm_ozaki_bufferSize"] = (Status, [c_int, c_int, c_int, c_int, c_int, c_size_t_p])
SIGNATURES["calaman_gemm_ozaki_d"] = (Status, _GEMM + [c_int, c_void_p, c_size_t])
SIGNATURES["calaman_gemm_ozaki_z"] = (Status, _GEMM + [c_int, c_void_p, c_size_t])
SIGNATURES["calaman_gemm_ozaki_wait_check"] = (Status, [c_void_p, ctypes.c_longlong, c_void_p, c_size_t,
                                                        c_int_p])
SIGNATURES["calaman_expm_noalloc_d"] = (Status, [_H, c_void_p, c_int, c_void_p, c_int, c_void_p,
                                                 c_int, c_int_p, ctypes.POINTER(ExpmPlan)])
# expm_batched: blas, solver, stream, batch, h_n, h_A, h_lda, h_E, h_lde, work, bytes, info, plans
_BATCHED = [_H, _H, c_void_p, c_int, c_int_p, ctypes.POINTER(c_void_p), c_int_p,
            ctypes.POINTER(c_void_p), c_int_p, c_void_p, c_size_t, c_int_p, ctypes.POINTER(ExpmPlan)]
# expm_vjp_batched: blas, solver, stream, batch, h_n, h_A, h_lda, h_G, h_ldg, h_gradA, h_ldga,
#                   h_expA, h_lde, work, bytes, info, plans
_PP = ctypes.POINTER(c_void_p)
_VJPB = [_H, _H, c_void_p, c_int, c_int_p, _PP, c_int_p, _PP, c_int_p, _PP, c_int_p, _PP, c_int_p,
         c_void_p, c_size_t, c_int_p, ctypes.POINTER(ExpmPlan)]
for _suf in ("s", "d"):
    SIGNATURES[f"calaman_expm_batched_bufferSize_{_suf}"] = (Status, [_H, c_int, c_int_p, c_size_t_p])
    SIGNATURES[f"calaman_expm_batched_{_suf}"] = (Status, _BATCHED)
    SIGNATURES[f"calaman_expm_vjp_batched_bufferSize_{_suf}"] = (Status, [_H, c_int, c_int_p, c_size_t_p])
    SIGNATURES[f"calaman_expm_vjp_batched_{_suf}"] = (Status, _VJPB)
SIGNATURES["calaman_gebal_bufferSize"] = (Status, [c_int, c_int_p])
for _suf in ("s", "d", "c", "z"):
    # gebal: stream, job, n, A, lda, ilo, ihi, scale, work, max_sweeps, sweeps
    SIGNATURES[f"calaman_gebal_{_suf}"] = (Status, [c_void_p, c_int, c_int, c_void_p, c_int, c_int_p,
                                                   c_int_p, c_void_p, c_void_p, c_int, c_int_p])
    SIGNATURES[f"calaman_expm_balanced_bufferSize_{_suf}"] = (Status, [_H, c_int, c_size_t_p])
    SIGNATURES[f"calaman_expm_balanced_{_suf}"] = (Status, _EXPM)
for _suf in ("s", "d", "c", "z"):
    # expm_herm: blas, solver, stream, uplo, n, A, lda, E, lde, work, bytes, info
    SIGNATURES[f"calaman_expm_herm_bufferSize_{_suf}"] = (Status, [_H, c_int, c_int, c_size_t_p])
    SIGNATURES[f"calaman_expm_herm_{_suf}"] = (Status, [_H, _H, c_void_p, c_int, c_int, c_void_p, c_int,
                                                       c_void_p, c_int, c_void_p, c_size_t, c_int_p])
    # heevd: stream, uplo, n, A, lda, w, work, bytes, info
    SIGNATURES[f"calaman_heevd_bufferSize_{_suf}"] = (Status, [c_int, c_int, c_size_t_p])
    SIGNATURES[f"calaman_heevd_{_suf}"] = (Status, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                                   c_void_p, c_size_t, c_int_p])
for _suf in ("s", "d", "c", "z"):
    # geodesic points: blas, solver, stream, n, W, ldw, H, ldh, step, num_samples, Wout, work, bytes, info
    SIGNATURES[f"calaman_geodesic_points_bufferSize_{_suf}"] = (Status, [_H, c_int, c_int, c_size_t_p])
    SIGNATURES[f"calaman_geodesic_points_{_suf}"] = (Status, [_H, _H, c_void_p, c_int, c_void_p, c_int,
                                                             c_void_p, c_int, c_double, c_int, c_void_p,
                                                             c_void_p, c_size_t, c_int_p])
for _suf, _real in (("s", c_float), ("d", c_double)):
    # lacn2: blas, n, v, x, work, bytes, est (host), kase (host), isave[3] (host)
    SIGNATURES[f"calaman_lacn2_bufferSize_{_suf}"] = (c_size_t, [c_int])
    SIGNATURES[f"calaman_lacn2_{_suf}"] = (Status, [_H, c_int, c_void_p, c_void_p, c_void_p, c_size_t,
                                                   ctypes.POINTER(_real), c_int_p, c_int_p])
SIGNATURES["calamanSetFloatSplit"] = (Status, [_H, c_int])
SIGNATURES["calamanGetFloatSplit"] = (Status, [_H, c_int_p])

_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m calaman_g_b200.build` "
                "(the matrix-exponential path has no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def declared_symbols(header: str | None = None) -> list[str]:
    """Every function name declared in include/calaman_b200.h."""
    import re

    header = header or os.path.join(HERE, "..", "include", "calaman_b200.h")
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(calaman\w*)\s*\(", text)))
