"""Generate ``lacn2.json``: traces of LAPACK's own xLACN2 on the operators of
``lacn2_cases.py``. Run: ``python tests/golden/make_lacn2_golden.py``.

The reference's lacn2 (src/lapack/lacn2/interface.cppm) restates LAPACK's
DLACN2/SLACN2, and its test suite compares it with the Fortran routine called
by symbol (src/lapack/lacn2/README.md:40-47). The same pin is made here: the
LAPACK inside the OpenBLAS that scipy bundles is driven through its LAPACKE
entry point (scipy_LAPACKE_{s,d}lacn2_work: no NaN screening, 32-bit integers) on each seeded
operator, and the kase sequence, isave states, estimate and final v are
recorded. The products are computed by ``lacn2_cases.operators`` and rounded
to the working precision, exactly as the oracle's driver does.
"""
from __future__ import annotations

import ctypes
import glob
import json
import os

import numpy as np
import scipy

from lacn2_cases import CASES, make_matrix, operators

HERE = os.path.dirname(os.path.abspath(__file__))


def _lapacke():
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                  "libscipy_openblas*.so*"))
    if not libs:
        raise SystemExit("scipy's bundled OpenBLAS not found")
    return ctypes.CDLL(libs[0])


def trace(lib, a, single):
    n = a.shape[0]
    dt, ct = (np.float32, ctypes.c_float) if single else (np.float64, ctypes.c_double)
    fn = lib.scipy_LAPACKE_slacn2_work if single else lib.scipy_LAPACKE_dlacn2_work
    fn.restype = ctypes.c_int
    rp = ctypes.POINTER(ct)
    v, x = np.zeros(n, dt), np.zeros(n, dt)
    isgn = np.zeros(n, np.int32)
    est, kase = ct(0), ctypes.c_int(0)
    isave = (ctypes.c_int * 3)()
    apply, apply_t = operators(a)
    kases, isaves = [], []
    for _ in range(64):
        rc = fn(n, v.ctypes.data_as(rp), x.ctypes.data_as(rp),
                isgn.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(est),
                ctypes.byref(kase), isave)
        assert rc == 0
        kases.append(kase.value)
        isaves.append(list(isave))
        if kase.value == 0:
            break
        y = apply(x.astype(np.float64)) if kase.value == 1 else apply_t(x.astype(np.float64))
        x[:] = y.astype(dt)
    return {"kases": kases, "isaves": isaves, "est": float(est.value),
            "v": [float(t) for t in v]}


def main():
    lib = _lapacke()
    out = {}
    for name, kind, n, seed, single in CASES:
        a = make_matrix(kind, n, seed)
        if single:
            a = a.astype(np.float32).astype(np.float64)
        t = trace(lib, a, single)
        t.update({"kind": kind, "n": n, "seed": seed, "single": single,
                  "norm1": float(np.abs(a).sum(axis=0).max())})
        out[name] = t
    with open(os.path.join(HERE, "lacn2.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {len(out)} traces")


if __name__ == "__main__":
    main()
