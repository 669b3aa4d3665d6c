"""Oracle parity at the benchmark workloads themselves, on the benchmark's own
generators and seeds (bench.make_matrix, bench.batched_spec,
bench.batched_matrix), through the C ABI:

  float64 256 x 256, ||A||_1 = 4                     <= 1e-12 vs the oracle
  complex128 1024 x 1024, A = -iH (GUE), ||A||_1 = 50  <= 1e-12, plan (13, 4),
                                                     ||U^H U - I||_F <= 1e-12 n
  float32 4096 x 4096, ||A||_1 = 8                   <= 1e-6 vs exp(A) in FP64
  float64 2048 x 2048, ||A||_1 = 6                   <= 1e-12 vs the oracle
  8192 matrices, n on {16..256}, ||A||_1 in [0.1, 100]:
      FP64 tier vs the oracle on a subsample covering every size and both
      s = 0 and s > 0 (<= 1e-12); FP32 tier vs FP64 tier on all 8192 (<= 1e-6)

The tolerances follow the expm contract (src/expm/expm.cppm:87-174) and the
reference's accuracy check (test/expm/expm_tests.cpp:206-228); the 1e-6 bar of
the single-precision workloads is measured against FP64. The oracle runs on
every host thread."""
import ctypes
import os

import numpy as np
import pytest

import bench
from helpers import Runner, rel_frob

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
MIXED_REL = 1e-6


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


@pytest.fixture(scope="module")
def orc(oracle):
    oracle.set_threads(os.cpu_count() or 1)
    yield oracle
    oracle.set_threads(1)


def _single(run, orc, name):
    cfg = bench.CONFIGS[name]
    a = bench.make_matrix(cfg)
    st, plan, e, _, info = run.expm(a, cfg["suf"])
    assert st.ok and list(info) == [0, 0], (st, info)
    return cfg, a, plan, e


def test_fp64_256_norm4(run, orc):
    cfg, a, plan, e = _single(run, orc, "expm_f64_256")
    ref, oplan, _ = orc.expm(a)
    assert (plan.m, plan.s, plan.num_gemms) == (oplan.m, oplan.s, oplan.num_gemms) == (13, 0, 6)
    assert rel_frob(e, ref) <= FP64_REL


def test_complex128_1024_gue_norm50(run, orc):
    cfg, a, plan, e = _single(run, orc, "expm_c128_1024")
    ref, oplan, _ = orc.expm(a)
    assert (plan.m, plan.s) == (oplan.m, oplan.s) == (13, 4)
    assert rel_frob(e, ref) <= FP64_REL
    n = cfg["n"]
    assert np.linalg.norm(e.conj().T @ e - np.eye(n)) <= 1e-12 * n  # exp(-iH) is unitary


def test_float32_4096_norm8(run, orc):
    cfg, a, plan, e = _single(run, orc, "expm_f32_4096")
    # the single tier's plan is the reference's float ladder (theta at u = 2^-24)
    want_plan = orc.expm_plan(float(np.abs(a.astype(np.float64)).sum(axis=0).max()), single=True)
    assert (plan.m, plan.s) == (want_plan.m, want_plan.s) == (13, 0)
    exact, _, _ = orc.expm(a.astype(np.float64))  # exp(A) in FP64 on the FP64 ladder
    assert rel_frob(e.astype(np.float64), exact) <= MIXED_REL


def test_fp64_2048_norm6(run, orc):
    cfg, a, plan, e = _single(run, orc, "expm_f64_2048")
    ref, oplan, _ = orc.expm(a)
    assert (plan.m, plan.s) == (oplan.m, oplan.s) == (13, 1)
    assert rel_frob(e, ref) <= FP64_REL


def _c4():
    cfg = bench.CONFIGS["expm_batched_f32_8192"]
    sizes, norms = bench.batched_spec(cfg, cfg["count"])
    return cfg, sizes, norms


def _subsample(sizes, norms, per_bucket=18):
    """Indices of the benchmark batch: for every size, the same number of
    matrices with s = 0 and with s > 0 on the FP64 ladder (theta_13 = 5.37),
    first in batch order."""
    pick = []
    for n in sorted(set(int(x) for x in sizes)):
        lo = [i for i in range(len(sizes)) if sizes[i] == n and norms[i] <= 5.371920351148152]
        hi = [i for i in range(len(sizes)) if sizes[i] == n and norms[i] > 5.371920351148152]
        pick += lo[: per_bucket // 2] + hi[: per_bucket // 2]
    return sorted(pick)


def test_batched_benchmark_fp64_tier_subsample(run, orc):
    cfg, sizes, norms = _c4()
    idx = _subsample(sizes, norms)
    assert len(idx) >= 256
    mats = [bench.batched_matrix(int(sizes[i]), float(norms[i]), i).astype(np.float64) for i in idx]
    st, plans, outs, _, info = run.batched(mats, "d")
    assert st.ok and (info == 0).all()
    seen = set()
    for a, e, p in zip(mats, outs, plans):
        ref, op, _ = orc.expm(a)
        assert (p.m, p.s) == (op.m, op.s)
        assert rel_frob(e, ref) <= FP64_REL, (a.shape[0], p.m, p.s)
        seen.add((a.shape[0], p.s > 0))
    assert len(seen) == 2 * 16  # every size, with and without squarings


def test_batched_benchmark_fp32_tier_all_8192(run):
    """The whole benchmark batch: FP32 tier against the FP64 tier (the same
    float32 values widened), worst relative Frobenius error over all 8192."""
    cfg, sizes, norms = _c4()
    mats = bench.batched_workload(cfg)
    assert len(mats) == 8192
    st64, p64, o64, _, i64 = run.batched([m.astype(np.float64) for m in mats], "d")
    st32, p32, o32, _, i32 = run.batched(mats, "s")
    assert st64.ok and st32.ok and (i64 == 0).all() and (i32 == 0).all()
    worst = max(rel_frob(a.astype(np.float64), b) for a, b in zip(o32, o64))
    assert worst <= MIXED_REL, worst
    assert any(p.s > 0 for p in p32) and any(p.s == 0 for p in p32)
