#!/usr/bin/env python
"""Benchmark of the B200 matrix-exponential path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config expm_batched_f32_8192] [--no-cpu] [--cpu-threads T]

Default workload: 8192 float32 matrices, n uniform on {16, 32, ..., 256},
N(0,1) entries rescaled to a 1-norm log-uniform in [0.1, 100] (seeded
synthetic data). One step = one calaman_expm_batched_s call over the whole
batch (the mixed tier: per-matrix (m, s), error <= 1e-6 against FP64). The
same matrices, widened, also go through the plain FP64 tier
(calaman_expm_batched_d) in the same run: `vs_fp64_tier` is the ratio of the
two, the comparison the metric names. `--config` selects the single-matrix
workloads (one calaman_expm_<t> call per step; the complex128 1024 x 1024
A = -iH (GUE), 1-norm 50 case is `expm_c128_1024`), the adjoint and the
other entry points.

Printed (rank 0, one JSON line):
  value       units/s over all ranks, inputs resident in HBM (single
              matrices: L2 flushed, 256 MiB write, untimed, before every
              timed step; batches: inputs larger than L2), no
              instrumentation in the timed steps;
  e2e         the same through the C ABI with pinned host buffers: H2D of
              the inputs, the call, D2H of the results, all timed;
  roofline    dense-product throughput from a separate instrumented call
              (CUDA events around every GEMM launch, algorithmic flops)
              against the FP64 tensor peak measured in this run (cuBLAS
              GEMM, 4096^3) or, for the single-precision tiers, the measured
              BF16 peak (frac_executed counts the executed BF16 products);
  cpu_baseline  the reference algorithm restated in FP64 with its products on
              numpy's BLAS and its solve on LAPACK (the bundled OpenBLAS) on
              this host's cores, on a bounded sample of the same workload;
              the C oracle (fixed evaluation order) checks the result.
With torchrun (N > 1) every rank runs its own replica of a single-matrix
workload, or its cost-balanced share of a batch N times the size (weak
scaling), and value = units over all ranks / max over ranks of the timed
seconds. `--gpus N` without a launcher re-runs itself under
torch.distributed.run with N ranks.
`--impl reference` times that CPU restatement alone.
`--cpu-threads T` limits both CPU legs to T host threads (1: the
single-threaded baseline); the default uses every host thread.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "expm/s & TFLOP/s at rel err<=1e-6 vs FP64"
# the metric's own comparison: the mixed batched tier against the plain FP64
# tier on the same 8192 matrices
DEFAULT_CONFIG = "expm_batched_f32_8192"

CONFIGS = {
    # name: (n, type suffix, 1-norm, generator)
    "expm_c128_1024": dict(n=1024, suf="z", norm=50.0, gen="gue",
                           desc="complex128 1024x1024, A=-iH (GUE), ||A||_1=50"),
    "expm_f64_256": dict(n=256, suf="d", norm=4.0, gen="gauss",
                         desc="float64 256x256, N(0,1) rescaled to ||A||_1=4"),
    "expm_f64_2048": dict(n=2048, suf="d", norm=6.0, gen="gauss",
                          desc="float64 2048x2048, N(0,1) rescaled to ||A||_1=6"),
    "expm_f32_4096": dict(n=4096, suf="s", norm=8.0, gen="gauss",
                          desc="float32 4096x4096, N(0,1)/sqrt(n) rescaled to ||A||_1=8"),
    "expm_balanced_f64_1024": dict(n=1024, suf="d", norm=1.0e4, gen="scaled", entry="expm_balanced",
                                   desc="float64 1024x1024, N(0,1) under a random power-of-two "
                                        "similarity (2^-12..2^12), ||A||_1=1e4, balanced expm"),
    "expm_herm_c128_1024": dict(n=1024, suf="z", norm=50.0, gen="herm", entry="expm_herm",
                                desc="complex128 1024x1024 Hermitian H=(X+X^H)/2 (GUE), ||H||_1=50, "
                                     "expm_herm (eigendecomposition route)"),
    "geodesic_c128_1024_p6": dict(kind="geodesic", n=1024, suf="z", samples=6, scale=10.0, step=0.1,
                                  desc="cg_unitary geodesic trial points W_j = exp(j mu H) W, j = 1..5 "
                                       "(Table 1 search, P + 1 = 6 samples), complex128 1024x1024, W "
                                       "unitary (QR of complex N(0,1)), H skew-Hermitian with ||H||_2 = 10, "
                                       "mu = 0.1"),
    "geodesic_c128_1024_dft31": dict(kind="geodesic", n=1024, suf="z", samples=31, scale=10.0, step=0.02,
                                     desc="the same with the Table 2 (DFT) sample count, 31 samples, "
                                          "mu = 0.02"),
    "expm_batched_f32_8192": dict(kind="batched", count=8192, nmax=256, suf="s",
                                  desc="8192 float32 matrices, n uniform on {16,32,...,256}, "
                                       "N(0,1) rescaled to ||A||_1 log-uniform in [0.1,100]"),
    "expm_batched_f64_8192": dict(kind="batched", count=8192, nmax=256, suf="d",
                                  desc="the same 8192 matrices in float64 (plain FP64 tier)"),
    "expm_batched_f32_2048": dict(kind="batched", count=2048, nmax=256, suf="s",
                                  desc="the first 2048 matrices of the 8192-matrix batch (a profiling case: "
                                       "inputs above L2, a few GB on the device)"),
    "lu_c128_1024": dict(kind="lu", n=1024, suf="z", norm=50.0, gen="gue",
                         desc="LU with partial pivoting + 1024-RHS solve of the complex128 1024x1024 GUE "
                              "matrix (the factor and solve expm runs on q), beside cuSOLVER's getrf/getrs "
                              "(torch.linalg.lu_factor / lu_solve) on the same box"),
    "lu_f32_4096": dict(kind="lu", n=4096, suf="s", norm=8.0, gen="gauss",
                        desc="LU with partial pivoting + 4096-RHS solve of the float32 4096x4096 matrix, "
                             "beside cuSOLVER's getrf/getrs (torch.linalg.lu_factor / lu_solve)"),
    "expm_vjp_f64_2048": dict(kind="vjp", n=2048, suf="d", norm=6.0,
                              desc="loss <G, expm(A)>, float64 2048x2048, A and G N(0,1), "
                                   "A rescaled to ||A||_1=6"),
    "expm_vjp_f32_128x512": dict(kind="vjp", n=128, count=512, suf="s", norm=6.0,
                                 desc="loss <G, expm(A)>, 512 float32 128x128 pairs, A and G "
                                      "N(0,1), A rescaled to ||A||_1=6"),
}
NP = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
ELEM_BYTES = {"s": 4, "d": 8, "c": 8, "z": 16}


def make_matrix(cfg, seed=20261203):
    rng = np.random.default_rng(seed)
    n = cfg["n"]
    if cfg["gen"] in ("gue", "herm"):
        x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        a = (x + x.conj().T) / 2
        if cfg["gen"] == "gue":
            a = -1j * a
    elif cfg["gen"] == "scaled":
        d = 2.0 ** rng.integers(-12, 13, n)
        a = (rng.standard_normal((n, n)) * d[:, None]) / d[None, :]
    else:
        a = rng.standard_normal((n, n)) / np.sqrt(n)
    a = a * (cfg["norm"] / np.abs(a).sum(axis=0).max())
    return np.asfortranarray(a.astype(NP[cfg["suf"]]))


def batched_spec(cfg, count, seed=20261204):
    """Sizes and 1-norms of the batched workload: n uniform on {16, 32, ...,
    nmax}, 1-norm log-uniform in [0.1, 100]."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, cfg["nmax"] // 16 + 1, count) * 16
    norms = np.exp(rng.uniform(np.log(0.1), np.log(100.0), count))
    return sizes, norms


def batched_shard(lib, cfg, world, rank):
    """This rank's matrices of a global batch of world x count (weak
    scaling): the cost-balanced partition every rank computes alike from the
    plans the library picks (calaman_expm_plan_*, host-side). Returns
    (indices, global count)."""
    from calaman_g_b200.shard import expm_cost, partition

    total = world * cfg["count"]
    sizes, norms = batched_spec(cfg, total)
    plan_fn = lib.calaman_expm_plan_s if cfg["suf"] == "s" else lib.calaman_expm_plan_d
    costs = []
    for n_, t_ in zip(sizes, norms):
        p_ = plan_fn(float(t_))
        costs.append(expm_cost(int(n_), p_.m, p_.s))
    return partition(costs, world)[rank], total


def batched_matrix(n, norm, i, seed=20261204):
    """Matrix i of the batched workload: N(0,1) entries from its own seeded
    stream (so any rank can draw any matrix), rescaled to its 1-norm, float32
    values (the float64 tier gets the same values widened)."""
    a = np.random.default_rng([seed, int(i)]).standard_normal((n, n))
    return (a * (norm / np.abs(a).sum(axis=0).max())).astype(np.float32)


def batched_workload(cfg, indices=None, total=None):
    sizes, norms = batched_spec(cfg, total or cfg["count"])
    idx = range(len(sizes)) if indices is None else indices
    return [batched_matrix(int(sizes[i]), float(norms[i]), i) for i in idx]


def vjp_pair(n, norm, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a = a * (norm / np.abs(a).sum(axis=0).max())
    g = rng.standard_normal((n, n))
    return a, g


def geodesic_inputs(cfg, seed=20261205):
    """W unitary (QR of complex N(0,1)), H skew-Hermitian rescaled to spectral norm `scale`."""
    rng = np.random.default_rng(seed)
    n = cfg["n"]
    w, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    y = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = (y - y.conj().T) / 2
    h = h * (cfg["scale"] / np.linalg.norm(h, 2))
    return np.asfortranarray(w), np.asfortranarray(h)


def vjp_flops(n, m, s):
    """Algorithmic flops of one adjoint: (19 + 3s) products at m = 13 (else
    3 per power + 3), one LU, two n-RHS solves."""
    pim = {3: 1, 5: 2, 7: 3, 9: 4, 13: 3}[m]
    gemms = 3 * pim + (6 if m == 13 else 0) + 4 + 3 * s
    return gemms * 2.0 * n ** 3 + (2.0 / 3.0) * n ** 3 + 2 * 2.0 * n ** 3


def herm_flops(n, cplx):
    """Algorithmic flops of the eigendecomposition route: Householder
    tridiagonalisation (4/3 n^3), back-transformation of the eigenvectors
    (2 n^3) and the product M U^H (2 n^3), x4 for complex, plus the
    divide-and-conquer merges' real products (8/3 n^3 summed over levels)."""
    return (4.0 if cplx else 1.0) * (4.0 / 3.0 + 4.0) * n ** 3 + (8.0 / 3.0) * n ** 3


def expm_flops(n, m, s, cplx):
    pim = {3: 2, 5: 3, 7: 4, 9: 5, 13: 6}[m]
    f = (pim + s) * 2.0 * n ** 3 + (2.0 / 3.0) * n ** 3 + 2.0 * n ** 3
    return f * (4.0 if cplx else 1.0)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the first sample before the timed region starts, so a region
            # shorter than the sampling period still has one
            t0 = time.time()
            while not self.rows and self.proc.poll() is None and time.time() - t0 < 3.0:
                time.sleep(0.01)
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------------------------------------------------------------------
CPU_THREADS = 0  # host threads of the CPU legs; 0: every host thread


def cpu_threads() -> int:
    return CPU_THREADS if CPU_THREADS > 0 else (os.cpu_count() or 1)


def threads_phrase(n: int) -> str:
    return "1 thread" if n == 1 else f"{n} threads"


# ---- CPU legs over many small matrices: one single-threaded worker per host
# thread, the matrices spread over the workers (largest first) -------------
_POOL_ITEMS, _POOL_SINGLE = None, False


def _pool_init(items, single):
    global _POOL_ITEMS, _POOL_SINGLE
    from threadpoolctl import threadpool_limits

    from oracle import oracle as O

    threadpool_limits(limits=1)
    O.set_threads(1)
    _POOL_ITEMS, _POOL_SINGLE = items, single


def _pool_expm(i):
    from oracle import oracle as O

    O.expm_blas(_POOL_ITEMS[i], single=_POOL_SINGLE)
    return i


def _pool_ready(_):
    time.sleep(0.2)  # held long enough that every task lands on a worker of its own
    return os.getpid()


def _pool_vjp(i):
    from oracle import oracle as O

    a, g = _POOL_ITEMS[i]
    O.expm_vjp_frechet(a, g, single=_POOL_SINGLE)
    return i


class MatrixPool:
    """A process pool over a fixed sample of matrices (or adjoint pairs),
    started with spawn (no worker inherits a CUDA context), every worker
    started before any timing; run() evaluates the whole sample once. Each
    pass has a time limit, so a pool whose workers cannot start raises
    instead of waiting for good."""

    LIMIT_S = 600.0

    def __init__(self, items, sizes, single, workers):
        import concurrent.futures as cf
        import multiprocessing as mp

        self.order = sorted(range(len(items)), key=lambda i: -sizes[i])
        self.ex = cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"),
                                         initializer=_pool_init, initargs=(items, single))
        # the executor starts workers on demand: one blocking task per worker
        # brings them all up now
        list(self.ex.map(_pool_ready, range(workers), timeout=self.LIMIT_S))

    def run(self, fn):
        for _ in self.ex.map(fn, self.order, chunksize=1, timeout=self.LIMIT_S):
            pass

    def close(self):
        self.ex.shutdown()


CPU_FORM = ("the reference algorithm restated with its products on numpy's BLAS and its solve "
            "on LAPACK xGESV (bundled OpenBLAS), FP64")


def cpu_baseline(a, cfg, min_seconds=8.0, max_reps=3):
    """The CPU baseline on all host threads: whole calls of the timing
    restatement (oracle.expm_blas: the reference algorithm with GEMM through
    BLAS and LU through LAPACK) on the same matrix until min_seconds; then
    one untimed call of the C oracle, whose result the accuracy check uses."""
    from oracle import oracle as O

    cores = cpu_threads()
    O.set_threads(cores)
    single = cfg["suf"] in "sc"
    x = a.astype(np.complex128 if cfg["suf"] in "cz" else np.float64)
    reps, t0 = 0, time.perf_counter()
    while True:
        if cfg.get("entry") == "expm_balanced":
            O.expm_balanced(x, single=single, blas=True)
        elif cfg.get("entry") == "expm_herm":
            O.expm_herm(x)
        else:
            O.expm_blas(x, single=single)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= max_reps:
            break
    if cfg.get("entry") == "expm_balanced":
        result = O.expm_balanced(x, single=single)[0]
    elif cfg.get("entry") == "expm_herm":
        result = O.expm_herm(x)
    else:
        result = O.expm(x, single=single)[0]
    form = ("LAPACK xHEEVD through numpy, then the column scale and one product on BLAS"
            if cfg.get("entry") == "expm_herm" else CPU_FORM)
    return {"value": reps / el, "unit": "expm/s", "cores": cores, "kind": "port",
            "sample": f"{reps} full expm call(s) of the benchmark matrix ({cfg['desc']}), "
                      f"{el:.1f} s, {form}, {threads_phrase(cores)}"}, result


def run_reference(args, cfg):
    """The reference algorithm's CPU form on the same workload, all host
    threads, rank 0 only: the FP64 restatement with its products on numpy's
    BLAS and its solve on LAPACK (oracle.expm_blas; the C oracle's gebal
    sweep for the balanced config, xHEEVD for expm_herm). Batched: each step
    is the first 8 matrices per host thread, spread over single-threaded
    worker processes (32 in order on one thread); adjoint: the numpy
    restatement of the adjoint (FP64), one 2048^2 pair on threaded BLAS, or
    4 pairs of 128^2 per host thread over the workers."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    cores = cpu_threads()
    O.set_threads(cores)
    kind = cfg.get("kind", "single")
    dtype = {"z": "c128", "d": "f64", "s": "f32", "c": "c64"}[cfg["suf"]]
    single = cfg["suf"] in "sc"
    pool = None
    if kind == "batched":
        count = 32 if cores == 1 else 8 * cores
        mats = [m.astype(np.float64) for m in batched_workload(cfg, range(count))]
        per_step, unit = len(mats), "expm/s"
        if cores == 1:
            def one():
                for m in mats:
                    O.expm_blas(m, single=single)
        else:
            pool = MatrixPool(mats, [m.shape[0] ** 3 for m in mats], single, cores)

            def one():
                pool.run(_pool_expm)
        sample = (f"the first {count} matrices of the batch per step"
                  + (f", spread over {cores} single-threaded worker processes" if pool else ""))
        plan_info = None
    elif kind == "geodesic":
        w, hmat = geodesic_inputs(cfg)
        per_step, unit = 1, "search/s"

        def one():
            O.geodesic_points(w, hmat, cfg["step"], cfg["samples"], blas=True)
        sample = ("the trial points of one search per step (general expm, then the power chain and "
                  "products, all on numpy's threaded BLAS)")
        plan_info = None
    elif kind == "vjp":
        k = 1 if cfg["n"] > 512 else (8 if cores == 1 else 4 * cores)
        pairs = [vjp_pair(cfg["n"], cfg["norm"], 7000 + i) for i in range(k)]
        per_step, unit = k, "vjp/s"
        if k == 1 or cores == 1:
            def one():
                for a, g in pairs:
                    O.expm_vjp_frechet(a, g, single=single)
        else:
            pool = MatrixPool(pairs, [1] * k, single, cores)

            def one():
                pool.run(_pool_vjp)
        sample = (f"{k} adjoint(s) per step (numpy restatement of the adjoint)"
                  + (f", spread over {cores} single-threaded worker processes" if pool else ""))
        plan_info = None
    else:
        x = make_matrix(cfg).astype(np.complex128 if cfg["suf"] in "cz" else np.float64)
        per_step, unit = 1, "expm/s"
        holder = {}

        if cfg.get("entry") == "expm_balanced":
            def one():
                holder["plan"] = O.expm_balanced(x, single=single, blas=True)[1]
        elif cfg.get("entry") == "expm_herm":
            def one():
                O.expm_herm(x)
        else:
            def one():
                holder["plan"] = O.expm_blas(x, single=single)[1]
        sample = "one full expm of the benchmark matrix per step"
        if cfg.get("entry") == "expm_herm":
            sample += " (eigendecomposition route: LAPACK zheevd through numpy, threaded BLAS)"
        plan_info = holder if cfg.get("entry") != "expm_herm" else None
    for _ in range(max(args.warmup, 1 if pool else 0)):  # a pool's workers start in its first pass
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    el = time.perf_counter() - t0
    if pool:
        pool.close()
    value = per_step * args.steps / el
    config = {"workload": args.config, "desc": cfg["desc"]}
    if plan_info:
        config["plan"] = {"m": plan_info["plan"].m, "s": plan_info["plan"].s}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)", "config": config,
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port",
                         "sample": f"{sample}; {args.steps} timed steps after {args.warmup} "
                                   f"warm-up; {CPU_FORM}; {threads_phrase(cores)}"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if kind == "single" and plan_info:
        line["tflops"] = expm_flops(cfg["n"], plan_info["plan"].m, plan_info["plan"].s,
                                    cfg["suf"] in "cz") * value / 1e12
    elif kind == "single":
        line["tflops"] = herm_flops(cfg["n"], cfg["suf"] in "cz") * value / 1e12
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def measure_fp64_peak(torch, dev, cplx):
    """cuBLAS (torch.matmul) FP64 GEMM throughput at 4096^3: the FP64 tensor
    denominator (the driver's peak file carries no FP64 figure)."""
    n = 4096
    dt = torch.complex128 if cplx else torch.float64
    a = torch.randn(n, n, dtype=dt, device=dev)
    b = torch.randn(n, n, dtype=dt, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    flops = (8.0 if cplx else 2.0) * n ** 3
    del a, b
    return flops / (best * 1e-3) / 1e12


def read_traffic(name):
    """dram bytes per dense-product launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{name}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_ours(args, cfg):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    from calaman_g_b200 import capi

    lib = capi.load()
    suf, n = cfg["suf"], cfg["n"]
    cplx = suf in "cz"
    a = make_matrix(cfg)

    baseline, oracle_result = (None, None)
    if rank == 0 and world == 1 and not args.no_cpu:
        baseline, oracle_result = cpu_baseline(a, cfg)

    tdt = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}[suf]
    host_a = torch.from_numpy(np.ascontiguousarray(a.T).reshape(-1)).to(tdt).pin_memory()
    host_e = torch.empty_like(host_a).pin_memory()
    dA = host_a.to(dev)
    dE = torch.empty_like(dA)
    stream = torch.cuda.Stream(device=dev)
    h = ctypes.c_void_p()
    assert lib.calamanCreate(ctypes.byref(h)).ok
    assert lib.calamanSetStream(h, ctypes.c_void_p(stream.cuda_stream)).ok
    nb = ctypes.c_size_t()
    entry = cfg.get("entry", "expm")
    herm = entry == "expm_herm"
    if herm:
        assert getattr(lib, f"calaman_{entry}_bufferSize_{suf}")(h, capi.FILL_LOWER, n, ctypes.byref(nb)).ok
    else:
        assert getattr(lib, f"calaman_{entry}_bufferSize_{suf}")(h, n, ctypes.byref(nb)).ok
    work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    info = torch.zeros(2, dtype=torch.int32, device=dev)
    infop = ctypes.cast(info.data_ptr(), capi.c_int_p)
    plan = capi.ExpmPlan()
    fn = getattr(lib, f"calaman_{entry}_{suf}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        if herm:
            st = fn(h, h, ctypes.c_void_p(stream.cuda_stream), capi.FILL_LOWER, n,
                    ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(dE.data_ptr()), n,
                    ctypes.c_void_p(work.data_ptr()), nb.value, infop)
        else:
            st = fn(h, h, ctypes.c_void_p(stream.cuda_stream), n, ctypes.c_void_p(dA.data_ptr()), n,
                    ctypes.c_void_p(dE.data_ptr()), n, ctypes.c_void_p(work.data_ptr()), nb.value,
                    infop, ctypes.byref(plan))
        if not st.ok:
            raise RuntimeError(f"{entry} failed: {st!r}")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()

    # ---- timed: inputs resident, L2 flushed before each step ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.calamanGetLaunchCount()
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                starts[i].record(stream)
                step()
                ends[i].record(stream)
        torch.cuda.synchronize()
        launches = lib.calamanGetLaunchCount() - launches0
        total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
        # instrumented steps (not in value): CUDA events around every GEMM launch
        assert lib.calamanSetKernelTiming(h, 1).ok
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                step()
        torch.cuda.synchronize()
        kt = capi.KernelTiming()
        assert lib.calamanGetKernelTiming(h, ctypes.byref(kt)).ok
        lib.calamanSetKernelTiming(h, 0)

        # ---- e2e: pinned host in, pinned host out, through the C ABI ----
        e2e_ms = 0.0
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
                dA.copy_(host_a, non_blocking=True)
                step()
                host_e.copy_(dE, non_blocking=True)
                e.record(stream)
                e.synchronize()
                e2e_ms += s.elapsed_time(e)
    torch.cuda.synchronize()
    if info.cpu().tolist() != [0, 0]:
        raise RuntimeError(f"LU reported info {info.cpu().tolist()}")

    t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, e2e_ms = t.tolist()
    value = world * args.steps / (total_ms * 1e-3)
    e2e_value = world * args.steps / (e2e_ms * 1e-3)

    if rank == 0:
        flops = herm_flops(n, cplx) if herm else expm_flops(n, plan.m, plan.s, cplx)
        achieved = kt.gemm_flops / (kt.gemm_ms * 1e-3) / 1e12 if kt.gemm_ms > 0 else None
        oz_digits = 7 if (suf in "dz" and n >= 1536) else 0  # the library's default policy
        if suf == "s":
            # split-BF16 x6 tensor-core products: six BF16 products per FP32 product
            peak, peak_src = _bf16_peak()
            executed = 6.0 * achieved if achieved else None
        elif oz_digits:
            # Ozaki-scheme products on the INT8 tensor cores: digits (digits + 1) / 2
            # int8 products per real product (complex: 4 real products' worth)
            peak = measure_fp64_peak(torch, dev, cplx)
            peak_src = ("cuBLAS complex128/float64 GEMM 4096^3 measured in this run: the FP64 peak the "
                        "emulated products are measured against")
            pairs = oz_digits * (oz_digits + 1) / 2
            executed = (pairs * (1.0 if cplx else 1.0) * achieved) if achieved else None
        else:
            peak = measure_fp64_peak(torch, dev, cplx)
            peak_src = ("cuBLAS complex128/float64 GEMM 4096^3 measured in this run "
                        "(MEASURED_PEAKS.json has no FP64 figure)")
            # complex products run as three real products (Gauss): 6/8 of the
            # algorithmic flops are executed on the tensor cores
            executed = (0.75 * achieved if cplx else achieved) if achieved else None
        got = host_e.numpy().reshape(n, n).T
        acc = {}
        if oracle_result is not None:
            acc["rel_frob_vs_oracle"] = float(np.linalg.norm(got - oracle_result)
                                              / np.linalg.norm(oracle_result))
        if cfg["gen"] == "gue":
            g = got.astype(np.complex128)
            acc["unitarity_frob"] = float(np.linalg.norm(g.conj().T @ g - np.eye(n)))
        line = {
            "metric": METRIC, "value": value, "unit": "expm/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"z": "c128", "d": "f64", "s": "f32", "c": "c64"}[suf],
            "data": "synthetic (seeded)",
            "config": {"workload": args.config, "desc": cfg["desc"],
                       "plan": None if herm else {"m": plan.m, "s": plan.s,
                                                   "num_gemms": plan.num_gemms},
                       "l2": "flushed before every timed step (256 MiB write, untimed)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "tflops": flops * value / 1e12,
            "algorithmic_flops_per_expm": flops,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if achieved else None,
                         "executed_tflops": executed,
                         "frac_executed": (executed / (2.0 * _bf16_peak()[0]) if oz_digits else executed / peak)
                         if executed else None,
                         "products": (f"Ozaki INT8 tensor cores, {oz_digits} digits (frac_executed: int8 "
                                      "ops against twice the measured BF16 peak)") if oz_digits else
                                     ("split-BF16 x6 tensor cores" if suf == "s" else "FP64 tensor cores"),
                         "traffic": read_traffic(f"zgemm_{n}" if cplx else f"dgemm_{n}"),
                         "kernel": "dense products (every GEMM launch of instrumented steps run "
                                   "after the timed ones); achieved and frac: algorithmic flops "
                                   "(2n^3 real, 8n^3 complex per product); frac_executed: the "
                                   "flops the tensor cores execute (3 real products per complex "
                                   "one; 6 BF16 products per split-BF16 FP32 one)",
                         "launches": kt.gemm_launches, "kernel_ms_per_step": kt.gemm_ms / args.steps,
                         "peak_source": peak_src},
            "cpu_baseline": baseline,
            "e2e": {"value": e2e_value, "unit": "expm/s",
                    "h2d_bytes_per_step": n * n * ELEM_BYTES[suf],
                    "d2h_bytes_per_step": n * n * ELEM_BYTES[suf]},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    lib.calamanDestroy(h)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_lu(args, cfg):
    """One step = calaman_getrf + calaman_getrs with n right-hand sides on the
    workload matrix (the factor and solve of expm's q); the same factor and
    solve by cuSOLVER (torch.linalg.lu_factor + lu_solve) timed the same way
    on the same box, as a yardstick. Rank 0 only; L2 flushed before each step."""
    torch, world, rank, local, dev, dist = _init_dist()
    from calaman_g_b200 import capi

    lib = capi.load()
    suf, n = cfg["suf"], cfg["n"]
    tdt = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}[suf]
    a = make_matrix(cfg)
    rng = np.random.default_rng(7)
    b = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if suf in "cz" else 0)
    dA0 = torch.from_numpy(np.ascontiguousarray(a.T).reshape(-1)).to(tdt).to(dev)  # column-major
    dB = torch.from_numpy(np.ascontiguousarray(b.T).reshape(-1)).to(tdt).to(dev)
    dA = torch.empty_like(dA0)
    dX = torch.empty_like(dB)
    nb = ctypes.c_size_t()
    assert lib.calaman_getrf_bufferSize(n, ctypes.byref(nb)).ok
    scratch = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
    info = torch.zeros(2, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    getrf, getrs = getattr(lib, f"calaman_getrf_{suf}"), getattr(lib, f"calaman_getrs_{suf}")
    infp = ctypes.cast(info.data_ptr(), capi.c_int_p)
    infp1 = ctypes.cast(info.data_ptr() + 4, capi.c_int_p)

    def ours():
        dA.copy_(dA0)
        assert getrf(sp, n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(scratch.data_ptr()), infp).ok
        assert getrs(sp, n, n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(scratch.data_ptr()),
                     ctypes.c_void_p(dB.data_ptr()), n, ctypes.c_void_p(dX.data_ptr()), n, infp1).ok

    Am = dA0.view(n, n).t()  # the matrix (row-major view of the column-major buffer)
    Bm = dB.view(n, n).t()

    def library():
        lu, piv = torch.linalg.lu_factor(Am)
        return torch.linalg.lu_solve(lu, piv, Bm)

    def timed(fn):
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                fn()
        torch.cuda.synchronize()
        tot = 0.0
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                flush.zero_()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                fn()
                s1.record(stream)
                s1.synchronize()
                tot += s0.elapsed_time(s1)
        return tot
    with ClockSampler(local) as clocks:
        ms_ours = timed(ours)
        ms_lib = timed(library)
    torch.cuda.synchronize()
    # the solution against the library's (both solve the same system)
    x = dX.view(n, n).t()
    with torch.cuda.stream(stream):
        xl = library()
    torch.cuda.synchronize()
    rel = float((x - xl).abs().norm() / xl.abs().norm())
    resid = float((Am @ x - Bm).abs().norm() / (Am.abs().norm() * x.abs().norm()))
    if rank == 0:
        flops = (8.0 / 3.0 if suf not in "cz" else 4 * 8.0 / 3.0) * n ** 3  # (2/3) n^3 + 2 n^3, x4 complex
        line = {
            "metric": "LU + n-RHS solve per second (factor and solve of expm's q)", "value": args.steps / (ms_ours * 1e-3),
            "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_ours / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"z": "c128", "d": "f64", "s": "f32", "c": "c64"}[suf], "data": "synthetic (seeded)",
            "config": {"workload": args.config, "desc": cfg["desc"], "l2": "flushed before every timed step"},
            "tflops": flops * args.steps / (ms_ours * 1e-3) / 1e12,
            "cusolver": {"value": args.steps / (ms_lib * 1e-3), "ms_per_step": ms_lib / args.steps,
                         "entry": "torch.linalg.lu_factor + torch.linalg.lu_solve (cuSOLVER getrf / getrs), "
                                  "a yardstick only: nothing in the library calls it"},
            "vs_cusolver": ms_lib / ms_ours,
            "accuracy": {"rel_vs_cusolver_solution": rel, "backward_residual": resid},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def _init_dist():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    return torch, world, rank, local, dev, dist


def _max_over_ranks(torch, dist, dev, values):
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def _bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "MEASURED_PEAKS.json bf16_tflops (burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback 1.59 PFLOP/s (no MEASURED_PEAKS.json)"


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


def hbm_min(ns, esz, ms_per_step):
    """The batch's minimum-HBM-traffic bound: every matrix read once and its
    exponential written once (2 n^2 elements each), over the step time."""
    peak, src = _hbm_peak()
    nbytes = 2 * sum(n * n for n in ns) * esz
    gbs = nbytes / (ms_per_step * 1e-3) / 1e9
    return {"bytes_per_step": nbytes, "achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
            "unit": "GB/s", "peak_source": src,
            "what": "each matrix read once and its exponential written once, per GPU"}


# sub-batches of the batched end-to-end pipelines (--e2e-parts): measured on a
# B200, the 8192-matrix expm gave 231k / 253k / 264k expm/s end to end with
# 4 / 8 / 16, the 512-pair adjoint 168k / 151k vjp/s with 4 / 8
E2E_PARTS_EXPM = 16
E2E_PARTS_VJP = 4


def _sub_batches(lib, capi, torch, dev, suf, ns, offs, dA, dE, host_in, host_out, info, parts):
    """Split the batch into `parts` contiguous sub-batches of about equal sum n^3,
    each with its own handle, stream, workspace and views of the batch buffers."""
    cost = np.cumsum([n ** 3 for n in ns], dtype=np.float64)
    bounds = [0]
    for k in range(1, parts):
        bounds.append(int(np.searchsorted(cost, cost[-1] * k / parts)) + 1)
    bounds.append(len(ns))
    esz = dA.element_size()
    total = dA.numel()
    fn = getattr(lib, f"calaman_expm_batched_{suf}")
    out = []
    for k in range(parts):
        i0, i1 = bounds[k], bounds[k + 1]
        if i1 <= i0:
            continue
        cnt = i1 - i0
        e0 = offs[i0]
        e1 = offs[i1] if i1 < len(ns) else total
        s_ = torch.cuda.Stream(device=dev)
        h = ctypes.c_void_p()
        assert lib.calamanCreate(ctypes.byref(h)).ok
        assert lib.calamanSetStream(h, ctypes.c_void_p(s_.cuda_stream)).ok
        IntArr, PtrArr = ctypes.c_int * cnt, ctypes.c_void_p * cnt
        h_n = IntArr(*ns[i0:i1])
        h_A = PtrArr(*[dA.data_ptr() + o * esz for o in offs[i0:i1]])
        h_E = PtrArr(*[dE.data_ptr() + o * esz for o in offs[i0:i1]])
        intp = ctypes.cast(h_n, capi.c_int_p)
        nb = ctypes.c_size_t()
        assert getattr(lib, f"calaman_expm_batched_bufferSize_{suf}")(h, cnt, intp, ctypes.byref(nb)).ok
        work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
        plans = (capi.ExpmPlan * cnt)()
        infop = ctypes.cast(info.data_ptr() + 2 * i0 * 4, capi.c_int_p)

        def call(h=h, s_=s_, cnt=cnt, intp=intp, h_A=h_A, h_E=h_E, work=work, nb=nb, infop=infop,
                 plans=plans):
            st = fn(h, h, ctypes.c_void_p(s_.cuda_stream), cnt, intp,
                    ctypes.cast(h_A, ctypes.POINTER(ctypes.c_void_p)), intp,
                    ctypes.cast(h_E, ctypes.POINTER(ctypes.c_void_p)), intp,
                    ctypes.c_void_p(work.data_ptr()), nb.value, infop, plans)
            if not st.ok:
                raise RuntimeError(f"expm_batched failed: {st!r}")

        out.append({"stream": s_, "h": h, "call": call, "work": work, "plans": plans,
                    "din": dA[e0:e1], "dout": dE[e0:e1], "hin": host_in[e0:e1], "hout": host_out[e0:e1],
                    "done": torch.cuda.Event()})
    return out


def _vjp_sub_batches(lib, capi, torch, dev, suf, n, count, dA, dG, dD, host_a, host_g, host_d, parts):
    """`parts` equal sub-batches of the packed n x n pairs, each with its own
    handle, stream, workspace and views of the pair buffers."""
    esz = dA.element_size()
    nn = n * n
    fn = getattr(lib, f"calaman_expm_vjp_batched_{suf}")
    PP = ctypes.POINTER(ctypes.c_void_p)
    out = []
    for k in range(parts):
        i0, i1 = count * k // parts, count * (k + 1) // parts
        cnt = i1 - i0
        if cnt <= 0:
            continue
        s_ = torch.cuda.Stream(device=dev)
        h = ctypes.c_void_p()
        assert lib.calamanCreate(ctypes.byref(h)).ok
        assert lib.calamanSetStream(h, ctypes.c_void_p(s_.cuda_stream)).ok
        IntArr, PtrArr = ctypes.c_int * cnt, ctypes.c_void_p * cnt
        h_n = IntArr(*([n] * cnt))
        ip = ctypes.cast(h_n, capi.c_int_p)
        h_A = PtrArr(*[dA.data_ptr() + i * nn * esz for i in range(i0, i1)])
        h_G = PtrArr(*[dG.data_ptr() + i * nn * esz for i in range(i0, i1)])
        h_D = PtrArr(*[dD.data_ptr() + i * nn * esz for i in range(i0, i1)])
        nb = ctypes.c_size_t()
        assert getattr(lib, f"calaman_expm_vjp_batched_bufferSize_{suf}")(h, cnt, ip, ctypes.byref(nb)).ok
        work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
        info = torch.zeros(2 * cnt, dtype=torch.int32, device=dev)
        plans = (capi.ExpmPlan * cnt)()

        def call(h=h, s_=s_, cnt=cnt, ip=ip, h_A=h_A, h_G=h_G, h_D=h_D, work=work, nb=nb, info=info,
                 plans=plans):
            st = fn(h, h, ctypes.c_void_p(s_.cuda_stream), cnt, ip, ctypes.cast(h_A, PP), ip,
                    ctypes.cast(h_G, PP), ip, ctypes.cast(h_D, PP), ip, None, ip,
                    ctypes.c_void_p(work.data_ptr()), nb.value, ctypes.cast(info.data_ptr(), capi.c_int_p),
                    plans)
            if not st.ok:
                raise RuntimeError(f"expm_vjp_batched failed: {st!r}")

        sl = slice(i0 * nn, i1 * nn)
        out.append({"stream": s_, "h": h, "call": call, "work": work, "info": info, "plans": plans,
                    "da": dA.view(-1)[sl], "dg": dG.view(-1)[sl], "dd": dD.view(-1)[sl],
                    "ha": host_a.view(-1)[sl], "hg": host_g.view(-1)[sl], "hd": host_d.view(-1)[sl],
                    "done": torch.cuda.Event()})
    return out


def _batched_entry(lib, capi, torch, dev, suf, ns, offs, dIn, dOut, stream, info):
    """A calaman_expm_batched_<suf> call over every matrix of the batch:
    returns (call, plans, handle, workspace)."""
    count = len(ns)
    esz = dIn.element_size()
    IntArr, PtrArr = ctypes.c_int * count, ctypes.c_void_p * count
    h_n = IntArr(*ns)
    h_A = PtrArr(*[dIn.data_ptr() + o * esz for o in offs])
    h_E = PtrArr(*[dOut.data_ptr() + o * esz for o in offs])
    h = ctypes.c_void_p()
    assert lib.calamanCreate(ctypes.byref(h)).ok
    assert lib.calamanSetStream(h, ctypes.c_void_p(stream.cuda_stream)).ok
    nb = ctypes.c_size_t()
    intp = ctypes.cast(h_n, capi.c_int_p)
    assert getattr(lib, f"calaman_expm_batched_bufferSize_{suf}")(h, count, intp, ctypes.byref(nb)).ok
    work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    plans = (capi.ExpmPlan * count)()
    fn = getattr(lib, f"calaman_expm_batched_{suf}")

    def call():
        st = fn(h, h, ctypes.c_void_p(stream.cuda_stream), count, intp,
                ctypes.cast(h_A, ctypes.POINTER(ctypes.c_void_p)), intp,
                ctypes.cast(h_E, ctypes.POINTER(ctypes.c_void_p)), intp,
                ctypes.c_void_p(work.data_ptr()), nb.value,
                ctypes.cast(info.data_ptr(), capi.c_int_p), plans)
        if not st.ok:
            raise RuntimeError(f"expm_batched_{suf} failed: {st!r}")

    call._keep = (h_n, h_A, h_E)
    return call, plans, h, work


def _time_steps(torch, stream, call, steps):
    """CUDA-event time (ms) of `steps` back-to-back calls on `stream`."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for i in range(steps):
            starts[i].record(stream)
            call()
            ends[i].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in zip(starts, ends))


def _plain_fp64_pass(lib, capi, torch, dev, stream, ns, offs, dIn, dOut):
    """CUDA-event time (ms) of calaman_expm_d called once per matrix over the
    whole batch, after a warm-up over its first matrices."""
    h = ctypes.c_void_p()
    assert lib.calamanCreate(ctypes.byref(h)).ok
    assert lib.calamanSetStream(h, ctypes.c_void_p(stream.cuda_stream)).ok
    nb = ctypes.c_size_t()
    assert lib.calaman_expm_bufferSize_d(h, max(ns), ctypes.byref(nb)).ok
    work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    info = torch.zeros(2, dtype=torch.int32, device=dev)
    infop = ctypes.cast(info.data_ptr(), capi.c_int_p)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def one(i):
        n = ns[i]
        st = lib.calaman_expm_d(h, h, sp, n, ctypes.c_void_p(dIn.data_ptr() + offs[i] * 8), n,
                                ctypes.c_void_p(dOut.data_ptr() + offs[i] * 8), n,
                                ctypes.c_void_p(work.data_ptr()), nb.value, infop, None)
        if not st.ok:
            raise RuntimeError(f"expm_d failed: {st!r}")

    for i in range(min(64, len(ns))):
        one(i)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for i in range(len(ns)):
        one(i)
    b.record(stream)
    torch.cuda.synchronize()
    lib.calamanDestroy(h)
    return a.elapsed_time(b)


def run_batched(args, cfg):
    """One step = one calaman_expm_batched_<t> call over the whole batch.
    Under torchrun the batch is split across ranks (matrices are
    independent; balanced by sum n^3), no collective on the data path.

    For the mixed tier (float32 in/out) the same matrices, widened to
    float64, also go through the plain FP64 tier in the same run, timed the
    same way: `vs_fp64_tier` = mixed value / FP64-tier value, the ratio the
    metric names, and `accuracy` = the mixed tier's worst relative Frobenius
    error against the FP64 tier over every matrix.

    `value` is timed with no instrumentation; the roofline's kernel figures
    come from a separate pass with CUDA events around every grouped-GEMM
    launch (calamanSetKernelTiming)."""
    torch, world, rank, local, dev, dist = _init_dist()
    from calaman_g_b200 import capi

    lib = capi.load()
    suf = cfg["suf"]
    if world > 1:
        # weak scaling: a global batch of world x count matrices, partitioned
        # across the ranks by algorithmic cost (no data-path collective)
        mine, total = batched_shard(lib, cfg, world, rank)
        mats = batched_workload(cfg, mine, total)
    else:
        mats = batched_workload(cfg)
    count = len(mats)
    ns = [m.shape[0] for m in mats]
    tdt = torch.float32 if suf == "s" else torch.float64
    npdt = np.float32 if suf == "s" else np.float64
    offs, at = [], 0
    for n in ns:
        offs.append(at)
        at += ((n * n + 63) // 64) * 64
    host_in = torch.empty(at, dtype=tdt).pin_memory()
    hv = host_in.numpy()
    for m, o in zip(mats, offs):
        n = m.shape[0]
        hv[o:o + n * n] = np.ascontiguousarray(m.T).reshape(-1).astype(npdt)
    host_out = torch.empty_like(host_in).pin_memory()
    dA = host_in.to(dev)
    dE = torch.empty_like(dA)
    esz = dA.element_size()
    stream = torch.cuda.Stream(device=dev)
    info = torch.zeros(2 * count, dtype=torch.int32, device=dev)
    step, plans, h, work = _batched_entry(lib, capi, torch, dev, suf, ns, offs, dA, dE, stream, info)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.calamanGetLaunchCount()
    with ClockSampler(local) as clocks:
        # ---- value: inputs resident in HBM (larger than L2), no instrumentation
        total_ms = _time_steps(torch, stream, step, args.steps)
        launches = lib.calamanGetLaunchCount() - launches0
        # ---- e2e as a user would pipeline it: the batch in sub-batches on their own
        # streams (one handle each), so one sub-batch's copies overlap another's
        # compute; every step still copies all inputs in and all results out
        subs = _sub_batches(lib, capi, torch, dev, suf, ns, offs, dA, dE, host_in, host_out, info,
                            args.e2e_parts or E2E_PARTS_EXPM)
        e2e_ms = 0.0
        for i in range(args.warmup + args.steps):  # warm-up steps first, untimed
            a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a_ev.record(stream)
            for sb in subs:
                sb["stream"].wait_event(a_ev)
                with torch.cuda.stream(sb["stream"]):
                    sb["din"].copy_(sb["hin"], non_blocking=True)
                    sb["call"]()
                    sb["hout"].copy_(sb["dout"], non_blocking=True)
                    sb["done"].record(sb["stream"])
            for sb in subs:
                stream.wait_event(sb["done"])
            b_ev.record(stream)
            b_ev.synchronize()
            if i >= args.warmup:
                e2e_ms += a_ev.elapsed_time(b_ev)
        for sb in subs:
            lib.calamanDestroy(sb["h"])
        # ---- the plain FP64 tier on the same matrices, timed the same way
        fp64_ms = plain_ms = None
        if suf == "s":
            h64in = torch.from_numpy(host_in.numpy().astype(np.float64)).to(dev)
            e64 = torch.empty_like(h64in)
            info64 = torch.zeros(2 * count, dtype=torch.int32, device=dev)
            step64, plans64, h64, w64 = _batched_entry(lib, capi, torch, dev, "d", ns, offs, h64in, e64,
                                                       stream, info64)
            with torch.cuda.stream(stream):
                for _ in range(args.warmup):
                    step64()
            torch.cuda.synchronize()
            fp64_ms = _time_steps(torch, stream, step64, args.steps)
            # ---- the plain FP64 GPU expm: calaman_expm_d once per matrix, the
            # reference's one-matrix-per-call API (each call reads its 1-norm
            # back, one stream synchronisation per matrix); one pass over the batch
            if not args.no_plain:
                plain_ms = _plain_fp64_pass(lib, capi, torch, dev, stream, ns, offs, h64in, e64)
    # ---- instrumented pass (not timed into value): CUDA events around every
    # grouped-GEMM launch give the dense products' own throughput
    assert lib.calamanSetKernelTiming(h, 1).ok
    with torch.cuda.stream(stream):
        step()
    torch.cuda.synchronize()
    kt = capi.KernelTiming()
    assert lib.calamanGetKernelTiming(h, ctypes.byref(kt)).ok
    lib.calamanSetKernelTiming(h, 0)
    if any(info.cpu().tolist()):
        raise RuntimeError("an LU reported a zero pivot")
    reduced = [total_ms, e2e_ms] + ([fp64_ms] if fp64_ms is not None else [])
    reduced = _max_over_ranks(torch, dist, dev, reduced)
    total_ms, e2e_ms = reduced[0], reduced[1]
    if fp64_ms is not None:
        fp64_ms = reduced[2]
    total_count = count
    if dist:
        tc = torch.tensor([count], dtype=torch.float64, device=dev)
        dist.all_reduce(tc)
        total_count = int(tc.item())
    value = total_count * args.steps / (total_ms * 1e-3)
    e2e_value = total_count * args.steps / (e2e_ms * 1e-3)
    if rank == 0:
        pl = list(plans)
        flops = sum(expm_flops(n, p.m, p.s, False) for n, p in zip(ns, pl))
        peak64 = measure_fp64_peak(torch, dev, False)
        achieved = kt.gemm_flops / (kt.gemm_ms * 1e-3) / 1e12 if kt.gemm_ms > 0 else None
        acc = {}
        fp64_tier = None
        if suf == "s":
            # the mixed tier against the FP64 tier (same widened values), all matrices
            with torch.cuda.stream(stream):
                step()
                host_out.copy_(dE, non_blocking=True)
            torch.cuda.synchronize()
            out32 = host_out.numpy()
            ref = e64.cpu().numpy()
            worst = 0.0
            for n, o in zip(ns, offs):
                x, y = out32[o:o + n * n].astype(np.float64), ref[o:o + n * n]
                worst = max(worst, float(np.linalg.norm(x - y) / np.linalg.norm(y)))
            acc["max_rel_frob_vs_fp64_tier"] = worst
            acc["bar"] = 1e-6
            v64 = total_count * args.steps / (fp64_ms * 1e-3)
            flops64 = sum(expm_flops(n, p.m, p.s, False) for n, p in zip(ns, list(plans64)))
            fp64_tier = {"value": v64, "unit": "expm/s", "ms_per_step": fp64_ms / args.steps,
                         "tflops": flops64 * v64 / count / 1e12,
                         "entry": "calaman_expm_batched_d (every product on the FP64 tensor cores, "
                                  "FP64 LU), the same matrices widened to float64"}
            if plain_ms is not None and world == 1:
                vp_ = count / (plain_ms * 1e-3)
                fp64_tier["plain_expm"] = {
                    "value": vp_, "unit": "expm/s", "ms_per_batch": plain_ms,
                    "entry": "calaman_expm_d once per matrix over the same float64 matrices (one pass): "
                             "the one-matrix-per-call FP64 expm, as the reference evaluates it"}
            lib.calamanDestroy(h64)
            del w64, h64in, e64
        baseline = None
        if world == 1 and not args.no_cpu:
            baseline = batched_cpu_sample(mats, suf, seconds=10.0)
        n_s_pos = sum(1 for p in pl if p.s > 0)
        line = {
            "metric": METRIC, "value": value, "unit": "expm/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if suf == "s" else "f64", "data": "synthetic (seeded)",
            "config": {"workload": args.config, "desc": cfg["desc"], "matrices": count,
                       "algorithmic_flops_per_batch": flops,
                       "matrices_with_squarings": n_s_pos,
                       "l2": "inputs (%.0f MB) larger than L2" % (host_in.numel() * esz / 1e6),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "tflops": flops * value / count / 1e12,
        }
        if fp64_tier:
            line["vs_fp64_tier"] = value / fp64_tier["value"]
            if "plain_expm" in fp64_tier:
                line["vs_plain_fp64_expm"] = value / fp64_tier["plain_expm"]["value"]
            line["fp64_tier"] = fp64_tier
        line.update({
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64 if achieved else None,
                         "flops": "algorithmic (2 n^3 per product)", "traffic": None,
                         "kernel": "grouped dense-product phases (every grouped GEMM launch of one "
                                   "instrumented call), against the FP64 tensor peak",
                         "launches": kt.gemm_launches, "kernel_ms_per_call": kt.gemm_ms,
                         "peak_source": "cuBLAS float64 GEMM 4096^3 measured in this run "
                                        "(MEASURED_PEAKS.json has no FP64 figure)"},
            "hbm_min": hbm_min(ns, esz, total_ms / args.steps),
            "cpu_baseline": baseline,
            "e2e": {"value": e2e_value, "unit": "expm/s",
                    "h2d_bytes_per_step": sum(n * n for n in ns) * esz,
                    "d2h_bytes_per_step": sum(n * n for n in ns) * esz,
                    "pipeline": f"{args.e2e_parts or E2E_PARTS_EXPM} sub-batches of equal sum n^3, one handle and stream "
                                "each, copies overlapping compute"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "accuracy": acc,
        })
        print(json.dumps(line), flush=True)
    lib.calamanDestroy(h)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def batched_cpu_sample(mats, suf, seconds=10.0):
    """The timing restatement (oracle.expm_blas) on the first matrices of the
    batch: one thread, matrices in order until `seconds` pass; more threads,
    the first 16 per thread spread over single-threaded worker processes,
    whole passes over them until `seconds` pass (after a warm-up pass)."""
    from oracle import oracle as O

    cores = cpu_threads()
    O.set_threads(cores)
    if cores > 1:
        sample = [m.astype(np.float64) for m in mats[:16 * cores]]
        pool = MatrixPool(sample, [m.shape[0] ** 3 for m in sample], suf == "s", cores)
        pool.run(_pool_expm)
        passes, t0 = 0, time.perf_counter()
        while True:
            pool.run(_pool_expm)
            passes += 1
            el = time.perf_counter() - t0
            if el >= seconds:
                break
        pool.close()
        return {"value": passes * len(sample) / el, "unit": "expm/s", "cores": cores, "kind": "port",
                "sample": f"{passes} passes over the first {len(sample)} matrices of the batch ({el:.1f} s) "
                          f"on {cores} single-threaded worker processes, {CPU_FORM}"}
    done, t0 = 0, time.perf_counter()
    for m in mats:
        O.expm_blas(m.astype(np.float64), single=suf == "s")
        done += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    return {"value": done / el, "unit": "expm/s", "cores": cores, "kind": "port",
            "sample": f"the first {done} matrices of the batch ({el:.1f} s), {CPU_FORM}, "
                      f"{threads_phrase(cores)}"}


def vjp_cpu_sample(pairs, single, seconds=10.0):
    """The CPU baseline of the adjoint: the numpy restatement (FP64) of what
    the library computes. One pair: whole calls on threaded BLAS until
    `seconds` pass (3 at most); many pairs: passes over the first 4 per host
    thread, spread over single-threaded worker processes (in order on one
    thread), until `seconds` pass."""
    from oracle import oracle as O

    cores = cpu_threads()
    O.set_threads(cores)
    if len(pairs) > 1 and cores > 1:
        sample = pairs[:4 * cores]
        pool = MatrixPool(sample, [1] * len(sample), single, cores)
        pool.run(_pool_vjp)
        done, t0 = 0, time.perf_counter()
        while True:
            pool.run(_pool_vjp)
            done += len(sample)
            el = time.perf_counter() - t0
            if el >= seconds:
                break
        pool.close()
        where = f"{len(sample)} pairs per pass on {cores} single-threaded worker processes"
    else:
        done, t0 = 0, time.perf_counter()
        while True:
            a, g = pairs[done % len(pairs)]
            O.expm_vjp_frechet(a, g, single=single)
            done += 1
            el = time.perf_counter() - t0
            if el >= seconds or (len(pairs) == 1 and done >= 3):
                break
        where = threads_phrase(cores)
    return {"value": done / el, "unit": "vjp/s", "cores": cores, "kind": "port",
            "sample": f"{done} adjoint(s) ({el:.1f} s), the numpy restatement of the adjoint (FP64), {where}"}


def run_vjp(args, cfg):
    """One step = the adjoint of expm for the whole workload through the C ABI:
    one calaman_expm_vjp_<t> call (2048^2), or one calaman_expm_vjp_batched_<t>
    call over the 512 pairs of 128^2."""
    torch, world, rank, local, dev, dist = _init_dist()
    from calaman_g_b200 import capi

    lib = capi.load()
    suf, n = cfg["suf"], cfg["n"]
    count = cfg.get("count", 1)
    tdt = torch.float32 if suf == "s" else torch.float64
    pairs = [vjp_pair(n, cfg["norm"], 7000 + i) for i in range(count)]
    host_a = torch.stack([torch.from_numpy(np.ascontiguousarray(a.T)) for a, _ in pairs]).to(tdt).pin_memory()
    host_g = torch.stack([torch.from_numpy(np.ascontiguousarray(g.T)) for _, g in pairs]).to(tdt).pin_memory()
    host_d = torch.empty_like(host_a).pin_memory()
    dA, dG = host_a.to(dev), host_g.to(dev)
    dD = torch.empty_like(dA)
    stream = torch.cuda.Stream(device=dev)
    h = ctypes.c_void_p()
    assert lib.calamanCreate(ctypes.byref(h)).ok
    assert lib.calamanSetStream(h, ctypes.c_void_p(stream.cuda_stream)).ok
    nb = ctypes.c_size_t()
    esz = dA.element_size()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    plan = capi.ExpmPlan()
    if count == 1:
        # one pair: calaman_expm_vjp_<t>
        assert getattr(lib, f"calaman_expm_vjp_bufferSize_{suf}")(h, n, ctypes.byref(nb)).ok
        work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
        info = torch.zeros(2, dtype=torch.int32, device=dev)
        fn = getattr(lib, f"calaman_expm_vjp_{suf}")

        def step():
            st = fn(h, h, ctypes.c_void_p(stream.cuda_stream), n, ctypes.c_void_p(dA.data_ptr()), n,
                    ctypes.c_void_p(dG.data_ptr()), n, ctypes.c_void_p(dD.data_ptr()), n, None, n,
                    ctypes.c_void_p(work.data_ptr()), nb.value,
                    ctypes.cast(info.data_ptr(), capi.c_int_p), ctypes.byref(plan))
            if not st.ok:
                raise RuntimeError(f"expm_vjp failed: {st!r}")
    else:
        # many pairs: one calaman_expm_vjp_batched_<t> call per step
        IntArr, PtrArr = ctypes.c_int * count, ctypes.c_void_p * count
        PP = ctypes.POINTER(ctypes.c_void_p)
        h_n = IntArr(*([n] * count))
        ip = ctypes.cast(h_n, capi.c_int_p)
        h_A = PtrArr(*[dA.data_ptr() + i * n * n * esz for i in range(count)])
        h_G = PtrArr(*[dG.data_ptr() + i * n * n * esz for i in range(count)])
        h_D = PtrArr(*[dD.data_ptr() + i * n * n * esz for i in range(count)])
        assert getattr(lib, f"calaman_expm_vjp_batched_bufferSize_{suf}")(h, count, ip, ctypes.byref(nb)).ok
        work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
        info = torch.zeros(2 * count, dtype=torch.int32, device=dev)
        plans = (capi.ExpmPlan * count)()
        fn = getattr(lib, f"calaman_expm_vjp_batched_{suf}")

        def step():
            st = fn(h, h, ctypes.c_void_p(stream.cuda_stream), count, ip, ctypes.cast(h_A, PP), ip,
                    ctypes.cast(h_G, PP), ip, ctypes.cast(h_D, PP), ip, None, ip,
                    ctypes.c_void_p(work.data_ptr()), nb.value,
                    ctypes.cast(info.data_ptr(), capi.c_int_p), plans)
            if not st.ok:
                raise RuntimeError(f"expm_vjp_batched failed: {st!r}")
            plan.m, plan.s, plan.num_gemms = plans[0].m, plans[0].s, plans[0].num_gemms

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.calamanGetLaunchCount()
    assert lib.calamanSetKernelTiming(h, 1).ok
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                starts[i].record(stream)
                step()
                ends[i].record(stream)
        torch.cuda.synchronize()
        launches = lib.calamanGetLaunchCount() - launches0
        kt = capi.KernelTiming()
        assert lib.calamanGetKernelTiming(h, ctypes.byref(kt)).ok
        lib.calamanSetKernelTiming(h, 0)
        total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
        e2e_ms = 0.0
        if count == 1:
            with torch.cuda.stream(stream):
                for i in range(args.steps):
                    a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a_ev.record(stream)
                    dA.copy_(host_a, non_blocking=True)
                    dG.copy_(host_g, non_blocking=True)
                    step()
                    host_d.copy_(dD, non_blocking=True)
                    b_ev.record(stream)
                    b_ev.synchronize()
                    e2e_ms += a_ev.elapsed_time(b_ev)
        else:
            # as for the batched expm: sub-batches on their own streams, copies
            # overlapping compute, every input in and every gradient out each step
            subs = _vjp_sub_batches(lib, capi, torch, dev, suf, n, count, dA, dG, dD, host_a, host_g,
                                    host_d, args.e2e_parts or E2E_PARTS_VJP)
            for i in range(args.warmup + args.steps):  # warm-up steps first, untimed
                a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a_ev.record(stream)
                for sb in subs:
                    sb["stream"].wait_event(a_ev)
                    with torch.cuda.stream(sb["stream"]):
                        sb["da"].copy_(sb["ha"], non_blocking=True)
                        sb["dg"].copy_(sb["hg"], non_blocking=True)
                        sb["call"]()
                        sb["hd"].copy_(sb["dd"], non_blocking=True)
                        sb["done"].record(sb["stream"])
                for sb in subs:
                    stream.wait_event(sb["done"])
                b_ev.record(stream)
                b_ev.synchronize()
                if i >= args.warmup:
                    e2e_ms += a_ev.elapsed_time(b_ev)
            for sb in subs:
                lib.calamanDestroy(sb["h"])
    torch.cuda.synchronize()
    total_ms, e2e_ms = _max_over_ranks(torch, dist, dev, [total_ms, e2e_ms])
    value = world * count * args.steps / (total_ms * 1e-3)
    e2e_value = world * count * args.steps / (e2e_ms * 1e-3)
    if rank == 0:
        flops = vjp_flops(n, plan.m, plan.s)
        if suf == "s":
            peak, peak_src = _bf16_peak()
        else:
            peak, peak_src = measure_fp64_peak(torch, dev, False), "cuBLAS float64 GEMM 4096^3 in this run"
        achieved = kt.gemm_flops / (kt.gemm_ms * 1e-3) / 1e12 if kt.gemm_ms > 0 else None
        acc = {}
        from oracle import oracle as O

        k = 0 if n > 512 else min(count, 4)
        for i in range(k):
            a, g = pairs[i]
            ref, _, _ = O.expm_vjp_frechet(a.astype(np.float32).astype(np.float64) if suf == "s" else a,
                                           g.astype(np.float32).astype(np.float64) if suf == "s" else g,
                                           single=suf == "s")
            got = host_d[i].numpy().T.astype(np.float64)
            acc.setdefault("rel_frob_vs_oracle", []).append(
                float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
        baseline = None
        if world == 1 and not args.no_cpu:
            baseline = vjp_cpu_sample(pairs, suf == "s")
        line = {
            "metric": METRIC.replace("expm/s", "vjp/s"), "value": value, "unit": "vjp/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if suf == "s" else "f64", "data": "synthetic (seeded)",
            "config": {"workload": args.config, "desc": cfg["desc"], "pairs": count,
                       "plan": {"m": plan.m, "s": plan.s},
                       "algorithmic_flops_per_vjp": flops,
                       "l2": "flushed before every timed step (256 MiB write, untimed)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "tflops": flops * value / 1e12,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if achieved else None, "traffic": None,
                         "kernel": "dense products (every GEMM launch in the timed steps)",
                         "launches": kt.gemm_launches, "kernel_ms_per_step": kt.gemm_ms / args.steps,
                         "peak_source": peak_src},
            "cpu_baseline": baseline,
            "e2e": {"value": e2e_value, "unit": "vjp/s",
                    "h2d_bytes_per_step": 2 * count * n * n * esz,
                    "d2h_bytes_per_step": count * n * n * esz,
                    "pipeline": (f"{args.e2e_parts or E2E_PARTS_VJP} sub-batches, one handle and stream each, copies "
                                 "overlapping compute") if count > 1 else "one call"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    lib.calamanDestroy(h)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_geodesic(args, cfg):
    """One step = the trial points of one line search through
    calaman_geodesic_points_z (one Hermitian eigensolve, one wide product).
    Replicas under torchrun."""
    torch, world, rank, local, dev, dist = _init_dist()
    from calaman_g_b200 import capi

    lib = capi.load()
    n, num = cfg["n"], cfg["samples"]
    w, hmat = geodesic_inputs(cfg)
    host_w = torch.from_numpy(np.ascontiguousarray(w.T).reshape(-1)).pin_memory()
    host_h = torch.from_numpy(np.ascontiguousarray(hmat.T).reshape(-1)).pin_memory()
    host_o = torch.empty((num - 1) * n * n, dtype=torch.complex128).pin_memory()
    dW, dH = host_w.to(dev), host_h.to(dev)
    dO = torch.empty((num - 1) * n * n, dtype=torch.complex128, device=dev)
    stream = torch.cuda.Stream(device=dev)
    h = ctypes.c_void_p()
    assert lib.calamanCreate(ctypes.byref(h)).ok
    assert lib.calamanSetStream(h, ctypes.c_void_p(stream.cuda_stream)).ok
    nb = ctypes.c_size_t()
    assert lib.calaman_geodesic_points_bufferSize_z(h, n, num, ctypes.byref(nb)).ok
    work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        st = lib.calaman_geodesic_points_z(h, h, ctypes.c_void_p(stream.cuda_stream), n,
                                           ctypes.c_void_p(dW.data_ptr()), n, ctypes.c_void_p(dH.data_ptr()), n,
                                           float(cfg["step"]), num, ctypes.c_void_p(dO.data_ptr()),
                                           ctypes.c_void_p(work.data_ptr()), nb.value,
                                           ctypes.cast(info.data_ptr(), capi.c_int_p))
        if not st.ok:
            raise RuntimeError(f"geodesic_points failed: {st!r}")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.calamanGetLaunchCount()
    assert lib.calamanSetKernelTiming(h, 1).ok
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                starts[i].record(stream)
                step()
                ends[i].record(stream)
        torch.cuda.synchronize()
        launches = lib.calamanGetLaunchCount() - launches0
        kt = capi.KernelTiming()
        assert lib.calamanGetKernelTiming(h, ctypes.byref(kt)).ok
        lib.calamanSetKernelTiming(h, 0)
        total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
        e2e_ms = 0.0
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a_ev.record(stream)
                dW.copy_(host_w, non_blocking=True)
                dH.copy_(host_h, non_blocking=True)
                step()
                host_o.copy_(dO, non_blocking=True)
                b_ev.record(stream)
                b_ev.synchronize()
                e2e_ms += a_ev.elapsed_time(b_ev)
    torch.cuda.synchronize()
    if info.item() != 0:
        raise RuntimeError(f"geodesic_points reported info {info.item()}")
    total_ms, e2e_ms = _max_over_ranks(torch, dist, dev, [total_ms, e2e_ms])
    value = world * args.steps / (total_ms * 1e-3)
    e2e_value = world * args.steps / (e2e_ms * 1e-3)
    if rank == 0:
        peak = measure_fp64_peak(torch, dev, True)
        achieved = kt.gemm_flops / (kt.gemm_ms * 1e-3) / 1e12 if kt.gemm_ms > 0 else None
        baseline, acc = None, {}
        if world == 1 and not args.no_cpu:
            from oracle import oracle as O

            cores = cpu_threads()
            O.set_threads(cores)
            t0 = time.perf_counter()
            O.geodesic_points(w, hmat, cfg["step"], num, blas=True)
            el = time.perf_counter() - t0
            baseline = {"value": 1.0 / el, "unit": "search/s", "cores": cores, "kind": "port",
                        "sample": f"one search's trial points in the reference's order (general expm, "
                                  f"power chain, products, all on numpy's BLAS), {el:.1f} s, "
                                  f"{threads_phrase(cores)}"}
            ref = O.geodesic_points(w, hmat, cfg["step"], num)  # the checker: the C oracle's expm
            got = host_o.numpy()
            worst = 0.0
            for j, r in enumerate(ref):
                g = got[j * n * n:(j + 1) * n * n].reshape(n, n).T
                worst = max(worst, float(np.linalg.norm(g - r) / np.linalg.norm(r)))
            acc["max_rel_frob_vs_oracle"] = worst
        flops = herm_flops(n, True) - 8.0 * n ** 3 + 8.0 * n ** 3 * (1 + (num - 1))
        line = {
            "metric": METRIC, "value": value, "unit": "search/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded)",
            "config": {"workload": args.config, "desc": cfg["desc"], "samples": num,
                       "l2": "flushed before every timed step (256 MiB write, untimed)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "tflops": flops * value / world / 1e12,
            "algorithmic_flops_per_search": flops,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if achieved else None, "traffic": None,
                         "kernel": "dense products (every GEMM launch in the timed steps)",
                         "launches": kt.gemm_launches, "kernel_ms_per_step": kt.gemm_ms / args.steps,
                         "peak_source": "cuBLAS complex128 GEMM 4096^3 measured in this run"},
            "cpu_baseline": baseline,
            "e2e": {"value": e2e_value, "unit": "search/s", "h2d_bytes_per_step": 2 * n * n * 16,
                    "d2h_bytes_per_step": (num - 1) * n * n * 16},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    lib.calamanDestroy(h)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _relaunch_under_torchrun(nproc):
    """`--gpus N` without a launcher: run this same command as N ranks of one
    node under torch.distributed.run (rendezvous on 127.0.0.1)."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__),
           *sys.argv[1:]]
    sys.stdout.flush()
    os.execv(sys.executable, cmd)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    p.add_argument("--e2e-parts", type=int, default=0,
                   help="sub-batches of the batched end-to-end pipelines (copies of one overlap another's compute; 0: 16 for the batched expm, 4 for the batched adjoint)")
    p.add_argument("--no-plain", action="store_true",
                   help="batched workloads: skip the per-matrix FP64 expm pass (for profiling runs)")
    p.add_argument("--cpu-threads", type=int, default=0,
                   help="host threads of the CPU baseline and the reference arm (numpy's "
                        "BLAS and the C oracle's workers); 0: every host thread")
    args = p.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        _relaunch_under_torchrun(args.gpus)
    global CPU_THREADS
    CPU_THREADS = max(0, args.cpu_threads)
    if CPU_THREADS:
        # numpy's BLAS (the timed restatements) obeys the same limit as the
        # C oracle's own workers
        from threadpoolctl import threadpool_limits

        threadpool_limits(limits=CPU_THREADS)
    cfg = CONFIGS[args.config]
    kind = cfg.get("kind", "single")
    if args.impl == "reference":
        run_reference(args, cfg)
    elif kind == "batched":
        run_batched(args, cfg)
    elif kind == "vjp":
        run_vjp(args, cfg)
    elif kind == "geodesic":
        run_geodesic(args, cfg)
    elif kind == "lu":
        run_lu(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
