"""bench.py's reference arm on the CPU: the JSON line it prints for the
driver (one line, `impl` reference, the line's own value as cpu_baseline and
e2e with no host<->device bytes) and the host-thread limit of its CPU legs."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_line(*extra):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--config", "expm_f64_256", "--steps", "1", "--warmup", "0", *extra],
                       capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_line_contract():
    d = _reference_line()
    assert d["impl"] == "reference"
    assert d["unit"] == "expm/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "expm_f64_256"
    assert d["config"]["plan"] == {"m": 13, "s": 0}  # the C1 matrix, 1-norm 4
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["cores"] == (os.cpu_count() or 1)
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_single_thread():
    d = _reference_line("--cpu-threads", "1")
    assert d["cpu_baseline"]["cores"] == 1
    assert d["cpu_baseline"]["sample"].endswith("1 thread")
    assert "BLAS" in d["cpu_baseline"]["sample"]
    assert d["value"] > 0


def test_hbm_min_bound():
    """The batched line's minimum-HBM-traffic figure: 2 n^2 elements per
    matrix over the step time, against the measured copy bandwidth."""
    sys.path.insert(0, ROOT)
    import bench

    peak, _ = bench._hbm_peak()
    d = bench.hbm_min([16, 256], 4, 2.0)
    assert d["bytes_per_step"] == 2 * (16 * 16 + 256 * 256) * 4
    assert abs(d["achieved_gbs"] - d["bytes_per_step"] / 2e-3 / 1e9) < 1e-12
    assert d["peak_gbs"] == peak and abs(d["frac"] - d["achieved_gbs"] / peak) < 1e-15


def test_batched_reference_spreads_over_workers():
    """More than one host thread: the batched sample runs on single-threaded
    worker processes (spawned), one step = 8 matrices per thread."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--config", "expm_batched_f32_8192", "--steps", "1", "--warmup", "0",
                        "--cpu-threads", "2"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    assert d["cpu_baseline"]["cores"] == 2 and d["value"] > 0
    assert "the first 16 matrices" in d["cpu_baseline"]["sample"]
    assert "2 single-threaded worker processes" in d["cpu_baseline"]["sample"]


def test_vjp_cpu_sample_one_thread():
    """The adjoint lines' CPU baseline: the numpy restatement, timed whole."""
    sys.path.insert(0, ROOT)
    import bench

    pairs = [bench.vjp_pair(64, 6.0, 7000 + i) for i in range(3)]
    old = bench.CPU_THREADS
    bench.CPU_THREADS = 1
    try:
        d = bench.vjp_cpu_sample(pairs, True, seconds=0.2)
    finally:
        bench.CPU_THREADS = old
    assert d["unit"] == "vjp/s" and d["value"] > 0 and d["cores"] == 1 and d["kind"] == "port"
    assert d["sample"].endswith("1 thread")
