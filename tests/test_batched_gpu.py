"""GPU parity of expm_batched through the C ABI: every matrix of a batch of
mixed sizes and norms against the FP64 oracle (FP64 tier within 1e-12,
relative Frobenius) with the plan expm picks for it, the FP32 tier against
the oracle on the single-precision plan, against the FP64 batched tier on
the batched benchmark workload, padding, and the argument checks."""
import numpy as np
import pytest

from helpers import Runner, c4_batch, gaussian_scaled, rel_frob, scaled_random

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
SINGLE_REL = 5e-6


@pytest.fixture(scope="module")
def run(cuda):
    r = Runner()
    yield r
    r.close()


def mixed_batch(seed):
    cases = [(1, 0.3), (2, 1.0), (5, 4.0), (16, 0.01), (17, 0.2), (31, 0.9), (33, 2.0),
             (64, 5.0), (65, 30.0), (100, 2.0), (127, 12.0), (129, 0.5), (200, 80.0),
             (255, 6.0), (256, 40.0), (256, 0.1)]
    return [gaussian_scaled(n, t, seed + i) for i, (n, t) in enumerate(cases)]


def test_fp64_mixed_batch_matches_oracle(run, oracle):
    mats = mixed_batch(100)
    st, plans, outs, _, info = run.batched(mats, "d")
    assert st.ok, st
    assert (info == 0).all()
    for a, e, p in zip(mats, outs, plans):
        ref, op, _ = oracle.expm(a)
        assert (p.m, p.s, p.num_gemms) == (op.m, op.s, op.num_gemms)
        assert rel_frob(e, ref) <= FP64_REL, (a.shape[0], p.m, p.s)


def test_fp64_batch_matches_single_matrix_path(run):
    mats = mixed_batch(200)
    st, _, outs, _, _ = run.batched(mats, "d")
    assert st.ok
    for a, e in zip(mats, outs):
        st1, _, e1, _, _ = run.expm(a, "d")
        assert st1.ok and rel_frob(e, e1) <= 1e-13


def test_fp32_mixed_batch_matches_oracle(run, oracle):
    mats = [m.astype(np.float32) for m in mixed_batch(300)]
    st, plans, outs, _, _ = run.batched(mats, "s")
    assert st.ok
    for a, e, p in zip(mats, outs, plans):
        ref, op, _ = oracle.expm(a, single=True)
        assert (p.m, p.s) == (op.m, op.s)
        assert rel_frob(e, ref) <= SINGLE_REL, (a.shape[0], p.m, p.s)


def test_padding_and_leading_dimensions(run, oracle):
    mats = [scaled_random(n, 3.0, 400 + n) for n in (7, 40, 130)]
    lds = [9, 41, 133]
    ldes = [8, 45, 131]
    st, _, outs, fulls, _ = run.batched(mats, "d", lds=lds, ldes=ldes)
    assert st.ok
    for a, e, f, ld in zip(mats, outs, fulls, ldes):
        n = a.shape[0]
        assert rel_frob(e, oracle.expm(a)[0]) <= FP64_REL
        assert np.all(f.reshape(n, ld)[:, n:] == -123.5)


def test_argument_checks(run):
    ok = [gaussian_scaled(8, 1.0, 1)]
    st, *_ = run.batched([gaussian_scaled(257, 1.0, 2)], "d")
    assert st.code == run.capi.NOT_SUPPORTED
    bad = [gaussian_scaled(8, 1.0, 3), gaussian_scaled(9, 1.0, 4)]
    bad[1][3, 4] = np.inf
    st, _, outs, _, _ = run.batched(bad, "d")
    assert st.code == run.capi.INVALID_VALUE
    assert all(np.all(o == -123.5) for o in outs)  # nothing written
    st, *_ = run.batched(ok, "d", lwork=256)
    assert st.code == run.capi.ALLOC_FAILED
    st, *_ = run.batched([], "d")
    assert st.ok


def test_fp32_benchmark_workload_against_fp64_tier(run):
    """The batched benchmark's distribution (n on {16..256}, ||A||_1
    log-uniform in [0.1, 100]), FP32 tier against the FP64 tier."""
    mats = [m.astype(np.float32) for m in c4_batch(512, 2024)]
    st64, p64, o64, _, _ = run.batched([m.astype(np.float64) for m in mats], "d")
    st32, p32, o32, _, _ = run.batched(mats, "s")
    assert st64.ok and st32.ok
    worst = max(rel_frob(a, b) for a, b in zip(o32, o64))
    assert worst <= 1e-6, worst


def test_graph_replay_matches_direct_launches(run):
    """The batched call captures its launches as a CUDA graph when its
    configuration repeats, then replays it: the results stay identical to the
    directly launched call's, and the replays count their kernels."""
    import ctypes

    mats = [m.astype(np.float32) for m in c4_batch(96, 77)]
    en, cached = ctypes.c_int(-1), ctypes.c_int(-1)
    assert run.lib.calamanSetBatchedGraphs(run.h, 0).ok
    st0, _, o0, _, _ = run.batched(mats, "s")
    assert run.lib.calamanSetBatchedGraphs(run.h, 1).ok
    try:
        # run.batched allocates fresh buffers each call; keep one set so the
        # configuration repeats
        import torch

        from helpers import _dev, colmajor_buffer, from_buffer

        ns = [m.shape[0] for m in mats]
        dA = [_dev(colmajor_buffer(m, n, "s")) for m, n in zip(mats, ns)]
        dE = [torch.empty(n * n, dtype=torch.float32, device="cuda") for n in ns]
        b = len(mats)
        IntArr, PtrArr = ctypes.c_int * b, ctypes.c_void_p * b
        h_n = IntArr(*ns)
        h_A = PtrArr(*[t.data_ptr() for t in dA])
        h_E = PtrArr(*[t.data_ptr() for t in dE])
        nb = ctypes.c_size_t()
        assert run.lib.calaman_expm_batched_bufferSize_s(run.h, b, ctypes.cast(h_n, run.capi.c_int_p),
                                                         ctypes.byref(nb)).ok
        w = run.workspace(nb.value)
        info = torch.zeros(2 * b, dtype=torch.int32, device="cuda")
        side = torch.cuda.Stream()  # a capturable (non-default) stream
        torch.cuda.synchronize()
        outs = []
        for call in range(4):
            before = run.lib.calamanGetLaunchCount()
            st = run.lib.calaman_expm_batched_s(
                run.h, run.h, ctypes.c_void_p(side.cuda_stream), b, ctypes.cast(h_n, run.capi.c_int_p),
                ctypes.cast(h_A, ctypes.POINTER(ctypes.c_void_p)), ctypes.cast(h_n, run.capi.c_int_p),
                ctypes.cast(h_E, ctypes.POINTER(ctypes.c_void_p)), ctypes.cast(h_n, run.capi.c_int_p),
                ctypes.c_void_p(w.data_ptr()), nb.value, ctypes.cast(info.data_ptr(), run.capi.c_int_p), None)
            torch.cuda.synchronize()
            assert st.ok, st
            assert run.lib.calamanGetLaunchCount() - before > 0
            outs.append([from_buffer(t.cpu().numpy(), n, n) for t, n in zip(dE, ns)])
            assert run.lib.calamanGetBatchedGraphs(run.h, ctypes.byref(en), ctypes.byref(cached)).ok
            if call >= 1:
                assert en.value == 1 and cached.value >= 1
        for o in outs:
            assert all(np.array_equal(x, y) for x, y in zip(o, o0))
    finally:
        run.lib.calamanSetBatchedGraphs(run.h, 1)


def test_schedule_setting_and_the_tuner(run, oracle):
    import ctypes

    lu = (ctypes.c_int * 17)()
    tc = ctypes.c_int()
    assert run.lib.calamanGetBatchedTuning(run.h, lu, ctypes.byref(tc)).ok
    default = list(lu), tc.value
    bad = (ctypes.c_int * 17)(*([256] * 17))
    bad[10] = 64  # fewer threads than rows (n = 160)
    assert run.lib.calamanSetBatchedTuning(run.h, bad, 1).code == 7
    assert run.lib.calamanSetBatchedTuning(run.h, None, 0).code == 7
    mats = mixed_batch(500)
    ref = [oracle.expm(a)[0] for a in mats]
    try:
        # every LU on 256-thread CTAs, FP32 products on the SIMT kernel below n = 129
        all256 = (ctypes.c_int * 17)(*([256] * 17))
        assert run.lib.calamanSetBatchedTuning(run.h, all256, 129).ok
        st, _, o64, _, _ = run.batched(mats, "d")
        assert st.ok and all(rel_frob(e, r) <= FP64_REL for e, r in zip(o64, ref))
        st, _, o32, _, _ = run.batched([m.astype(np.float32) for m in mats], "s")
        assert st.ok and all(rel_frob(e.astype(np.float64), r) <= SINGLE_REL for e, r in zip(o32, ref))
        # the tuner on a small batch per size: a valid schedule, kept in the handle
        count = 8
        nb = run.lib.calamanTuneBatched_bufferSize(count)
        w = run.workspace(nb)
        assert run.lib.calamanTuneBatched(run.h, count, ctypes.c_void_p(w.data_ptr()), nb, lu,
                                          ctypes.byref(tc)).ok
        assert all(lu[b] in (64, 128, 256) and lu[b] >= 16 * b for b in range(1, 17))
        assert 1 <= tc.value <= 257
        st, _, o32, _, _ = run.batched([m.astype(np.float32) for m in mats], "s")
        assert st.ok and all(rel_frob(e.astype(np.float64), r) <= SINGLE_REL for e, r in zip(o32, ref))
    finally:
        run.lib.calamanSetBatchedTuning(run.h, (ctypes.c_int * 17)(*default[0]), default[1])
