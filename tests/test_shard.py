"""The batched tier's multi-rank host path on CPU: the cost-balanced
partition of a batch across ranks, and a two-rank gloo job in which every rank
evaluates its shard (with the oracle, no GPU) and rank 0 gathers the results,
which must equal a single-process evaluation of the whole batch."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from calaman_g_b200.shard import expm_cost, partition

from helpers import gaussian_scaled


def test_partition_covers_and_balances():
    rng = np.random.default_rng(3)
    costs = list(rng.uniform(1.0, 100.0, 257))
    for world in (1, 2, 3, 8):
        shards = partition(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
    assert partition(costs, 4) == partition(list(costs), 4)  # deterministic


def test_expm_cost_matches_flop_formula():
    assert expm_cost(256, 13, 0) == pytest.approx(2.461e8, rel=2e-3)
    assert expm_cost(2, 3, 0) == (2 + 0) * 16 + (2 / 3) * 8 + 16


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O

        mats = [gaussian_scaled(n, t, 50 + i) for i, (n, t) in
                enumerate([(5, 0.1), (9, 3.0), (12, 40.0), (7, 1.0), (16, 8.0), (3, 0.5)])]
        plans = [O.expm_plan(O.norm1(a)) for a in mats]
        costs = [expm_cost(a.shape[0], p.m, p.s) for a, p in zip(mats, plans)]
        mine = partition(costs, world)[rank]
        results = {i: O.expm(mats[i])[0] for i in mine}
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(results, gathered, dst=0)
        if rank == 0:
            merged = {}
            for part in gathered:
                assert not (set(part) & set(merged))
                merged.update(part)
            assert sorted(merged) == list(range(len(mats)))
            ok = all(np.array_equal(merged[i], O.expm(mats[i])[0]) for i in range(len(mats)))
            out.put(ok)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shards_match_single_process():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert out.get(timeout=5) is True


def _bench_worker(rank, world, port, out):
    """What bench.py does for a batched workload under torchrun: each rank
    takes its share of the global batch from the plans the library picks."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from calaman_g_b200 import capi

        lib = capi.load()
        cfg = dict(bench.CONFIGS["expm_batched_f32_8192"], count=48)
        mine, total = bench.batched_shard(lib, cfg, world, rank)
        sizes, norms = bench.batched_spec(cfg, total)
        plans = [lib.calaman_expm_plan_s(float(norms[i])) for i in mine]
        mats = bench.batched_workload(cfg, mine, total)
        local = {"idx": mine, "n": [m.shape[0] for m in mats],
                 "plans": [(p.m, p.s) for p in plans],
                 "cost": sum(expm_cost(int(sizes[i]), p.m, p.s) for i, p in zip(mine, plans))}
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        if rank == 0:
            allidx = sorted(i for g in gathered for i in g["idx"])
            ok = allidx == list(range(total))                      # the shards cover the batch
            ok &= sum(len(g["idx"]) for g in gathered) == total    # disjointly
            ok &= all(g["n"] == [int(sizes[i]) for i in g["idx"]] for g in gathered)
            from oracle import oracle as O
            want = {i: O.expm_plan(float(norms[i]), single=True) for i in range(total)}
            ok &= all((m, s_) == (want[i].m, want[i].s)
                      for g in gathered for i, (m, s_) in zip(g["idx"], g["plans"]))
            costs = [g["cost"] for g in gathered]
            ok &= max(costs) <= 1.2 * min(costs)                   # balanced
            out.put(bool(ok))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_bench_shards_are_the_batch():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 30500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    assert out.get(timeout=5) is True
