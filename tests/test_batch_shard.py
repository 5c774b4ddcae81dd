"""Batched uneven solves sharded across ranks (CPU, gloo world size 2).

Instances are independent, so each rank solves its own share with no
collective in the solve; the per-instance results are gathered on the host
afterwards.  These tests check the split (every instance on exactly one rank,
work balanced) and the gather (every rank ends with all instances' results in
index order) without a GPU: the per-instance "solve" is a host stand-in.
"""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from simul_b200 import batch_bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_covers_every_instance_once_and_balances_work():
    specs = batch_bench.instance_specs(64, 32, 96, seed=0)
    for world in (1, 2, 3, 8):
        parts = [batch_bench.shard(specs, r, world) for r in range(world)]
        ids = sorted(s[0] for p in parts for s in p)
        assert ids == list(range(64))
        work = [sum(s[1] ** 3 for s in p) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest instance
        assert max(work) - sum(work) / world <= max(s[1] ** 3 for s in specs)
        for p in parts:
            assert [s[0] for s in p] == sorted(s[0] for s in p)


def test_shard_with_more_ranks_than_instances():
    specs = batch_bench.instance_specs(3, 32, 40, seed=1)
    parts = [batch_bench.shard(specs, r, 5) for r in range(5)]
    assert sorted(s[0] for p in parts for s in p) == [0, 1, 2]
    assert sum(1 for p in parts if not p) == 2


def _stand_in_result(spec, rank):
    idx, n, seed, case, strain = spec
    return {"idx": idx, "n": n, "case": case, "tets": 5 * n ** 3, "rank": rank, "converged": True,
            "wall_ms": float(n), "rank_wall_s": 0.0, "cg_iterations": idx * 7}


def _gather_worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from simul_b200 import batch_bench as bb
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        specs = bb.instance_specs(10, 32, 96, seed=3)
        local = [_stand_in_result(sp, rank) for sp in bb.shard(specs, rank, world)]
        per = bb.gather_results(local, world)
        out.put((rank, [(r["idx"], r["rank"], r["cg_iterations"]) for r in per]))
    finally:
        dist.destroy_process_group()


def test_gather_results_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    specs = batch_bench.instance_specs(10, 32, 96, seed=3)
    owner = {s[0]: r for r in range(2) for s in batch_bench.shard(specs, r, 2)}
    want = [(i, owner[i], i * 7) for i in range(10)]
    assert got[0] == want and got[1] == want
    assert {r for _, r, _ in want} == {0, 1}
