"""Batched uneven solves: many seeded vertebral bodies of different sizes and
load cases solved concurrently on one GPU; reports solves/s and p50/p99
per-instance solve time.

    python -m simul_b200.batch_bench --instances 64 --n-min 32 --n-max 96

Instances: grid sizes drawn uniformly from [n-min, n-max] voxels per axis,
per-instance modulus fields (cortical shell 12 GPa, lognormal core), J2
(yield 100 MPa, H = 0.02 E).  Load case per instance, drawn from: axial
compression 1-3 % of the height (prescribed top-face displacement), or a
7.5 N m (7,500 N mm) flexion / extension / lateral-bending / torsion moment.
A moment is applied as an equivalent linear nodal force couple on the top-face
nodes (a rigid top plate is not modelled); the bottom face is fixed.
All data are seeded synthetic inputs.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import time
from concurrent.futures import ProcessPoolExecutor, ThreadPoolExecutor

import numpy as np

CASES = ("axial", "flexion", "extension", "lateral_bending", "torsion")
MOMENT = 7500.0  # N mm


def _make_case(args):
    """Host-side generation of one instance (runs in a worker process)."""
    idx, n, seed, case, strain = args
    from simul_b200 import meshgen
    v = meshgen.vertebral_body(n=n, seed=seed, axial_strain=strain)
    X = v.X
    fixed = v.fixed_mask.copy()
    vals = v.fixed_vals.copy()
    f = np.zeros_like(X)
    if case != "axial":
        top = np.isclose(X[:, 2], X[:, 2].max())
        fixed[top] = False
        vals[top] = 0.0
        f = meshgen.top_moment_forces(X, top, case, MOMENT)
    return {"idx": idx, "n": n, "seed": seed, "case": case, "strain": strain, "X": X, "conn": v.conn,
            "E": v.E, "fixed": fixed, "vals": vals, "f": f, "tets": int(v.n_elements)}


def instance_specs(instances, n_min, n_max, seed):
    """The seeded instance list: (index, grid size, mesh seed, load case, axial strain)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(instances):
        n = int(rng.integers(n_min, n_max + 1))
        case = CASES[int(rng.integers(0, len(CASES)))]
        specs.append((i, n, 1000 + i, case, float(rng.uniform(0.01, 0.03))))
    return specs


def shard(specs, rank, world):
    """This rank's share of the instances.  Instances are independent, so
    they are split across ranks with no collective in the solve: largest
    first (work grows as n^3), each to the rank with the least work so far
    (ties to the lower rank).  Every rank computes the same split."""
    load = [0] * world
    mine = []
    for sp in sorted(specs, key=lambda s: (-s[1] ** 3, s[0])):
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += sp[1] ** 3
        if r == rank:
            mine.append(sp)
    return sorted(mine, key=lambda s: s[0])


def gather_results(local, world):
    """Per-instance result dicts of all ranks, ordered by instance index (a
    host gather after the solves; world 1 returns ``local`` sorted)."""
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, local)
        local = [r for part in parts for r in part]
    return sorted(local, key=lambda r: r["idx"])


def run(instances=64, n_min=32, n_max=96, load_steps=10, threads=0, seed=0, precond="two_level",
        sequential=False, workers=16, coarse_cell=4, coarse_bf16=True, coarse_reuse=0, device=0,
        rank=0, world=1, extrapolate=True):
    """Generates the seeded instances, solves them as one batch after a
    one-step warm-up pass, and returns solves/s, p50/p99 per-instance wall
    time and iteration counts (one dict).  With world > 1 (one process per
    GPU, torch.distributed initialised) each rank solves its ``shard`` and
    the per-instance results are gathered; the batch time is the slowest
    rank's."""
    all_specs = instance_specs(instances, n_min, n_max, seed)
    specs = shard(all_specs, rank, world) if world > 1 else all_specs
    t0 = time.perf_counter()
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        cases = sorted(ex.map(_make_case, specs), key=lambda d: d["idx"])
    t_gen = time.perf_counter() - t0

    import torch
    from simul_b200 import batch
    from simul_b200 import fem as B
    dev = torch.device(device) if isinstance(device, str) else torch.device("cuda", device)
    torch.cuda.init()

    def build(d):
        mat = B.J2Plasticity(d["E"], 0.3, 100.0, hardening_modulus=0.02 * d["E"])
        inst = batch.BatchInstance(d["X"], d["conn"], mat, d["fixed"], d["vals"], d["f"], device=dev,
                                   coarse_cell=coarse_cell, coarse_bf16=bool(coarse_bf16),
                                   coarse_reuse=coarse_reuse)
        inst.mesh.set_extrapolation(bool(extrapolate))
        return inst

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=8) as ex:
        insts = list(ex.map(build, cases))
    t_setup = time.perf_counter() - t0

    def reset():
        """Every instance back to rest: u = 0, no plastic history."""
        for inst in insts:
            inst.reset()
        torch.cuda.synchronize()

    out = {"instances": []}
    wall = 0.0
    if insts:   # a rank may hold no instance when there are more ranks than instances
        # warm-up pass (graph capture, matvec-variant timing, coarse set-up), then reset
        batch.solve_batch(insts, load_steps=1, precond=precond, n_threads=threads)
        reset()
        t0 = time.perf_counter()
        out = batch.solve_batch(insts, load_steps=load_steps, precond=precond, n_threads=threads)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    local = [dict(r, idx=d["idx"], n=d["n"], case=d["case"], tets=d["tets"], rank=rank, rank_wall_s=wall)
             for r, d in zip(out["instances"], cases)]
    per = gather_results(local, world)
    wall = max(r["rank_wall_s"] for r in per)
    ms = np.array([r["wall_ms"] for r in per])
    res = {"instances": instances, "n_range": [n_min, n_max], "tets_total": int(sum(r["tets"] for r in per)),
           "tets_min": int(min(r["tets"] for r in per)), "tets_max": int(max(r["tets"] for r in per)),
           "cases": {c: sum(1 for r in per if r["case"] == c) for c in CASES},
           "load_steps": load_steps, "precond": precond, "extrapolate": bool(extrapolate),
           "coarse": {"cell_voxels": coarse_cell, "inverse": "bf16" if coarse_bf16 else "f32",
                      "reuse": coarse_reuse},
           "all_converged": bool(all(r["converged"] for r in per)),
           "batch_wall_s": wall, "solves_per_s": instances / wall,
           "p50_instance_ms": float(np.percentile(ms, 50)), "p99_instance_ms": float(np.percentile(ms, 99)),
           "newton_iterations": int(sum(r["newton_iterations"] for r in per)),
           "cg_iterations": int(sum(r["cg_iterations"] for r in per)),
           "host_generation_s": t_gen, "host_setup_s": t_setup}
    if world > 1:
        res["ranks"] = world
        res["instances_per_rank"] = [sum(1 for r in per if r["rank"] == k) for k in range(world)]
    if sequential and world == 1:
        reset()
        t0 = time.perf_counter()
        out2 = batch.solve_batch(insts, load_steps=load_steps, precond=precond, n_threads=1)
        torch.cuda.synchronize()
        res["sequential_wall_s"] = time.perf_counter() - t0
        res["sequential_solves_per_s"] = instances / res["sequential_wall_s"]
        res["sequential_all_converged"] = bool(all(r["converged"] for r in out2["instances"]))
    del insts
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--n-min", type=int, default=32)
    ap.add_argument("--n-max", type=int, default=96)
    ap.add_argument("--load-steps", type=int, default=10)
    ap.add_argument("--threads", type=int, default=0, help="host workers (0: one per instance)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precond", default="two_level", choices=["jacobi", "two_level"])
    ap.add_argument("--sequential", action="store_true", help="also time the instances one after another")
    ap.add_argument("--workers", type=int, default=16, help="host processes generating meshes")
    ap.add_argument("--coarse-cell", type=int, default=4, help="two-level lattice cell edge in voxels")
    ap.add_argument("--coarse-bf16", type=int, default=1, help="packed BF16 coarse inverse")
    ap.add_argument("--coarse-reuse", type=int, default=0,
                    help="coarse operator: 0 once per solve from rest (small-strain J2), -1 adaptive")
    ap.add_argument("--extrapolate", type=int, default=1, help="load-step extrapolation of the Newton start")
    args = ap.parse_args(argv)
    print(json.dumps(run(instances=args.instances, n_min=args.n_min, n_max=args.n_max, load_steps=args.load_steps,
                         threads=args.threads, seed=args.seed, precond=args.precond, sequential=args.sequential,
                         workers=args.workers, coarse_cell=args.coarse_cell, coarse_bf16=bool(args.coarse_bf16),
                         coarse_reuse=args.coarse_reuse, extrapolate=bool(args.extrapolate))))


if __name__ == "__main__":
    main()
