"""Synthetic motion segment: the four moment load cases as a batch.

    python -m simul_b200.motion_segment_bench --n 80 --moment 750

Two vertebral bodies (J2, per-element modulus), an intervertebral disc
(hyperelastic Mooney-Rivlin matrix C10 = 0.18, C01 = 0.045 MPa, D1 from
nu = 0.45, two fibre families at +-30 degrees from horizontal in the x-z
plane, 500 MPa) and a titanium pedicle-screw cylinder (E = 110 GPa, nu = 0.3)
on one voxel grid (``meshgen.motion_segment``).  Bottom face fixed; flexion,
extension, lateral bending and torsion moments on the top face as equivalent
nodal force couples, each instance its own context, solved concurrently by
``fem_batch_solve`` with the two-level preconditioner.  Seeded synthetic data.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

CASES = ("flexion", "extension", "lateral_bending", "torsion")


def disc_material():
    from simul_b200 import fem as B
    fib = np.array([[np.cos(np.pi / 6), 0.0, np.sin(np.pi / 6)], [np.cos(np.pi / 6), 0.0, -np.sin(np.pi / 6)]])
    mu = 2.0 * (0.18 + 0.045)
    K = 2.0 * mu * (1.0 + 0.45) / (3.0 * (1.0 - 2.0 * 0.45))
    return B.FibreReinforcedMooneyRivlin(0.18, 0.045, 2.0 / K, fib, 500.0)


def materials(E):
    from simul_b200 import fem as B
    return {0: B.J2Plasticity(E, 0.3, 100.0, hardening_modulus=0.02 * E), 1: disc_material(),
            2: B.LinearElastic(110e3, 0.3)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=80, help="voxels across the 32 mm extent")
    ap.add_argument("--moment", type=float, default=750.0, help="N mm")
    ap.add_argument("--load-steps", type=int, default=5)
    ap.add_argument("--precond", default="two_level", choices=["jacobi", "two_level"])
    ap.add_argument("--line-search", default="reference", choices=["reference", "guarded", "none"])
    ap.add_argument("--max-iterations", type=int, default=50)
    ap.add_argument("--coarse-cell", type=int, default=8)
    ap.add_argument("--coarse-reuse", type=int, default=-1,
                    help="coarse operator: 0 once per state, -1 adaptive refresh, k every k PCG solves")
    ap.add_argument("--recurrence", type=int, default=1, help="two-level CG direction by recurrence")
    ap.add_argument("--block-smoother", type=int, default=1, help="two-level nodal block smoother")
    ap.add_argument("--cases", nargs="+", default=list(CASES), choices=list(CASES),
                    help="moment cases solved as one batch")
    ap.add_argument("--extrapolate", type=int, default=0, help="load-step extrapolation of the Newton start")
    args = ap.parse_args(argv)
    from simul_b200 import batch, meshgen
    import torch
    t0 = time.perf_counter()
    ms = meshgen.motion_segment(n=args.n)
    ids = ms.info["material_ids"]
    top = np.isclose(ms.X[:, 2], ms.X[:, 2].max())
    t_gen = time.perf_counter() - t0
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    insts = [batch.BatchInstance(ms.X, ms.conn, materials(ms.E), ms.fixed_mask, None,
                                 meshgen.top_moment_forces(ms.X, top, case, args.moment), device=dev,
                                 material_ids=ids, coarse_cell=args.coarse_cell) for case in args.cases]
    for inst in insts:
        inst.mesh.set_coarse_options(reuse=args.coarse_reuse)
        inst.mesh.set_direction_recurrence(bool(args.recurrence))
        inst.mesh.set_block_smoother(bool(args.block_smoother))
        inst.mesh.set_extrapolation(bool(args.extrapolate))
    t_setup = time.perf_counter() - t0
    kw = dict(precond=args.precond, line_search=args.line_search, max_iterations=args.max_iterations)
    batch.solve_batch(insts, load_steps=1, **kw)      # warm-up
    for inst in insts:
        inst.reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = batch.solve_batch(insts, load_steps=args.load_steps, **kw)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    res = {"tets": int(ms.n_elements), "nodes": int(ms.n_nodes), "disc_tets": ms.info["disc_elements"],
           "screw_tets": ms.info["screw_elements"], "moment_N_mm": args.moment, "load_steps": args.load_steps,
           "precond": args.precond, "line_search": args.line_search, "batch_wall_s": wall,
           "coarse": {"cell_voxels": args.coarse_cell, "reuse": args.coarse_reuse},
           "direction_recurrence": bool(args.recurrence), "block_smoother": bool(args.block_smoother),
           "host_generation_s": t_gen, "host_setup_s": t_setup,
           "cases": {}}
    for case, inst, r in zip(args.cases, insts, out["instances"]):
        u = inst.mesh.u.cpu().numpy()
        res["cases"][case] = {**r, "max_u_mm": float(np.abs(u).max()),
                              "top_mean_u_mm": u[top].mean(axis=0).round(6).tolist()}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
