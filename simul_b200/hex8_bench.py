"""HEX8 vertebral-body static solve: the headline workload's geometry and
loading with one 8-node hexahedron (2 x 2 x 2 Gauss points) per voxel.

Synthetic vertebral body at ``--n`` voxels per axis (h = 32/n mm), J2
plasticity (yield 100 MPa, H = 0.02 E), bottom face fixed, top face pushed
2 % of the height in ``--load-steps`` steps, each Newton solve to ``--tol``.
After ``--warmup`` untimed sequences, each timed sequence starts from rest
(history reset) and is timed with CUDA events on the solve stream; an L2-sized
buffer is rewritten between sequences.  Prints one JSON line per
preconditioner.

    python -m simul_b200.hex8_bench --n 64 --precond two_level jacobi
"""
from __future__ import annotations

import argparse
import json

import numpy as np

L2_FLUSH_BYTES = 256 << 20


def run(n=64, precond="two_level", load_steps=20, tol=1e-8, warmup=1, steps=3, coarse_cell=4,
        whole_solve_graph=True, body=None, device="cuda:0", extrapolate=True) -> dict:
    """Times ``steps`` sequences of ``load_steps`` solves from rest after
    ``warmup`` untimed ones; returns the median and the solve counts."""
    import torch

    from simul_b200 import fem as B
    from simul_b200 import meshgen

    dev = torch.device(device)
    v = body if body is not None else meshgen.vertebral_body(n, seed=0, element="hex8")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    mesh = B.FEMesh(v.n_nodes, v.n_elements, B.ElementType.HEX8, device=dev)
    mesh.initialize_from_numpy(v.X, v.conn)
    mesh.set_coarse_options(cell=coarse_cell, bf16=True, reuse=0, inverse="tf32", max_nodes=6144)
    mesh.set_whole_solve_graph(bool(whole_solve_graph))
    mesh.set_extrapolation(bool(extrapolate))
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    solver = B.StaticSolver(mesh, mat, tol=tol, precond=precond)
    idx = np.where(v.fixed_mask.reshape(-1))[0]
    vals = v.fixed_vals.reshape(-1)[idx]

    def sequence():
        mesh.u.zero_()
        mat.reset_state()
        st = {"newton": 0, "cg": 0, "converged": True}
        for k in range(1, load_steps + 1):
            mesh.set_fixed_dofs(idx, vals * (k / load_steps))
            r = solver.solve(verbose=False)
            st["newton"] += r["iterations"]
            st["cg"] += r["cg_iterations"]
            st["converged"] &= bool(r["converged"])
        return st

    for _ in range(warmup):
        sequence()
    torch.cuda.synchronize()
    times, st = [], None
    for _ in range(steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = sequence()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    out = {"element": "hex8", "n": n, "hexes": int(v.n_elements), "nodes": int(v.n_nodes), "precond": precond,
           "load_steps": load_steps, "tol": tol, "seconds": float(np.median(times)), "seconds_all": times, **st,
           "coarse": mesh.coarse_info() if precond == "two_level" else None, "data": "synthetic"}
    del solver, mesh
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--load-steps", type=int, default=20)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precond", nargs="+", default=["two_level", "jacobi"],
                    choices=["two_level", "jacobi"])
    ap.add_argument("--coarse-cell", type=int, default=4)
    ap.add_argument("--whole-solve-graph", type=int, default=1,
                    help="0: fixed-size iteration graphs (kernel profilers cannot see into the conditional graph)")
    args = ap.parse_args(argv)

    from simul_b200 import meshgen

    v = meshgen.vertebral_body(args.n, seed=0, element="hex8")
    for pc in args.precond:
        print(json.dumps(run(args.n, pc, args.load_steps, args.tol, args.warmup, args.steps, args.coarse_cell,
                             bool(args.whole_solve_graph), body=v)), flush=True)


if __name__ == "__main__":
    main()
