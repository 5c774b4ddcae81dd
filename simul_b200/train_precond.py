"""Trains the learned preconditioner on synthetic vertebral bodies and saves it.

    python -m simul_b200.train_precond --out simul_b200/weights/mpnn_vertebra.npz

Training data are (residual, correction) pairs produced by the library's
Jacobi-PCG at tangent states of the plain J2 solve: for each training body
(seeds ``--seeds``, ``--n`` voxels per axis) the elastic state and the state
after half of the compression.  The loss is the preconditioner's A-norm error
with the two-level coarse correction included, so the network learns what
the coarse lattice misses.  The bodies here never include the benchmark's
seed-0 body, which stays held out.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np
import torch

from . import learned, meshgen
from . import fem as B


def _state(n, seed, frac, dev, load_steps=20, cell=8):
    v = meshgen.vertebral_body(n=n, seed=seed)
    mesh = B.FEMesh(v.n_nodes, v.n_elements, device=dev)
    mesh.initialize_from_numpy(v.X, v.conn)
    mesh.set_coarse_options(cell=cell)
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    idx = np.where(v.fixed_mask.reshape(-1))[0]
    k_end = int(round(frac * load_steps))
    if k_end == 0:
        mesh.set_fixed_dofs(idx, np.zeros(idx.size))
        mat.compute_nodal_forces(mesh)
    else:
        solver = B.StaticSolver(mesh, mat, tol=1e-8, precond="two_level")
        for k in range(1, k_end + 1):
            mesh.set_fixed_dofs(idx, (v.fixed_vals * (k / load_steps)).reshape(-1)[idx])
            solver.solve(verbose=False)
        mat.compute_nodal_forces(mesh)
    return v, mesh


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "weights" / "mpnn_vertebra.npz"))
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--seeds", type=int, nargs="+", default=[1, 2, 3])
    ap.add_argument("--fracs", type=float, nargs="+", default=[0.0, 0.5])
    ap.add_argument("--pairs", type=int, default=48)
    ap.add_argument("--rounds", type=int, default=4)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--init-seed", type=int, default=0)
    args = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    states = []
    for seed in args.seeds:
        for frac in args.fracs:
            v, mesh = _state(args.n, seed, frac, dev)
            learned.set_weights(mesh, learned.init_weights(seed=args.init_seed))
            rng = np.random.default_rng(1000 * seed + int(100 * frac))
            R, E = learned.solver_pairs(mesh, learned.random_rhs(v.X, v.fixed_mask, args.pairs, rng))
            states.append((mesh, R, E))
    t_data = time.perf_counter() - t0
    w = learned.init_weights(seed=args.init_seed)
    log = []
    for rnd in range(args.rounds):
        for k, (mesh, R, E) in enumerate(states):
            learned.set_weights(mesh, w)
            res = learned.train(mesh, R, E, steps=args.steps, batch=args.batch,
                                lr=args.lr * (0.5 ** (rnd // 2)), seed=rnd, reset_optimizer=(rnd == 0))
            w = learned.get_weights(mesh)
            log.append({"round": rnd, "state": k, **res})
    evals = []
    for mesh, R, E in states:
        learned.set_weights(mesh, w)
        evals.append(learned.evaluate(mesh, R[:8], E[:8]))
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    learned.save(args.out, w)
    print(json.dumps({"out": args.out, "states": len(states), "pairs_per_state": args.pairs,
                      "data_s": t_data, "total_s": time.perf_counter() - t0,
                      "final_losses": evals, "last_rounds": log[-len(states):]}))


if __name__ == "__main__":
    main()
