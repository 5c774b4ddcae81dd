"""Small, self-terminating workload for kernel profiling (ncu) and timing.

Builds the synthetic vertebral body at ``--n`` voxels per axis (five TET4
per voxel, or one HEX8 per voxel with ``--element hex8``), binds J2
plasticity, evaluates the FP64 residual at a plastic state (top face pushed
``--strain`` of the height, which yields the cortical shell), and launches each
hot kernel ``--reps`` times through ``fem_profile_kernels``: the tangent matvec
(the variant given by ``--variant``), the FP64 residual, the CG update and the
CG direction update; optionally the learned network's forward pass
(``--learned weights.npz``) and one two-level PCG solve (``--two-level``,
4-voxel cells with the packed BF16 coarse inverse by default, run as
fixed-size iteration graphs so a kernel profiler sees every launch).  The
per-launch CUDA-event times are printed as one JSON line.  With ``--reps 3`` and ``-k``/``-c`` filters an ncu capture of one kernel
ends in seconds.

    python -m simul_b200.profile_case --n 64 --variant fused --reps 3
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--variant", default="fused", choices=["fused", "two_phase", "element_block", "warp_agg", "persistent"])
    ap.add_argument("--block-size", type=int, default=0, help="element-block variant: elements per block")
    ap.add_argument("--element", default="tet4", choices=["tet4", "hex8"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--strain", type=float, default=0.004)
    ap.add_argument("--nodes-per-block", type=int, default=0)
    ap.add_argument("--residual", default="two_phase", choices=["two_phase", "fused"],
                    help="TET4 FP64 residual variant")
    ap.add_argument("--learned", default="", help="weights file: also run the network forward --reps times")
    ap.add_argument("--two-level", action="store_true", help="also run one two-level PCG solve (rtol 1e-6)")
    ap.add_argument("--coarse-cell", type=int, default=4, help="two-level: lattice cell edge in voxels")
    ap.add_argument("--coarse-bf16", type=int, default=1, help="two-level: BF16 packed coarse inverse")
    args = ap.parse_args(argv)

    import torch

    from simul_b200 import _lib, meshgen
    from simul_b200 import fem as B

    v = meshgen.vertebral_body(n=args.n, seed=0, element=args.element)
    et = B.ElementType.HEX8 if args.element == "hex8" else B.ElementType.TET4
    mesh = B.FEMesh(v.n_nodes, v.n_elements, et, device=0, nodes_per_block=args.nodes_per_block)
    mesh.initialize_from_numpy(v.X, v.conn)
    if args.element == "tet4":
        mesh.set_matvec_variant(args.variant, block_size=args.block_size if args.variant == "element_block" else None)
        mesh.set_residual_variant(args.residual)
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    idx = np.where(v.fixed_mask.reshape(-1))[0]
    vals = (v.fixed_vals * (args.strain / 0.02)).reshape(-1)
    mesh.set_fixed_dofs(idx, vals[idx])
    # a smooth compression field with the prescribed values on the boundary
    top = v.X[:, 2].max()
    u = np.zeros_like(v.X)
    u[:, 2] = -args.strain * v.X[:, 2] * (top / max(top, 1e-30))
    mesh.u.copy_(torch.from_numpy(u))
    mat.compute_nodal_forces(mesh)
    ms = (C.c_double * 4)()
    rc = _lib.load().fem_profile_kernels(mesh.ctx, args.reps, ms)
    if rc != 0:
        raise RuntimeError(_lib.last_error(mesh.ctx))
    torch.cuda.synchronize()
    extra = {}
    if args.learned:
        from simul_b200 import learned
        learned.set_weights(mesh, learned.load(args.learned))
        r = torch.randn(v.n_nodes, 3, dtype=torch.float32, device=mesh.device)
        z = torch.empty_like(r)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.reps):
            rc = _lib.load().fem_mpnn_forward(mesh.ctx, B._ptr(r), B._ptr(z))
            if rc != 0:
                raise RuntimeError(_lib.last_error(mesh.ctx))
        e1.record()
        e1.synchronize()
        extra["mpnn_forward_ms"] = e0.elapsed_time(e1) / args.reps
    if args.two_level:
        mesh.set_coarse_options(cell=args.coarse_cell, bf16=bool(args.coarse_bf16))
        mesh.set_whole_solve_graph(False)   # kernel profilers cannot see into the conditional graph
        rhs = torch.randn(v.n_nodes, 3, dtype=torch.float64, device=mesh.device)
        du = torch.zeros_like(rhs)
        it, rel = C.c_int32(), C.c_double()
        rc = _lib.load().fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, B._ptr(rhs),
                                 B._ptr(du), 1e-6, 5000, C.byref(it), C.byref(rel))
        if rc not in (0, _lib.FEM_NOT_CONVERGED):
            raise RuntimeError(_lib.last_error(mesh.ctx))
        extra["two_level_iterations"] = it.value
        extra["coarse"] = mesh.coarse_info()
    info = mesh.info()
    print(json.dumps({"n": args.n, "element": args.element, "elements": info["n_elements"],
                      "nodes": info["n_nodes"], "variant": "two_phase" if args.element == "hex8" else args.variant,
                      "reps": args.reps, "block_size": mesh.stats()["element_block_size"],
                      "ms": {"matvec": ms[0], "residual": ms[1], "cg_update": ms[2], "cg_direction": ms[3]},
                      **extra}))


if __name__ == "__main__":
    main()
