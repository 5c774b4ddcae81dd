#!/usr/bin/env python
"""Time-to-1e-8 residual of the synthetic vertebral-body J2 static solve on B200.

Workload (one "step"): the 64^3-voxel, 0.5 mm vertebral body (566,000 TET4,
121,023 nodes), J2 plasticity with per-element E (cortical 12 GPa shell,
lognormal core around 300 MPa), bottom fixed, top face compressed 2 % in 20
load steps, every load step solved by Newton (FP64 residual) + Jacobi-PCG
(FP32 matvecs, FP64 dots) to 1e-8 relative residual.  Each step starts from
u = 0 and zero plastic history.  Inputs are seeded synthetic data.

``value`` is the device time of one full solve (CUDA events on the solver's
stream, L2 flushed before every timed step, inputs resident in HBM);
``e2e`` is the same solve through the public API with the per-solve inputs
copied from pinned host memory and the displacement copied back.
``--impl reference`` times the CPU restatement of the same method (the
reference itself, Python 3.13 + Taichi, cannot run in this image).

One process per GPU (torchrun for N > 1): every rank solves its own replica
(the single-mesh solve does not shard); ``value`` is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-8 residual: learned-FPCG vs Jacobi-PCG (1 B200); elem GB/s"
UNIT = "s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", "--grid", dest="n", type=int, default=64, help="voxels per axis of the vertebral grid")
    ap.add_argument("--load-steps", type=int, default=20)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--precond", default="two_level", choices=["jacobi", "two_level", "learned"],
                    help="preconditioner of the timed solve; Jacobi-PCG is timed beside it")
    ap.add_argument("--weights", default=os.path.join(ROOT, "simul_b200", "weights", "mpnn_vertebra.npz"),
                    help="learned-preconditioner weights (simul_b200.train_precond)")
    ap.add_argument("--learned-coarse", type=int, default=1, help="learned: add the coarse correction")
    ap.add_argument("--matvec-variant", default="auto", choices=["auto", "fused", "two_phase", "element_block", "warp_agg", "persistent"],
                    help="tangent-matvec variant (auto: timed on the first solve)")
    ap.add_argument("--no-jacobi-baseline", action="store_true")
    ap.add_argument("--no-hex8", action="store_true", help="skip the HEX8 form of the workload (reported beside)")
    ap.add_argument("--coarse-reuse", type=int, default=0,
                    help="coarse operator rebuilds: 0 once per solve from rest (this small-strain J2 path: "
                         "the first operator serves the whole load path), k every k PCG solves, -1 adaptive")
    ap.add_argument("--coarse-cell", type=int, default=4,
                    help="coarse lattice cell edge in voxels (4: 7,728 coarse DOFs on the n = 64 body)")
    ap.add_argument("--coarse-bf16", type=int, default=1,
                    help="store the coarse inverse in BF16 (packed lower block triangle)")
    ap.add_argument("--whole-solve-graph", type=int, default=1,
                    help="1: one graph launch per PCG solve; 0: fixed-size iteration graphs (for kernel profilers)")
    ap.add_argument("--pdl", type=int, default=1, help="programmatic dependent launches in the CG graphs")
    ap.add_argument("--coarse-inverse", default="tf32",
                    choices=["f32", "f64", "tf32", "trsm_syrk", "potri", "trsm_syrk_f32", "trsm_syrk_tf32"],
                    help="precision of the coarse operator's Cholesky, triangular inverse and product")
    ap.add_argument("--coarse-max-nodes", type=int, default=6144, help="cap on the coarse lattice's nodes")
    ap.add_argument("--block-smoother", type=int, default=1,
                    help="two-level smoother: 1 nodal 3x3 block inverse, 0 diagonal inverse")
    ap.add_argument("--fused-step", type=int, default=0,
                    help="1: CG work after each matvec as one cooperative kernel; 0: kernel chain")
    ap.add_argument("--extrapolate", type=int, default=1,
                    help="1: each load step's Newton starts from the last step's change of u repeated "
                         "(convergence test unchanged); 0: from the previous state, the change of the "
                         "prescribed values carried by a first linear solve")
    ap.add_argument("--cg-rtol-min", type=float, default=1e-5, help="inexact-Newton forcing term floor")
    ap.add_argument("--cg-rtol-max", type=float, default=1e-1, help="inexact-Newton forcing term cap")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the keys reported beside the headline (1M-tet point, n = 128 roofline, batch)")
    ap.add_argument("--n-large", type=int, default=78,
                    help="the vertebral body solved beside the headline (78: ~1.02 M tets)")
    ap.add_argument("--n-roofline", type=int, default=128,
                    help="matvec roofline also reported at this size (beyond L2)")
    ap.add_argument("--batch-instances", type=int, default=16, help="batched uneven solves reported beside")
    return ap.parse_args()


def max_over_ranks(x: float, device, ws: int) -> float:
    """Max of a per-rank timing over all ranks (any backend; identity at N=1)."""
    if ws <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def world():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload_config(args, v):
    return {"workload": f"vertebral_body_n{args.n}_j2_{args.load_steps}steps",
            "voxels": int(v.info["n_voxels"]), "tets": int(v.n_elements), "nodes": int(v.n_nodes),
            "h_mm": v.info["h"], "load_steps": args.load_steps, "tol": args.tol,
            "material": "J2 sigma_y=100 MPa H=0.02E, E shell 12 GPa / core lognormal(300 MPa, 0.3)",
            "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas"}


class ClockSampler:
    """nvidia-smi samples (200 ms) over the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def matvec_bytes(n_elements, n_nodes):
    """Algorithmic bytes of one J2 tangent matvec launch.

    Per element: connectivity 16, tangent payload 32 (n, theta, gamma2),
    material id 1 + modulus scale 4, node-block slot entries 16.  Per node:
    coordinates 16 (float4), x 12, y 12, slot row pointer 4, fixed mask 1.
    """
    return n_elements * (16 + 32 + 5 + 16) + n_nodes * (16 + 12 + 12 + 4 + 1)


def residual_bytes(n_elements, n_nodes):
    """Algorithmic bytes of one FP64 J2 residual launch: per element conn 16,
    id+scale 5, slots 16, history read 56 + trial write 56, payload write 32;
    per node X 24, u 24, f_ext 24, R 24, row 4, mask 1."""
    return n_elements * (16 + 5 + 16 + 56 + 56 + 32) + n_nodes * (24 + 24 + 24 + 24 + 4 + 1)


def load_traffic():
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        try:
            return json.load(open(path))
        except ValueError:
            return {}
    return {}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


def learned_info(mesh, args):
    import ctypes as C
    from simul_b200 import _lib
    st = (C.c_int64 * 4)()
    _lib.load().fem_learned_stats(mesh.ctx, st)
    return {"weights": os.path.relpath(args.weights, ROOT), "coarse_correction": bool(args.learned_coarse),
            "fallbacks_to_jacobi_pcg": int(st[0]), "fpcg_steps": int(st[2]),
            "steps_with_jacobi_direction": int(st[3]),
            "network": "4-layer message passing, width 64, BF16 tcgen05 dense layers, FP32 accumulation"}


def build_inputs(args):
    from simul_b200 import meshgen
    return meshgen.vertebral_body(n=args.n, seed=0)


def cpu_path(args, v, threads, steps=None, on_step=None):
    """The C++/OpenMP FP64 restatement of the plain method (Newton + Jacobi-PCG)
    over the load path from rest: load steps 1..``steps`` (default all), each
    to ``tol``, J2 history carried from step to step.  ``on_step(k, dt, info,
    solver)`` sees every step.  Returns the solver (its u after the last step)
    and the per-step (seconds, info)."""
    from oracle.cpu_solver import CpuSolver
    s = CpuSolver(v.X, v.conn, "j2", v.E, 0.3, sigma_y=100.0, H_ratio=0.02, threads=threads)
    out = []
    for k in range(1, (steps or args.load_steps) + 1):
        t = time.perf_counter()
        info = s.solve(v.fixed_mask, v.fixed_vals * (k / args.load_steps), v.f_ext, tol=args.tol)
        dt = time.perf_counter() - t
        out.append((dt, info))
        if on_step is not None:
            on_step(k, dt, info, s)
    return s, out


def reference_arm(args, rank, ws):
    """One bench step = one load step of the CPU restatement's load path, in
    order from rest (J2 history carried).  At least one full path is timed:
    with ``--steps`` below the number of load steps the whole path still
    runs (one full solve is the metric's unit); more steps start the path
    again.  ``value`` = the mean load-step time times the number of load
    steps, i.e. the measured time of a full path."""
    if rank != 0:
        return
    v = build_inputs(args)
    from oracle.cpu_solver import CpuSolver
    threads = args.cpu_threads or os.cpu_count() or 1
    # warm-up: the first load steps of a separate path (page-in, OpenMP start-up)
    warm = CpuSolver(v.X, v.conn, "j2", v.E, 0.3, sigma_y=100.0, H_ratio=0.02, threads=threads)
    for k in range(1, min(args.warmup, args.load_steps) + 1):
        warm.solve(v.fixed_mask, v.fixed_vals * (k / args.load_steps), v.f_ext, tol=args.tol)
    nthreads = warm.n_threads
    del warm
    times, newton, cg, conv = [], 0, 0, True
    s = None
    n_timed = max(args.steps, args.load_steps)
    for i in range(n_timed):
        k = i % args.load_steps + 1
        if k == 1:
            s = CpuSolver(v.X, v.conn, "j2", v.E, 0.3, sigma_y=100.0, H_ratio=0.02, threads=threads)
        t = time.perf_counter()
        info = s.solve(v.fixed_mask, v.fixed_vals * (k / args.load_steps), v.f_ext, tol=args.tol)
        times.append(time.perf_counter() - t)
        newton += info["iterations"]
        cg += info["cg_iterations"]
        conv &= info["converged"]
    per_step = float(np.mean(times))
    value = per_step * args.load_steps
    sample = (f"{n_timed} load steps timed one by one in path order from rest ({newton} Newton / {cg} CG "
              f"iterations, all converged: {conv}); value = their mean x {args.load_steps}"
              + (f", i.e. the measured time of the full {args.load_steps}-step path"
                 if n_timed % args.load_steps == 0 else " (the last path partial)"))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "load_steps_timed": n_timed, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
            "step": "one load step of the path (the metric's unit, one full solve, is load_steps of them)",
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded vertebral body)", "config": workload_config(args, v),
            "method": "Newton (FP64) + Jacobi-PCG (FP64), C++/OpenMP restatement",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_note": "the reference's Taichi ti.cpu path cannot run here (no taichi, Python 3.12 "
                              "vs >=3.13); this arm times oracle/cpu_fem.cpp, a C++/OpenMP restatement "
                              "of the plain method (the reference itself factorises an assembled tangent "
                              "with SuperLU, which does not finish at this size in minutes)"}
    print(json.dumps(line), flush=True)


def configure(mesh, args):
    """The timed method's solver options on a mesh."""
    mesh.set_coarse_options(cell=args.coarse_cell, reuse=args.coarse_reuse, bf16=bool(args.coarse_bf16),
                            inverse=args.coarse_inverse, max_nodes=args.coarse_max_nodes)
    if args.matvec_variant != "auto":
        mesh.set_matvec_variant(args.matvec_variant)
    mesh.set_fused_step(bool(args.fused_step))
    mesh.set_whole_solve_graph(bool(args.whole_solve_graph))
    mesh.set_programmatic_launch(bool(args.pdl))
    mesh.set_block_smoother(bool(args.block_smoother))
    mesh.set_extrapolation(bool(args.extrapolate))


def size_point(args, n, dev, jacobi=True):
    """The same workload at n voxels per axis: one warm-up and one timed full
    solve with the timed method, and (``jacobi``) the same with Jacobi-PCG."""
    import torch
    from simul_b200 import fem as B
    from simul_b200 import meshgen
    v = meshgen.vertebral_body(n=n, seed=0)
    mesh = B.FEMesh(v.n_nodes, v.n_elements, device=dev)
    mesh.initialize_from_numpy(v.X, v.conn)
    configure(mesh, args)
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    fixed_full = torch.from_numpy(v.fixed_vals).to(dev)
    fixed_mask = torch.from_numpy(v.fixed_mask.astype(np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    out = {"n": n, "tets": int(v.n_elements), "nodes": int(v.n_nodes)}
    for name, pc in [(args.precond, args.precond)] + ([("jacobi_pcg", "jacobi")] if jacobi else []):
        solver = B.StaticSolver(mesh, mat, tol=args.tol, precond=pc, cg_rtol_min=args.cg_rtol_min,
                                cg_rtol_max=args.cg_rtol_max)
        for rep in range(2):
            mesh.u.zero_()
            mat.reset_state()
            mesh.fixed.copy_(fixed_mask)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = {"newton": 0, "cg": 0, "conv": True, "rel": 0.0}
            for k in range(1, args.load_steps + 1):
                mesh.fixed_value.copy_(fixed_full * (k / args.load_steps))
                mesh._bc_dirty = True
                r = solver.solve(verbose=False)
                st["newton"] += r["iterations"]
                st["cg"] += r["cg_iterations"]
                st["conv"] &= r["converged"]
                st["rel"] = max(st["rel"], r["relative_residual"])
            e1.record(stream)
            e1.synchronize()
        out[name] = {"s": e0.elapsed_time(e1) / 1e3, "newton_iterations": st["newton"], "cg_iterations": st["cg"],
                     "all_converged": bool(st["conv"]), "max_relative_residual": st["rel"],
                     "timed_once_after_one_warmup": True}
        del solver
    if jacobi:
        out["speedup_vs_jacobi_pcg"] = out["jacobi_pcg"]["s"] / out[args.precond]["s"]
    del mesh
    torch.cuda.empty_cache()
    return out


def roofline_point(args, n, dev):
    """Tangent-matvec roofline at n voxels per axis (its working set beyond the
    126 MB L2): CUDA-event time per launch at a plastic state of the
    workload (fem_profile_kernels, 50 launches) against the algorithmic bytes."""
    import ctypes as C
    import torch
    from simul_b200 import _lib
    from simul_b200 import fem as B
    from simul_b200 import meshgen
    v = meshgen.vertebral_body(n=n, seed=0)
    mesh = B.FEMesh(v.n_nodes, v.n_elements, device=dev)
    mesh.initialize_from_numpy(v.X, v.conn)
    configure(mesh, args)
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    idx = np.where(v.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, (v.fixed_vals * 0.2).reshape(-1)[idx])
    u = np.zeros_like(v.X)
    u[:, 2] = -0.004 * v.X[:, 2]
    mesh.u.copy_(torch.from_numpy(u))
    mat.compute_nodal_forces(mesh)
    # the variant choice the solver makes (timed on a first PCG solve)
    rhs = torch.zeros(v.n_nodes, 3, dtype=torch.float64, device=dev)
    rhs[:, 2] = 1.0
    du = torch.zeros_like(rhs)
    it, rel = C.c_int32(), C.c_double()
    _lib.load().fem_pcg(mesh.ctx, _lib.FEM_PRECOND_JACOBI, B._ptr(rhs), B._ptr(du), 1e-2, 50, C.byref(it),
                        C.byref(rel))
    kms = (C.c_double * 4)()
    rc = _lib.load().fem_profile_kernels(mesh.ctx, 50, kms)
    peak, peak_src = measured_peaks()
    st = mesh.stats()
    b = matvec_bytes(v.n_elements, v.n_nodes)
    out = {"n": n, "tets": int(v.n_elements), "nodes": int(v.n_nodes), "variant": st["matvec_variant"],
           "matvec_ms": kms[0] if rc == 0 else None, "algorithmic_bytes": b}
    if rc == 0:
        ach = b / (kms[0] * 1e-3) / 1e9
        out.update({"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_source": peak_src,
                    "residual_ms": kms[1],
                    "residual_achieved": residual_bytes(v.n_elements, v.n_nodes) / (kms[1] * 1e-3) / 1e9})
    del mesh
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    rank, ws, local = world()
    if args.impl == "reference":
        if ws > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=timedelta(seconds=600))
        reference_arm(args, rank, ws)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    import ctypes as C

    from simul_b200 import _lib
    from simul_b200 import fem as B

    v = build_inputs(args)
    mesh = B.FEMesh(v.n_nodes, v.n_elements, device=local)
    mesh.initialize_from_numpy(v.X, v.conn)
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    solver = B.StaticSolver(mesh, mat, tol=args.tol, precond=args.precond, cg_rtol_min=args.cg_rtol_min,
                            cg_rtol_max=args.cg_rtol_max)
    configure(mesh, args)
    if args.precond == "learned":
        from simul_b200 import learned
        learned.set_weights(mesh, learned.load(args.weights))
        learned.set_coarse(mesh, bool(args.learned_coarse))
    fixed_full = torch.from_numpy(v.fixed_vals).to(dev)
    fixed_mask = torch.from_numpy(v.fixed_mask.astype(np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def solve_all(solver=solver):
        """One full solve from rest: all load steps, each to tol."""
        mesh.u.zero_()
        mat.reset_state()
        mesh.fixed.copy_(fixed_mask)
        stats = {"newton": 0, "cg": 0, "converged": True, "max_rel": 0.0}
        for k in range(1, args.load_steps + 1):
            mesh.fixed_value.copy_(fixed_full * (k / args.load_steps))
            mesh._bc_dirty = True
            r = solver.solve(verbose=False)
            stats["newton"] += r["iterations"]
            stats["cg"] += r["cg_iterations"]
            stats["converged"] &= r["converged"]
            stats["max_rel"] = max(stats["max_rel"], r["relative_residual"])
        return stats

    for _ in range(args.warmup):
        solve_all()
    torch.cuda.synchronize()

    props = torch.cuda.get_device_properties(dev)
    gid = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local)
    clocks = ClockSampler(gid)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = mesh.stats()["launches"]
    step_ms = []
    last = None
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        last = solve_all()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier()
    launches = mesh.stats()["launches"] - launches0
    clk = clocks.stop()
    ms = float(np.mean(step_ms))
    ms = max_over_ranks(ms, dev, ws)

    # end to end through the public API: per-solve inputs from pinned host memory
    h_fixed = torch.from_numpy(v.fixed_vals).pin_memory()
    h_mask = torch.from_numpy(v.fixed_mask.astype(np.int32)).pin_memory()
    h_fext = torch.from_numpy(v.f_ext).pin_memory()
    h_u = torch.empty(v.n_nodes, 3, dtype=torch.float64).pin_memory()
    d_fixed = torch.empty_like(fixed_full)
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_fixed.copy_(h_fixed, non_blocking=True)
        mesh.fixed.copy_(h_mask, non_blocking=True)
        mesh.f_ext.copy_(h_fext, non_blocking=True)
        mesh.u.zero_()
        mat.reset_state()
        for k in range(1, args.load_steps + 1):
            mesh.fixed_value.copy_(d_fixed * (k / args.load_steps))
            mesh._bc_dirty = True
            solver.solve(verbose=False)
        h_u.copy_(mesh.u, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    h2d = h_fixed.numel() * 8 + h_mask.numel() * 4 + h_fext.numel() * 8
    d2h = h_u.numel() * 8
    e2e_s = float(np.mean(e2e_ms)) / 1e3
    e2e_s = max_over_ranks(e2e_s, dev, ws)

    # the plain method timed beside the chosen one (same mesh, same clocks regime)
    jac = None
    if args.precond != "jacobi" and not args.no_jacobi_baseline:
        jsolver = B.StaticSolver(mesh, mat, tol=args.tol, precond="jacobi")
        solve_all(jsolver)
        torch.cuda.synchronize()
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        jl = solve_all(jsolver)
        e1.record(stream)
        e1.synchronize()
        jms = e0.elapsed_time(e1)
        jms = max_over_ranks(jms, dev, ws)
        jac = {"s": jms / 1e3, "newton_iterations": jl["newton"], "cg_iterations": jl["cg"],
               "all_converged": bool(jl["converged"]), "max_relative_residual": jl["max_rel"],
               "speedup_of_timed_method": jms / ms, "timed_once_after_one_warmup": True}
        del jsolver

    # learned flexible PCG timed beside it (held-out trained weights), when available
    lrn = None
    if args.precond != "learned" and not args.no_jacobi_baseline and os.path.exists(args.weights):
        from simul_b200 import learned as L
        L.set_weights(mesh, L.load(args.weights))
        L.set_coarse(mesh, bool(args.learned_coarse))
        lsolver = B.StaticSolver(mesh, mat, tol=args.tol, precond="learned")
        solve_all(lsolver)
        torch.cuda.synchronize()
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ll = solve_all(lsolver)
        e1.record(stream)
        e1.synchronize()
        lms = max_over_ranks(e0.elapsed_time(e1), dev, ws)
        lrn = {"s": lms / 1e3, "newton_iterations": ll["newton"], "cg_iterations": ll["cg"],
               "all_converged": bool(ll["converged"]), "max_relative_residual": ll["max_rel"],
               "vs_jacobi_pcg": (jac["s"] * 1e3 / lms) if jac else None, "timed_once_after_one_warmup": True,
               **learned_info(mesh, args)}
        del lsolver

    # roofline of the dominant kernel (tangent matvec), CUDA events on the solver stream
    kms = (C.c_double * 4)()
    rc = _lib.load().fem_profile_kernels(mesh.ctx, 200, kms)
    mv_ms = kms[0] if rc == 0 else None
    info = mesh.info()
    peak, peak_src = measured_peaks()
    b_mv = matvec_bytes(info["n_elements"], info["n_nodes"])
    achieved = b_mv / (mv_ms * 1e-3) / 1e9 if mv_ms else None
    st = mesh.stats()
    variant = st["matvec_variant"]
    traffic = load_traffic().get(f"matvec_{variant}_j2_n{args.n}")
    traffic_warm = load_traffic().get(f"matvec_{variant}_j2_n{args.n}_warm")
    line = {"metric": METRIC, "value": ms / 1e3, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "job_solves_per_s": ws / (ms / 1e3),
            "warmup": args.warmup, "ms_per_step": ms, "step_ms": [round(t, 3) for t in step_ms],
            "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 matvec / f64 residual+dots",
            "data": "synthetic (seeded vertebral body)", "config": workload_config(args, v),
            "method": {"learned": "Newton (FP64 residual) + learned flexible PCG (FP32 matvec, FP64 dots)",
                       "two_level": "Newton (FP64 residual) + two-level PCG: Jacobi + trilinear Galerkin "
                                    "coarse correction (FP32 matvec, FP64 dots)",
                       "jacobi": "Newton (FP64 residual) + Jacobi-PCG (FP32 matvec, FP64 dots)"}[args.precond],
            "learned_fpcg_s": (ms / 1e3) if args.precond == "learned" else (lrn["s"] if lrn else None),
            "learned": (learned_info(mesh, args) if args.precond == "learned" else lrn),
            "jacobi_pcg": jac,
            "coarse": ({**mesh.coarse_info(), "reuse": args.coarse_reuse, "inverse_dtype": "bf16" if args.coarse_bf16 else "f32"}
                       if args.precond in ("two_level", "learned") else None),
            "solve": {"newton_iterations": last["newton"], "cg_iterations": last["cg"],
                      "all_converged": bool(last["converged"]), "max_relative_residual": last["max_rel"],
                      "cg_ms_per_iteration": (ms / last["cg"]) if last["cg"] else None},
            "clocks": clk,
            "e2e": {"value": e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "step_ms": [round(t, 3) for t in e2e_ms]},
            "gpu_launches": int(launches // max(args.steps, 1)),
            "kernel_ms": {"matvec": kms[0], "residual": kms[1], "cg_update": kms[2], "cg_direction": kms[3]},
            "matvec_variant": {"chosen": variant, "ns_per_launch": st["matvec_ns"]},
            "fused_step": mesh.step_info(),
            "whole_solve_graphs": {"available": st["whole_solve_graph_available"],
                                   "pcg_solves_as_one_launch": st["whole_solve_graphs"]},
            "roofline": {"bound": "hbm", "kernel": {
                "fused": "matvec_kernel<J2> (fused node-block)",
                "two_phase": "elem_mv_kernel<J2> + node_gather_kernel (two-phase)",
                "element_block": "eb_matvec_kernel<J2> + eb_complete_kernel (element-block)",
                "warp_agg": "elem_wagg_kernel<J2> + node_gather_kernel (warp-aggregated two-phase)",
                "persistent": "elem_mv_persist_kernel<J2> + node_gather_persist_kernel (persistent two-phase)"}.get(variant, variant),
                         "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "frac_nominal_8tbs": (achieved / 8000.0) if achieved else None,
                         "peak_source": peak_src, "algorithmic_bytes": b_mv,
                         "traffic": traffic,
                         "traffic_note": "ncu cold-cache capture (caches flushed before each kernel)",
                         "traffic_warm": traffic_warm,
                         "residual_achieved": residual_bytes(info["n_elements"], info["n_nodes"]) / (kms[1] * 1e-3) / 1e9
                         if rc == 0 else None}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = args.cpu_threads or os.cpu_count() or 1
        # the timed method's displacement after the first and the last load step
        mesh.u.zero_()
        mat.reset_state()
        mesh.fixed.copy_(fixed_mask)
        u_gpu, rel_gpu = {}, {}
        for k in range(1, args.load_steps + 1):
            mesh.fixed_value.copy_(fixed_full * (k / args.load_steps))
            mesh._bc_dirty = True
            r = solver.solve(verbose=False)
            if k in (1, args.load_steps):
                u_gpu[k], rel_gpu[k] = mesh.get_displacements(), r["relative_residual"]
        # the CPU restatement over the same full path (one measured path: the
        # CPU baseline), compared with the GPU after steps 1 and load_steps
        u_cpu, rel_cpu = {}, {}

        def keep(k, dt, info, s):
            if k in (1, args.load_steps):
                u_cpu[k], rel_cpu[k] = s.u.copy(), info["relative_residual"]

        t0 = time.perf_counter()
        cs, steps = cpu_path(args, v, threads, on_step=keep)
        cpu_s = time.perf_counter() - t0
        acc = {}
        for k in sorted(u_gpu):
            acc[f"load_step_{k}"] = {
                "u_rel_l2": float(np.linalg.norm(u_gpu[k] - u_cpu[k]) / max(np.linalg.norm(u_cpu[k]), 1e-300)),
                "gpu_relative_residual": rel_gpu[k], "cpu_relative_residual": rel_cpu[k]}
        line["accuracy"] = {"reference": "oracle/cpu_fem.cpp: FP64 Newton + Jacobi-PCG over the same load path "
                                         "to the same tol", **acc}
        line["cpu_baseline"] = {"value": cpu_s, "unit": UNIT, "cores": cs.n_threads, "kind": "port",
                                "sample": f"the full {args.load_steps}-step path from rest, timed once "
                                          f"({sum(i['iterations'] for _, i in steps)} Newton / "
                                          f"{sum(i['cg_iterations'] for _, i in steps)} CG iterations, all "
                                          f"converged: {all(i['converged'] for _, i in steps)}); C++/OpenMP "
                                          f"FP64 restatement of the plain method (Newton + Jacobi-PCG), the "
                                          f"same code --impl reference times"}
    if rank == 0 and ws == 1 and not args.no_hex8:
        # the same body and loading with one HEX8 per voxel (the reference's
        # FEMAdapter / labelmap element), two-level PCG, one warm-up sequence
        try:
            from simul_b200 import hex8_bench
            h = hex8_bench.run(n=args.n, precond="two_level", load_steps=args.load_steps, tol=args.tol, warmup=1,
                               steps=1, device=str(dev))
            line["hex8"] = {"workload": f"vertebral body n={args.n} as HEX8 (one hexahedron per voxel), J2, "
                                        f"{args.load_steps} steps to {args.tol:g}",
                            "value": h["seconds"], "unit": UNIT, "hexes": h["hexes"], "nodes": h["nodes"],
                            "newton_iterations": h["newton"], "cg_iterations": h["cg"],
                            "all_converged": h["converged"]}
        except Exception as exc:  # reported, never fatal to the headline line
            line["hex8"] = {"error": repr(exc)}
    if rank == 0 and ws == 1 and not args.no_extras:
        # beside the headline, each reported, never fatal to it: the north
        # star's 1M-tet point, the matvec roofline beyond L2, batched solves
        for key, fn in (("vertebra_1m_tets", lambda: size_point(args, args.n_large, dev)),
                        ("roofline_large", lambda: roofline_point(args, args.n_roofline, dev))):
            try:
                line[key] = fn()
            except Exception as exc:
                line[key] = {"error": repr(exc)}
    if not args.no_extras:
        # batched uneven solves: the instances are sharded across the ranks
        # (every rank takes part; the per-instance results are gathered)
        from simul_b200 import batch_bench
        try:
            bres = batch_bench.run(instances=args.batch_instances, n_min=32, n_max=64, load_steps=10, seed=0,
                                   workers=8, device=str(dev), rank=rank, world=ws)
        except Exception as exc:  # reported, never fatal to the headline line
            bres = {"error": repr(exc)}
        if rank == 0 and "error" in bres:
            line["batch"] = bres
        elif rank == 0:
            line["batch"] = bres
            line["batch"]["note"] = ("the batched uneven-solves workload at reduced scale: instances with grid "
                                     "sizes 32-64 voxels per axis, 10 load steps, sharded across "
                                     f"{ws} rank(s) (the full 64-instance, 32-96 run: "
                                     "python -m simul_b200.batch_bench)")
    if rank == 0:
        print(json.dumps(line), flush=True)
    del solver, mesh
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
