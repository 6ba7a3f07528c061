"""Benchmark of the shape-gradient hot path (one JSON line on rank 0).

One step = one shape-gradient evaluation: freestream start, SSP-RK3 time
loop, lift/drag and J = -C_L + beta C_D, adjoint solve (BiCGSTAB to a true
relres <= 1e-8 or the workload's iteration cap), shape gradient dJ/d(m, p, t)
by the perturbed-residual pairs.
Default workload ("large"): NACA 0012, seeded O-grid of ~2.0M triangles
(first cell 1e-4 chord, growth 1.1), M = 0.85, AoA = 1.25 deg, FP64,
20,000 SSP-RK3 steps at CFL 0.3, then one 500-iteration BiCGSTAB restart
chunk with the reference's identity preconditioner: on this mesh and
impulsive-start state neither that solver (it diverges) nor the block-ILU(0)
one reaches 1e-8, so the evaluation does the reference's own fixed chunk of
work and the line reports the relres it reached.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl o2f|reference]

Under torchrun (N > 1) every rank evaluates a replica of the workload (weak scaling,
no data-path collective); the max over ranks of the device time is reported.
``--impl reference`` times the reference's own OpenMP CPU code (oracle/_ref)
on the same mesh on rank 0 and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "shape-gradient evals/s (state+adjoint) vs plain FP64 GPU at dJ rel err≤1e-4"
# Adjoint iteration cap per evaluation (one restart chunk of the reference's
# solver, src/shape_optimization.cpp:691) for the wall-refined workloads,
# where BiCGSTAB does not reach 1e-8; "small" converges (about 350-550
# iterations with block ILU(0)).  The reference arm extrapolates with the
# iteration count of the GPU path (the cap, or 350 for "small").
ADJOINT_CAP = {"large": 500, "mixed": 500, "small": 100000}
ADJOINT_ITERS = {"large": 500, "mixed": 500, "small": 350}


# DRAM bytes per launch of the dominant kernel from one ncu capture
# (k_cell_gradient on the 502,656-cell mesh: 131.1 MB read + written),
# scaled by cells to each workload; None where no capture applies.
TRAFFIC_PER_CELL = {"cell_gradient": 131.1e6 / 502656}


def naca_name(spec) -> str:
    """Four-digit NACA designation (p digit 0 for a symmetric section)."""
    m = int(round(spec.m * 100))
    p = int(round(spec.p * 10)) if m else 0
    return f"{m}{p}{int(round(spec.t * 100)):02d}"


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The largest of every rank's x (each rank times its own replica; the
    job takes as long as the slowest).  world == 1: x itself."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, evals_per_rank: int, seconds: float) -> float:
    """Whole-job evaluations per second: every rank evaluates its own
    candidate (weak scaling), timed by the slowest rank."""
    return world * evals_per_rank / seconds


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def workload(name: str):
    from optimisation2forme_b200 import SimulationParams
    from optimisation2forme_b200.meshgen import config_mesh, naca_ogrid
    spec, flow = config_mesh(name)
    mesh = naca_ogrid(spec)
    # CFL / diffusive time-step bound / preconditioner shift per workload: the
    # 1e-4-chord wall layers need the thermal dt bound and CFL <= 0.5 (0.3 on
    # the 2M-cell mesh) for the reference scheme to stay finite over 20k steps.
    # Adjoint: block ILU(0) where BiCGSTAB converges (the 20k-cell case); on
    # the wall-refined meshes no preconditioner reaches 1e-8, and the fixed
    # 500-iteration chunk runs the reference's identity-preconditioned solver.
    cfl, rk_steps, dt_mode, precond = {"small": (0.5, 2000, "reference", "ilu0"),
                                       "mixed": (0.5, 20000, "thermal", "none"),
                                       "large": (0.3, 20000, "thermal", "none")}[name]
    # Reference physics at the reference's own viscosity (mu = 1.8e-5): the
    # reference's viscous operator diverges at the configs' Reynolds numbers.
    params = SimulationParams(viscosity=1.8e-5, inflow_velocity=flow["mach"], aoa_deg=flow["aoa"], cfl_number=cfl,
                              final_time=1e30, limiter_k=5.0, adjoint_precond=precond, dt_mode=dt_mode,
                              verbosity=0)
    shape = dict(m=spec.m, p=spec.p, t=spec.t, pos_x=spec.pos_x, c=spec.chord)
    return spec, flow, mesh, params, shape, rk_steps


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        rows = [[x.strip() for x in line.split(",")] for line in self.path.read_text().splitlines()]
        rows = [r for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def kernel_bytes(nc, ne, nv, nnz) -> dict:
    """Algorithmic bytes per launch of each kernel class (FP64): the unique
    elements each kernel must read and write once (nc, ne, nv: cells, edges,
    vertices; nnz: vertex-cell pairs)."""
    return {
        "vertex_state": nv * (4 + 1 + 32) + nnz * (4 + 8) + nc * 32,
        "cell_gradient": nc * (16 + 32 + 32 + 32 + 8) + ne * (8 + 8 + 1 + 32 + 16 + 64) + nv * 32,
        "vertex_visc": nv * (4 + 1 + 40) + nnz * (4 + 8) + nc * 40,
        "edge_flux": ne * (32 + 64 + 8 + 1 + 32 + 40) + nv * 40,
        "cell_residual": nc * (16 + 32 + 32 + 32) + ne * (32 + 40 + 32),
        "jt_apply": nc * (16 + 32 + 32 + 32) + ne * (256 + 32 + 8 + 1),
        "jt_blocks": ne * (64 + 32 + 1 + 256),
    }


def residual_bytes(nc, ne, nv, nnz) -> int:
    """Compulsory bytes of one fully fused residual (w = g = 8 bytes):
    Nc(8w+3g) + Ne(16+5g) + Nv*4 + sum(valence)(4+g)."""
    w = g = 8
    return nc * (8 * w + 3 * g) + ne * (16 + 5 * g) + nv * 4 + nnz * (4 + g)


RESIDUAL_KERNELS = ("vertex_state", "cell_gradient", "vertex_visc", "edge_flux", "cell_residual")


def run_o2f(args, rank: int, world: int) -> dict | None:
    import torch
    from optimisation2forme_b200 import Solver, mesh_desc
    from optimisation2forme_b200._lib import ShapeParams

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    spec, flow, mesh, params, shape, rk_steps = workload(args.workload)
    if args.rk_steps is not None:
        rk_steps = args.rk_steps
    stream = torch.cuda.Stream()
    desc = mesh_desc(mesh["node_xy"], mesh["segments"], mesh["segment_bc"], mesh["cell_offsets"], mesh["cell_nodes"])
    s = Solver(params, desc=desc, stream=stream.cuda_stream)
    names = ["m", "p", "t"]
    sp = ShapeParams(shape["pos_x"], shape["c"], shape["m"], shape["p"], shape["t"])
    nnz = int(mesh["cell_offsets"][-1])  # sum of cell sizes == sum of vertex valences
    beta = 0.1
    last = {}

    cap = ADJOINT_CAP[args.workload]

    def adjoint_and_gradient():
        _, _, J = s.lift_drag(beta)
        a = s.solve_adjoint_system(beta, tol=args.adjoint_tol, max_iter=cap, restart=500, raise_on_failure=False)
        if a["status"] not in ("OK", "O2F_ERR_NOT_CONVERGED"):
            raise RuntimeError(f"adjoint solve failed: {a['status']}")
        g = s.compute_shape_gradient(names, sp, beta=beta, eps=1e-6)
        return {"J": J, "iters": a["iters"], "relres": a["relres"], "grad": g}

    def evaluation():
        s.initialize_freestream()
        s.time_loop(rk_steps)
        last.update(adjoint_and_gradient())

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        evaluation()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = s.timing()["kernel_launches"]
    with Clocks(dev) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            evaluation()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = s.timing()["kernel_launches"] - launches0
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = replica_throughput(world, args.steps, ms / 1e3)

    # End to end through the C ABI with host buffers: the initial state goes
    # host->device (pinned) each step, the final state and the gradient come back.
    e2e = None
    if not args.no_e2e:
        s.initialize_freestream()
        U0 = torch.from_numpy(s.get_state()).pin_memory().numpy()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            s.set_state(U0)
            s.time_loop(rk_steps)
            adjoint_and_gradient()
            Uf = s.get_state()
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0, world)
        e2e = {"value": replica_throughput(world, args.e2e_steps, dt), "unit": "evals/s", "h2d_bytes_per_step": int(U0.nbytes),
               "d2h_bytes_per_step": int(Uf.nbytes + 8 * s.n_cells * 4 + 8 * len(names) + 24)}

    # Per-kernel launch durations (CUDA events on the solver's stream) about
    # the state the timed evaluations left.
    prof = s.profile_kernels(20)
    kb = kernel_bytes(s.n_cells, s.n_edges, s.n_vertices, nnz)
    per_eval = {k: 3 * rk_steps + 7 for k in RESIDUAL_KERNELS}
    per_eval.update(jt_apply=2 * int(last.get("iters", 0)) + 2, jt_blocks=1)
    share = {k: prof[k] * per_eval[k] for k in per_eval}
    dom = max(share, key=share.get)
    peaks = load_peaks()
    achieved = kb[dom] / (prof[dom] / 1e3) / 1e9
    traffic = args.traffic
    if traffic is None and dom in TRAFFIC_PER_CELL:
        traffic = round(TRAFFIC_PER_CELL[dom] * s.n_cells)
    res_ms = sum(prof[k] for k in RESIDUAL_KERNELS)
    res_gbs = residual_bytes(s.n_cells, s.n_edges, s.n_vertices, nnz) / (res_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                "peak_source": peaks["source"], "bytes_per_launch": kb[dom], "launch_ms": round(prof[dom], 5),
                "residual": {"ms": round(res_ms, 4), "algorithmic_GBs": round(res_gbs, 1),
                             "frac": round(res_gbs / peaks["hbm_gbs"], 4)},
                "kernel_ms": {k: round(v, 5) for k, v in prof.items()}}
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded NACA O-grid, freestream start)",
        "config": {"workload": f"{args.workload}: NACA {naca_name(spec)} O-grid, {s.n_cells} triangles, "
                               f"M={flow['mach']:.3f}, "
                               f"AoA={flow['aoa']:.2f}, {rk_steps} SSP-RK3 steps, adjoint tol {args.adjoint_tol}, "
                               "dJ/d(m,p,t)",
                   "cells": s.n_cells, "edges": s.n_edges, "rk_steps": rk_steps, "cfl": params.cfl_number,
                   "dt_mode": params.dt_mode, "viscosity": params.viscosity,
                   "adjoint": f"BiCGSTAB, preconditioner {params.adjoint_precond}, cap {cap} iterations",
                   "adjoint_iters": last.get("iters"), "adjoint_relres": last.get("relres"), "J": last.get("J"),
                   "grad": [float(g) for g in last.get("grad", [])],
                   "l2": "inputs larger than L2 (working set > 126 MB)" if s.n_cells > 400000 else "working set fits L2",
                   "parallelism": f"replicas x{world}"},
        "roofline": roofline,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    if e2e:
        line["e2e"] = e2e
    s.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, mesh, rk_steps, int(last.get("iters", 0)))
    return line if rank == 0 else None


def batch_candidates(n: int = 16, seed: int = 0):
    """Seeded candidates of uneven size for the batched path: NACA (m, p, t)
    in [0, 0.06] x [0.2, 0.6] x [0.08, 0.18], M in [0.5, 0.8], AoA in [0, 4]
    deg, O-grids of about 25k-150k triangles (first cell 1e-3 chord)."""
    from optimisation2forme_b200 import SimulationParams
    from optimisation2forme_b200.meshgen import OGridSpec, naca_ogrid
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ns = int(rng.integers(100, 250)) * 2
        nl = int(rng.integers(60, 150))
        spec = OGridSpec(m=float(rng.uniform(0, 0.06)), p=float(rng.uniform(0.2, 0.6)), t=float(rng.uniform(0.08, 0.18)),
                         n_surface=ns, n_layers=nl, first_height=1e-3, growth=1.1, seed=seed + i)
        params = SimulationParams(viscosity=1.8e-5, inflow_velocity=float(rng.uniform(0.5, 0.8)),
                                  aoa_deg=float(rng.uniform(0, 4)), cfl_number=0.5, final_time=1e30, limiter_k=5.0,
                                  adjoint_precond="none", dt_mode="thermal", verbosity=0)
        out.append((spec, naca_ogrid(spec), params))
    return out


def run_batch(args) -> dict:
    """Candidates advanced by the batched time loop (one grouped launch per
    phase for all of them) vs the same candidates one context at a time; each
    evaluation = RK3 steps + a 100-iteration adjoint chunk + dJ/d(m,p,t)."""
    import torch
    from optimisation2forme_b200 import Batch, Solver, mesh_desc
    from optimisation2forme_b200._lib import ShapeParams
    torch.cuda.set_device(0)
    rk_steps = args.rk_steps or 2000
    cands = batch_candidates()
    ctxs = [Solver(p, desc=mesh_desc(m["node_xy"], m["segments"], m["segment_bc"], m["cell_offsets"],
                                    m["cell_nodes"])) for _, m, p in cands]
    cells = [c.n_cells for c in ctxs]
    shapes = [ShapeParams(sp.pos_x, sp.chord, sp.m, sp.p, sp.t) for sp, _, _ in cands]

    def adjoint_and_gradient():
        for s, sh in zip(ctxs, shapes):
            s.solve_adjoint_system(0.1, tol=1e-8, max_iter=100, restart=100, raise_on_failure=False)
            s.compute_shape_gradient(["m", "p", "t"], sh, beta=0.1)

    def batched(b):
        for s in ctxs:
            s.initialize_freestream()
        b.time_loop(rk_steps)
        adjoint_and_gradient()

    def sequential():
        for s in ctxs:
            s.initialize_freestream()
            s.time_loop(rk_steps, raise_on_failure=False)
        adjoint_and_gradient()

    b = Batch(ctxs)
    tuned = b.tune(reps=5)
    for s in ctxs:
        s.initialize_freestream()
    finite = sum(r["status"] == "OK" for r in b.time_loop(rk_steps))
    times = {}
    for name, fn in (("batched", lambda: batched(b)), ("sequential", sequential)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fn()
        torch.cuda.synchronize()
        times[name] = (time.perf_counter() - t0) / args.steps
    b.close()
    n = len(ctxs)
    return {"metric": "batched shape-gradient evals/s (uneven candidates)", "value": n / times["batched"],
            "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * times["batched"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded NACA O-grids)",
            "config": {"workload": f"batch: {n} candidates, {sum(cells)} triangles ({min(cells)}-{max(cells)} each), "
                                   f"{rk_steps} SSP-RK3 steps + 100 BiCGSTAB iterations + dJ/d(m,p,t)",
                       "candidates_finite": finite,
                       "sequential_evals_per_s": n / times["sequential"],
                       "batched_over_sequential": times["sequential"] / times["batched"],
                       "tuned": {k: list(v) for k, v in tuned.items()}}}


def reference_times(mesh: dict, reps: int, threads: int) -> dict:
    """Per-call times of the reference's own computeResidual and
    applyJacobianTranspose (oracle/_ref, OpenMP) on the workload mesh."""
    from oracle import ref
    if not ref.available():
        raise RuntimeError("reference build oracle/_ref is not present")
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        ref.write_binary_mesh(td / "mesh.bin", mesh)
        cfg = ref.write_config(td / "cfg.txt", mesh=str(td / "mesh.bin"), viscosity=1.8e-5, inflow_velocity=0.85)
        out = ref.run("bench", cfg, reps, exact=False, threads=threads, capture=True)["stdout"]
    return json.loads(out.strip().splitlines()[-1])


def eval_seconds(t_res: float, t_jt: float, rk_steps: int, adj_iters: int) -> float:
    """One evaluation of the reference's CPU path: 3 residuals per RK3 step,
    2 J^T products per BiCGSTAB iteration, 7 residuals for J and the gradient
    (RK update, dt reduction and vector updates not counted)."""
    return rk_steps * 3 * t_res + adj_iters * 2 * t_jt + 7 * t_res


def cpu_baseline(args, mesh, rk_steps, adj_iters) -> dict:
    threads = os.cpu_count() or 1
    t0 = time.time()
    r = reference_times(mesh, args.cpu_reps, threads)
    wall = time.time() - t0
    t_res, t_jt = statistics.median(r["residual_s"]), statistics.median(r["jt_s"])
    return {"value": 1.0 / eval_seconds(t_res, t_jt, rk_steps, adj_iters), "unit": "evals/s", "cores": r["threads"],
            "kind": "reference",
            "sample": f"reference computeResidual x{args.cpu_reps} and applyJacobianTranspose x{args.cpu_reps} on the "
                      f"same {r['cells']}-cell mesh (medians {t_res:.3f} s, {t_jt:.3f} s; {wall:.0f} s wall incl. "
                      f"mesh build); eval = {rk_steps}x3 residuals + {adj_iters}x2 J^T products + 7 residuals "
                      "(adjoint iterations of the GPU path)"}


def run_reference(args, rank: int, world: int) -> dict | None:
    if rank != 0:
        return None
    spec, flow, mesh, params, shape, rk_steps = workload(args.workload)
    if args.rk_steps is not None:
        rk_steps = args.rk_steps
    threads = os.cpu_count() or 1
    iters = ADJOINT_ITERS[args.workload]
    # One process builds the mesh once and times warmup+steps samples; the
    # first `warmup` samples are discarded.
    r = reference_times(mesh, args.warmup + args.steps, threads)
    vals = [1.0 / eval_seconds(a, b, rk_steps, iters)
            for a, b in zip(r["residual_s"][args.warmup:], r["jt_s"][args.warmup:])]
    v = statistics.median(vals)
    return {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded NACA O-grid)", "impl": "reference",
            "config": {"workload": f"{args.workload}: {r['cells']} triangles, {rk_steps} SSP-RK3 steps + adjoint "
                                   f"({iters} BiCGSTAB iterations) + dJ/d(m,p,t)",
                       "parallelism": f"OpenMP {r['threads']} threads"},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": r["threads"], "kind": "reference",
                             "sample": "per step: one reference computeResidual and one applyJacobianTranspose "
                                       "timed on the same mesh, extrapolated to one evaluation"},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="o2f", choices=["o2f", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "mixed", "small", "batch"])
    ap.add_argument("--rk-steps", type=int, default=None)
    ap.add_argument("--adjoint-tol", type=float, default=1e-8)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--traffic", type=float, default=None, help="ncu DRAM bytes per launch of the dominant kernel")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    use_pg = world > 1 and args.impl == "o2f"
    if use_pg:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800))
    try:
        if args.workload == "batch":
            line = run_batch(args) if rank == 0 and args.impl == "o2f" else None
        else:
            line = run_reference(args, rank, world) if args.impl == "reference" else run_o2f(args, rank, world)
    finally:
        if use_pg:
            import torch
            torch.distributed.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
