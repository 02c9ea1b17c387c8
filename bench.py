"""Benchmark of the B200 kinetic backend: one CIS iteration of the tube case per step.

Workload (the 3-D tube case, plain FP64 on the GPU): O-grid hex tube of radius 1 and length 5 with a downstream
reservoir, 134,528 cells; inlet p = 1, outlet p = 0.01, T = 1, diffuse walls; delta = 10, omega = 0.81; uniform
32^3 velocity grid on [-5, 5]^3 (the parity variant of the case's velocity grid); default strong CIS settings
(octant sweep order, 4 inner sweeps with wall refresh, 2 block passes, discrete equilibrium). Synthetic: the mesh
and the uniform initial state are generated here; f (35 GB in FP64) is far larger than L2, so no flush is needed.

A step = KineticSolver.sweep(): moments, cell parameters (discrete-equilibrium Newton), pressure-boundary inflow,
boundary sums, then 4 x (gradient, residual, 2 LU-SGS block passes) with wall refreshes.
metric = cell-velocity updates per second = n_cells * n_velocities * inner_sweeps / step time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32|mixed] [--impl b200|reference]
Under torchrun (N > 1) every rank runs an independent replica of the case on its own GPU (value = all ranks'
updates / the slowest rank's time); with --shard the ranks split one case's velocities instead (strong scaling).

The default line (one GPU) also carries, besides the FP64 figures and every kernel's roofline: the mixed-precision
leg on the same tube, the adjoint / forward ratio on the channel of the adjoint check (median of 3), the reference's
own CUDA backend rebuilt for sm_100a on the same tube and GPU, and the reference's CPU path on the host cores.
Other metrics: --time-to-mdot (solve time to M_dot within 1e-4 of the converged FP64 value, FP64 against mixed),
--adjoint (the channel adjoint with finite differences, --adjoint-fd), --tube-adjoint (the mixed-precision tube
adjoint at a per-face wall-temperature field, checked by FP64 directional differences).
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


# DRAM bytes (read + write) per (cell, velocity) per launch from ncu captures of the tube case at 62,848 cells x
# 12^3 velocities (profiles/gradient_residual_sweep_tiles_tube63k_12cube_fp64.md, FP64;
# profiles/residual_tube63k_12cube_mixed.md, mixed); the LU-SGS figure is that of the first block pass. Scaled by
# the units of a full launch for roofline.traffic.
# ncu DRAM bytes per (cell, velocity) of one launch on the 62,848-cell tube at 12^3 (the gradient_residual_sweep_tiles_*
# and sweep_tiles_moments_* summaries); the block passes: the mean of pass 1 and pass 2 (one launch each, with the
# stored diagonal)
DRAM_BYTES_PER_UNIT = {("fp64", "k_gradient"): 36.4, ("fp64", "k_residual"): 56.7, ("fp64", "k_sweep_tiles"): 66.65,
                       ("mixed", "k_gradient"): 16.8, ("mixed", "k_residual"): 23.7}
DRAM_SOURCE = "ncu DRAM bytes per cell-velocity of the 62,848-cell 12^3 capture, scaled to this launch"
# thread instructions per (cell, velocity) (smsp__inst_executed.sum x 32 / units) from the same captures: gradient,
# residual, first and second LU-SGS block pass of the tile kernel
INSTR_PER_UNIT = {"fp64": (697.0, 450.5, 440.6, 472.4), "mixed": (439.5, 443.8, 364.7, 373.3)}
B200_SMS = 148
ISSUE_PER_SM_CLOCK = 4 * 32  # 4 schedulers, one warp instruction (32 threads) each per cycle


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.file = None

    def __enter__(self):
        if self.dev < 0:
            return self
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": sorted(reasons)}


def max_over_ranks(values, ws, device="cuda"):
    """Element-wise maximum of per-rank timings over all ranks (every rank gets it); identity for one rank."""
    if ws <= 1:
        return [float(x) for x in values]
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x) for x in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0
    import datetime

    import torch.distributed as dist

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    import torch

    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, ws, local


def build_case(args):
    from gsis_sim_b200 import tube

    t0 = time.time()
    from gsis_sim_b200 import kinetic_setup as ks

    mesh_kw = None if args.nx == 100 else {"n_x": args.nx}
    grid = ks.VelocityGrid.clustered((args.nv,) * 3, 6.0, 2.0) if args.grid == "clustered" else None
    setup, host = tube.tube_case(delta=10.0, nv=args.nv, precision=args.precision, mesh_kw=mesh_kw, grid=grid)
    return setup, host, time.time() - t0


# the bounded same-grid sample of the reference's CPU path: the tube geometry (radius 1, length 5, reservoir) on a
# coarse O-grid (8 x 8 core, 5 + 6 rings, 4 tube layers, 1 reservoir layer: 1,312 cells) with the benchmark's
# velocity grid, so that one CIS iteration takes seconds on the host cores
COARSE_TUBE = dict(n_c=8, n_r=5, n_x=4, n_o=6, n_xr=1)


def cpu_baseline(args, steps=None, warmup=1, nv=None, coarse=True):
    """The reference's own CPU kinetic path (oracle/_ref/libgsisref.so: KineticSolver + OpenMP CpuBackend) timed on a
    bounded sample: the benchmark's velocity grid on the coarse tube mesh (coarse=True), or the benchmark mesh with a
    reduced velocity grid (coarse=False). Falls back to the C port of oracle/ where the library is absent."""
    from gsis_sim_b200 import tube

    nv_s = nv or args.nv
    cores = os.cpu_count() or 1
    mesh = tube.tube_mesh(**(COARSE_TUBE if coarse else {}))
    steps = args.cpu_steps if steps is None else max(1, steps)
    what = ("coarse tube mesh (same geometry, 8x8 core, 4 tube + 1 reservoir layers)" if coarse else
            "benchmark tube mesh")
    sample = f"{what}: {mesh.n_cells:,} cells x {nv_s}^3 velocities, {steps} CIS iteration(s), {args.precision}"
    prec = args.precision if args.precision != "mixed" else "fp32"
    try:
        from oracle import ref

        if not ref.available():
            raise FileNotFoundError("oracle/_ref/libgsisref.so not built")
        rm = ref.RefMesh.from_arrays(mesh.as_dict())
        case = ref.RefCase(rm, ref.tube_spec(nv_s, prec))
        case.init_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
        for _ in range(max(1, warmup)):
            case.sweep()
        fails = []
        t0 = time.perf_counter()
        for _ in range(steps):
            case.sweep()
            fails.append(int(case.backend.deq_counts()[1]))
        dt = (time.perf_counter() - t0) / steps
        kind = "reference"
        inner = case.inner_sweeps
        nc = case.setup.n_cells
    except (FileNotFoundError, OSError) as e:
        from oracle.kinetic_oracle import OracleBackend
        from gsis_sim_b200.solver import KineticSolver

        setup, host = tube.tube_case(delta=10.0, nv=nv_s, precision=prec,
                                     mesh_kw=COARSE_TUBE if coarse else None)
        be = OracleBackend(setup)
        sol = KineticSolver(setup, host, be)
        sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
        for _ in range(max(1, warmup)):
            sol.sweep()
        fails = []
        t0 = time.perf_counter()
        for _ in range(steps):
            sol.sweep()
            fails.append(int(be.deq_counts()[1]))
        dt = (time.perf_counter() - t0) / steps
        kind = "port"
        inner = host.inner_sweeps
        nc = setup.n_cells
        sample += f" (reference library unavailable: {e})"
    if any(fails):
        sample += (f"; the discrete equilibrium failed in up to {max(fails)} cells per iteration on this grid "
                   f"(collisionless fallback there)")
    value = nc * nv_s ** 3 * inner / dt
    return {"value": value, "unit": "cell*velocity updates/s", "cores": cores, "kind": kind, "sample": sample,
            "seconds_per_iteration": dt}


def run_reference_arm(args, rank):
    if rank != 0:
        return
    cb = cpu_baseline(args, steps=args.steps, warmup=args.warmup)
    line = {"impl": "reference", "metric": "cell_velocity_updates_per_s", "value": cb["value"],
            "unit": cb["unit"], "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * cb["seconds_per_iteration"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32", "mixed": "f32"}[args.precision],
            "data": "synthetic", "config": workload_config(args),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args, cb_nv=None, n_cells=134528):
    grid = (f"uniform {args.nv}^3 velocities on [-5,5]^3" if getattr(args, "grid", "uniform") == "uniform" else
            f"clustered (sinh, stretch 2) {args.nv}^3 velocities on [-6,6]^3 with quadrature weights")
    return {"workload": f"kinetic CIS iteration, O-grid tube + reservoir {n_cells} cells, {grid}, delta 10, "
                        f"{args.precision}",
            "cells": n_cells, "velocities": (cb_nv or args.nv) ** 3, "inner_sweeps": 4, "block_passes": 2,
            "sweep_order": "octant", "equilibrium": "discrete",
            "l2": "no flush: f and the work arrays (tens of GB) exceed the 126 MB L2"}


def mdot_of_last_prepare(sol):
    """M_dot of the state the last CIS iteration started from (the patch sums of its prepare step; the same formula as
    KineticSolver.mass_flow without an extra prepare)."""
    import math

    from gsis_sim_b200.solver import T_MASS_FLOW_INLET, T_PRESSURE_INLET, T_PRESSURE_OUTLET, T_VACUUM

    pm = sol.info.patch_mass_flow
    mdot_in = -sum(pm[p] for p in range(len(pm)) if sol.ptype[p] in (T_PRESSURE_INLET, T_MASS_FLOW_INLET))
    mdot_out = sum(pm[p] for p in range(len(pm)) if sol.ptype[p] in (T_PRESSURE_OUTLET, T_VACUUM))
    return 0.5 * (mdot_in + mdot_out) * math.sqrt(2.0 / math.pi)


def settle_time(hist, ref, tol):
    """Wall time of the first iteration after which every recorded M_dot stays within tol of ref (None if never)."""
    t = None
    for (tw, m, _) in hist:
        if abs(m - ref) <= tol * abs(ref):
            if t is None:
                t = tw
        else:
            t = None
    return t


def run_time_to_mdot(args, local):
    """Solve time to M_dot within --mdot-tol of the converged FP64 M_dot, FP64 against mixed precision, plain CIS
    iterations through the public host loop (wall clock, host logic included). The FP64 run continues until M_dot
    changes by less than 1e-8 (relative) per iteration over 5 iterations, or --max-iters; its last M_dot is the
    reference. Each iteration's M_dot is that of the state it started from (the patch sums of its prepare step)."""
    import numpy as np
    import torch

    from gsis_sim_b200.backend import B200Backend
    from gsis_sim_b200.solver import KineticSolver

    torch.cuda.set_device(local)
    out = {}
    ref = args.mdot_fp64
    precisions = ("mixed",) if ref is not None else ("fp64", "mixed")
    for prec in precisions:
        args.precision = prec
        setup, host, _ = build_case(args)
        n_cells = setup.n_cells
        with B200Backend(setup, device=local) as be:
            sol = KineticSolver(setup, host, be)
            sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
            hist = []
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for it in range(args.max_iters):
                info = sol.sweep()
                hist.append((time.perf_counter() - t0, mdot_of_last_prepare(sol), info.residual))
                if prec == "fp64" and len(hist) > 6:
                    ch = [abs(hist[-k][1] - hist[-k - 1][1]) / abs(hist[-1][1]) for k in range(1, 6)]
                    if max(ch) < 1e-8:
                        break
                if prec == "mixed" and ref is not None and len(hist) > 10:
                    # stop once M_dot has stayed within a hundredth of the tolerance for 10 iterations
                    if all(abs(h[1] - ref) <= 0.01 * args.mdot_tol * abs(ref) for h in hist[-10:]):
                        break
        if prec == "fp64":
            ref = hist[-1][1]
        out[prec] = hist
        if args.history:
            np.savetxt(f"{args.history}_{prec}.txt", np.array(hist), header="wall_s mdot residual")
    t64 = settle_time(out["fp64"], ref, args.mdot_tol) if "fp64" in out else args.fp64_seconds
    tmx = settle_time(out["mixed"], ref, args.mdot_tol)
    line = {"metric": f"solve time to M_dot within {args.mdot_tol:g} of the converged FP64 M_dot (mixed)",
            "value": tmx, "unit": "s", "higher_is_better": False, "fp64_seconds": t64,
            "speedup_mixed_vs_fp64": (t64 / tmx) if (t64 and tmx) else None, "mdot_fp64_converged": ref,
            "mdot_mixed_final": out["mixed"][-1][1],
            "mdot_mixed_rel_error": abs(out["mixed"][-1][1] - ref) / abs(ref),
            "iterations": {k: len(v) for k, v in out.items()},
            "fp64_from": "this run" if "fp64" in out else "--mdot-fp64 / --fp64-seconds of an earlier FP64 run",
            "seconds_per_iteration": {k: out[k][-1][0] / len(out[k]) for k in out},
            "final_residual": {k: out[k][-1][2] for k in out},
            "data": "synthetic", "config": workload_config(args, n_cells=n_cells)}
    line["config"]["workload"] = line["config"]["workload"].replace(", mixed", "")
    print(json.dumps(line), flush=True)


# the adjoint's discretisation choices: the reference's defaults (discrete equilibrium, "limited" pressure-boundary
# reconstruction) or the simpler continuous equilibrium with the owner cell's state at pressure faces
ADJ_SCHEMES = {"default": dict(equilibrium="discrete", pressure_boundary_reconstruction="limited"),
               "continuous-cell": dict(equilibrium="continuous", pressure_boundary_reconstruction="cell")}


def channel_case(delta=5.0, Tw=1.0, nv=24, n=(64, 32, 1), alpha=1.0, scheme="default"):
    """Pressure-driven channel: box n[0] x n[1] x 1 on x in [0, 4], y in [0, 1], one cell thick with periodic sides;
    inlet p 1, outlet p 0.5, T 1; walls at T_w with accommodation alpha (diffuse at 1); nv^3 uniform velocities on
    [-5, 5]^3; FP64; the equilibrium and pressure-boundary reconstruction of ADJ_SCHEMES[scheme]."""
    from gsis_sim_b200 import kinetic_setup as ks
    from gsis_sim_b200.mesh import box_mesh

    m = box_mesh(n, (0.0, 0.0, 0.0), (4.0, 1.0, 1.0 / n[1]), ("inlet", "outlet", "wall", "wall", "side", "side"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "pressure_outlet", p=0.5),
           ks.BC("wall", "diffuse_wall", T=Tw, alpha=alpha), ks.BC("side", "periodic_slab")]
    kp = ks.KineticParams(precision="fp64", **ADJ_SCHEMES[scheme])
    return ks.build_kinetic_setup(m, ks.Gas(omega=0.81), ks.Conditions(L_ref=1.0, T0=273.15, delta_rp=delta), bcs,
                                  ks.VelocityGrid(n=(nv, nv, nv)), kp)


def converge_channel(setup, host, local, tol, max_iters):
    """Plain CIS from rest to a residual below tol; returns (solver, wall seconds, iterations)."""
    import torch

    from gsis_sim_b200.backend import B200Backend
    from gsis_sim_b200.solver import KineticSolver

    be = B200Backend(setup, device=local)
    sol = KineticSolver(setup, host, be)
    sol.initialize_uniform(0.75, (0.0, 0.0, 0.0), 1.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    it = 0
    for it in range(1, max_iters + 1):
        if sol.sweep().residual < tol:
            break
    sol.prepare()
    torch.cuda.synchronize()
    return sol, time.perf_counter() - t0, it


def wall_temperature_field(prob, seed=2026, sigma=0.02):
    """Seeded N(1, sigma^2) temperature per diffuse wall face (the order of prob.wall_faces)."""
    import numpy as np

    return 1.0 + sigma * np.random.default_rng(seed).standard_normal(len(prob.wall_faces))


def tube_adjoint(args, local):
    """dM_dot/dT_w per wall face on the tube (delta 10, --nv^3 velocities, the reference's discrete equilibrium,
    "cell" pressure-boundary reconstruction) at a seeded N(1, 0.02^2) wall-temperature field, by the mixed-precision
    adjoint: the mixed forward solve to --fwd-tol and the mixed adjoint solve to --adj-tol, timed through the public
    host loops (wall clock). The gradient is checked against central differences of FP64 forward solves along
    --fd-directions seeded random unit directions of the per-face field, on the coarse tube of the same geometry
    (--fd-mesh coarse: 1,312 cells; a full-size FP64 solve takes minutes, 16 of them hours) or on the same mesh."""
    import numpy as np
    import torch

    from gsis_sim_b200 import tube
    from gsis_sim_b200.adjoint import KineticAdjoint, MassFlowProblem

    torch.cuda.set_device(local)

    def case(precision, mesh_kw):
        return tube.tube_case(delta=10.0, nv=args.nv, precision=precision, pressure_boundary_reconstruction="cell",
                              mesh_kw=mesh_kw)

    def mixed_gradient(mesh_kw, timed):
        setup, host = case("mixed", mesh_kw)
        prob = MassFlowProblem(setup, host, tol=args.fwd_tol, max_iterations=args.max_iters, device=local,
                               stall_iterations=args.stall, polish_iterations=args.polish)
        Tw = wall_temperature_field(prob)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol, J = prob.solve(prob.delta0, Tw)
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        it_fwd = sol.iteration
        r_fwd = prob.last_residual
        # FP64 defect correction of the mixed state (MassFlowProblem.polish_state), counted with the adjoint
        t0 = time.perf_counter()
        sol = prob.polish_state(sol, prob.delta0)
        torch.cuda.synchronize()
        t_pol = time.perf_counter() - t0
        t0 = time.perf_counter()
        ka = KineticAdjoint(sol)
        res = ka.solve(tol=args.adj_tol, max_iterations=args.adj_max_iters, stall_iterations=args.stall)
        torch.cuda.synchronize()
        t_adj = time.perf_counter() - t0 + t_pol
        ka.close()
        prob.release(sol)
        out = {"cells": setup.n_cells, "velocities": setup.nv, "wall_faces": len(prob.wall_faces), "M_dot": J,
               "forward_seconds": t_fwd, "forward_iterations": it_fwd, "forward_residual": r_fwd,
               "polish_seconds": t_pol, "polish_residuals": prob.last_polish, "adjoint_seconds": t_adj,
               "adjoint_iterations": res.iterations, "adjoint_residual": res.residual,
               "ratio": t_adj / t_fwd}
        return out, res.dJ_dTw[prob.wall_faces].copy(), Tw, setup, host

    if args.adj_mesh == "coarse":
        mk_full = dict(COARSE_TUBE)
    else:
        mk_full = None if args.nx == 100 else {"n_x": args.nx}
    main_run, g_main, _, _, _ = mixed_gradient(mk_full, True)
    line = {"metric": "adjoint / forward wall-time ratio, mixed precision, dM_dot/dT_w per wall face",
            "value": main_run["ratio"], "unit": "x", "higher_is_better": False, "dtype": DTYPES["mixed"],
            "data": "synthetic", "run": main_run,
            "dM_dot_dT_w": {"sum": float(g_main.sum()), "max_abs": float(np.abs(g_main).max())},
            "config": {"workload": f"kinetic CIS, O-grid tube + reservoir {main_run['cells']} cells, inlet p 1 / "
                                   f"outlet p 0.01, diffuse walls at T_w ~ N(1, 0.02^2) per face (seed 2026), "
                                   f"delta 10, {args.nv}^3 velocities on [-5,5]^3, discrete equilibrium",
                       "forward_tol": args.fwd_tol, "adjoint_tol": args.adj_tol}}
    if args.fd_mesh != "none":
        mk = dict(COARSE_TUBE) if args.fd_mesh == "coarse" else mk_full
        if args.fd_mesh == "coarse" and args.adj_mesh != "coarse":
            fd_run, g, Tw, _, _ = mixed_gradient(mk, False)
        else:
            fd_run, g, Tw = main_run, g_main, None
        s64, h64 = case("fp64", mk)
        prob = MassFlowProblem(s64, h64, tol=1e-12, max_iterations=max(args.max_iters, 4000), device=local)
        if Tw is None:
            Tw = wall_temperature_field(prob)
        # the FP64 adjoint at the FP64 fixed point on the same mesh and field
        t0 = time.perf_counter()
        sol, _ = prob.solve(prob.delta0, Tw)
        ka = KineticAdjoint(sol)
        r64 = ka.solve(tol=1e-10, max_iterations=max(args.adj_max_iters, 4000))
        ka.close()
        prob.release(sol)
        g64 = r64.dJ_dTw[prob.wall_faces]
        line["fp64_adjoint"] = {"max_rel_difference": float(np.abs(g - g64).max() / np.abs(g64).max()),
                                "sum_rel_difference": float(abs(g.sum() - g64.sum()) / abs(g64.sum())),
                                "iterations": r64.iterations, "residual": r64.residual,
                                "seconds": time.perf_counter() - t0}
        rng = np.random.default_rng(7)
        h = args.fd_tw_step
        dirs = []
        t0 = time.perf_counter()
        for _ in range(args.fd_directions):
            v = rng.standard_normal(len(prob.wall_faces))
            v /= np.linalg.norm(v)
            Js = []
            for sgn in (1.0, -1.0):
                sol, Jv = prob.solve(prob.delta0, Tw + sgn * h * v)
                prob.release(sol)
                Js.append(Jv)
            fd = (Js[0] - Js[1]) / (2 * h)
            ad = float(g @ v)
            ad64 = float(g64 @ v)
            dirs.append({"adjoint": ad, "fd": fd, "rel_error": abs(ad - fd) / abs(fd),
                         "fp64_adjoint": ad64, "fp64_rel_error": abs(ad64 - fd) / abs(fd)})
        line["fd_check"] = {"mesh": "coarse tube (same geometry), 1,312 cells" if mk == COARSE_TUBE
                            else "the tube above", "run": fd_run, "step": h, "directions": dirs,
                            "max_rel_error": max(d["rel_error"] for d in dirs),
                            "max_rel_error_fp64_adjoint": max(d["fp64_rel_error"] for d in dirs),
                            "max_error_over_gradient_norm": max(abs(d["adjoint"] - d["fd"]) for d in dirs) /
                            float(np.linalg.norm(g)),
                            "fd_seconds": time.perf_counter() - t0,
                            "fd_solver": "FP64 forward, residual 1e-12, central differences"}
    return line


def run_adjoint(args, local):
    print(json.dumps(adjoint_ratio(args, local)), flush=True)


def adjoint_ratio(args, local):
    """Adjoint / forward wall-time ratio on the channel (or, --adjoint-case tube, on the tube mesh): the forward CIS
    solve from rest to residual --fwd-tol, then
    the adjoint solve of dM_dot/d(delta, T_w) to --adj-tol (both through the public host loops, wall clock). With
    --adjoint-fd also finite differences of the forward solver: central in delta (step --fd-step relative) and, on the
    channel, central in a uniform wall temperature (step --fd-step) and second-order one-sided from below in a
    uniform accommodation (alpha = 1 - h, 1 - 2h, h = 1e-4; Maxwell-wall solves)."""
    import numpy as np
    import torch

    from gsis_sim_b200.adjoint import KineticAdjoint

    torch.cuda.set_device(local)
    if args.adjoint_case == "tube":
        from gsis_sim_b200 import tube

        delta = 10.0

        def make(d):
            return tube.tube_case(delta=d, nv=args.adj_nv, precision="fp64", **ADJ_SCHEMES[args.adj_scheme])

        workload = (f"kinetic CIS, O-grid tube + reservoir 134528 cells, inlet p 1 / outlet p 0.01, diffuse walls, "
                    f"{args.adj_nv}^3 velocities on [-5,5]^3, delta 10, {args.adj_scheme} scheme")
    else:
        delta = 5.0

        def make(d, Tw=1.0, alpha=1.0):
            return channel_case(delta=d, nv=args.adj_nv, Tw=Tw, alpha=alpha, scheme=args.adj_scheme)

        workload = (f"kinetic CIS, channel 64x32x1 cells x in [0,4], inlet p 1 / outlet p 0.5, diffuse walls, "
                    f"{args.adj_nv}^3 velocities on [-5,5]^3, delta 5, {args.adj_scheme} scheme")
    setup, host = make(delta)
    sol, t_fwd, it_fwd = converge_channel(setup, host, local, args.fwd_tol, args.max_iters)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ka = KineticAdjoint(sol)
    hist = []
    res = ka.solve(tol=args.adj_tol, max_iterations=args.max_iters, inner=args.adj_inner,
                   callback=lambda it, r: hist.append(r))
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t0
    mu0 = float(setup["mu0"])
    dJ_ddelta = res.dJ_ddelta(mu0, delta)
    ka.close()
    sol.backend.close()
    line = {"metric": "adjoint / forward wall-time ratio (dM_dot / d(delta, T_w per wall face, alpha at 1))",
            "value": t_adj / t_fwd, "unit": "x", "higher_is_better": False,
            "forward_seconds": t_fwd, "forward_iterations": it_fwd, "adjoint_seconds": t_adj,
            "adjoint_iterations": res.iterations,
            "adjoint_inner_sweeps": int(args.adj_inner or host.inner_sweeps),
            "adjoint_residual": res.residual,
            "adjoint_residual_history": [hist[i] for i in range(0, len(hist), max(1, len(hist) // 20))],
            "M_dot": res.J, "dM_dot_d_alpha": float(np.nansum(res.dJ_dalpha)),
            "dM_dot_d_delta": dJ_ddelta, "dM_dot_dT_w_sum": float(np.sum(res.dJ_dTw)),
            "dM_dot_dT_w_max_abs": float(np.max(np.abs(res.dJ_dTw))),
            "n_wall_faces": int(np.count_nonzero(res.dJ_dTw)), "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload, "cells": setup.n_cells, "velocities": setup.nv,
                       "forward_tol": args.fwd_tol, "adjoint_tol": args.adj_tol,
                       "scheme": dict(ADJ_SCHEMES[args.adj_scheme])}}
    if args.adjoint_fd:
        h = args.fd_step

        def mdot(*a, **kw):
            sp, hp = make(*a, **kw)
            sp_sol = converge_channel(sp, hp, local, args.fwd_tol, args.max_iters)[0]
            J = sp_sol.mass_flow()[2]
            sp_sol.backend.close()
            return J

        fd = (mdot(delta * (1 + h)) - mdot(delta * (1 - h))) / (2 * h * delta)
        line["fd_step"] = h
        line["dM_dot_d_delta_fd"] = fd
        line["fd_rel_error"] = abs(dJ_ddelta - fd) / abs(fd)
        if args.adjoint_case == "channel":
            fd_T = (mdot(delta, Tw=1 + h) - mdot(delta, Tw=1 - h)) / (2 * h)
            line["dM_dot_dT_w_sum_fd"] = fd_T
            line["fd_T_w_rel_error"] = abs(line["dM_dot_dT_w_sum"] - fd_T) / abs(fd_T)
            ha = 1e-4
            fd_a = (3 * res.J - 4 * mdot(delta, alpha=1 - ha) + mdot(delta, alpha=1 - 2 * ha)) / (2 * ha)
            line["dM_dot_d_alpha_fd"] = fd_a
            line["fd_alpha_rel_error"] = abs(line["dM_dot_d_alpha"] - fd_a) / abs(fd_a)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "mixed"])
    ap.add_argument("--nv", type=int, default=32)
    ap.add_argument("--grid", default="uniform", choices=["uniform", "clustered"],
                    help="uniform nv^3 on [-5,5]^3 (the parity grid) or sinh-clustered nv^3 on [-6,6]^3 with weights")
    ap.add_argument("--cpu-nv", type=int, default=8)
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision, adjoint and reference-GPU legs of the default line")
    # smaller variants of the tube case for profiler captures (the benchmark itself uses the defaults)
    ap.add_argument("--nx", type=int, default=100, help="axial cells of the tube (100: 134,528 cells)")
    ap.add_argument("--velocity-chunk", type=int, default=None, help="velocities per chunk (default: all that fit)")
    # second headline metric: solve time to M_dot within a tolerance of the converged FP64 M_dot, mixed vs FP64
    ap.add_argument("--shard", action="store_true",
                    help="split the case's velocities over the ranks (strong scaling) instead of one replica per rank")
    ap.add_argument("--time-to-mdot", action="store_true")
    ap.add_argument("--mdot-tol", type=float, default=1e-4)
    ap.add_argument("--mdot-fp64", type=float, default=None,
                    help="--time-to-mdot: the converged FP64 M_dot of an earlier run (then only the mixed solve runs)")
    ap.add_argument("--fp64-seconds", type=float, default=None,
                    help="--time-to-mdot with --mdot-fp64: that run's FP64 time to the tolerance")
    ap.add_argument("--max-iters", type=int, default=2000)
    ap.add_argument("--history", default=None, help="write per-iteration (wall s, M_dot, residual) to <prefix>_<prec>.txt")
    # third headline metric: adjoint / forward wall-time ratio on the channel
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--adjoint-fd", action="store_true",
                    help="with --adjoint: also finite differences in delta and, on the channel, wall T and alpha")
    ap.add_argument("--fd-step", type=float, default=1e-6, help="relative step of the central differences")
    ap.add_argument("--adj-nv", type=int, default=24)
    ap.add_argument("--adjoint-case", default="channel", choices=["channel", "tube"])
    ap.add_argument("--adj-scheme", default="default", choices=sorted(ADJ_SCHEMES),
                    help="equilibrium and pressure-boundary reconstruction of the adjoint legs (default: the "
                         "reference's defaults, discrete equilibrium and limited reconstruction)")
    ap.add_argument("--adj-inner", type=int, default=None, help="adjoint sweeps per coupling update (default: the "
                    "set-up's inner_sweeps, as the forward)")
    ap.add_argument("--fwd-tol", type=float, default=1e-10)
    ap.add_argument("--adj-tol", type=float, default=1e-10)
    # the tube adjoint in mixed precision (per-wall-face temperature gradient)
    ap.add_argument("--tube-adjoint", action="store_true",
                    help="mixed-precision adjoint of the tube with a seeded N(1, 0.02^2) wall-temperature field: "
                    "adjoint / forward time on the tube (--nx, --nv), directional FP64 differences on the coarse tube")
    ap.add_argument("--fd-directions", type=int, default=8)
    ap.add_argument("--adj-mesh", default="full", choices=["full", "coarse"],
                    help="mesh of the timed tube adjoint: the benchmark tube (--nx) or the 1,312-cell coarse tube")
    ap.add_argument("--adj-max-iters", type=int, default=2000, help="outer iterations of the adjoint solve at most")
    ap.add_argument("--polish", type=int, default=20,
                    help="--tube-adjoint: FP64 CIS iterations from the converged mixed state before the adjoint")
    ap.add_argument("--stall", type=int, default=None,
                    help="--tube-adjoint: stop the mixed solves at their FP32 floor (no 1%% progress in this many "
                    "iterations)")
    ap.add_argument("--fd-mesh", default="coarse", choices=["coarse", "same", "none"])
    ap.add_argument("--fd-tw-step", type=float, default=1e-5, help="step of the directional wall-temperature differences")
    args = ap.parse_args()

    rank, ws, local = dist_init() if args.gpus > 1 or int(os.environ.get("WORLD_SIZE", "1")) > 1 else (0, 1, 0)
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.time_to_mdot:
        if rank == 0:
            run_time_to_mdot(args, local)
        return
    if args.adjoint:
        if rank == 0:
            run_adjoint(args, local)
        return
    if args.tube_adjoint:
        if rank == 0:
            print(json.dumps(tube_adjoint(args, local)), flush=True)
        return

    import torch

    torch.cuda.set_device(local)
    run = time_iterations(args, args.precision, ws, rank, local)
    nc, nv, inner = run["n_cells"], run["nv"], run["inner"]
    jobs = 1 if args.shard else ws  # sharded: one case over all ranks; replicas: one case per rank
    updates = float(nc) * nv * inner * args.steps
    value = updates * jobs / run["device_s"]
    e2e = updates * jobs / run["wall_s"]
    hbm, peak_kind = peaks()
    kern = kernel_rooflines(run, args.precision, args.steps, hbm)
    dom = max(kern, key=lambda k: kern[k]["seconds_per_step"])
    d = kern[dom]
    line = {
        "metric": "cell_velocity_updates_per_s", "value": value, "unit": "cell*velocity updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * run["wall_s"] / args.steps,
        "higher_is_better": True, "scaling": "strong" if args.shard else "weak", "vs_baseline": None,
        "dtype": DTYPES[args.precision], "data": "synthetic",
        "config": dict(workload_config(args, n_cells=nc),
                       parallelism=(f"velocity shards x{ws}" if args.shard else f"replicas x{ws}")),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": d["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                     "frac": d["achieved_gbs"] / hbm, "peak_source": peak_kind, "traffic": d["traffic"],
                     "traffic_source": d["traffic_source"],
                     "algorithmic_bytes_per_launch": d["bytes_per_launch"], "avg_launch_ms": d["avg_launch_ms"],
                     "kernels": kern,
                     "step": step_fraction(run, args.precision, args.steps, hbm)},
        "e2e": {"value": e2e, "unit": "cell*velocity updates/s", "h2d_bytes_per_step": run["h2d"],
                "d2h_bytes_per_step": run["d2h"]},
        "gpu_launches": run["launches"], "clocks": run["clocks"],
        "phase_seconds_per_step": {k: v / args.steps for k, v in run["timings"].items()},
        "mass_flow": run["mass_flow"], "setup_seconds": run["setup_s"],
    }
    if ws == 1 and rank == 0 and not args.no_extras:
        # the other parts of the headline metric on the same box: mixed precision on the same tube, the adjoint /
        # forward ratio, and the reference's own CUDA backend rebuilt for sm_100a
        line["mixed"] = mixed_leg(args, local, hbm)
        line["adjoint"] = adjoint_leg(args, local)
        line["gpu_baseline"] = gpu_baseline(args, run)
    if rank == 0 and not args.no_cpu_baseline:
        # same velocity grid on the coarse tube (the headline CPU rate), and the benchmark mesh on an 8^3 grid
        line["cpu_baseline"] = cpu_baseline(args)
        line["cpu_baseline"].pop("seconds_per_iteration", None)
        full = cpu_baseline(args, nv=args.cpu_nv, coarse=False)
        full.pop("seconds_per_iteration", None)
        line["cpu_baseline"]["benchmark_mesh_sample"] = full
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


DTYPES = {"fp64": "f64", "fp32": "f32", "mixed": "f32 (f, gradient, LU-SGS) / f64 (residual, sums)"}


def time_iterations(args, precision, ws=1, rank=0, local=0, steps=None, warmup=None, clocks=True):
    """K CIS iterations of the tube case through the public host loop (host buffers, H2D/D2H inside the timed region),
    after W untimed ones; device time from the backend's CUDA events, wall time max over ranks."""
    import torch

    from gsis_sim_b200.backend import B200Backend
    from gsis_sim_b200.solver import KineticSolver

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    prev = args.precision
    args.precision = precision
    setup, host, t_setup = build_case(args)
    args.precision = prev
    nc, nv = setup.n_cells, setup.nv
    inner = host.inner_sweeps
    if args.shard and ws > 1:
        # one velocity shard of the case per rank; moments, boundary sums and residuals all-reduced (NCCL)
        from gsis_sim_b200 import shard

        ranges = shard.shard_ranges(setup, ws)
        local_be = B200Backend(shard.shard_setup(setup, *ranges[rank]), device=local,
                               velocity_chunk=args.velocity_chunk)
        be = shard.ShardedBackend(setup, [local_be], [ranges[rank]], shard.torch_allreduce(device="cuda"),
                                  device=True, device_allreduce=shard.torch_device_allreduce())
    else:
        be = B200Backend(setup, device=local, velocity_chunk=args.velocity_chunk)
    sol = KineticSolver(setup, host, be)
    sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    for _ in range(warmup):
        sol.sweep()
    be.take_timings()
    launches0 = be.launch_count()

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local if clocks else -1) as clk:
        t0 = time.perf_counter()
        for _ in range(steps):
            sol.sweep()
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t0
    barrier()
    timings = be.take_timings()
    launches = be.launch_count() - launches0
    device_busy = sum(timings.values())
    # per-step host<->device traffic of the host loop (moments, deq flags, inflow tables, boundary sums, residuals,
    # discrete-Maxwellian inflow states)
    nb = setup.n_bfaces
    n_pres = len(sol.pres_faces)
    per_prepare_d2h = 15 * nc * 8 + nc * 4 + 20 * nb * 8 + n_pres * (5 * 8 + 4)
    per_prepare_h2d = 2 * nb * 6 * 8 + n_pres * 5 * 8
    bytes_d2h = per_prepare_d2h + inner * nc * 8 + (inner - 1) * 20 * nb * 8
    bytes_h2d = per_prepare_h2d + (inner - 1) * nb * 6 * 8
    t_wall, device_busy = max_over_ranks([t_wall, device_busy], ws)
    out = {"n_cells": nc, "nv": nv, "inner": inner, "passes": int(setup["block_passes"]), "device_s": device_busy,
           "wall_s": t_wall, "timings": timings, "launches": launches, "clocks": clk.summary() if clocks else None,
           "h2d": bytes_h2d, "d2h": bytes_d2h, "mass_flow": sol.mass_flow()[2], "setup_s": t_setup,
           "lout_bytes_per_unit": lout_bytes_per_unit(setup, 8 if precision == "fp64" else 4)}
    be.close()
    return out


def lout_bytes_per_unit(setup, s):
    """Algorithmic bytes of the out-of-block coupling kernel per (cell, velocity) of the mesh: for every cell with a
    neighbour in another RCB block, read R and write R + Lout (2 s), and read Delta f of each such neighbour (s)."""
    import numpy as np

    off = np.asarray(setup["csr_offsets"], np.int64)
    other = np.asarray(setup["csr_other"], np.int64)
    bo = np.asarray(setup["block_offsets"], np.int64)
    nc = len(off) - 1
    block = np.searchsorted(bo, np.arange(nc), side="right") - 1
    owner = np.repeat(np.arange(nc), np.diff(off))
    out = (other >= 0) & (block[np.maximum(other, 0)] != block[owner])
    n_entries = int(out.sum())
    n_cells = int(len(np.unique(owner[out])))
    return (2 * n_cells + n_entries) * s / nc


def sweep_kernel_bytes(s, passes):
    """The LU-SGS block-pass kernel the backend runs (KIN_SWEEP_KERNEL) and its algorithmic bytes per launch and
    (cell, velocity), averaged over the passes of one inner sweep."""
    sel = os.environ.get("KIN_SWEEP_KERNEL", "")
    if sel.startswith("resident"):
        # resident block pass: read R and write Delta f (2 s); the last pass reads R and reads and writes f (3 s);
        # the out-of-block coupling of a later pass is the separate k_lout
        return ("k_sweep_resident", (2 * s * (passes - 1) + 3 * s) / passes,
                "read R, write Delta f; last pass read R, read + write f")
    name = "k_sweep_pass" if sel == "legacy" else "k_sweep_tiles"
    # first pass: read R, write Delta f (2 s); a middle pass also reads the previous pass (3 s); the last pass reads
    # R and the previous pass and reads and writes f (4 s); a single pass reads R and reads and writes f (3 s)
    if passes == 1:
        return name, 3 * s, "read R, read + write f"
    return (name, (2 * s + 3 * s * (passes - 2) + 4 * s) / passes,
            "read R (+ previous pass), write Delta f; last pass read R + previous pass, read + write f")


def kernel_rooflines(run, precision, steps, hbm):
    """Per kernel: device seconds per step, launches, algorithmic bytes per launch (per (cell, velocity) figure x the
    cells x velocities a launch processes) over its average launch time, against the measured HBM peak."""
    s = 8 if precision == "fp64" else 4
    units = float(run["n_cells"]) * run["nv"]
    inner, passes = run["inner"], run["passes"]
    t = run["timings"]
    n_sweeps = inner * steps
    kern = {}
    # gradient: read f, write the three components (4 s)
    kern["k_gradient"] = (t["gradient"], n_sweeps, 4 * s, "read f, write g_x, g_y, g_z")
    # residual: read f, g_x, g_y, g_z, write R (5 s); the mixed defect scheme (KIN_MIXED_RESIDUAL=defect): first
    # sweep FP64 residual (5 s) + defect store (read f, g, R; write the defect: 6 s), further sweeps FP32 residual +
    # defect (read f, g, defect; write R: 6 s)
    if precision == "mixed" and os.environ.get("KIN_MIXED_RESIDUAL", "") == "defect":
        kern["k_residual"] = (t["residual"], n_sweeps, (11 * s + 6 * s * (inner - 1)) / inner,
                              "mixed defect scheme: per inner sweep on average")
    else:
        kern["k_residual"] = (t["residual"], n_sweeps, 5 * s, "read f, g_x, g_y, g_z, write R")
    name, b_pass, what = sweep_kernel_bytes(s, passes)
    kern[name] = (t["sweep_forward"], n_sweeps * passes, b_pass, what)
    if t.get("sweep_backward", 0.0) > 0.0:
        # coupling of a later pass: read R and write R + Lout for the surface cells, read Delta f of their
        # out-of-block neighbours (per (cell, velocity) of the whole mesh: the surface share)
        share = run.get("lout_bytes_per_unit")
        kern["k_lout"] = (t["sweep_backward"], n_sweeps * (passes - 1), share if share else 3 * s,
                          "read R + out-of-block Delta f, write R + Lout (surface cells)")
    out = {}
    for k, (sec, launches, b_unit, what) in kern.items():
        if launches <= 0 or sec <= 0:
            continue
        t_launch = sec / launches
        b_launch = b_unit * units
        per_unit = DRAM_BYTES_PER_UNIT.get((precision, k))
        out[k] = {"seconds_per_step": sec / steps, "launches_per_step": launches / steps,
                  "avg_launch_ms": 1e3 * t_launch, "bytes_per_unit": b_unit, "bytes_per_launch": b_launch,
                  "achieved_gbs": b_launch / t_launch / 1e9, "frac": b_launch / t_launch / 1e9 / hbm,
                  "algorithmic_bytes": what,
                  "traffic": per_unit * units if per_unit is not None else None,
                  "traffic_source": (DRAM_SOURCE if per_unit is not None else None)}
    return out


def step_fraction(run, precision, steps, hbm):
    """The whole CIS iteration against the path's algorithmic bytes: per inner sweep and (cell, velocity)
    3 s_F + 2 s_W, plus 3 s_W per further block pass, plus s_F for the moments per iteration."""
    s = 8 if precision == "fp64" else 4
    units = float(run["n_cells"]) * run["nv"]
    per_unit = run["inner"] * (3 * s + 2 * s + 3 * s * (run["passes"] - 1)) + s
    t_step = run["device_s"] / steps
    achieved = per_unit * units / t_step / 1e9
    out = {"bytes_per_unit_per_iteration": per_unit, "seconds_per_iteration": t_step, "achieved": achieved,
           "frac": achieved / hbm}
    instr = INSTR_PER_UNIT.get(precision)
    if instr is not None and run["passes"] == 2 and not os.environ.get("KIN_SWEEP_KERNEL"):
        # the issue-rate bound: the sweeps at one instruction per scheduler per cycle, the other phases as measured
        t = run["timings"]
        sweep_phases = sum(t.get(k, 0.0) for k in ("gradient", "residual", "sweep_forward", "sweep_backward"))
        other = max(0.0, (run["device_s"] - sweep_phases) / steps)
        rate = B200_SMS * ISSUE_PER_SM_CLOCK * sm_max_mhz() * 1e6
        t_min = run["inner"] * sum(instr) * units / rate + other
        bound = per_unit * units / t_min / 1e9 / hbm
        out["issue_bound"] = {"thread_instructions_per_unit_per_inner_sweep": sum(instr),
                              "issue_rate_per_s": rate, "min_seconds_per_iteration": t_min, "max_frac": bound,
                              "frac_of_bound": out["frac"] / bound,
                              "source": "ncu instruction counts of the 62,848-cell 12^3 capture"}
    return out


def sm_max_mhz():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f).get("sm_max_mhz", 1965.0))
    return 1965.0


def mixed_leg(args, local, hbm):
    """Mixed precision on the same tube and grid: updates/s (device and wall) and seconds per CIS iteration."""
    steps = max(3, min(args.steps, 5))
    run = time_iterations(args, "mixed", local=local, steps=steps, warmup=max(3, min(args.warmup, 3)),
                          clocks=False)
    updates = float(run["n_cells"]) * run["nv"] * run["inner"] * steps
    return {"value": updates / run["device_s"], "e2e": updates / run["wall_s"], "unit": "cell*velocity updates/s",
            "seconds_per_iteration": run["device_s"] / steps, "wall_seconds_per_iteration": run["wall_s"] / steps,
            "steps": steps, "phase_seconds_per_step": {k: v / steps for k, v in run["timings"].items()},
            "kernels": kernel_rooflines(run, "mixed", steps, hbm), "step": step_fraction(run, "mixed", steps, hbm),
            "mass_flow": run["mass_flow"]}


def adjoint_leg(args, local, repeats=3):
    """Adjoint / forward wall-time ratio on the channel of the adjoint check (median of repeats)."""
    ratios, fwd, adj = [], [], []
    for _ in range(repeats):
        r = adjoint_ratio(args, local)
        ratios.append(r["value"])
        fwd.append(r["forward_seconds"])
        adj.append(r["adjoint_seconds"])
    return {"value": statistics.median(ratios), "unit": "x", "repeats": ratios, "forward_seconds": fwd,
            "adjoint_seconds": adj, "workload": r["config"]["workload"], "bound": "<= 2 (north star)",
            "gradients": {k: r[k] for k in ("dM_dot_d_delta", "dM_dot_dT_w_sum", "dM_dot_d_alpha")}}


def gpu_baseline(args, run):
    """The reference's own CudaBackend (src/kinetic/kinetic_backend_cuda.cpp, kinetic_cuda_kernels.cu) rebuilt
    unchanged for sm_100a (oracle/Makefile target refcuda) under the reference KineticSolver, on the same tube, grid
    and precision, on the same GPU after this repository's backend is released: one warm-up and one timed CIS
    iteration, with the reference's per-phase device times."""
    try:
        from oracle import ref
        from gsis_sim_b200 import tube

        if not (ref.available() and ref.available(refcuda=True)):
            return {"unavailable": "oracle/_ref/libgsisrefcuda.so not built"}
        prec = args.precision if args.precision != "mixed" else "fp32"
        rm = ref.RefMesh.from_arrays(tube.tube_mesh().as_dict())
        case = ref.RefCase(rm, ref.tube_spec(args.nv, prec), refcuda=True)
        case.init_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
        case.sweep()
        t0 = time.perf_counter()
        case.sweep()
        dt = time.perf_counter() - t0
        ph = case.last_timings()
        nc, inner = case.setup.n_cells, case.inner_sweeps
        del case
        ours = {k: v / args.steps for k, v in run["timings"].items()}
        # the reference times its forward and backward sweep kernels apart; here one kernel runs both (the
        # coupling kernel of the resident variant is the backward slot), so the sweep is compared as a whole
        def merged(d):
            m = {k: v for k, v in d.items() if k not in ("sweep_forward", "sweep_backward")}
            m["sweep"] = d.get("sweep_forward", 0.0) + d.get("sweep_backward", 0.0)
            return m

        ph_m, ours_m = merged(ph), merged(ours)
        out = {"kind": "reference CudaBackend rebuilt for sm_100a", "value": nc * args.nv ** 3 * inner / dt,
               "unit": "cell*velocity updates/s", "seconds_per_iteration": dt, "phase_seconds": ph,
               "speedup_per_phase": {k: (ph_m[k] / ours_m[k]) if ours_m.get(k) else None for k in ph_m},
               "speedup_iteration": dt / (run["wall_s"] / args.steps)}
        return out
    except Exception as e:  # the baseline is reported, not required
        return {"unavailable": f"{type(e).__name__}: {e}"}


if __name__ == "__main__":
    main()
