"""Benchmark: steady SIMPLE outer iterations on the 1M-cell polyhedral cube cavity.

Workload (the reference's 3D polyhedral cavity configuration): unit cube,
100^3 = 1,000,000 Voronoi cells of a jittered lattice (jitter 0.3h, seed
20261007, ~13.8 faces per cell), lid u = 1 on plus_y, other walls no-slip,
rho = 1, mu = 1e-3, linearUpwind convection, least-squares gradients, corrected
diffusion, 2 non-orthogonal correctors, relaxation U 0.7 / p 0.3, momentum
BiCGStab + Jacobi and pressure CG + AMG, both to rtol 1e-10.  A step is one
SIMPLE outer iteration (the unit of cell-iters/s); the first outer iterations
are warm-up.  Synthetic mesh and initial state (fields at rest); the working
set (~1.5 GB of geometry, matrices and fields) is far larger than L2, so no
L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--cells 1000000]

Under torchrun (N > 1) every rank solves its own copy of the case (independent
requests: replicas, weak scaling); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-iters/s (steady SIMPLE outer iterations, 1M-cell polyhedral cube cavity)"
SEED = 20261007


def case_settings():
    return dict(rho=1.0, mu=1e-3, alpha_u=0.7, alpha_p=0.3, non_orthogonal_corrections=2,
                interpolation="linear", gradient="leastSquares", convection="linearUpwind", diffusion="corrected",
                rtol=1e-10, atol=1e-14)


def simple_config(n_side: int, world: int) -> dict:
    """The cavity workload's `config`, shared by both arms so their lines name the same case."""
    s = case_settings()
    return {"workload": f"steady SIMPLE, {n_side ** 3}-cell jittered-Voronoi cube cavity (n={n_side}^3)",
            "cells": n_side ** 3, "nu": s["mu"], "lid": 1.0, "convection": s["convection"],
            "gradient": s["gradient"], "diffusion": s["diffusion"],
            "non_orthogonal_corrections": s["non_orthogonal_corrections"], "solver_rtol": s["rtol"],
            "momentum": "bcgs+jacobi", "pressure": "cg+amg", "precision": "fp64",
            "l2": "working set >> 126 MB L2, no flush", "parallelism": f"replicas x{world}"}


def mesh_for(n: int):
    """Generate (or reuse from /tmp) the jittered-Voronoi cube of n^3 cells."""
    from babelsim_b200 import meshgen
    path = os.path.join(tempfile.gettempdir(), f"bsg_voronoi_{n}_{SEED}.npz")
    if os.path.exists(path):
        d = np.load(path)
        return meshgen.PolyMesh(d["vertices"], None, d["owner"], d["neighbour"], d["patch"],
                                ["minus_x", "plus_x", "minus_y", "plus_y", "minus_z", "plus_z"], ["wall"] * 6,
                                offsets=d["offsets"], ids=d["ids"])
    pm = meshgen.voronoi_cube(n, 0.3, SEED)
    np.savez(path, vertices=pm.vertices, owner=pm.owner, neighbour=pm.neighbour, patch=pm.patch,
             offsets=pm.offsets, ids=pm.ids)
    return pm


def build_simple(bsg, mesh, s, precision=0, boundaries=True, momentum_precision=0):
    opts = bsg.options(s["interpolation"], s["gradient"], s["convection"], s["diffusion"])
    sim = bsg.Simple(mesh, s["rho"], s["mu"], s["alpha_u"], s["alpha_p"], s["non_orthogonal_corrections"],
                     1e-8, 1e-7, 1e-6, 1e-6, opts, opts,
                     bsg.solver_config("bcgs", "bjacobi", s["atol"], s["rtol"], 1000, precision=momentum_precision),
                     bsg.solver_config("cg", "hypre", s["atol"], s["rtol"], 1000, precision=precision))
    if not boundaries:  # the caller sets boundaries (and segments) before the fields
        return sim
    for patch in range(6):
        sim.set_boundary("U", patch, "fixedValue", (1.0, 0.0, 0.0) if patch == 3 else (0.0, 0.0, 0.0))
        sim.set_boundary("p", patch, "zeroGradient")
    n = mesh.n_cells
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    return sim


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region (entering
    waits, at most 3 s, for the first sample, so sampling is already running when timing starts)."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.start = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
            return self
        deadline = time.time() + 3.0
        while not self.rows and time.time() < deadline and self.proc.poll() is None:
            time.sleep(0.02)
        self.start = len(self.rows)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = self.rows[self.start:] or self.rows  # samples taken after timing started
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(name, N, nnz_off, amg_rows):
    """Bytes each instrumented kernel must move (each array counted once; FP64 8 B, int32 4 B)."""
    matrix = 8 * N + 4 * (N + 1) + 12 * nnz_off          # diag, row pointers, values + columns
    if name == "cg_spmv_dot":
        return matrix + 8 * N + 8 * N                     # read p, write q
    if name == "bicgstab3_spmv_dot":
        return matrix + 24 * N * 3                        # read x(3), write y(3), read r0(3) for the dot
    if name == "cg_update_norm":
        return 8 * N * 6                                  # x, r, p, q read; x, r write
    if name == "amg_pre_smooth_restrict_l0":
        # x = w b / d; x' = x + w (b - A x) / d; coarse b = sum over aggregate of (b - A x')
        return (8 * 3 * N) + (matrix + 8 * 5 * N) + (matrix + 8 * 2 * N + 4 * N + 4 * amg_rows + 8 * amg_rows)
    if name == "amg_prolong_post_smooth_l0":
        return (matrix + 8 * 4 * N + 4 * N + 8 * amg_rows) + (matrix + 8 * 4 * N)
    return None


# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte,
# measured by one ncu capture of the kernel: kPcgSell, first pressure solve of the
# 512000-cell Voronoi cavity of the same generator and settings (30 CG iterations),
# 15.58 GB of DRAM traffic for 17.10 GB of algorithmic bytes.  Both grow with cells
# and CG iterations in proportion, so the ratio scales the 1M-cell launches.
DRAM_PER_ALGORITHMIC_BYTE = {"pcg_amg_persistent": 0.911}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Side of the Voronoi cube the CPU runs: a bounded sample of the 1M-cell workload
# (same generator, seed, physics and solver controls, 48^3 = 110592 cells) that the
# reference's sources finish in about half a minute on one core.
CPU_SAMPLE_SIDE = 48


def cpu_baseline(seconds_budget=25.0, iterations=4, n=CPU_SAMPLE_SIDE):
    """The reference's own sources (oracle/_ref) on a bounded sample of the workload, 1 core:
    `iterations` outer iterations of the n^3-cell Voronoi cube, the first one excluded."""
    exe = os.path.join(ROOT, "oracle", "_ref", "babelsim-oracle")
    if not os.path.exists(exe):
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import write_case  # noqa: E402  (case writer shared with the fixture generator)
    from babelsim_b200 import meshgen
    s = case_settings()
    pm = meshgen.voronoi_cube(n, 0.3, SEED)
    work = tempfile.mkdtemp(prefix="bsg_cpu_baseline_")
    U = [("fixedValue", (1.0, 0.0, 0.0) if p == 3 else (0.0, 0.0, 0.0)) for p in range(6)]
    P = [("zeroGradient", 0.0)] * 6
    methods = {"momentum": dict(interpolation="linear", gradient=s["gradient"], convection=s["convection"],
                                diffusion=s["diffusion"])}
    methods["pressureCorrection"] = dict(methods["momentum"])
    sol = {"maxIterations": iterations, "velocityRelaxation": s["alpha_u"], "pressureRelaxation": s["alpha_p"],
           "nonOrthogonalCorrections": s["non_orthogonal_corrections"], "continuityTolerance": 1e-8,
           "velocityTolerance": 1e-7, "momentumTolerance": 1e-6, "pressureCorrectionTolerance": 1e-6,
           "equation.momentum.kspType": "bcgs", "equation.momentum.pcType": "bjacobi",
           "equation.momentum.absoluteTolerance": s["atol"], "equation.momentum.relativeTolerance": s["rtol"],
           "equation.momentum.maxIterations": 1000, "equation.pressureCorrection.kspType": "cg",
           "equation.pressureCorrection.pcType": "hypre", "equation.pressureCorrection.absoluteTolerance": s["atol"],
           "equation.pressureCorrection.relativeTolerance": s["rtol"],
           "equation.pressureCorrection.maxIterations": 20000}
    write_case(work, pm, U, P, methods, sol, {"density": s["rho"], "dynamicViscosity": s["mu"]})
    out = os.path.join(work, "out")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    res = subprocess.run([exe, work, out], env=env, capture_output=True, text=True,
                         timeout=max(60.0, 10 * seconds_budget))
    if not os.path.exists(os.path.join(out, "run.json")):
        raise RuntimeError(f"reference run failed (exit {res.returncode}): {res.stderr[-300:]}")
    info = json.load(open(os.path.join(out, "run.json")))
    intervals = max(int(info["reported_iteration_intervals"]), 1)
    secs = float(info["iteration_compute_seconds"]) or float(info["solver_seconds"])
    value = pm.n_cells * intervals / secs
    return {"value": value, "unit": "cell-iters/s", "cores": 1, "kind": "reference", "cells": pm.n_cells,
            "sample": f"reference finite-volume sources (runSimple, operators, procedural equations) with a CPU "
                      f"stand-in for the PETSc/Hypre backend (CG + aggregation AMG and BiCGStab + ILU(0), "
                      f"preconditioners lagged per equation as PetscLinearSystem lags them), {pm.n_cells}-cell "
                      f"Voronoi cube (same generator and settings as the device workload), {iterations} outer "
                      f"iterations, first excluded, exit {res.returncode}",
            "linear_solve_seconds": info.get("linear_solve_seconds"), "krylov_iterations": info.get("krylov_iterations"),
            "preconditioner_setups": info.get("preconditioner_setups")}


# Phase ids of the persistent pressure solver's timeline (bsg_context_phase_log).
PHASE_NAMES = {1: "initial residual", 2: "CG product + p.q", 3: "x, r update + norm (+ level-0 residual)",
               4: "level-0 post sweep + r.z", 50: "coarsest solve"}


def pressure_phases(ctx, sim, iterations=2):
    """Device time between the persistent pressure solver's grid barriers over `iterations` more
    outer iterations (device %globaltimer), per CG iteration and phase."""
    ctx.phase_log(1 << 20)
    sim.iterate(iterations)
    ctx.synchronize()
    ent = ctx.phase_log_read()
    ctx.phase_log(0)
    acc, cg = {}, 0
    for k in range(1, len(ent)):
        pid = int(ent[k, 0])
        if pid == 1:
            continue  # the gap before a launch's first barrier includes the host's work between solves
        cg += pid == 2
        acc[pid] = acc.get(pid, 0.0) + (ent[k, 1] - ent[k - 1, 1]) / 1e3
    cg = max(cg, 1)

    def name(pid):
        if pid in PHASE_NAMES:
            return PHASE_NAMES[pid]
        kind = {1: "pre-smooth", 3: "residual", 6: "first post sweep", 8: "post sweep + prolong"}.get(pid // 10, None)
        if pid >= 100:
            return f"restrict {pid - 100}->{pid - 99}"
        return f"level {pid % 10} {kind}" if kind else str(pid)
    out = {name(p): round(v / cg, 2) for p, v in sorted(acc.items())}
    out["total"] = round(sum(acc.values()) / cg, 2)
    out["cg_iterations"] = cg
    return out


def device_on_sample(bsg, ctx, s, warmup, steps=5):
    """The device path on the CPU baseline's own sample (the same mesh and settings), so the
    two throughputs can be compared case for case as well as per cell."""
    mesh = bsg.Mesh.from_polyhedral(ctx, mesh_for(CPU_SAMPLE_SIDE))
    sim = build_simple(bsg, mesh, s)
    sim.iterate(max(warmup, 3))
    ctx.synchronize()
    ctx.record(6)
    sim.iterate(steps)
    ctx.record(7)
    ms = ctx.elapsed_ms(6, 7)
    out = {"cells": mesh.n_cells, "value": mesh.n_cells * steps / (ms / 1e3), "unit": "cell-iters/s",
           "ms_per_step": ms / steps, "steps": steps}
    sim.close()
    mesh.close()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # the bounded sample: --steps timed outer iterations (at most 5, so the run stays within a
    # few minutes) after one excluded first iteration
    timed = max(1, min(args.steps, 5))
    cb = cpu_baseline(iterations=timed + 1)
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/babelsim-oracle was not built here"}))
        return
    config = simple_config(CPU_SAMPLE_SIDE, args.gpus)
    config["parallelism"] = "1 process, 1 core (the reference is MPI-parallel; no MPI on this host)"
    config["sample_of"] = (f"the {max(2, round(args.cells ** (1.0 / 3.0))) ** 3}-cell device workload: same "
                           f"generator, seed, physics and solver controls, fewer cells; cell-iters/s is per cell")
    line = {"metric": METRIC, "value": cb["value"], "unit": cb["unit"], "n_gpus": args.gpus, "steps": timed,
            "warmup": 1, "ms_per_step": cb["cells"] / cb["value"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_serving(args):
    """Serving workload: a seeded Poisson stream of steady SIMPLE cavity requests (hex and
    jittered-Voronoi cubes, cells log-uniform, lid speed uniform 0.5-2, nu log-uniform 1e-3-1e-2),
    admitted under an HBM budget and served with continuous batching (babelsim_b200.serve)."""
    import babelsim_b200 as bsg
    from babelsim_b200 import meshgen, serve
    rng = np.random.default_rng(SEED)
    pool = {("hex", n): meshgen.hex_box(n, n, n) for n in (16, 20, 26, 32, 40, 46)}
    for n in (16, 24, 32):
        pool[("voronoi", n)] = meshgen.voronoi_cube(n, 0.3, SEED + n)
    keys = sorted(pool, key=lambda k: pool[k].n_cells)
    sizes = np.array([pool[k].n_cells for k in keys], float)
    reqs, t = [], 0.0
    for i in range(args.requests):
        target = np.exp(rng.uniform(np.log(4000), np.log(1e5)))
        k = keys[int(np.argmin(np.abs(np.log(sizes) - np.log(target))))]
        t += rng.exponential(1.0 / args.arrival_rate)
        reqs.append(serve.Request(i, t, pool[k], speed=float(rng.uniform(0.5, 2.0)),
                                  nu=float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-2)))),
                                  max_iterations=args.max_outer, tolerance=args.tolerance))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        # requests shard across GPUs (each its own admission loop, no data exchanged); one gather at the end
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    mine = serve.shard(reqs, world, rank)
    ctx = bsg.Context(int(os.environ.get("LOCAL_RANK", "0")))
    srv = serve.Server(ctx, hbm_budget=150 * 2**30, slots=args.slots, solver_precision=args.precision,
                       batched=not args.unbatched, trace=args.trace)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    res = srv.run(mine)
    wall = time.perf_counter() - t0
    if dist:
        gathered = [None] * world
        dist.all_gather_object(gathered, ([(r.id, r.cells, r.arrival, r.admitted, r.finished, r.iterations,
                                            r.converged) for r in res], wall))
        dist.destroy_process_group()
        if rank != 0:
            ctx.close()
            return
        res = sorted((serve.Result(*t) for g in gathered for t in g[0]), key=lambda r: r.id)
        wall = max(g[1] for g in gathered)
    out = serve.summary(res, wall)
    alone, ratio = None, None
    if world == 1:
        # each request solved alone on the same GPU (arrival at 0, nothing else running)
        alone = []
        for r in reqs:
            solo = serve.Server(ctx, hbm_budget=150 * 2**30, slots=1, solver_precision=args.precision,
                                batched=not args.unbatched)
            rr = solo.run([serve.Request(r.id, 0.0, r.mesh, r.speed, r.nu, r.max_iterations, r.tolerance)])[0]
            alone.append(rr.latency)
            if args.trace:
                print(f"serve: alone {r.id} {rr.iterations} {rr.latency:.3f}", file=sys.stderr, flush=True)
        ratio = np.array([res[i].latency / alone[i] for i in range(len(reqs))])
    line = {"metric": "served solves/s (steady SIMPLE cavity requests)", "value": out["solves_per_s"],
            "unit": "solves/s", "n_gpus": world, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "scaling": "strong",
            "config": {"workload": f"{args.requests} seeded requests, cells log-uniform 4k-100k (hex and "
                                   f"jittered-Voronoi cubes), Poisson arrivals {args.arrival_rate}/s, "
                                   f"{args.slots} slots, 150 GiB budget, outer tolerance {args.tolerance} or "
                                   f"{args.max_outer} iterations, pressure V-cycle "
                                   f"{'fp32' if args.precision == 2 else 'fp64'}, "
                                   f"{'one solve per request' if args.unbatched else 'cohorts as block-diagonal batches'}",
                       "slots": args.slots, "batched": not args.unbatched},
            "p50_latency_s": out["p50_latency_s"], "p99_latency_s": out["p99_latency_s"],
            "converged": out["converged"], "cell_iters_per_s": out["cell_iters_per_s"], "wall_s": wall,
            "parallelism": f"requests sharded over {world} GPU(s) by predicted cell-iterations, no data exchange",
            "isolated_solve_s": None if alone is None else {"p50": float(np.percentile(alone, 50)),
                                                            "p99": float(np.percentile(alone, 99))},
            "latency_over_isolated": None if ratio is None else {"p50": float(np.percentile(ratio, 50)),
                                                                 "p99": float(np.percentile(ratio, 99))},
            "p99_latency_over_isolated_p99": None if alone is None else
            out["p99_latency_s"] / float(np.percentile(alone, 99))}
    print(json.dumps(line))
    ctx.close()


def _reference_run(case_writer, steps_label):
    """Run the reference's own sources (oracle/_ref) on a case written by `case_writer(dir)`;
    returns (seconds, run info)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "babelsim-oracle")
    if not os.path.exists(exe):
        return None, None
    work = tempfile.mkdtemp(prefix=f"bsg_ref_{steps_label}_")
    case_writer(work)
    out = os.path.join(work, "out")
    res = subprocess.run([exe, work, out], env=dict(os.environ, OMP_NUM_THREADS="1"), capture_output=True,
                         text=True, timeout=900)
    if not os.path.exists(os.path.join(out, "run.json")):
        raise RuntimeError(f"reference run failed (exit {res.returncode}): {res.stderr[-300:]}")
    info = json.load(open(os.path.join(out, "run.json")))
    return float(info["solver_seconds"]), info


def run_piso_cylinder(args):
    """Transient PISO (BDF2, 2 correctors, 1 non-orthogonal corrector) past a cylinder D = 1 on a
    hex O-grid (radial growth 1.05 to 15 D), nu 0.01, inlet u = 1; metric cell-steps/s.  The
    default dt 0.001 keeps the Courant number near the cylinder below 1 on the 2000-cell
    circumference (dt 0.005 gives about 3 there and the impulsive start diverges)."""
    import babelsim_b200 as bsg
    from babelsim_b200 import meshgen
    n_theta, n_r = args.theta_cells, args.radial_cells
    poly = meshgen.cylinder_ogrid(n_theta, n_r, 0.5, 15.0, 1.05)
    ctx = bsg.Context(int(os.environ.get("LOCAL_RANK", "0")))
    mesh = bsg.Mesh.from_polyhedral(ctx, poly)
    N = mesh.n_cells
    o = bsg.options("linear", "leastSquares", "linearUpwind", "corrected")
    steps = args.steps
    out = {}
    for precision in (0, 2):
        sim = bsg.Piso(mesh, 1.0, 0.01, 1.0, 1, 2, None, None, 1, 1e-7, 1e-7, 1e-6, 1e-7, "bdf2", 0.0, 1e9, args.dt,
                       o, o, bsg.solver_config("bcgs", "bjacobi", 1e-12, 1e-8, 1000),
                       bsg.solver_config("cg", "hypre", 1e-13, 1e-9, 1500, precision=precision))
        bcsU = [("fixedValue", (0, 0, 0)), ("fixedValue", (1, 0, 0)), ("zeroGradient", 0), ("symmetry", 0),
                ("symmetry", 0)]
        bcsP = [("zeroGradient", 0), ("zeroGradient", 0), ("fixedValue", 0), ("symmetry", 0), ("symmetry", 0)]
        for pi, (t, v) in enumerate(bcsU):
            sim.set_boundary("U", pi, t, v)
        for pi, (t, v) in enumerate(bcsP):
            sim.set_boundary("p", pi, t, v)
        U0 = np.zeros((N, 3))
        U0[:, 0] = 1.0
        sim.set_fields(U0, np.zeros(N))
        sim.advance(max(args.warmup, 3))
        ctx.synchronize()
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
            ctx.record(0)
            rep = sim.advance(steps)
            ctx.record(1)
            ms = ctx.elapsed_ms(0, 1)
        out[precision] = (ms, rep, clocks.summary())
        sim.close()
    ms, rep, clk = out[0]
    # the reference's own runPiso on a 10x smaller O-grid, 4 steps, 1 core
    from make_golden import write_case  # noqa: E402
    small = meshgen.cylinder_ogrid(max(n_theta // 4, 16), max(n_r // 2, 8), 0.5, 15.0, 1.05 ** 2)
    bU = [("fixedValue", (0.0, 0.0, 0.0)), ("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0)),
          ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    bP = [("zeroGradient", 0.0), ("zeroGradient", 0.0), ("fixedValue", 0.0), ("symmetry", 0.0), ("symmetry", 0.0)]
    meth = {"momentum": dict(interpolation="linear", gradient="leastSquares", convection="linearUpwind",
                             diffusion="corrected")}
    meth["pressureCorrection"] = dict(meth["momentum"])
    sol = {"maxIterations": 1, "nCorrectors": 2, "nonOrthogonalCorrections": 1, "velocityRelaxation": 1.0,
           "continuityTolerance": 1e-7, "velocityTolerance": 1e-7, "momentumTolerance": 1e-6,
           "pressureCorrectionTolerance": 1e-7, "equation.momentum.kspType": "bcgs",
           "equation.momentum.pcType": "bjacobi", "equation.momentum.absoluteTolerance": 1e-12,
           "equation.momentum.relativeTolerance": 1e-8, "equation.momentum.maxIterations": 1000,
           "equation.pressureCorrection.kspType": "cg", "equation.pressureCorrection.pcType": "hypre",
           "equation.pressureCorrection.absoluteTolerance": 1e-13,
           "equation.pressureCorrection.relativeTolerance": 1e-9,
           "equation.pressureCorrection.maxIterations": 1500}
    cb = None
    try:
        secs, info = _reference_run(lambda d: write_case(d, small, bU, bP, meth, sol, {"density": 1.0,
                                    "dynamicViscosity": 0.01}, solver="piso", time="bdf2",
                                    control=(0.0, 4 * args.dt, args.dt)), "piso")
        if secs:
            cb = {"value": small.n_cells * 4 / secs, "unit": "cell-steps/s", "cores": 1, "kind": "reference",
                  "sample": f"reference runPiso, {small.n_cells}-cell O-grid, 4 steps (whole run timed), "
                            f"status {info['status']}"}
    except Exception as exc:  # the baseline is reported, never required for the GPU number
        cb = {"value": None, "error": str(exc)[:200]}
    line = {"metric": "cell-steps/s (transient PISO, BDF2, flow past a cylinder)", "value": N * steps / (ms / 1e3),
            "unit": "cell-steps/s", "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 3),
            "ms_per_step": ms / steps, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"PISO cylinder O-grid {n_theta}x{n_r} = {N} cells, radial growth 1.05 to 15 D, "
                                   f"Re 100, dt {args.dt}, 2 correctors, 1 non-orthogonal corrector",
                       "cells": N},
            "mixed_precision": {"value": N * steps / (out[2][0] / 1e3), "unit": "cell-steps/s",
                                "precision": "fp64 flexible PCG + fp32 AMG V-cycle"},
            "cpu_baseline": cb, "clocks": clk,
            "last_report": {"courant_max": rep.courant_max, "mass": rep.mass, "coupling": rep.coupling,
                            "pressure_iterations": rep.pressure_iterations,
                            "momentum_iterations": rep.momentum_iterations}}
    print(json.dumps(line))
    mesh.close()
    ctx.close()


def batched_cases():
    """Uneven cavity cases of the batched workload: jittered-Voronoi cubes (the 1M-cell
    workload's generator) and hex boxes, lid speed uniform 0.5-2 and viscosity log-uniform
    1e-3-1e-2 from a seeded stream (the serving stream's distributions)."""
    from babelsim_b200 import meshgen
    rng = np.random.default_rng(SEED + 1)
    meshes = [meshgen.voronoi_cube(n, 0.3, SEED + n) for n in (16, 20, 24, 28, 32, 40)]
    meshes += [meshgen.hex_box(n, n, n, flat=True) for n in (20, 32)]
    return [(m, float(rng.uniform(0.5, 2.0)), float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-2)))))
            for m in meshes]


def run_batched(args):
    """Block-diagonal batching: the uneven cases of batched_cases() advanced as one batch (one set
    of launches per outer iteration, all pressure systems in one persistent launch per attempt)
    against the same cases one after another, each with its own launches on the whole GPU."""
    import babelsim_b200 as bsg
    from babelsim_b200 import meshgen
    s = case_settings()
    cases = batched_cases()
    ctx = bsg.Context(int(os.environ.get("LOCAL_RANK", "0")))
    warm, steps = max(args.warmup, 3), args.steps

    def configure(sim, patch0, lid):
        for patch in range(6):
            sim.set_boundary("U", patch0 + patch, "fixedValue", (lid, 0.0, 0.0) if patch == 3 else (0.0, 0.0, 0.0))
            sim.set_boundary("p", patch0 + patch, "zeroGradient")

    def simple(mesh, mu, precision):
        t = dict(s, mu=mu)
        return build_simple(bsg, mesh, t, precision=precision, boundaries=False)

    # one after another: each case alone, its own kernels on the whole GPU
    seq_ms, seq_fields, cells = 0.0, [], 0
    for poly, lid, mu in cases:
        mesh = bsg.Mesh.from_polyhedral(ctx, poly)
        sim = simple(mesh, mu, 0)
        configure(sim, 0, lid)
        sim.set_fields(np.zeros((mesh.n_cells, 3)), np.zeros(mesh.n_cells))
        sim.iterate(warm)
        ctx.synchronize()
        ctx.record(0)
        sim.iterate(steps)
        ctx.record(1)
        seq_ms += ctx.elapsed_ms(0, 1)
        seq_fields.append(sim.fields()[:2])
        cells += mesh.n_cells
        sim.close()
        mesh.close()
    seq_value = cells * steps / (seq_ms / 1e3)
    poly, offsets, patches = meshgen.concatenate([c[0] for c in cases])
    mesh = bsg.Mesh.from_polyhedral(ctx, poly)
    out = {}
    for precision in (0, 2):
        sim = simple(mesh, cases[0][2], precision)
        sim.set_segments(offsets, [c[2] for c in cases])
        for k, (_, lid, _) in enumerate(cases):
            configure(sim, int(patches[k]), lid)
        sim.set_fields(np.zeros((mesh.n_cells, 3)), np.zeros(mesh.n_cells))
        sim.iterate(warm)
        ctx.synchronize()
        launches0 = ctx.launches()
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
            ctx.record(2)
            sim.iterate(steps)
            ctx.record(3)
            ms = ctx.elapsed_ms(2, 3)
        U, p, _ = sim.fields()
        dev = []
        for k, (Us, ps) in enumerate(seq_fields):
            a, b = int(offsets[k]), int(offsets[k + 1])
            dev.append(max(float(np.linalg.norm(U[a:b] - Us) / max(np.linalg.norm(Us), 1e-300)),
                           float(np.linalg.norm(p[a:b] - ps) / max(np.linalg.norm(ps), 1e-300))))
        out[precision] = {"value": cells * steps / (ms / 1e3), "ms_per_step": ms / steps,
                          "launches_per_step": (ctx.launches() - launches0) / steps, "clocks": clocks.summary(),
                          "max_rel_l2_vs_one_after_another": max(dev)}
        sim.close()
    mesh.close()
    ctx.close()
    b64 = out[0]
    line = {"metric": "cell-iters/s (uneven steady SIMPLE cavities, block-diagonal batch)", "value": b64["value"],
            "unit": "cell-iters/s", "n_gpus": 1, "steps": steps, "warmup": warm, "ms_per_step": b64["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{len(cases)} cavities, {cells} cells in total (jittered-Voronoi cubes "
                                   f"16^3-40^3 and hex boxes 20^3, 32^3), lid 0.5-2, nu 1e-3-1e-2, linearUpwind, "
                                   f"least squares, corrected diffusion, 2 non-orthogonal correctors, pressure CG + "
                                   f"AMG and momentum BiCGStab to rtol 1e-10", "cases": len(cases), "cells": cells},
            "one_after_another": {"value": seq_value, "ms_per_step": seq_ms / steps},
            "speedup_vs_one_after_another": b64["value"] / seq_value,
            "launches_per_step": b64["launches_per_step"], "clocks": b64["clocks"],
            "max_rel_l2_vs_one_after_another": b64["max_rel_l2_vs_one_after_another"],
            "fp32_vcycle": {"value": out[2]["value"], "ms_per_step": out[2]["ms_per_step"],
                            "vs_fp64_batch": out[2]["value"] / b64["value"],
                            "max_rel_l2_vs_fp64_one_after_another": out[2]["max_rel_l2_vs_one_after_another"]}}
    print(json.dumps(line))


def run_komega_channel(args):
    """Steady SIMPLE with k-omega in a plane channel (2 pi x 2 x pi, tanh wall clustering),
    inlet/outlet (the reference has no periodic patches), nu 1e-4; metric cell-iters/s."""
    import babelsim_b200 as bsg
    from babelsim_b200 import meshgen
    nx, ny, nz = args.channel_cells
    poly = meshgen.channel(nx, ny, nz)
    ctx = bsg.Context(int(os.environ.get("LOCAL_RANK", "0")))
    mesh = bsg.Mesh.from_polyhedral(ctx, poly)
    N = mesh.n_cells
    o = bsg.options("linear", "greenGauss", "linearUpwind", "orthogonal")
    t = bsg.options("linear", "greenGauss", "upwind", "orthogonal")
    sim = bsg.Simple(mesh, 1.0, 1e-4, 0.7, 0.3, 0, 1e-8, 1e-7, 1e-6, 1e-6, o, o,
                     bsg.solver_config("bcgs", "bjacobi", 1e-14, 1e-8, 1000),
                     bsg.solver_config("cg", "hypre", 1e-14, 1e-8, 1000))
    sim.enable_komega(k_transport=t, omega_transport=t,
                      k_solver=bsg.solver_config("bcgs", "bjacobi", 1e-18, 1e-8, 1000),
                      omega_solver=bsg.solver_config("bcgs", "bjacobi", 1e-18, 1e-8, 1000))
    U = [("fixedValue", (1.0, 0, 0)), ("zeroGradient", 0), ("fixedValue", (0, 0, 0)), ("fixedValue", (0, 0, 0)),
         ("symmetry", 0), ("symmetry", 0)]
    P = [("zeroGradient", 0), ("fixedValue", 0), ("zeroGradient", 0), ("zeroGradient", 0), ("symmetry", 0),
         ("symmetry", 0)]
    K = [("fixedValue", 3.75e-3), ("zeroGradient", 0), ("fixedValue", 1e-12), ("fixedValue", 1e-12),
         ("symmetry", 0), ("symmetry", 0)]
    W = [("fixedValue", 10.0), ("zeroGradient", 0), ("fixedValue", 1e4), ("fixedValue", 1e4), ("symmetry", 0),
         ("symmetry", 0)]
    for name, bcs in (("U", U), ("p", P), ("k", K), ("omega", W)):
        for pi, (tp, v) in enumerate(bcs):
            sim.set_boundary(name, pi, tp, v)
    sim.set_turbulence_fields(np.full(N, 3.75e-3), np.full(N, 10.0))
    U0 = np.zeros((N, 3))
    U0[:, 0] = 1.0
    sim.set_fields(U0, np.zeros(N))
    sim.iterate(max(args.warmup, 3))
    ctx.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        ctx.record(0)
        rep = sim.iterate(args.steps)
        ctx.record(1)
        ms = ctx.elapsed_ms(0, 1)
    line = {"metric": "cell-iters/s (steady SIMPLE + k-omega, plane channel)", "value": N * args.steps / (ms / 1e3),
            "unit": "cell-iters/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"k-omega channel {nx}x{ny}x{nz} = {N} cells, tanh wall clustering, "
                                   "inlet/outlet, nu 1e-4", "cells": N},
            "clocks": clocks.summary(),
            "last_report": {"status": rep.status, "rU": rep.rU, "turbulence_change": rep.turbulence_change,
                            "pressure_iterations": rep.pressure_iterations}}
    print(json.dumps(line))
    sim.close()
    mesh.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cells", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison run")
    ap.add_argument("--phases", action="store_true", help="add the pressure solver's phase timeline to the line")
    ap.add_argument("--workload", default="cavity", choices=["cavity", "serving", "piso-cylinder", "komega-channel", "batched"])
    ap.add_argument("--theta-cells", type=int, default=2000)
    ap.add_argument("--dt", type=float, default=0.001)
    ap.add_argument("--radial-cells", type=int, default=100)
    ap.add_argument("--channel-cells", type=int, nargs=3, default=[200, 160, 125])
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--arrival-rate", type=float, default=8.0)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--max-outer", type=int, default=150)
    ap.add_argument("--tolerance", type=float, default=1e-4, help="serving: outer-loop tolerance")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 2], help="serving: pressure V-cycle precision")
    ap.add_argument("--unbatched", action="store_true", help="serving: one solve per request, no cohorts")
    ap.add_argument("--trace", action="store_true", help="serving: print admissions and retirements to stderr")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "piso-cylinder":
        sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
        return run_piso_cylinder(args)
    if args.workload == "komega-channel":
        return run_komega_channel(args)
    if args.workload == "batched":
        return run_batched(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    import babelsim_b200 as bsg
    n_side = max(2, round(args.cells ** (1.0 / 3.0)))
    t0 = time.time()
    poly = mesh_for(n_side)
    t_mesh = time.time() - t0
    ctx = bsg.Context(local)
    # Mesh ingest (Mesh::polyhedral): geometry on the device, and at N=1 the host geometry beside it.
    t0 = time.perf_counter()
    mesh = bsg.Mesh.from_polyhedral(ctx, poly)
    ingest = {"device_geometry_s": round(time.perf_counter() - t0, 3)}
    if world == 1:
        t0 = time.perf_counter()
        host_mesh = bsg.Mesh.from_polyhedral(ctx, poly, host_geometry=True)
        ingest["host_geometry_s"] = round(time.perf_counter() - t0, 3)
        host_mesh.close()
    N, F, Fi = mesh.n_cells, mesh.n_faces, mesh.n_interior
    s = case_settings()
    sim = build_simple(bsg, mesh, s)
    sim.iterate(max(args.warmup, 3))
    ctx.synchronize()
    if dist:
        dist.barrier()
    launches0 = ctx.launches()
    with ClockSampler(local) as clocks:
        ctx.record(0)
        rep = sim.iterate(args.steps)
        ctx.record(1)
        ms = ctx.elapsed_ms(0, 1)
    launches = ctx.launches() - launches0
    if dist:
        import torch
        t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    steps_done = args.steps
    value = world * N * steps_done / (ms / 1e3)
    # Live per-kernel timing of one more outer iteration (CUDA events on the library's stream).
    ctx.profile(True)
    sim.iterate(1)
    prof = ctx.profile_report()
    ctx.profile(False)
    amg_rows = int(N / 4)

    def launch_bytes(name, rec):
        if rec[2] > 0:  # algorithmic bytes the library declared for these launches
            return rec[2] / rec[0]
        return algorithmic_bytes(name, N, 2 * Fi, amg_rows)

    phases = pressure_phases(ctx, sim) if args.phases else None
    candidates = {k: v for k, v in prof.items() if launch_bytes(k, v)}
    top = max(candidates, key=lambda k: candidates[k][1]) if candidates else None
    peak, peak_kind = load_peaks()
    roofline = None
    if top:
        cnt, tot = candidates[top][0], candidates[top][1]
        avg_s = tot / cnt / 1e3
        ab = launch_bytes(top, candidates[top])
        achieved = ab / avg_s / 1e9
        ratio = DRAM_PER_ALGORITHMIC_BYTE.get(top)
        roofline = {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 3),
                    "traffic": round(ratio * ab) if ratio else None, "algorithmic_bytes_per_launch": round(ab),
                    "avg_launch_us": round(avg_s * 1e6, 2), "launches_per_step": cnt,
                    "share_of_step": round(tot / sum(v[1] for v in prof.values()), 3)}
        if candidates[top][3] > 0:
            roofline["units_per_launch"] = round(candidates[top][3] / cnt, 1)
    # End to end through the C ABI with host buffers: every step copies U, p, phi in from
    # pinned host memory, runs one outer iteration and copies them back out.
    import torch
    Uh = torch.zeros((N, 3), dtype=torch.float64).pin_memory().numpy()
    ph = torch.zeros(N, dtype=torch.float64).pin_memory().numpy()
    phih = torch.zeros(F, dtype=torch.float64).pin_memory().numpy()
    sim.fields_into(Uh, ph, phih)
    e2e_steps = max(2, min(args.steps, 5))
    ctx.synchronize()
    ctx.record(2)
    for _ in range(e2e_steps):
        sim.load_state(Uh, ph, phih)
        sim.iterate(1)
        sim.fields_into(Uh, ph, phih)
    ctx.record(3)
    e2e_ms = ctx.elapsed_ms(2, 3)
    if dist:
        t = torch.tensor([e2e_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    bytes_io = 8 * (3 * N + N + F)
    e2e = {"value": world * N * e2e_steps / (e2e_ms / 1e3), "unit": "cell-iters/s", "h2d_bytes_per_step": bytes_io,
           "d2h_bytes_per_step": bytes_io, "steps": e2e_steps}
    # Mixed precision (FP32 inner PCG + FP32 V-cycle inside FP64 iterative refinement, pressure
    # solves) from the same initial state and for the same number of outer iterations; its
    # fields are compared with the FP64 run's.
    mixed = None
    if not args.no_mixed:
        U64, p64, _ = sim.fields()
        steps64 = sim.iterate(0).iterations  # every outer iteration of the FP64 run so far
        mixed = {}
        for mode, label in ((2, "fp64 flexible PCG + fp32 AMG V-cycle"),
                            (1, "fp32 inner PCG + fp32 AMG V-cycle, fp64 refinement"),
                            ("1_momentum", "fp32 inner BiCGStab in fp64 refinement for momentum, fp64 pressure"),
                            ("1_all", "fp32 inner iterations in fp64 refinement for pressure (PCG + AMG) "
                                      "and momentum (BiCGStab)")):
            sim.close()
            sim = build_simple(bsg, mesh, s, precision={"1_all": 1, "1_momentum": 0}.get(mode, mode),
                               momentum_precision=1 if mode in ("1_all", "1_momentum") else 0)
            sim.iterate(max(args.warmup, 3))
            ctx.synchronize()
            ctx.record(4)
            sim.iterate(steps_done)
            ctx.record(5)
            mms = ctx.elapsed_ms(4, 5)
            if dist:
                t = torch.tensor([mms], device=f"cuda:{local}", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                mms = float(t.item())
            sim.iterate(steps64 - max(args.warmup, 3) - steps_done)
            U32, p32, _ = sim.fields()
            mixed[f"precision_{mode}"] = {
                "value": world * N * steps_done / (mms / 1e3), "unit": "cell-iters/s", "ms_per_step": mms / steps_done,
                "precision": label, "vs_fp64_value": round(ms / mms, 3),
                "rel_l2_vs_fp64_after_%d_iterations" % steps64: {
                    "U": float(np.linalg.norm(U32 - U64) / np.linalg.norm(U64)),
                    "p": float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))}}
    cb = None
    same_sample = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline()
        except Exception as exc:  # the baseline is reported, never required for the GPU number
            cb = {"value": None, "error": str(exc)[:200]}
        same_sample = device_on_sample(bsg, ctx, s, args.warmup)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cell-iters/s", "n_gpus": world, "steps": steps_done,
                "warmup": max(args.warmup, 3), "ms_per_step": ms / steps_done, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": simple_config(n_side, world),
                "mesh": {"cells": N, "faces": F, "interior_faces": Fi, "generation_seconds": round(t_mesh, 1)},
                "roofline": roofline, "cpu_baseline": cb, "device_on_cpu_sample": same_sample, "e2e": e2e,
                "mixed_precision": mixed,
                "gpu_launches": launches, "mesh_ingest": ingest,
                "clocks": clocks.summary(), "profile_ms_one_step": {k: round(v[1], 3) for k, v in prof.items()},
                "pressure_phases_us_per_cg_iteration": phases,
                "pressure_iterations_per_solve": round(prof["pcg_amg_persistent"][3] / prof["pcg_amg_persistent"][0], 1)
                if "pcg_amg_persistent" in prof else None,
                "last_report": {"momentum_iterations": rep.momentum_iterations,
                                "pressure_iterations": rep.pressure_iterations, "rU": rep.rU, "dU": rep.dU,
                                "mass": rep.mass}}
        print(json.dumps(line))
    sim.close()
    mesh.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
