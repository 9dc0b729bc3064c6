#!/usr/bin/env python
"""Throughput of the PARIS per-timestep grid core on B200.

One step = vofsweeps (CIAM, three split sweeps) -> linfunc(rho) -> the
predicted velocity u* into u (stand-in for the momentum predictor, which is
outside this path) -> SetupPoisson -> NewSolver to ||r||_2/||b||_2 < 1e-10
from p = 0 -> project_velocity, on the 256^3 periodic unit cube with 64 drops
of radius U[0.03,0.08] at density ratio 1000 and a seeded Gaussian u*
(unit variance, 3 Jacobi smoothing sweeps).  `value` uses the mixed-precision
multigrid (FP32 V(2,2) cycles preconditioning an FP64 flexible CG) with
inputs resident in HBM; `fp64_steps_per_s` the same algorithm all in FP64;
`pressure_error` compares the two solutions step by step and the mixed one
with the oracle's FP64 solution once; `e2e` is the same step through the
C-ABI with host buffers (u* uploaded, u,v,w,cvof downloaded every step).
`--impl reference` times the reference algorithm (the CPU restatement in
oracle/) on the host cores.

`--workload rising_bubble` times instead the full explicit Navier-Stokes step
(momentum predictor, VOF, heights, curvature, CSF, projection) on a gas
bubble of radius 0.125 rising in liquid in the walled box [0,1]x[0,1]x[0,2]
at 512x512x1024, with the time step of TimeStepSize (CFL 0.5, MaxDt 5e-4).

Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s @256³ VOF+MG projection, mixed vs FP64 MG at 1e-10 residual"
REL_TOL = 1e-10
NU = [2, 2, 4, 1, 2]   # pre/post sweeps of the B200 V-cycle; sweeps from level NU[3] down (--nu1 --nu2 --nu-coarse --coarse-from --coarse-to)
OMEGA = [1.1, 1.25]   # relaxation factor of its red-black smoother on the finest level and below it (--beta --beta-coarse)
REF_BETA = 1.2  # the reference's default BETA (paris.f90:3553), for its own multigrid


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="projection", choices=["projection", "rising_bubble"])
    ap.add_argument("--grid", "--n", dest="n", type=int, default=None,
                    help="cells per direction (projection: 256; rising_bubble: 512 across, twice that in z); "
                         "under torchrun use --grid, which its own options cannot be confused with")
    ap.add_argument("--pcg", type=int, default=1, help="1: FP64 flexible CG preconditioned by the V-cycle, 0: defect correction")
    ap.add_argument("--beta", type=float, default=1.1,
                    help="relaxation factor of the B200 multigrid's red-black smoother (the reference's BETA)")
    ap.add_argument("--beta-coarse", type=float, default=1.25,
                    help="the smoother's relaxation factor on the levels below the finest (0: --beta)")
    ap.add_argument("--nu-coarse", type=int, default=4,
                    help="pre/post sweeps of the B200 V-cycle on the levels from --coarse-from down (0: --nu1/--nu2)")
    ap.add_argument("--coarse-from", type=int, default=1, help="first level (0 = finest) that takes --nu-coarse")
    ap.add_argument("--coarse-to", type=int, default=2, help="last level that takes --nu-coarse (0: every coarser level)")
    ap.add_argument("--nu1", type=int, default=2, help="pre-smoothing sweeps of the B200 V-cycle")
    ap.add_argument("--nu2", type=int, default=2, help="post-smoothing sweeps of the B200 V-cycle")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds of reference V-cycles in the cpu_baseline sample step")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="--impl reference: seconds of reference V-cycles over all timed steps")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-only", action="store_true", help="a few profiled steps, no JSON timing")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU; replicas only (the grid core does not shard)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
def load_pkg():
    import __graft_entry__
    return __graft_entry__.load_package()


def workload(pkg, n, device=0):
    capi, wl = pkg.capi, pkg.workloads
    desc = capi.make_desc((n, n, n), rho1=1.0, rho2=1000.0, device=device)
    cen, rad = wl.drop_layout(64, rmin=0.03, rmax=0.08, seed=0, h=1.0 / n)
    us = wl.smoothed_gaussian_faces((n, n, n), seed=1)
    umax = max(float(np.abs(a).max()) for a in us)
    dt = 0.25 * (1.0 / n) / umax
    return desc, cen, rad, us, dt


# algorithmic HBM bytes per cell of each labelled kernel (cells as recorded
# by the profiler: the grid cells the launch processes)
ALGO_BYTES = {
    "pcg_matvec_fp64": 40.0,      # d 8 + 3 faces 24 + q 8
    "pcg_update_fp64(z32)": 56.0, # p r/w 16 + d 8 + r r/w 16 + q 8 + rhs (FP32) 4 + z (FP32) 4
    "pcg_update_fp64(z64)": 64.0,
    "pcg_rz(z32)": 12.0,          # r 8 + z 4
    "pcg_rz(z64)": 16.0,
    "pcg_dir(z32)": 20.0,         # z 4 + d r/w 16
    "pcg_dir(z64)": 24.0,
    "mg_sweep_f32": 24.0,         # fused red-black sweep: x in 4 + 3 faces 12 + rhs 4 + x out 4
    "mg_sweep_f64": 48.0,
    "mg_sweep_zero_f32": 20.0,    # first sweep from x = 0: no iterate read
    "mg_sweep_zero_f64": 40.0,
    "mg_sweep_lower_f32": 24.0,   # levels below the finest: the same bytes, served from L2
    "mg_sweep_lower_f64": 48.0,
    "mg_sweep_pair_f32": 24.0,    # two sweeps in one pass: the bytes of one sweep
    "mg_sweep_pair_f64": 48.0,
    "mg_sweep_pair_zero_f32": 20.0,
    "mg_sweep_pair_zero_f64": 40.0,
    "mg_sweep_pair_lower_f32": 24.0,
    "mg_sweep_pair_lower_f64": 48.0,
    "mg_smooth_f32": 12.0,        # half of a red-black sweep: (p 4 + 3 faces 12 + rhs 4 + p write 4)/2
    "mg_smooth_f64": 24.0,
    "mg_restrict_f32": 20.5,      # x 4 + b 4 + 3 faces 12 + coarse rhs 4/8
    "mg_restrict_f64": 41.0,
    "mg_prolong_f32": 8.5,        # x read+write 8 + coarse 4/8
    "mg_prolong_f64": 17.0,
    "mg_residual_fp64(r32)": 52.0,  # 3 faces + rhs 32 + p 8 + r (FP32) 4 + r (FP64, the CG's) 8
    "mg_residual_fp64(r64)": 56.0,
    "mg_correct_f32": 20.0,       # p read+write 16 + correction 4
    "mg_correct_f64": 24.0,
    "mg_coef0": 36.0,             # FP64 faces 24 -> FP32 faces 12
    "vof_sweep": 25.0,            # c 8 + u_d 8 + new c 8 + flag 1
    "setup_poisson": 64.0,        # u,v,w,rho 32 + 3 faces + rhs 32
    "project_velocity": 64.0,     # p,rho 16 + u,v,w read+write 48
    "linfunc": 16.0,              # cvof 8 + rho 8 (ghosted cells)
    # the rest of a full Navier-Stokes step (rising-bubble workload)
    "mom_convection": 48.0,       # u,v,w 24 + du,dv,dw 24
    "mom_diffusion": 88.0,        # u,v,w,rho,mu 40 + du,dv,dw read+write 48
    "volume_force": 56.0,         # rho 8 + du,dv,dw read+write 48
    "advance_velocity": 72.0,     # u,v,w read+write 48 + du,dv,dw 24
    "surface_force": 72.0,        # cvof, kappa, rho 24 + du,dv,dw read+write 48
    "heights_pass1": 25.0,        # per direction: cvof 8 + flag 1 + two height arrays 16
    "vmax": 24.0,                 # u,v,w
    "calc_stats": 57.0,           # u,v,w,rho,p,cvof,mu 56 + flag 1
}


def gpu_step(gpu, capi, k, dt, mode, pcg):
    gpu.vof_sweeps(k, dt)
    gpu.linfunc(capi.F_RHO)
    for dst, src in ((capi.F_U, capi.F_USTAR), (capi.F_V, capi.F_VSTAR), (capi.F_W, capi.F_WSTAR)):
        gpu.copy_field(dst, src)
    gpu.setup_poisson(dt)
    gpu.fill_field(capi.F_P, 0.0)
    r = gpu.new_solver(0.0, maxit=200, mode=mode, rel_tol=REL_TOL, pcg=pcg, nu1=NU[0], nu2=NU[1], beta=OMEGA[0],
                       nu_coarse=NU[2], coarse_from=NU[3], coarse_to=NU[4], beta_coarse=OMEGA[1])
    gpu.project_velocity(dt)
    return r


def _rel_diff(a, b):
    """||(a - mean a) - (b - mean b)||_2 / ||b - mean b||_2 and the same in
    max-abs (the pressure of the periodic problem is fixed up to a constant)."""
    da, db = a - a.mean(), b - b.mean()
    e = da - db
    return float(np.linalg.norm(e) / np.linalg.norm(db)), float(np.abs(e).max() / np.abs(db).max())


def _residual_rel(A, p, b):
    """||b - A p||_2 / ||b||_2 on the host with the reference's 8-component A
    (periodic in all directions)."""
    r = b.copy()
    r -= A[6] * p
    r += A[0] * np.roll(p, 1, 2) + A[1] * np.roll(p, -1, 2) + A[2] * np.roll(p, 1, 1) + A[3] * np.roll(p, -1, 1) + \
        A[4] * np.roll(p, 1, 0) + A[5] * np.roll(p, -1, 0)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def pressure_error(gpu, capi, args, dt, reset, cpu_oracle):
    """The pressure of the mixed solver against the all-FP64 one, step by step
    on the same states (each step's matrix is solved by both from p = 0), and
    once, on the first step's matrix, against the oracle's FP64 solution
    (its restatement of the same multigrid in FP64, flexible CG to 1e-12).
    Untimed."""
    from oracle import pyoracle as orc
    reset()
    d = gpu.desc
    g = d.ng
    rows = []
    oracle = None
    for k in range(args.steps):
        gpu.vof_sweeps(k, dt)
        gpu.linfunc(capi.F_RHO)
        for dst, src in ((capi.F_U, capi.F_USTAR), (capi.F_V, capi.F_VSTAR), (capi.F_W, capi.F_WSTAR)):
            gpu.copy_field(dst, src)
        gpu.setup_poisson(dt)
        gpu.fill_field(capi.F_P, 0.0)
        rm = gpu.new_solver(0.0, maxit=200, mode=capi.MG_MIXED, rel_tol=REL_TOL, pcg=args.pcg, nu1=NU[0], nu2=NU[1], beta=OMEGA[0],
                       nu_coarse=NU[2], coarse_from=NU[3], coarse_to=NU[4], beta_coarse=OMEGA[1])
        pm = gpu.download(capi.F_P)
        gpu.fill_field(capi.F_P, 0.0)
        r64 = gpu.new_solver(0.0, maxit=200, mode=capi.MG_FP64, rel_tol=REL_TOL, pcg=args.pcg, nu1=NU[0], nu2=NU[1], beta=OMEGA[0],
                       nu_coarse=NU[2], coarse_from=NU[3], coarse_to=NU[4], beta_coarse=OMEGA[1])
        p64 = gpu.download(capi.F_P)
        pm_i, p64_i = pm[g:-g, g:-g, g:-g], p64[g:-g, g:-g, g:-g]
        l2, mx = _rel_diff(pm_i, p64_i)
        rows.append((l2, mx, rm.rel_res, r64.rel_res))
        if k == 0 and cpu_oracle:
            A = gpu.download(capi.F_A)
            p_int, it, _ = orc.fastmg_solve(d, A, np.zeros((d.nz, d.ny, d.nx)), 1e-12, maxit=100, mixed=False,
                                            pcg=True)
            ol2, omx = _rel_diff(pm_i, p_int)
            fl2, fmx = _rel_diff(p64_i, p_int)
            oracle = {"rel_l2_mixed": ol2, "rel_max_mixed": omx, "rel_l2_fp64": fl2, "rel_max_fp64": fmx,
                      "oracle_rel_res": _residual_rel(A, p_int, A[7]), "oracle_iterations": it,
                      "residual_of_mixed": _residual_rel(A, pm_i, A[7])}
            del A
        gpu.upload(capi.F_P, pm)
        gpu.project_velocity(dt)
    R = np.array(rows)
    return {"mixed_vs_fp64_rel_l2_max": float(R[:, 0].max()), "mixed_vs_fp64_rel_max_max": float(R[:, 1].max()),
            "rel_res_mixed_max": float(R[:, 2].max()), "rel_res_fp64_max": float(R[:, 3].max()),
            "tolerance": REL_TOL, "steps": len(rows), "vs_oracle_step0": oracle,
            "note": "pressure differences after removing the mean (the periodic problem fixes p up to a constant)"}


# DRAM bytes per cell of the dominant kernel measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of one 256^3 launch,
# 348.7 MB + 57.0 MB over 16,777,216 cells): fills roofline.traffic, scaled by
# the cells a launch processes
NCU_DRAM_BYTES_PER_CELL = {"mg_sweep_f32": (348.717568e6 + 57.026816e6) / 16777216}


def roofline(report, peak):
    rows = []
    for name, (n, ms, cells) in report.items():
        b = ALGO_BYTES.get(name)
        gbs = b * cells / (ms * 1e-3) / 1e9 if (b and ms > 0) else None
        rows.append({"kernel": name, "launches": n, "ms": round(ms, 4),
                     "algo_bytes_per_launch": (b * cells / n) if b else None,
                     "gbs": round(gbs, 1) if gbs else None,
                     "frac": round(gbs / peak, 3) if gbs else None})
    rows.sort(key=lambda r: -r["ms"])
    return rows


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
class CpuReference:
    """The reference algorithm on the host cores (the FP64 restatement in
    oracle/, OpenMP over all cores): vofsweeps, linfunc, SetupPoisson, the
    reference multigrid (NewSolverMG, MGsolver.f90:346-405: V-cycles from
    p = 0 until the RMS residual is below 1e-10 of the RMS right-hand side,
    with the reference's default relaxation factor BETA = 1.2) and
    project_velocity, on the same workload.

    The reference multigrid converges slowly at density ratio 1000: on this
    workload it needs 225 cycles at 64^3 (309 with BETA = 1), and more at
    higher resolution, so a complete step at 256^3 takes longer than a timing
    run can give it.  Each step therefore runs the
    V-cycles until the tolerance or until its time budget is spent, whichever
    comes first.  A step that stops at its budget has done less work than the
    reference needs, so the steps/s measured is an upper bound of the
    reference's: a measurement, not a model."""

    def __init__(self, pkg, desc, us, dt, cvof=None, flag=None, cen=None, rad=None):
        from oracle import pyoracle as orc
        self.orc, self.capi, self.desc, self.dt = orc, pkg.capi, desc, dt
        self.us = us
        if cvof is None:
            cvof, flag, _ = orc.init_spheres(desc, cen, rad, refinement=8)
        self.c, self.f = cvof.copy(), flag.copy()
        self.u = [a.copy() for a in us]
        self.cores = len(os.sched_getaffinity(0))
        self.log = []

    def step(self, k, budget_s):
        """One step with at most budget_s seconds of V-cycles (after the first
        cycle); returns its wall time."""
        orc, d = self.orc, self.desc
        t0 = time.perf_counter()
        orc.vofsweeps(d, k, self.dt, self.c, self.f, *self.u)
        rho = orc.linfunc(d, self.c, d.rho1, d.rho2, self.capi.MEAN_ARITH)
        self.u = [a.copy() for a in self.us]
        st, A = orc.setup_poisson(d, *self.u, rho, self.dt)
        rms_b = float(np.sqrt(np.mean(A[7] ** 2)))
        p = orc.zeros(d)
        ok, cycles, tres, _ = orc.new_solver_mg_timed(d, A, p, REL_TOL * rms_b, budget_s, beta=REF_BETA)
        orc.project_velocity(d, *self.u, p, rho, self.dt)
        t = time.perf_counter() - t0
        self.log.append({"s": round(t, 2), "cycles": cycles, "converged": bool(ok), "rel_res": tres / rms_b})
        return t


def projection_config(n, world):
    """The workload of both arms (the same dict)."""
    return {"workload": f"{n}^3 periodic unit cube, 64 drops r~U[0.03,0.08] (seed 0), rho 1000/1, smoothed Gaussian "
                        "u* (seed 1); per step CIAM vofsweeps, linfunc, SetupPoisson, the pressure solve from p=0 to "
                        "||r||/||b|| < 1e-10, project_velocity",
            "cells": n ** 3, "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (141 MB per field)"}


REF_SOLVER = "reference MG (MGsolver.f90 NewSolverMG, nrelax=3, BETA=1.2), FP64, on the host cores"


def run_reference(args, dist):
    pkg = load_pkg()
    if dist.rank != 0:
        return 0
    n = args.n
    desc, cen, rad, us, dt = workload(pkg, n)
    ref = CpuReference(pkg, desc, us, dt, cen=cen, rad=rad)
    # warm-up: the step's fixed work and one V-cycle each
    for k in range(args.warmup):
        ref.step(k, 1e-9)
    budget = args.ref_budget / max(1, args.steps)
    ts = [ref.step(args.warmup + k, budget) for k in range(args.steps)]
    t_mean = float(np.mean(ts))
    v = 1.0 / t_mean
    steps_log = ref.log[args.warmup:]
    conv = sum(1 for r in steps_log if r["converged"])
    sample = (f"each step complete at {n}^3 (VOF, linfunc, SetupPoisson, project_velocity) with reference V-cycles "
              f"until ||r||/||b|| < 1e-10 or a {budget:.1f} s budget: {conv} of {args.steps} steps converged, "
              f"{min(r['cycles'] for r in steps_log)}-{max(r['cycles'] for r in steps_log)} cycles per step, "
              f"residual reached <= {max(r['rel_res'] for r in steps_log):.2e}; "
              + ("steps/s as measured" if conv == args.steps else
                 "steps/s measured over the truncated steps, an upper bound of the reference's"))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mean * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": projection_config(n, args.gpus), "solver": REF_SOLVER,
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": ref.cores, "kind": "port", "sample": sample,
                         "upper_bound": conv < args.steps},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "steps_log": steps_log,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_b200(args, dist):
    import torch
    pkg = load_pkg()
    capi, runtime = pkg.capi, pkg.runtime
    dev = dist.local
    torch.cuda.set_device(dev)
    n = args.n
    desc, cen, rad, us, dt = workload(pkg, n, device=dev)
    gpu = runtime.ParisGpu(desc)
    gpu.init_spheres(cen, rad, refinement=8)
    for f, a in zip((capi.F_USTAR, capi.F_VSTAR, capi.F_WSTAR), us):
        gpu.upload(f, a)
    for dst, src in ((capi.F_U, capi.F_USTAR), (capi.F_V, capi.F_VSTAR), (capi.F_W, capi.F_WSTAR)):
        gpu.copy_field(dst, src)
    # initial projection gives the divergence-free velocity the first sweep uses
    gpu.linfunc(capi.F_RHO)
    gpu.setup_poisson(dt)
    gpu.fill_field(capi.F_P, 0.0)
    gpu.new_solver(0.0, maxit=200, mode=capi.MG_MIXED, rel_tol=REL_TOL, pcg=args.pcg, nu1=NU[0], nu2=NU[1], beta=OMEGA[0],
                       nu_coarse=NU[2], coarse_from=NU[3], coarse_to=NU[4], beta_coarse=OMEGA[1])
    gpu.project_velocity(dt)
    cvof0 = gpu.download(capi.F_CVOF) if (dist.rank == 0 and not args.no_cpu_baseline) else None
    flag0 = gpu.download(capi.F_VOF_FLAG) if cvof0 is not None else None
    stream = torch.cuda.ExternalStream(gpu.stream())
    peak, peak_kind = measured_peak()

    if args.profile_only:
        # the steps alone form the NVTX range "paris_steps" (ncu --nvtx-include)
        gpu.profile(True)
        gpu.sync()
        torch.cuda.nvtx.range_push("paris_steps")
        for k in range(max(1, args.steps)):
            gpu_step(gpu, capi, k, dt, capi.MG_MIXED, args.pcg)
        gpu.sync()
        torch.cuda.nvtx.range_pop()
        gpu.profile(False)
        rep = gpu.profile_report()
        if dist.rank == 0:
            print(json.dumps({"profile": roofline(rep, peak)}), flush=True)
        gpu.close()
        return 0

    # every timed run starts from the same state (the drops after the
    # initial projection), so the solvers see the same sequence of problems
    snap = {f: gpu.download(f) for f in (capi.F_CVOF, capi.F_VOF_FLAG, capi.F_U, capi.F_V, capi.F_W)}

    def reset():
        for f, a in snap.items():
            gpu.upload(f, a)
        gpu.sync()

    def timed(mode, steps, k0, pcg=args.pcg):
        reset()
        for k in range(args.warmup):
            gpu_step(gpu, capi, k0 + k, dt, mode, pcg)
        gpu.sync()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = []
        l0 = gpu.launch_count()
        e0.record(stream)
        for k in range(steps):
            r = gpu_step(gpu, capi, k0 + args.warmup + k, dt, mode, pcg)
            its.append(r.it)
        e1.record(stream)
        e1.synchronize()
        gpu.sync()
        launches = gpu.launch_count() - l0
        ms = dist.max(e0.elapsed_time(e1))
        dist.barrier()
        return ms, its, launches

    clocks = Clocks(dev)
    clocks.start()
    ms, its, launches = timed(capi.MG_MIXED, args.steps, 0)
    clk = clocks.stop()
    ms64, its64, _ = timed(capi.MG_FP64, args.steps, 0)
    msdc, itsdc, _ = timed(capi.MG_MIXED, args.steps, 0, pcg=1 - args.pcg)

    # per-kernel CUDA-event profile of the same step (separate, after timing)
    reset()
    gpu.profile(True)
    for k in range(2):
        gpu_step(gpu, capi, 2000 + k, dt, capi.MG_MIXED, args.pcg)
    gpu.profile(False)
    report = gpu.profile_report()
    rows = roofline(report, peak)
    top = rows[0]
    perr = pressure_error(gpu, capi, args, dt, reset, cpu_oracle=(dist.rank == 0 and not args.no_cpu_baseline))
    # summed kernel time per step (the rest of ms_per_step is the GPU waiting
    # on the host between launches)
    kernel_ms_per_step = sum(ms for _, ms, _ in report.values()) / 2

    # end to end through the C-ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        shape = us[0].shape
        h_in = [torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
        for h, a in zip(h_in, us):
            h[...] = a
        h_out = [torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
        e_steps = max(1, args.steps)
        ins = (capi.F_USTAR, capi.F_VSTAR, capi.F_WSTAR)
        outs = (capi.F_U, capi.F_V, capi.F_W, capi.F_CVOF)

        def e2e_run(pipelined):
            reset()
            dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            if pipelined:
                # step k+1's inputs go up while step k runs, step k's results come
                # down while step k+1 runs (paris_gpu_upload_async / _upload_commit /
                # _download_async)
                for f, h in zip(ins, h_in):
                    gpu.upload_async(f, h)
                for k in range(e_steps):
                    for f in ins:
                        gpu.upload_commit(f)
                    if k + 1 < e_steps:
                        for f, h in zip(ins, h_in):
                            gpu.upload_async(f, h)
                    gpu_step(gpu, capi, k, dt, capi.MG_MIXED, args.pcg)
                    for f, h in zip(outs, h_out):
                        gpu.download_async(f, h)
                gpu.sync_transfers()
            else:
                for k in range(e_steps):
                    for f, h in zip(ins, h_in):
                        gpu.upload_from(f, h)
                    gpu_step(gpu, capi, k, dt, capi.MG_MIXED, args.pcg)
                    for f, h in zip(outs, h_out):
                        gpu.download_into(f, h)
            e1.record(stream)
            e1.synchronize()
            wall = time.perf_counter() - t0
            ems = dist.max(e0.elapsed_time(e1))
            dist.barrier()
            return ems, wall

        ems, wall = e2e_run(True)
        ems_sync, _ = e2e_run(False)
        nb = int(np.prod(shape)) * 8
        e2e = {"value": dist.world * e_steps / (ems / 1e3), "unit": "steps/s", "h2d_bytes_per_step": 3 * nb,
               "d2h_bytes_per_step": 4 * nb, "steps": e_steps, "host_wall_s": round(wall, 3),
               "transfers": "pinned host buffers, asynchronous uploads and downloads overlapped with the steps",
               "sync_transfers_steps_per_s": dist.world * e_steps / (ems_sync / 1e3)}

    cpu = None
    if dist.rank == 0 and not args.no_cpu_baseline:
        ref = CpuReference(pkg, desc, us, dt, cvof=cvof0, flag=flag0)
        t = ref.step(1, args.cpu_budget)
        r = ref.log[-1]
        cpu = {"value": 1.0 / t, "unit": "steps/s", "cores": ref.cores, "kind": "port",
               "sample": f"one step at {n}^3 (VOF, linfunc, SetupPoisson, project_velocity) with reference "
                         f"V-cycles until ||r||/||b|| < 1e-10 or {args.cpu_budget:.0f} s: {r['cycles']} cycles, "
                         f"residual {r['rel_res']:.2e}, {t:.1f} s; "
                         + ("complete" if r["converged"] else "truncated, so the steps/s is an upper bound"),
               "upper_bound": not r["converged"]}
    gpu.close()
    if dist.rank != 0:
        return 0
    value = dist.world * args.steps / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": projection_config(n, dist.world),
        "solver": (f"B200 MG: FP32 red-black V({NU[0]},{NU[1]}) cycles" +
                   (f" ({NU[2]} sweeps each way on levels {NU[3]}.." + (str(NU[4]) if NU[4] else "coarsest") + ")"
                    if NU[2] else "") +
                   (f" (over-relaxed, factor {OMEGA[0]}" + (f"; {OMEGA[1]} below the finest level" if OMEGA[1] > 0 else "")
                    + ")" if OMEGA[0] != 1.0 or OMEGA[1] > 0 else "") + " in an FP64 " +
                   ("flexible-CG (preconditioner) loop" if args.pcg else "defect-correction loop")),
        "fp64_steps_per_s": dist.world * args.steps / (ms64 / 1e3),
        ("mixed_dc_steps_per_s" if args.pcg else "mixed_pcg_steps_per_s"): dist.world * args.steps / (msdc / 1e3),
        "mg_iterations": {"mixed": its, "fp64": its64, ("mixed_dc" if args.pcg else "mixed_pcg"): itsdc},
        "pressure_error": perr,
        "mcell_updates_per_s": value * n ** 3 / 1e6,
        "gpu_launches": launches,
        "kernel_ms_per_step": round(kernel_ms_per_step, 3),
        "roofline": {"bound": "hbm", "kernel": top["kernel"], "achieved": top["gbs"], "peak": peak,
                     "unit": "GB/s", "frac": top["frac"],
                     "traffic": (NCU_DRAM_BYTES_PER_CELL[top["kernel"]] * top["algo_bytes_per_launch"] /
                                 ALGO_BYTES[top["kernel"]] if top["kernel"] in NCU_DRAM_BYTES_PER_CELL else None),
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "algo_bytes_per_launch": top["algo_bytes_per_launch"]},
        "kernels": rows[:20],
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# rising bubble: the full explicit Navier-Stokes step
BUBBLE = {"radius": 0.125, "centre": (0.5, 0.5, 0.5), "rho_l": 1000.0, "rho_g": 1.0, "mu_l": 1e-3, "mu_g": 1e-5,
          "sigma": 0.0245, "gravity": (0.0, 0.0, -9.81), "cfl": 0.5, "max_dt": 5e-4}
BUBBLE_METRIC = "steps/s, rising bubble 512x512x1024, full NS step (mixed MG to 1e-9)"
# The pressure of this flow carries the hydrostatic field (|p| up to 1.4e4)
# and the face coefficients dt/(rho h^2) reach 131 in the gas at h = 1/512:
# p itself is stored to ~1e-12, which bounds the true residual near 1.2e-10
# of ||b||.  The solve stops at 1e-9, above that floor.
BUBBLE_REL_TOL = 1e-9


def bubble_desc(capi, n, device=0):
    """The walled box [0,1]x[0,1]x[0,2] at h = 1/n.  Phase 2 (cvof = 1, inside
    the sphere) is the gas, phase 1 the liquid: PARIS's input checks
    (paris.f90:3750-3773) then read dx^2 rho_l/(MaxDt mu_l) >= 6 and
    dx^3 rho_l/(MaxDt^2 sigma) >= 2, both met by MaxDt = 5e-4 at n = 512."""
    B = BUBBLE
    return capi.make_desc((n, n, 2 * n), length=(1.0, 1.0, 2.0), bc="wall", rho1=B["rho_l"], rho2=B["rho_g"],
                          mu1=B["mu_l"], mu2=B["mu_g"], sigma=B["sigma"], device=device)


def bubble_config(n, world=1):
    B = BUBBLE
    return {"workload": f"rising bubble: walled box [0,1]x[0,1]x[0,2] at {n}x{n}x{2 * n} (h=1/{n}), gas bubble "
                        f"R={B['radius']} at {B['centre']}, rho {B['rho_l']:g}/{B['rho_g']:g}, mu "
                        f"{B['mu_l']:g}/{B['mu_g']:g} (mu_l chosen: water-like), sigma {B['sigma']}, g=-9.81 in z; "
                        "full explicit NS step (QUICK convection, CIAM VOF, heights, curvature, CSF, explicit "
                        "viscosity, gravity, projection by the B200 mixed MG to ||r||/||b|| < 1e-9 from the "
                        f"previous p); dt from TimeStepSize (CFL {B['cfl']}, MaxDt {B['max_dt']}) each step",
            "cells": n * n * 2 * n, "parallelism": f"replicas x{world}", "l2": "inputs larger than L2"}


def bubble_cpu_sample(pkg, n_cpu, steps=2, warmup=1):
    """The reference step on the host cores (the oracle's ns_step, reference
    MG to the same relative residual) on the same bubble at n_cpu x n_cpu x
    2 n_cpu, from rest; returns (seconds per step, cells, cores)."""
    from oracle import pyoracle as orc
    capi, B = pkg.capi, BUBBLE
    d = bubble_desc(capi, n_cpu)
    cvof, flag, _ = orc.init_spheres(d, [B["centre"]], [B["radius"]], refinement=8)
    st = {"cvof": cvof, "flag": flag, "u": orc.zeros(d), "v": orc.zeros(d), "w": orc.zeros(d), "p": orc.zeros(d)}
    ts = []
    for k in range(1, warmup + steps + 1):
        t0 = time.perf_counter()
        dt, _ = orc.time_step_size(d, st["u"], st["v"], st["w"], B["cfl"], B["max_dt"])
        orc.ns_step(d, st, k, dt, gravity=B["gravity"], rel_tol=BUBBLE_REL_TOL, maxit=4000)
        if k > warmup:
            ts.append(time.perf_counter() - t0)
    return float(np.mean(ts)), n_cpu * n_cpu * 2 * n_cpu, len(os.sched_getaffinity(0))


def run_bubble_reference(args, dist):
    pkg = load_pkg()
    if dist.rank != 0:
        return 0
    n, n_cpu = args.n, min(args.n, 32)
    t, cells, cores = bubble_cpu_sample(pkg, n_cpu, steps=max(1, min(args.steps, 3)), warmup=min(args.warmup, 1))
    full = n * n * 2 * n
    v = cells / full / t   # steps/s at the full size, from the per-cell rate of the sample
    line = {
        "impl": "reference", "metric": BUBBLE_METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": bubble_config(n),
        "mcell_updates_per_s": cells / t / 1e6,
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"the oracle's step (reference MG) at {n_cpu}x{n_cpu}x{2 * n_cpu} from rest, "
                                   f"{t:.2f} s per step, scaled by cells to {n}x{n}x{2 * n}"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_bubble(args, dist):
    import torch
    pkg = load_pkg()
    capi, runtime, B = pkg.capi, pkg.runtime, BUBBLE
    dev = dist.local
    torch.cuda.set_device(dev)
    n = args.n
    gpu = runtime.ParisGpu(bubble_desc(capi, n, dev))
    gpu.init_spheres([B["centre"]], [B["radius"]], refinement=8)
    for f in (capi.F_U, capi.F_V, capi.F_W, capi.F_P):
        gpu.fill_field(f, 0.0)
    gpu.linfunc(capi.F_RHO)
    gpu.linfunc(capi.F_MU)
    stream = torch.cuda.ExternalStream(gpu.stream())
    peak, peak_kind = measured_peak()
    s0 = gpu.calc_stats(force_valid=0)
    k = [0]
    solve = {"max_error": 0.0, "rel_tol": BUBBLE_REL_TOL, "maxit": 200, "mode": capi.MG_MIXED, "pcg": 1,
             "beta": OMEGA[0], "nu1": NU[0], "nu2": NU[1], "nu_coarse": NU[2], "coarse_from": NU[3],
             "coarse_to": NU[4], "beta_coarse": OMEGA[1]}

    def step():
        dt, _ = gpu.time_step_size(B["cfl"], B["max_dt"])     # TimeStepSize, dtFlag 2
        k[0] += 1
        return dt, gpu.ns_step(k[0], dt, gravity=B["gravity"], solve=solve)

    if args.profile_only:
        for _ in range(args.warmup):
            step()
        gpu.profile(True)
        gpu.sync()
        torch.cuda.nvtx.range_push("paris_steps")
        for _ in range(max(1, args.steps)):
            step()
        gpu.sync()
        torch.cuda.nvtx.range_pop()
        gpu.profile(False)
        if dist.rank == 0:
            print(json.dumps({"profile": roofline(gpu.profile_report(), peak)}), flush=True)
        gpu.close()
        return 0

    for _ in range(args.warmup):
        step()
    gpu.sync()
    dist.barrier()
    clocks = Clocks(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dts, its = [], []
    l0 = gpu.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        dt, r = step()
        dts.append(dt)
        its.append(r.it)
    e1.record(stream)
    e1.synchronize()
    gpu.sync()
    clk = clocks.stop()
    launches = gpu.launch_count() - l0
    ms = dist.max(e0.elapsed_time(e1))
    dist.barrier()
    # per-kernel CUDA-event profile of two more steps
    gpu.profile(True)
    for _ in range(2):
        step()
    gpu.profile(False)
    report = gpu.profile_report()
    rows = roofline(report, peak)
    kernel_ms_per_step = sum(m for _, m, _ in report.values()) / 2
    # end to end: each step also reads back its statistics line, as the
    # reference's loop does with nstats = 1 (the state stays on the device)
    e_steps = max(1, min(args.steps, 10))
    opts = capi.make_stats_opts(gravity=B["gravity"])
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        step()
        s1 = gpu.calc_stats(opts)
    e1.record(stream)
    e1.synchronize()
    ems = dist.max(e0.elapsed_time(e1))
    dist.barrier()
    zc = gpu.download(capi.F_CVOF)
    g = 2
    cells = n * n * 2 * n
    vol0, vol1 = s0[9], s1[9]
    # bubble centre height: the cvof-weighted mean of z over the interior
    zcen = (np.arange(2 * n) + 0.5) / n
    ci = zc[g:-g, g:-g, g:-g]
    zbub = float((ci.sum(axis=(1, 2)) * zcen).sum() / ci.sum())
    cpu = None
    if dist.rank == 0 and not args.no_cpu_baseline:
        n_cpu = min(n, 32)
        t, ccells, cores = bubble_cpu_sample(pkg, n_cpu)
        cpu = {"value": ccells / cells / t, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": f"the oracle's step (reference MG) at {n_cpu}x{n_cpu}x{2 * n_cpu} from rest, "
                         f"{t:.2f} s per step, scaled by cells to {n}x{n}x{2 * n}"}
    gpu.close()
    if dist.rank != 0:
        return 0
    value = dist.world * args.steps / (ms / 1e3)
    top = rows[0]
    line = {
        "metric": BUBBLE_METRIC, "value": value, "unit": "steps/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic", "config": bubble_config(n, dist.world),
        "mcell_updates_per_s": value * cells / 1e6,
        "dt": [min(dts), max(dts)], "mg_iterations": its, "gpu_launches": launches,
        "kernel_ms_per_step": round(kernel_ms_per_step, 3),
        "gas_volume": {"initial": vol0, "final": vol1, "rel_change": abs(vol1 - vol0) / vol0},
        "bubble_centre_z": zbub,
        "roofline": {"bound": "hbm", "kernel": top["kernel"], "achieved": top["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": top["frac"], "traffic": None,
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "algo_bytes_per_launch": top["algo_bytes_per_launch"]},
        "kernels": rows[:20],
        "clocks": clk,
        "e2e": {"value": dist.world * e_steps / (ems / 1e3), "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8 * (capi.NSTATS + 2), "steps": e_steps,
                "note": "state resident on the device; per step the time step and the statistics line "
                        "come back to the host"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    NU[:] = [args.nu1, args.nu2, args.nu_coarse, args.coarse_from, args.coarse_to]
    OMEGA[:] = [args.beta, args.beta_coarse]
    if args.n is None:
        args.n = 512 if args.workload == "rising_bubble" else 256
    dist = Dist()
    try:
        if args.workload == "rising_bubble":
            rc = run_bubble_reference(args, dist) if args.impl == "reference" else run_bubble(args, dist)
        else:
            rc = run_reference(args, dist) if args.impl == "reference" else run_b200(args, dist)
    finally:
        dist.close()
    return rc


if __name__ == "__main__":
    sys.exit(main())
