#!/usr/bin/env python
"""Benchmark of the fully-coupled density-based step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload swept_wing_fp32|...]

Metric: cell-iterations per second (cells x nonlinear iterations / s) of
the implicit step (flux + residual, Roe Jacobian assembly, preconditioner
set-up, Krylov solve, field update, time-step control) on one workload.
`value` is device time of whole steps with the state resident in HBM
(CUDA events on the library's stream); `e2e` is the same metric through
the C ABI with the state copied host->device before and device->host
after every step.  Multi-GPU runs are independent replicas (the path does
not shard on one GPU's worth of mesh), one per rank, max time over ranks.

The `reference` arm times the CPU restatement of the reference's step
(the FP64 oracle; rhoDST itself needs foam-extend, absent on this box) on
the same workload and configuration.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def precision_desc(options: dict) -> str:
    prec = options.get("precision", "fp64")
    basis = "fp64" if basis_bytes(options) == 8 else "fp32"
    return (f"Jacobian/ILU {prec}, GMRES basis {basis}; residual, update, dots, Hessenberg "
            f"and norms fp64")


def workload(name: str):
    from rhodst_b200 import cases
    if name == "forward_step_2d":
        c = cases.forward_step_c1()
        desc = {"workload": "forward_step_2d", "mesh": "120x40 minus step, hex, one cell thick",
                "cells": c.mesh.n_cells, "internal_faces": c.mesh.n_internal_faces,
                "flux": "Kurganov", "reconstruction": "OSPRE/OSPREV", "ddt": "Euler, CFL 0.8 global dt",
                "solver": "GMRES(20), 1 restart cycle", "preconditioner": "block Jacobi",
                "precision": "fp64"}
        return c, desc
    if name.startswith("swept_wing"):
        prec = name.split("_")[-1] if name.count("_") >= 2 else "fp32"
        c = cases.swept_wing_c3(precision=prec)
        desc = {"workload": name, "mesh": "swept tapered NACA0012 wing, O-H hex 192x64x98",
                "cells": c.mesh.n_cells, "internal_faces": c.mesh.n_internal_faces,
                "flux": "HLLC", "reconstruction": "OSPRE/OSPREV", "ddt": "steadyStateDST local dt, CFL ramp 5->50",
                "solver": "GMRES(20), 1 restart cycle", "preconditioner": "subdomain block ILU(0)",
                "precision": precision_desc(c.options), "mach": 0.84, "alpha_deg": 3.06}
        return c, desc
    if name.startswith("naca0012_sa"):
        prec = name.split("_")[-1] if name.count("_") >= 2 else "fp64"
        c = cases.naca0012_turbulent().with_options(precision=prec)
        desc = {"workload": name, "mesh": "NACA0012 C-mesh 257x65, wall y+~1, far field 20 c",
                "cells": c.mesh.n_cells, "internal_faces": c.mesh.n_internal_faces,
                "flux": "AUSM+up", "reconstruction": "Venkatakrishnan", "turbulence": "SAneg",
                "ddt": "steadyStateDST local dt, CFL ramp 2->50", "solver": "GMRES(30), 1 restart cycle",
                "preconditioner": "subdomain block ILU(0)", "mach": 0.73, "alpha_deg": 2.3, "reynolds": 6.5e6,
                "precision": precision_desc(c.options)}
        return c, desc
    if name.startswith("forward_step_3d"):
        prec = name.split("_")[-1] if name.count("_") >= 3 else "fp32"
        c = cases.forward_step_3d_hybrid_c5(precision=prec)
        desc = {"workload": name, "mesh": "3D forward step, hybrid prism/tet from a 240x80x56 lattice, interior nodes "
                                          "jittered up to 25 % (seed 20240601)",
                "cells": c.mesh.n_cells, "internal_faces": c.mesh.n_internal_faces, "flux": "HLLC",
                "reconstruction": "Venkatakrishnan", "ddt": "steadyStateDST local dt, CFL 0.5->5",
                "solver": "GMRES(20), 1 restart cycle", "preconditioner": "subdomain block ILU(0)",
                "precision": precision_desc(c.options), "mach": 3.0}
        return c, desc
    raise SystemExit(f"unknown workload {name}")


# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        smax = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def traffic_per_launch(workload: str, kernel: str):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summary (profiles/traffic.json), or None when none was captured."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text()).get(workload, {})
    return d.get(kernel)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic (compulsory) bytes per launch of each kernel class; S = bytes
# per stored matrix scalar, Bk = N + 2F blocks, 4-byte column indices.
def algorithmic_bytes(kind: str, N: int, F: int, S: int, precon: str, vb: int = 8, m: int = 20) -> float:
    """Bytes one launch of a kernel class must move at least: S bytes per
    Jacobian/factor entry (8 fp64, 4 fp32, 2 bf16), vb per Krylov basis
    entry, m GMRES directions per restart cycle."""
    Bk = N + 2 * F
    if kind == "spmv":
        # matrix + column ids, x (a basis vector: vb per entry), y fp64
        return 25 * S * Bk + 4 * Bk + 5 * vb * N + 40 * N
    if kind == "precond":
        if precon == "diagonal":
            return 25 * S * N + 40 * N + 40 * N
        return 25 * S * Bk + 4 * Bk + 3 * 40 * N
    if kind == "flux":
        # q (64 B) + gradient (192 B) per cell, 72 B geometry + 40 B flux per face
        return 256 * N + 112 * F
    if kind == "assemble":
        return 25 * S * Bk + 4 * Bk + 104 * N + 72 * F
    if kind == "factor":
        return 2 * (25 * S * Bk + 4 * Bk) + 25 * S * N
    if kind == "orth":
        # one GMRES direction of CGS2 at the mean basis size J = (m+1)/2:
        # three passes over the J basis vectors (dots; axpy fused with the
        # second dots; axpy fused with the norm) and five passes over w
        # (read; read+write; read+write), w in fp64
        J = (m + 1) / 2.0
        return N * (3 * J * 5 * vb + 5 * 40)
    return 0.0


def basis_bytes(options: dict) -> int:
    """Bytes per Krylov basis entry: fp32 unless the Jacobian is fp64 (the
    library default), or as set by krylov.basis."""
    b = options.get("krylov", {}).get("basis") if isinstance(options.get("krylov"), dict) else options.get("krylov.basis")
    if b is None:
        b = "fp64" if options.get("precision", "fp64") == "fp64" else "fp32"
    return 8 if b == "fp64" else 4


def max_over_ranks(x: float) -> float:
    """The maximum of x over the ranks of the default process group (the
    job's time is its slowest rank's); x itself without one."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world):
    import torch
    import rhodst_b200
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    case, desc = workload(args.workload)
    opts = dict(case.options)
    opts["profile"] = False          # timed steps run without per-kernel events
    opts["device"] = dev             # the library's own CUDA runtime: name this rank's GPU
    s = rhodst_b200.Solver(case.mesh, case.bcs, opts)
    s.set_primitive(case.p, case.U, case.T)
    N, F = case.mesh.n_cells, case.mesh.n_internal_faces
    # L2 flush buffer (larger than the 126 MB L2), written on the library's stream
    stream = torch.cuda.ExternalStream(s.stream_handle())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB
    for _ in range(args.warmup):
        s.step(1)
    launches0 = s.launch_count()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms = []
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            s.step(1)                      # returns after its own stream synchronize
            step_ms.append(s.last_step_ms())
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches = s.launch_count() - launches0
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks(total_ms)
    value = world * N * args.steps / (total_ms * 1e-3)
    # kernel classes and the roofline of the dominant one: CUDA events around
    # each launch (on the library's stream) over a separate run of the same
    # number of steps (capped at 10), L2 flushed between steps as above
    s.set_profile(True)
    s.step(1)
    classes = ("spmv", "precond", "flux", "assemble", "factor", "orth", "update")
    stats0 = {k: s.kernel_stats(k) for k in classes}
    prof_steps = min(args.steps, 10)
    prof_ms = 0.0
    for _ in range(prof_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        s.step(1)
        prof_ms += s.last_step_ms()
    s.set_profile(False)
    stats = {k: tuple(np.subtract(s.kernel_stats(k), stats0[k])) for k in classes}
    prec0 = case.options.get("precision", "fp64")
    S0 = 8 if prec0 == "fp64" else (4 if prec0 == "fp32" else 2)
    pc0 = case.options["solvers"]["W"]["preconditioner"]
    vb0 = basis_bytes(case.options)
    m0 = int(case.options["solvers"]["W"].get("nDirections", 20))
    breakdown = {}
    for k, (nl_, ms_) in stats.items():
        if nl_ <= 0:
            continue
        by_ = algorithmic_bytes(k, N, F, S0, pc0, vb0, m0)
        breakdown[k] = {"launches": int(nl_), "avg_us": round(ms_ / nl_ * 1e3, 2),
                        "share_of_step": round(ms_ / max(prof_ms, 1e-9), 4),
                        "GBps": round(by_ / (ms_ / nl_ * 1e-3) / 1e9, 1) if by_ else None}
    dom = max(stats, key=lambda k: stats[k][1])
    n_l, ms_l = stats[dom]
    prec = case.options.get("precision", "fp64")
    S = 8 if prec == "fp64" else (4 if prec == "fp32" else 2)
    precon = case.options["solvers"]["W"]["preconditioner"]
    peak, peak_kind = measured_peaks()
    roof = None
    if n_l > 0 and ms_l > 0:
        by = algorithmic_bytes(dom, N, F, S, precon, vb0, m0)
        ach = by / (ms_l / n_l * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "peak_source": f"{peak_kind} hbm_gbs",
                "bytes_per_launch": by, "launches": int(n_l), "avg_launch_us": round(ms_l / n_l * 1e3, 3),
                "traffic": traffic_per_launch(args.workload, dom),
                "share_of_step": round(ms_l / max(prof_ms, 1e-9), 4),
                "note": "working set below L2 (126 MB): L2-resident bandwidth" if
                        (25 * S * (N + 2 * F)) < 100e6 else "HBM-resident"}
    # e2e through the C ABI with host buffers: H2D state, step, D2H state
    rho, rhoU, rhoE = s.conservative()
    e2e_steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.set_conservative(rho, rhoU, rhoE)
        s.step(1)
        rho, rhoU, rhoE = s.conservative()
    e2e_t = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * N * e2e_steps / e2e_t, "unit": "cell-iter/s",
           "h2d_bytes_per_step": int(rho.nbytes + rhoU.nbytes + rhoE.nbytes + 8 * 8 * N),
           "d2h_bytes_per_step": int(rho.nbytes + rhoU.nbytes + rhoE.nbytes)}
    line = {"metric": "cell_iterations_per_s", "value": value, "unit": "cell-iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == "fp64" else (f"f64 residual/dots/Hessenberg, {prec} Jacobian+ILU, "
                                                  f"{'f32' if vb0 == 4 else 'f64'} Krylov basis"),
            "data": "synthetic (generated mesh, uniform free-stream initial state)",
            "config": dict(desc, l2="flushed: 256 MB written between timed steps",
                           parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
            "clocks": clk.summary(), "e2e": e2e, "gpu_launches": int(launches), "roofline": roof,
            "kernels": breakdown, "kernels_profiled_ms_per_step": round(prof_ms / max(prof_steps, 1), 3)}
    return line, case, s


def _run_to_drop(case, opts, drop, max_steps, chunk=50):
    """Steps of a fresh context until ||R_rho V||_2 falls by `drop` from the
    first step's value (or max_steps): steps to the drop, device seconds,
    the drop history every `chunk` steps, the context."""
    import rhodst_b200
    s = rhodst_b200.Solver(case.mesh, case.bcs, dict(opts, profile=False))
    s.set_primitive(case.p, case.U, case.T, case.nuTilda)
    r0, steps, dev_ms, hit, hist = None, 0, 0.0, None, []
    while steps < max_steps and hit is None:
        reps = s.step(chunk)
        dev_ms += s.last_step_ms()
        for r in reps:
            steps += 1
            if r0 is None:
                r0 = r["res_l2"][0]
            if hit is None and r["res_l2"][0] <= drop * r0:
                hit = steps
        hist.append(float("%.3g" % (reps[-1]["res_l2"][0] / r0)))
    return {"steps": hit, "steps_run": steps, "device_s": dev_ms * 1e-3, "final_drop": hist[-1],
            "history_every_%d" % chunk: hist}, s


def convergence_and_adjoint(case, drop: float = 1e-10, max_steps: int = 1500):
    """Time to a density-residual drop of `drop`, FP64 against reduced
    precision, on three configurations:

    * wing, its own scheme (HLLC, OSPRE/OSPREV, local time step ramped to
      CFL 50), FP64 and FP32, up to 600 steps: where it stalls, the stall
      level and the history;
    * wing, first-order HLL at CFL 500 (a proxy that converges: the
      speed-up figures of mixed precision), FP64 / FP32 / BF16, with C_l
      and C_d of each;
    * C2, the 257x65 turbulent NACA0012 (SAneg, AUSM+up + Venkatakrishnan,
      CFL 50), FP64, up to 3000 steps;

    then the discrete adjoint of the pressure-drag coefficient at the proxy's
    FP64 converged state, solved to the same `drop`, its cost against that
    forward solve, and dJ/dMach, dJ/dalpha."""
    import math
    from rhodst_b200 import cases
    g = case.options["thermo"]
    U0 = np.asarray(case.U[0], dtype=float)
    c_inf = math.sqrt(g["Cp"] / (g["Cp"] - g["R"]) * g["R"] * 1.0)
    alpha = math.atan2(U0[1], U0[0])
    drag = (math.cos(alpha), math.sin(alpha), 0.0)
    lift = (-math.sin(alpha), math.cos(alpha), 0.0)
    patch = case.force_patch
    ref_area = 0.1 if case.name.startswith("naca") else 1.5 * 0.5 * (1.0 + 0.56)
    qA = 0.5 * (1.0 / (g["R"] * 1.0)) * float(U0 @ U0) * ref_area
    out = {"drop": drop}
    # the configuration's own scheme
    own = {"config": "the workload's own scheme: HLLC, OSPRE/OSPREV, local time step ramped to CFL 50",
           "max_steps": 600}
    for prec in ("fp64", "fp32"):
        r, s = _run_to_drop(case, dict(case.options, precision=prec), drop, 600)
        own[prec] = r
        s.close()
    out["own_scheme"] = own
    # first-order proxy
    first = {"fluxScheme": "HLL", "timeControls": dict(case.options["timeControls"], maxCo=500.0),
             "interpolationSchemes": {"reconstruct(rho)": "upwind", "reconstruct(U)": "upwind",
                                      "reconstruct(T)": "upwind"}}
    prox = {"config": "proxy: same mesh and free stream, HLL, first-order (upwind) reconstruction, CFL 500",
            "max_steps": max_steps}
    solvers = {}
    for prec in ("fp64", "fp32", "bf16"):
        r, s = _run_to_drop(case, dict(case.options, **first, precision=prec), drop, max_steps)
        f = s.forces(patch, lift, drag, 1.0, qA)
        r.update(Cl=f["Cl"], Cd=f["Cd"])
        prox[prec] = r
        solvers[prec] = s
    if prox["fp64"]["steps"] and prox["fp32"]["steps"]:
        prox["speedup_mixed_over_fp64"] = prox["fp64"]["device_s"] / prox["fp32"]["device_s"]
    if prox["fp64"]["steps"] and prox["bf16"]["steps"]:
        prox["speedup_bf16_over_fp64"] = prox["fp64"]["device_s"] / prox["bf16"]["device_s"]
    for p in ("fp32", "bf16"):
        prox[p + "_Cl_rel_diff"] = abs(prox[p]["Cl"] - prox["fp64"]["Cl"]) / abs(prox["fp64"]["Cl"])
        prox[p + "_Cd_rel_diff"] = abs(prox[p]["Cd"] - prox["fp64"]["Cd"]) / abs(prox["fp64"]["Cd"])
    out["first_order_proxy"] = prox
    # C2 as configured
    c2 = cases.naca0012_turbulent()
    r, s = _run_to_drop(c2, c2.options, drop, 3000)
    r["config"] = "C2: NACA0012 257x65, Re 6.5e6, SAneg, AUSM+up + Venkatakrishnan, CFL 50, GMRES(30) + ILU(0)"
    out["c2_airfoil_fp64"] = r
    s.close()
    # adjoint at the proxy's FP64 state, to the same drop
    rep, _ = solvers["fp64"].adjoint(patch, drag, p_ref=1.0, scale=1.0 / qA, rel_tol=drop, max_cycles=60,
                                     n_directions=30)
    from rhodst_b200.shape import freestream_derivatives
    dJ_dM, dJ_da = freestream_derivatives(rep["dJ_dU"], rep["force"], U0, c_inf, lift)
    out["adjoint"] = {"objective": f"pressure drag coefficient of patch {patch}", "J": rep["J"],
                      "device_s": rep["t_ms"] * 1e-3, "outer_iterations": rep["iterations"],
                      "residual_drop": rep["residual"] / rep["residual0"],
                      "cost_over_forward": rep["t_ms"] * 1e-3 / prox["fp64"]["device_s"],
                      "dJ_dMach": dJ_dM, "dJ_dalpha_per_rad": dJ_da}
    for s in solvers.values():
        s.close()
    return out


def cpu_baseline(case, budget_s: float, steps_max: int, warmup: int = 1):
    """The oracle (CPU FP64 restatement of the reference step) on a bounded
    sample of the same workload, on all host cores: cells split by RCB into
    one subdomain per thread with ILU(0) per subdomain -- the reference run
    on that many processors, whose ILU drops the couplings across processor
    patches -- and, for scale, one core with one subdomain (exact ILU(0))."""
    from tests.oracle_lib import OracleSolver, set_threads
    N = case.mesh.n_cells

    def timed(threads, parts, budget, w):
        set_threads(threads)
        o = OracleSolver(case.mesh, case.bcs, case.options, rcb_parts=parts)
        o.set_primitive(case.p, case.U, case.T)
        if w:
            o.step(w)
        n = 0
        t0 = time.perf_counter()
        while n < steps_max and (n == 0 or (time.perf_counter() - t0) < budget):
            o.step(1)
            n += 1
        return n, time.perf_counter() - t0

    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    n, dt = timed(cores, cores, budget_s, warmup)
    out = {"value": N * n / dt, "unit": "cell-iter/s", "cores": cores, "kind": "port",
           "sample": f"{n} steps of the same workload after {warmup} warm-up step(s), {dt:.2f} s, "
                     f"{cores} threads, RCB into {cores} subdomains with ILU(0) per subdomain"}
    n1, dt1 = timed(1, 1, budget_s / 3, 0)
    out["single_core"] = {"value": N * n1 / dt1, "cores": 1,
                          "sample": f"{n1} step(s), {dt1:.2f} s, 1 thread, one subdomain (exact ILU(0))"}
    set_threads(0)
    return out


def run_converge(args):
    """Steps until the density residual ||R_rho V||_2 drops by args.converge
    relative to the first step; reports device time, steps and forces."""
    import torch
    import rhodst_b200
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    case, desc = workload(args.workload)
    s = rhodst_b200.solver_for(case)
    N = case.mesh.n_cells
    chunk = 50
    r0 = None
    steps, dev_ms, hist = 0, 0.0, []
    t0 = time.perf_counter()
    while steps < args.max_steps:
        reps = s.step(chunk)
        dev_ms += s.last_step_ms()
        for r in reps:
            steps += 1
            if r0 is None:
                r0 = r["res_l2"][0]
            hist.append(r["res_l2"][0] / r0)
        if hist[-1] <= args.converge:
            break
    wall = time.perf_counter() - t0
    hit = next((i + 1 for i, h in enumerate(hist) if h <= args.converge), None)
    out = {"metric": "time_to_residual_drop", "workload": args.workload, "drop": args.converge,
           "reached": hit is not None, "steps_to_drop": hit, "steps_run": steps,
           "device_s": dev_ms * 1e-3, "wall_s": wall, "cells": N,
           "cell_iterations_per_s": N * steps / (dev_ms * 1e-3),
           "final_drop": hist[-1], "history_every_50": hist[::50], "config": desc}
    if case.force_patch:
        al = case.force_dirs
        g = case.options["thermo"]
        U = np.asarray(case.U[0])
        q = 0.5 * (1.0 / g["R"]) * float(U @ U)
        area = float(case.mesh.magSf[case.mesh.patch(case.force_patch).start:
                                     case.mesh.patch(case.force_patch).start + case.mesh.patch(case.force_patch).size].sum())
        # 2D: chord x span (1 x 0.1); wing: planform semi-span x mean chord
        ref_area = 0.1 if case.name.startswith("naca") else 1.5 * 0.5 * (1.0 + 0.56)
        out["forces"] = s.forces(case.force_patch, al["lift"], al["drag"], 1.0, q * ref_area)
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="swept_wing_fp32",
                    help="swept_wing_fp32 (default) | swept_wing_fp64 | swept_wing_bf16 | forward_step_2d | "
                         "naca0012_sa[_fp32]")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--converge", type=float, default=0.0,
                    help="run to this density-residual drop instead of timing fixed steps")
    ap.add_argument("--max-steps", type=int, default=5000)
    ap.add_argument("--no-convergence", dest="convergence", action="store_false",
                    help="skip the time-to-1e-10 (FP64 vs mixed) and adjoint-cost runs on the same mesh")
    args = ap.parse_args()
    if args.converge > 0:
        run_converge(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank != 0:
            return
        case, desc = workload(args.workload)
        cb = cpu_baseline(case, budget_s=args.cpu_budget, steps_max=args.steps, warmup=min(args.warmup, 3))
        line = {"impl": "reference", "metric": "cell_iterations_per_s", "value": cb["value"], "unit": "cell-iter/s",
                "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(desc, precision="fp64 throughout (the oracle has no reduced-precision storage)",
                               note="rhoDST needs foam-extend 4.1 (absent); CPU FP64 restatement timed "
                                    "on all host cores"),
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "cell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    line, case, _ = run_ours(args, rank, world)
    if rank == 0:
        inviscid = "transport" not in case.options and case.options.get("RASModel", "laminar") == "laminar"
        if world == 1 and args.convergence and case.force_patch in ("wing", "airfoil") and inviscid:
            line["time_to_residual_drop"] = convergence_and_adjoint(case)
        line["cpu_baseline"] = cpu_baseline(case, budget_s=args.cpu_budget, steps_max=1000, warmup=1)
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
