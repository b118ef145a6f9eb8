"""B200 library vs. CPU oracle: residual, assembled block system, full steps.

All comparisons are FP64 vs FP64 on the same seeded inputs.  Tolerances:
residual / assembly 1e-11 relative to the field's max magnitude (the only
differences are FMA contraction and per-face arithmetic order); step
trajectories 1e-10 relative per step (Krylov summation order differs:
SELL-ordered SpMV and CGS2 on the GPU vs. foam-ordered Amul and modified
Gram-Schmidt in the oracle)."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver

pytestmark = pytest.mark.gpu

SCHEMES = ["Kurganov", "HLL", "HLLC", "HLLCP", "AUSM+", "AUSM+up", "AUSM"]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def perturbed_state(case, seed=7, amp=0.05):
    """Smooth seeded perturbation of the initial primitive state, returned
    as conservative fields (exercises limiters in every direction)."""
    rng = np.random.default_rng(seed)
    C = case.mesh.C
    k = rng.uniform(1.0, 4.0, size=(5, 3))
    ph = rng.uniform(0, 2 * np.pi, size=5)
    modes = [np.sin(C @ k[i] * np.pi + ph[i]) for i in range(5)]
    p = case.p * (1 + amp * modes[0])
    T = case.T * (1 + amp * modes[1])
    U = case.U.copy()
    U[:, 0] *= 1 + amp * modes[2]
    U[:, 1] += amp * np.abs(case.U[:, 0]).max() * modes[3]
    g = case.options["thermo"]
    rho = p / (g["R"] * T)
    Cv = g["Cp"] - g["R"]
    rhoE = rho * (Cv * T + 0.5 * (U ** 2).sum(1))
    return rho, rho[:, None] * U, rhoE


def pair(case, partition=None):
    gpu = rhodst_b200.Solver(case.mesh, case.bcs, case.options)
    ora = OracleSolver(case.mesh, case.bcs, case.options, partition=partition)
    return gpu, ora


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("lim", [("OSPRE", "OSPREV"), ("vanLeer", "vanLeerV"), ("linear", "linear")])
def test_residual_parity(scheme, lim):
    case = cases.forward_step_c1().with_options(**{
        "fluxScheme": scheme,
        "interpolationSchemes.reconstruct(rho)": lim[0], "interpolationSchemes.reconstruct(T)": lim[0],
        "interpolationSchemes.reconstruct(U)": lim[1]})
    gpu, ora = pair(case)
    rho, rhoU, rhoE = perturbed_state(case)
    for s in (gpu, ora):
        s.set_conservative(rho, rhoU, rhoE)
    Rg, Ro = gpu.residual(), ora.residual()
    assert np.all(np.isfinite(Rg))
    for k in range(5):
        assert rel(Rg[:, k], Ro[:, k]) < 1e-11, (scheme, lim, k)


def test_assembly_parity():
    case = cases.forward_step_c1()
    gpu, ora = pair(case)
    rho, rhoU, rhoE = perturbed_state(case)
    for s in (gpu, ora):
        s.set_conservative(rho, rhoU, rhoE)
    dg, ug, lg, sg = gpu.assemble()
    do, uo, lo, so = ora.assemble()
    assert rel(dg, do) < 1e-11
    assert rel(ug, uo) < 1e-11
    assert rel(lg, lo) < 1e-11
    assert rel(sg, so) < 1e-11


def _run_pair(case, steps, partition=None, tol=1e-10):
    gpu, ora = pair(case, partition)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T)
    rg = gpu.step(steps)
    ro = ora.step(steps)
    for a, b in zip(rg, ro):
        assert abs(a["deltaT"] - b["deltaT"]) <= tol * abs(b["deltaT"])
        assert abs(a["res_mag"] - b["res_mag"]) <= tol * abs(b["res_mag"]), (a["res_mag"], b["res_mag"])
        assert a["lin_iterations"] == b["lin_iterations"]
    Wg, Wo = gpu.conservative(), ora.conservative()
    for a, b in zip(Wg, Wo):
        assert rel(a, b) < tol
    return rg, ro


def test_steps_gmres_jacobi():
    _run_pair(cases.forward_step_c1(), 20)


def test_steps_bicgstab_ilu_exact():
    case = cases.forward_step_c1(solver="BiCGStab", preconditioner="ILUC0", max_iter=4).with_options(
        **{"ilu.parts": 1, "solvers.W.minIter": 4})
    _run_pair(case, 5, tol=1e-9)


def test_steps_gmres_ilu_subdomains():
    case = cases.forward_step_c1(preconditioner="ILUC0", n_directions=10).with_options(**{"ilu.parts": 8})
    part = rhodst_b200.partition_cells(case.mesh.C, 8)
    _run_pair(case, 5, partition=part, tol=1e-9)


def test_tolerance_driven_restarts():
    case = cases.forward_step_c1(n_directions=5, max_iter=50).with_options(
        **{"solvers.W.tolerance": 1e-12, "solvers.W.minIter": 1})
    rg, ro = _run_pair(case, 3, tol=1e-9)
    assert rg[0]["lin_iterations"] > 1


def test_deterministic():
    case = cases.forward_step_c1()
    out = []
    for _ in range(2):
        s = rhodst_b200.solver_for(case)
        s.step(5)
        out.append(np.concatenate([x.ravel() for x in s.conservative()]))
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_mixed_precision_matrix(prec):
    """Reduced-precision Jacobian storage changes only the linear update:
    the residual R(W) stays FP64, so one step moves W by a near-identical
    increment."""
    base = cases.forward_step_c1()
    s64 = rhodst_b200.solver_for(base)
    sm = rhodst_b200.solver_for(base.with_options(precision=prec))
    s64.step(3)
    sm.step(3)
    W64, Wm = s64.conservative(), sm.conservative()
    tol = 1e-5 if prec == "fp32" else 1e-2
    for a, b in zip(Wm, W64):
        assert rel(a, b) < tol


def small_airfoil(**kw):
    c = cases.naca0012_inviscid(ni=129, nj=33, **kw)
    return c.with_options(**{"ilu.parts": 4})


@pytest.mark.parametrize("flux,lim", [("AUSM+up", "Venkatakrishnan"), ("HLLC", "OSPRE"), ("Kurganov", "vanLeer")])
def test_farfield_airfoil_residual(flux, lim):
    case = small_airfoil(flux=flux, limiter=lim)
    gpu, ora = pair(case, partition=rhodst_b200.partition_cells(case.mesh.C, 4))
    rho, rhoU, rhoE = perturbed_state(case, amp=0.02)
    for s in (gpu, ora):
        s.set_conservative(rho, rhoU, rhoE)
    Rg, Ro = gpu.residual(), ora.residual()
    for k in range(5):
        assert rel(Rg[:, k], Ro[:, k]) < 1e-11
    dg, ug, lg, sg = gpu.assemble()
    do, uo, lo, so = ora.assemble()
    assert rel(dg, do) < 1e-11 and rel(ug, uo) < 1e-11 and rel(lg, lo) < 1e-11


def test_farfield_airfoil_steps():
    case = small_airfoil()
    _run_pair(case, 10, partition=rhodst_b200.partition_cells(case.mesh.C, 4), tol=1e-9)


@pytest.mark.parametrize("neighbouring", [True, False])
def test_local_time_step_definitions(neighbouring):
    """Both local pseudo-time steps of setSteadyStateDeltaT: the face-based
    one with the per-cell ramped courant, the cell-centre one with the scalar
    courant (timeDST.C:218-273)."""
    case = small_airfoil().with_options(**{"timeControls.neighbouring": neighbouring})
    rg, ro = _run_pair(case, 8, partition=rhodst_b200.partition_cells(case.mesh.C, 4), tol=1e-9)
    for a, b in zip(rg, ro):
        assert abs(a["rdt_max"] - b["rdt_max"]) <= 1e-9 * abs(b["rdt_max"])


@pytest.mark.parametrize("adjust", [False, True])
def test_dual_time_steps(adjust):
    """Dual-time stepping (Dual::iterate + dual2ndDST + steadyCheck): the
    same inner-iteration counts, physical time steps, residuals and fields
    as the oracle over three physical steps."""
    case = cases.forward_step_c1().with_options(**{
        "timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
        "timeControls.adjustTimeStep": adjust, "controlDict.deltaT": 0.02})
    gpu, ora = pair(case)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T)
    rg, ro = gpu.step(3), ora.step(3)
    for a, b in zip(rg, ro):
        assert a["lin_iterations"] == b["lin_iterations"], (a["lin_iterations"], b["lin_iterations"])
        assert abs(a["deltaT"] - b["deltaT"]) <= 1e-10 * abs(b["deltaT"])
        assert abs(a["res_mag"] - b["res_mag"]) <= 1e-8 * abs(b["res_mag"]), (a["res_mag"], b["res_mag"])
    Wg, Wo = gpu.conservative(), ora.conservative()
    for a, b in zip(Wg, Wo):
        assert rel(a, b) < 1e-9


def test_wing_small_steps():
    case = cases.swept_wing_c3(n_around=48, n_normal=16, n_span=8, n_tip=4, ilu_parts=6)
    _run_pair(case, 4, partition=rhodst_b200.partition_cells(case.mesh.C, 6), tol=1e-9)


def test_forces_parity():
    case = small_airfoil()
    gpu, ora = pair(case, partition=rhodst_b200.partition_cells(case.mesh.C, 4))
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T)
        s.step(5)
    q = 0.5 * 1.4 * 0.73 ** 2   # 1/2 rho U^2 with rho = gamma (p = T = 1 normalised gas)
    fg = gpu.forces("airfoil", case.force_dirs["lift"], case.force_dirs["drag"], 1.0, q * 0.1)
    fo = ora.forces("airfoil", case.force_dirs["lift"], case.force_dirs["drag"], 1.0, q * 0.1)
    for k in ("Cl", "Cd", "Cm"):
        assert abs(fg[k] - fo[k]) <= 1e-9 * max(abs(fo[k]), 1e-3)


@pytest.mark.parametrize("fixed", [True, False])
def test_graphs_match_direct_launches(fixed):
    """CUDA-graph replay of the step gives bitwise the same trajectory as
    direct launches (fixed iteration count: one graph per step; tolerance
    driven: pre / iteration / post graphs with host convergence reads)."""
    case = cases.forward_step_c1(n_directions=5 if not fixed else 20, max_iter=1 if fixed else 20)
    if not fixed:
        case = case.with_options(**{"solvers.W.tolerance": 1e-11})
    out = []
    for graphs in (True, False):
        s = rhodst_b200.solver_for(case.with_options(graphs=graphs))
        rep = s.step(6)
        out.append((np.concatenate([x.ravel() for x in s.conservative()]),
                    [r["res_mag"] for r in rep], [r["lin_iterations"] for r in rep]))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]


def test_profile_counters():
    case = cases.forward_step_c1().with_options(profile=True)
    s = rhodst_b200.solver_for(case)
    s.step(3)
    n, ms = s.kernel_stats("spmv")
    assert n == 3 * 23 and ms > 0          # 20 directions + initial + final residual + W-form A.W
    assert s.launch_count() > 0 and s.last_step_ms() > 0


@pytest.mark.parametrize("flux,suth", [("AUSM+up", False), ("Kurganov", True), ("HLLC", False)])
def test_viscous_residual_and_assembly(flux, suth):
    case = cases.naca0012_laminar(flux=flux, sutherland=suth).with_options(**{"ilu.parts": 4})
    gpu, ora = pair(case, partition=rhodst_b200.partition_cells(case.mesh.C, 4))
    rho, rhoU, rhoE = perturbed_state(case, amp=0.02)
    for s in (gpu, ora):
        s.set_conservative(rho, rhoU, rhoE)
    Rg, Ro = gpu.residual(), ora.residual()
    for k in range(5):
        assert rel(Rg[:, k], Ro[:, k]) < 1e-11, k
    dg, ug, lg, sg = gpu.assemble()
    do, uo, lo, so = ora.assemble()
    assert rel(dg, do) < 1e-11 and rel(ug, uo) < 1e-11 and rel(lg, lo) < 1e-11


def test_viscous_steps():
    case = cases.naca0012_laminar().with_options(**{"ilu.parts": 4})
    _run_pair(case, 8, partition=rhodst_b200.partition_cells(case.mesh.C, 4), tol=1e-9)


def small_turbulent(model="SAneg"):
    c = cases.naca0012_turbulent(ni=129, nj=49, model=model)
    return c.with_options(**{"ilu.parts": 4})


@pytest.mark.parametrize("model", ["SAneg", "SARC1", "SARC2", "SpalartAllmaras"])
def test_sa_steps(model):
    case = small_turbulent(model)
    part = rhodst_b200.partition_cells(case.mesh.C, 4)
    gpu, ora = pair(case, partition=part)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T, case.nuTilda)
    rg, ro = gpu.step(6), ora.step(6)
    for a, b in zip(rg, ro):
        assert abs(a["res_mag"] - b["res_mag"]) <= 1e-9 * abs(b["res_mag"])
    pg, Ug, Tg, ng = gpu.primitive()
    po, Uo, To, no = ora.primitive()
    assert rel(pg, po) < 1e-9 and rel(Ug, Uo) < 1e-9 and rel(Tg, To) < 1e-9
    if model != "SARC1":
        assert rel(ng, no) < 1e-9
        return
    # SARC1's material derivative takes ddt(rho, S) = rDeltaT (rho S - rho0 S0)
    # with the local pseudo-time step: in the wall layer's tiny cells a huge
    # rDeltaT times a difference of nearly equal strain rates amplifies
    # rounding.  The oracle alone, built with and without FMA contraction,
    # differs there by 3.9e-5 after these six steps (2e-9 from 0.1 to 1 chord,
    # 7e-13 beyond); SARC2 by 6e-10 everywhere
    y = case.mesh.wall_distance
    away = y >= 0.1
    assert np.abs(ng - no)[away].max() <= 1e-7 * np.abs(no).max()
    assert rel(ng, no) < 1e-4


def test_rae2822_tutorial_steps():
    """The reference's RAE2822 tutorial (its own mesh, conditions and solver
    settings; SpalartAllmaras, BiCGStab + ILUC0 to 1e-10): five steps."""
    case = cases.rae2822().with_options(**{"ilu.parts": 8})
    part = rhodst_b200.partition_cells(case.mesh.C, 8)
    gpu, ora = pair(case, partition=part)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T, case.nuTilda)
    rg, ro = gpu.step(5), ora.step(5)
    for a, b in zip(rg, ro):
        assert abs(a["res_mag"] - b["res_mag"]) <= 1e-8 * abs(b["res_mag"])
    pg, Ug, Tg, ng = gpu.primitive()
    po, Uo, To, no = ora.primitive()
    assert rel(pg, po) < 1e-8 and rel(Ug, Uo) < 1e-8 and rel(Tg, To) < 1e-8 and rel(ng, no) < 1e-8


def test_sa_residual_with_mut():
    case = small_turbulent("SAneg")
    part = rhodst_b200.partition_cells(case.mesh.C, 4)
    gpu, ora = pair(case, partition=part)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T, case.nuTilda * 50.0)
    Rg, Ro = gpu.residual(), ora.residual()
    for k in range(5):
        assert rel(Rg[:, k], Ro[:, k]) < 1e-11
    dg, ug, lg, sg = gpu.assemble()
    do, uo, lo, so = ora.assemble()
    assert rel(dg, do) < 1e-11 and rel(ug, uo) < 1e-11
