"""B200 library vs. CPU oracle for the other selectable block preconditioners
and solvers: Cholesky (diagonal-based incomplete factorisation), Gauss-Seidel
sweeps, ILUCp with fill-in, and the stationary GaussSeidel / ILU solvers;
block AMG (preconditioner and solver); and the subdomain ILU(0) on
graph-bisection subdomains.

Both sides run the same subdomain partition (the GPU's RCB parts, passed to
the oracle), FP64 throughout.  Step trajectories agree to 1e-9 relative (the
factorisation and Krylov sums run in a different order: level-scheduled
rows and SELL-ordered SpMV on the GPU, cell order on the CPU).  The
stationary solvers run a fixed number of iterations (minIter = maxIter), so
the iteration counts match by construction and the states are compared."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import _abi, cases
from tests.oracle_lib import OracleSolver
from tests.test_oracle_block_solvers import split_channel_case

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def run_pair(case, steps, parts, tol=1e-9, graph=False):
    case = case.with_options(**{"ilu.parts": parts, "ilu.partition": "graph" if graph else "rcb"})
    part = rhodst_b200.partition_graph(case.mesh, parts) if graph else rhodst_b200.partition_cells(case.mesh.C, parts)
    gpu = rhodst_b200.Solver(case.mesh, case.bcs, case.options)
    ora = OracleSolver(case.mesh, case.bcs, case.options, partition=part)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T)
    rg, ro = gpu.step(steps), ora.step(steps)
    for a, b in zip(rg, ro):
        assert abs(a["deltaT"] - b["deltaT"]) <= tol * abs(b["deltaT"])
        assert abs(a["res_mag"] - b["res_mag"]) <= tol * abs(b["res_mag"]), (a["res_mag"], b["res_mag"])
        assert a["lin_iterations"] == b["lin_iterations"]
    for a, b in zip(gpu.conservative(), ora.conservative()):
        assert rel(a, b) < tol
    return rg, ro


def step_case(solver, precon, iters=1, **extra):
    """C1 with a linear solve the preconditioner shapes: iters fixed
    iterations (GMRES(5) cycles, BiCGStab or stationary iterations), far
    from converged, so the step's state depends on M^-1 itself."""
    return cases.forward_step_c1(solver=solver, preconditioner=precon, n_directions=5, max_iter=iters).with_options(
        **{"solvers.W.minIter": iters, **extra})


@pytest.mark.parametrize("solver,precon,extra", [
    ("BiCGStab", "Cholesky", {}),
    ("GMRES", "GaussSeidel", {}),
    ("GMRES", "GaussSeidel", {"solvers.W.nSweeps": 3}),
    ("BiCGStab", "ILUCp", {"solvers.W.fillInLevel": 1}),
    ("GMRES", "ILUCp", {"solvers.W.fillInLevel": 0}),
])
def test_preconditioned_steps(solver, precon, extra):
    run_pair(step_case(solver, precon, iters=2 if solver == "BiCGStab" else 1, **extra), 4, parts=8)


@pytest.mark.parametrize("solver,extra", [
    ("GMRES", {}),
    ("BiCGStab", {"solvers.W.nPreSweeps": 1, "solvers.W.nPostSweeps": 1, "amg.omega": 0.8}),
    ("GMRES", {"solvers.W.minCoarseEqns": 200, "amg.coarsestSweeps": 4}),
])
def test_amg_preconditioned_steps(solver, extra):
    """Block AMG (aggregation of the cell graph, Galerkin coarse blocks
    gathered on the device every step, damped block-Jacobi V-cycle)."""
    run_pair(step_case(solver, "AMG", iters=2 if solver == "BiCGStab" else 1, **extra), 4, parts=1)


@pytest.mark.parametrize("solver,extra", [("GaussSeidel", {}), ("GaussSeidel", {"solvers.W.nSweeps": 2}),
                                          ("ILU", {}), ("AMG", {})])
def test_stationary_solver_steps(solver, extra):
    rg, _ = run_pair(step_case(solver, "none", iters=6, **extra), 4, parts=8)
    assert all(r["lin_iterations"] == 6 for r in rg)


@pytest.mark.parametrize("precon", ["Cholesky", "ILUCp"])
def test_cell_triangles(precon):
    """On the centroid-split prism channel three cells are pairwise
    neighbours, so Cholesky keeps only pivot updates where ILU(0) also
    updates off-diagonal blocks, and ILUCp level 1 adds fill blocks that
    the factorisation writes (and must restart from zero every step)."""
    c = split_channel_case(8, 5)
    x, y = c.mesh.C[:, 0], c.mesh.C[:, 1]
    c.p = 1.0 + 0.2 * np.sin(2.1 * x + 0.3) * np.cos(2.7 * y)
    c.T = 1.0 + 0.1 * np.cos(1.3 * x - 2.2 * y)
    opts = {"fluxScheme": "HLL", "solvers.W.solver": "GMRES", "solvers.W.preconditioner": precon,
            "solvers.W.nDirections": 4, "solvers.W.maxIter": 1, "solvers.W.minIter": 1,
            "solvers.W.tolerance": 0.0}
    if precon == "ILUCp":
        opts["solvers.W.fillInLevel"] = 1
    run_pair(c.with_options(**opts), 4, parts=2)


def test_ilucp_wide_fill_steps():
    """fillInLevel 2 on the split channel: 10 lower / 9 upper factor blocks
    a cell, the sixteen-slot apply."""
    c = split_channel_case(8, 5)
    x, y = c.mesh.C[:, 0], c.mesh.C[:, 1]
    c.p = 1.0 + 0.2 * np.sin(2.1 * x + 0.3) * np.cos(2.7 * y)
    opts = {"fluxScheme": "HLL", "solvers.W.solver": "GMRES", "solvers.W.preconditioner": "ILUCp",
            "solvers.W.fillInLevel": 2, "solvers.W.nDirections": 4, "solvers.W.maxIter": 1,
            "solvers.W.minIter": 1, "solvers.W.tolerance": 0.0}
    run_pair(c.with_options(**opts), 4, parts=1)


def test_too_wide_fill_is_refused():
    c = step_case("GMRES", "ILUCp", **{"solvers.W.fillInLevel": 3, "ilu.parts": 1})
    with pytest.raises(_abi.RdstError) as e:
        rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    assert e.value.status == 6


@pytest.mark.parametrize("case_fn", [
    lambda: step_case("GMRES", "ILUC0"),
    lambda: cases.naca0012_inviscid(ni=129, nj=33, first_cell=2e-3, n_directions=10),
], ids=["C1", "airfoil"])
def test_graph_bisection_subdomains(case_fn):
    run_pair(case_fn(), 5, parts=16, graph=True)


def test_contexts_with_different_ilu_shapes_coexist():
    """The dynamic shared-memory limits of the record pack and the bulk
    apply belong to the kernels, not to a context: a context built later on
    a mesh with fewer factor blocks per row (2D quads: two lower and two
    upper) must not shrink them under an earlier context whose rows carry
    more (3D hexahedra: three and three)."""
    wing = cases.swept_wing_c3(n_around=32, n_normal=8, n_span=8, n_tip=4, precision="fp64").with_options(
        **{"ilu.parts": 4})
    s3 = rhodst_b200.Solver(wing.mesh, wing.bcs, wing.options)
    s3.set_primitive(wing.p, wing.U, wing.T)
    r_before = s3.step(1)[-1]["res_mag"]
    foil = cases.naca0012_inviscid(ni=65, nj=17).with_options(precision="fp64", **{"ilu.parts": 4})
    s2 = rhodst_b200.Solver(foil.mesh, foil.bcs, foil.options)
    s2.set_primitive(foil.p, foil.U, foil.T)
    s2.step(1)
    r_after = s3.step(1)[-1]["res_mag"]
    assert np.isfinite(r_before) and np.isfinite(r_after)
    s2.close()
    s3.close()
