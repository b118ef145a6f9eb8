"""The GPU linearization and adjoint against the CPU complex-step reference
(the oracle's residual and objective evaluated on complex numbers, h =
1e-30; independent code).

(1) Tangent products (dR/dW) u: GPU forward mode vs complex step, 1e-9
    relative (the two residual implementations agree to ~1e-11; the
    derivatives carry the same rounding), every scheme x reconstruction on
    the forward step and three combinations on the airfoil far field.  The
    boundary branches are the GPU's (rdst_boundary_branches).
(2) The adjoint gradient dJ/dU_patch (pressure drag of the airfoil) vs a
    complex-step reference gradient: the Jacobian assembled column by
    column by complex step (cells coloured so that each colour's columns
    do not overlap in any row), dR/dU_patch and dJ/dW by complex step,
    psi from a sparse direct solve of J^T psi = dJ/dW: 1e-8 relative, at
    converged first-order states (Kurganov and HLL).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import rhodst_b200
from tests.oracle_lib import ComplexStep, OracleSolver, conservative_array, distance2_colors
from tests.test_gpu_adjoint import SCHEMES, airfoil, converged, prepared, random_dirs, smooth_state, step_case

pytestmark = pytest.mark.gpu


def tangent_vs_cs(case, seed=5):
    W = smooth_state(case)
    s = prepared(case, W)
    o = OracleSolver(case.mesh, case.bcs, case.options)
    o.set_conservative(*W)
    u, _ = random_dirs(case.mesh.n_cells, W, seed=seed)
    Ju = s.tangent_product(u)
    _, dR = ComplexStep(o).residual(conservative_array(W), u, branches=s.boundary_branches())
    return np.abs(Ju - dR).max() / np.abs(dR).max()


@pytest.mark.parametrize("flux", SCHEMES)
@pytest.mark.parametrize("limiter", ["Venkatakrishnan", "OSPRE", "upwind"])
def test_tangent_matches_complex_step(flux, limiter):
    err = tangent_vs_cs(step_case(flux, limiter))
    assert err <= 1e-9, (flux, limiter, err)


@pytest.mark.parametrize("flux,limiter", [("AUSM+up", "Venkatakrishnan"), ("HLLC", "OSPRE"), ("Kurganov", "upwind")])
def test_tangent_matches_complex_step_far_field(flux, limiter):
    err = tangent_vs_cs(airfoil(flux=flux, limiter=limiter))
    assert err <= 1e-9, (flux, limiter, err)


def complex_step_adjoint(case, W, branches, patch, direction, p_ref, hops):
    """psi of the complex-step reference: the Jacobian assembled by
    coloured columns and dJ/dW by complex step, sparse direct solve of
    J^T psi = dJ/dW.  Returns (ComplexStep on the case's mesh, W as N x 5,
    psi as N x 5)."""
    o = OracleSolver(case.mesh, case.bcs, case.options)
    o.set_conservative(*W)
    cs = ComplexStep(o)
    Wa = conservative_array(W)
    N = case.mesh.n_cells
    color, adj = distance2_colors(case.mesh, hops)
    rows, cols, vals = [], [], []
    # cells whose rows a column j touches: j itself and its (hops/2)-hop neighbourhood
    reach = []
    for j in range(N):
        seen, front = {j}, [j]
        for _ in range(hops // 2):
            front = [y for x in front for y in adj[x] if y not in seen and not seen.add(y)]
        reach.append(seen)
    owner_of_row = {}
    for kc in range(int(color.max()) + 1):
        members = np.nonzero(color == kc)[0]
        row_col = {}
        for j in members:
            for i in reach[j]:
                row_col[i] = j
        for comp in range(5):
            u = np.zeros((N, 5))
            u[members, comp] = 1.0
            _, dR = cs.residual(Wa, u, branches=branches)
            for i, j in row_col.items():
                for r in range(5):
                    if dR[i, r] != 0.0:
                        rows.append(5 * i + r)
                        cols.append(5 * j + comp)
                        vals.append(dR[i, r])
    Jm = sp.csc_matrix((vals, (rows, cols)), shape=(5 * N, 5 * N))
    dJdW = np.zeros((N, 5))
    for comp in range(5):
        u = np.zeros((N, 5))
        u[:, comp] = 1.0
        _, _, cells = cs.objective(Wa, patch, direction, p_ref=p_ref, u=u, branches=branches, per_cell=True)
        dJdW[:, comp] = cells
    psi = spla.spsolve(Jm.T.tocsc(), dJdW.ravel())
    return cs, Wa, psi.reshape(N, 5)


def complex_step_gradient(case, W, branches, patch, direction, p_ref, hops):
    """dJ/dU_patch by complex step: dJ/dU = dJ/dU|explicit - psi^T dR/dU."""
    cs, Wa, psi = complex_step_adjoint(case, W, branches, patch, direction, p_ref, hops)
    N = case.mesh.n_cells
    dRdU = np.zeros((5 * N, 3))
    dJdU = np.zeros(3)
    for m in range(3):
        e = np.zeros(3)
        e[m] = 1.0
        _, dR = cs.residual(Wa, None, e, branches=branches)
        dRdU[:, m] = dR.ravel()
        dJdU[m] = cs.objective(Wa, patch, direction, p_ref=p_ref, dU=e, branches=branches)[1]
    return dJdU - dRdU.T @ psi.ravel()


@pytest.mark.parametrize("flux", ["Kurganov", "HLL"])
def test_adjoint_gradient_matches_complex_step(flux):
    alpha = np.radians(2.3)
    drag = (np.cos(alpha), np.sin(alpha), 0.0)
    c = airfoil(flux=flux, limiter="upwind")
    s, drop = converged(c)
    assert drop < 1e-11, drop
    W = s.conservative()
    rep, _ = s.adjoint("airfoil", drag, p_ref=1.0, scale=1.0, rel_tol=1e-12, max_cycles=60, n_directions=30)
    assert rep["residual"] <= 1e-11 * rep["residual0"], rep
    ref = complex_step_gradient(c, W, s.boundary_branches(), "airfoil", drag, 1.0, hops=2)
    g = rep["dJ_dU"]
    assert np.abs(g - ref)[:2].max() <= 1e-8 * np.abs(ref).max(), (g, ref)
