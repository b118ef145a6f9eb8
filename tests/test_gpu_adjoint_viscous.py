"""Discrete adjoint of the viscous residual (calcFields' laplacian(muEff, U),
div(tauMC) and div(sigmaDotU), baseFluxDST.C:229-250) at frozen turbulent
viscosity, on the B200.

(1) Duality: v . (J u) from the forward-mode linearization equals
    ((J^T v) . u) to 1e-10 on the laminar airfoil (constant viscosity and
    Sutherland's law, no-slip wall, characteristic far field) and on the
    Spalart-Allmaras airfoil with mu_t held (the residual of a state set
    with rdst_set_conservative keeps the mu_t of the last turbulence update).
(2) Tangent columns against central differences of the library's residual,
    1e-5, at cells next to the wall, the far field and inside.
(3) (dR/dU_patch)^T v against central differences of the residual with the
    far-field velocity moved (the no-slip wall's velocity is held).
(4) dJ/dU_patch . Uhat from rdst_adjoint against central differences of J
    at converged laminar states (first-order reconstruction), 1e-5.
"""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases
from tests.test_gpu_adjoint import converge, random_dirs, residual_at, smooth_state

pytestmark = pytest.mark.gpu


def laminar(flux="AUSM+up", limiter="vanLeer", sutherland=False, U_scale=None, **opts):
    c = cases.naca0012_laminar(ni=97, nj=25, flux=flux, limiter=limiter, sutherland=sutherland, first_cell=5e-3)
    if U_scale is not None:
        bcs = {k: dict(v) for k, v in c.bcs.items()}
        kind, U0 = bcs["farfield"]["U"]
        bcs["farfield"]["U"] = (kind, tuple(U_scale(np.asarray(U0, dtype=float))))
        c.bcs = bcs
    return c.with_options(**opts) if opts else c


def turbulent(flux="AUSM+up", limiter="Venkatakrishnan"):
    c = cases.naca0012_turbulent(ni=97, nj=25, flux=flux, limiter=limiter, first_cell=5e-3, reynolds=1e5)
    # a spatially varying nuTilda, so that mu_t is far from uniform
    C = c.mesh.C
    c.nuTilda = c.nuTilda * (1.0 + 200.0 * (1.0 + np.sin(3.0 * C[:, 0]) * np.cos(2.0 * C[:, 1])))
    return c


def prepared(case, W):
    """Solver at state W with mu_t from the case's nuTilda (set_primitive)
    and the boundary record of W."""
    s = rhodst_b200.solver_for(case)
    s.set_conservative(*W)
    s.residual()
    s.set_conservative(*W)
    return s


def dot_test(case, seed=11):
    W = smooth_state(case)
    s = prepared(case, W)
    u, v = random_dirs(case.mesh.n_cells, W, seed=seed)
    ATv, _ = s.adjoint_product(v)
    Ju = s.tangent_product(u)
    return float(np.sum(v * Ju)), float(np.sum(ATv * u))


@pytest.mark.parametrize("flux,limiter", [("AUSM+up", "vanLeer"), ("HLLC", "Venkatakrishnan"), ("Kurganov", "upwind"),
                                          ("HLLCP", "OSPRE")])
@pytest.mark.parametrize("sutherland", [False, True])
def test_viscous_adjoint_transposes_tangent(flux, limiter, sutherland):
    lhs, rhs = dot_test(laminar(flux=flux, limiter=limiter, sutherland=sutherland))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (flux, limiter, lhs, rhs)


@pytest.mark.parametrize("flux,limiter", [("AUSM+up", "Venkatakrishnan"), ("HLLC", "vanLeer")])
def test_frozen_turbulence_adjoint_transposes_tangent(flux, limiter):
    lhs, rhs = dot_test(turbulent(flux=flux, limiter=limiter))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (flux, limiter, lhs, rhs)


def test_viscous_terms_enter_the_linearization():
    """The viscous share of J u is not negligible on this mesh: the same
    product with the transport options removed differs."""
    c = laminar(sutherland=True)
    W = smooth_state(c)
    u, _ = random_dirs(c.mesh.n_cells, W, seed=4)
    Ju = prepared(c, W).tangent_product(u)
    inv = c.with_options()
    inv.options.pop("transport")
    inv.bcs = dict(inv.bcs)
    Ju0 = prepared(inv, W).tangent_product(u)
    assert np.abs(Ju - Ju0).max() > 1e-3 * np.abs(Ju).max()


@pytest.mark.parametrize("case_fn", [lambda: laminar(sutherland=True), lambda: turbulent()], ids=["laminar", "SA"])
def test_viscous_tangent_matches_central_differences(case_fn):
    case = case_fn()
    W = smooth_state(case)
    s = prepared(case, W)
    m = case.mesh
    N = m.n_cells
    cells = [int(np.asarray(m.owner)[P.start + P.size // 2]) for P in m.patches
             if P.size > 0 and P.name != "frontAndBack"] + [N // 2]
    Wf = np.concatenate([W[0][:, None], W[1], W[2][:, None]], 1)
    h = 1e-7
    for j in cells:
        for k in (0, 1, 2, 4):
            u = np.zeros((N, 5))
            u[j, k] = max(1.0, abs(Wf[j, k]))
            Ju = s.tangent_product(u)
            fd = (residual_at(s, W, u, h) - residual_at(s, W, u, -h)) / (2 * h)
            s.set_conservative(*W)
            err = np.abs(Ju - fd).max() / np.abs(fd).max()
            assert err <= 1e-5, (j, k, err)


def test_viscous_patch_velocity_derivative():
    c = laminar(sutherland=True)
    W = smooth_state(c)
    s = prepared(c, W)
    _, v = random_dirs(c.mesh.n_cells, W, seed=5)
    _, dU = s.adjoint_product(v)
    h = 1e-6
    for k in range(2):
        Rs = []
        for sgn in (1.0, -1.0):
            e = np.zeros(3)
            e[k] = sgn * h
            Rs.append(prepared(laminar(sutherland=True, U_scale=lambda U0, e=e: U0 + e), W).residual())
        fd = float(np.sum(v * (Rs[0] - Rs[1]) / (2 * h)))
        assert abs(fd - dU[k]) <= 1e-6 * max(abs(fd), abs(dU[k])), (k, fd, dU[k])


def test_viscous_adjoint_gradient_matches_central_differences():
    alpha = np.radians(1.0)
    drag = (np.cos(alpha), np.sin(alpha), 0.0)
    base = laminar(flux="Kurganov", limiter="upwind", sutherland=True)
    s, drop, r0 = converge(base)
    assert drop < 1e-11, drop
    W0 = s.conservative()
    rep, _ = s.adjoint("airfoil", drag, p_ref=1.0, rel_tol=1e-11, max_cycles=60)
    assert rep["residual"] <= 1e-10 * rep["residual0"], rep
    U0 = np.asarray(base.bcs["farfield"]["U"][1], dtype=float)
    uhat = U0 / np.linalg.norm(U0)
    grad = float(rep["dJ_dU"] @ uhat)
    h = 1e-6 * np.linalg.norm(U0)
    Js = []
    for sgn in (1.0, -1.0):
        ck = laminar(flux="Kurganov", limiter="upwind", sutherland=True, U_scale=lambda U, sgn=sgn: U + sgn * h * uhat)
        sk, dk, _ = converge(ck, W0=W0, r_ref=r0)
        assert dk < 1e-11, dk
        Js.append(sk.objective_gradient("airfoil", drag, p_ref=1.0)[0])
    fd = (Js[0] - Js[1]) / (2 * h)
    assert abs(grad - fd) <= 1e-5 * abs(fd), (grad, fd, rep)
