"""Discrete adjoint of the inviscid residual on the B200.

(1) Bookkeeping of the transposed product: for seeded random u, v,
    v . (dR/dW u) from the forward-mode (tangent) linearization of the
    residual must equal ((dR/dW)^T v) . u from the reverse (adjoint) pass,
    to rounding (1e-10 relative), for every flux scheme and reconstruction
    family, on the forward-step mesh (inlet, outlet, symmetry, slip walls)
    and the airfoil (characteristic far field).  Both take the branches of
    the primal evaluation, so limiter kinks do not enter.
(2) The linearization itself against central differences of the library's
    own residual: Jacobian columns (u = one component of one cell) at cells
    next to every patch and inside, 1e-5 relative per column (the central
    difference carries O(h^2) truncation and O(eps/h) rounding; a
    limiter branch that flips inside [-h, h] is avoided by the smooth state).
(3) Patch-velocity derivative (dR/dU_patch)^T v against central differences
    of the residual with the far-field velocity value moved by +-h.
(4) Full gradient: dJ/dU_patch from rdst_adjoint (pressure drag of the
    airfoil) against central differences of J at converged states
    (first-order reconstruction, which converges to round-off), 1e-5
    relative.
"""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases

pytestmark = pytest.mark.gpu

SCHEMES = ["Kurganov", "HLL", "HLLC", "HLLCP", "AUSM+", "AUSM+up", "AUSM"]


def airfoil(flux="HLLC", limiter="Venkatakrishnan", U_scale=None, **opts):
    c = cases.naca0012_inviscid(ni=97, nj=25, flux=flux, limiter=limiter, first_cell=5e-3)
    if U_scale is not None:
        bcs = {k: dict(v) for k, v in c.bcs.items()}
        kind, U0 = bcs["farfield"]["U"]
        bcs["farfield"]["U"] = (kind, tuple(U_scale(np.asarray(U0, dtype=float))))
        c.bcs = bcs
    if opts:
        c = c.with_options(**opts)
    return c


def step_case(flux, limiter):
    vlim = limiter if limiter in ("Venkatakrishnan", "upwind", "linear") else limiter + "V"
    return cases.forward_step_c1().with_options(**{
        "fluxScheme": flux, "interpolationSchemes.reconstruct(rho)": limiter,
        "interpolationSchemes.reconstruct(T)": limiter, "interpolationSchemes.reconstruct(U)": vlim})


def smooth_state(case, seed=3):
    """Seeded smooth perturbation of the case's initial state (conservative)."""
    rng = np.random.default_rng(seed)
    C = case.mesh.C
    k = rng.uniform(1.0, 4.0, size=(5, 3))
    ph = rng.uniform(0, 2 * np.pi, size=5)
    modes = [np.sin(C @ k[i] * np.pi + ph[i]) for i in range(5)]
    amp = 0.05
    p = case.p * (1 + amp * modes[0])
    T = case.T * (1 + amp * modes[1])
    U = case.U.copy()
    U[:, 0] *= 1 + amp * modes[2]
    U[:, 1] += amp * np.abs(case.U[:, 0]).max() * modes[3]
    # a z velocity too: an identically zero field ties every max/min of the
    # Venkatakrishnan limiter, a point where the limiter has no derivative
    U[:, 2] += amp * np.abs(case.U[:, 0]).max() * modes[4]
    g = case.options["thermo"]
    rho = p / (g["R"] * T)
    rhoE = rho * ((g["Cp"] - g["R"]) * T + 0.5 * (U ** 2).sum(1))
    return rho, rho[:, None] * U, rhoE


def prepared(case, W):
    s = rhodst_b200.Solver(case.mesh, case.bcs, case.options)
    s.set_conservative(*W)
    s.residual()                 # boundary mass fluxes of W
    s.set_conservative(*W)
    return s


def residual_at(s, W, u, h):
    """R(W + h u) with the boundary branches of W: the boundary mass fluxes
    and temperatures that choose in/outflow and sub/supersonic branches are
    refreshed at W first (as the adjoint holds them)."""
    rho, rhoU, rhoE = W
    s.set_conservative(rho, rhoU, rhoE)
    s.residual()
    s.set_conservative(rho + h * u[:, 0], rhoU + h * u[:, 1:4], rhoE + h * u[:, 4])
    return s.residual()


def random_dirs(N, W, seed):
    rng = np.random.default_rng(seed)
    rho, rhoU, rhoE = W
    scale = np.array([np.abs(rho).max(), *np.abs(rhoU).max(axis=0).clip(1e-3), np.abs(rhoE).max()])
    u = rng.uniform(-1, 1, size=(N, 5)) * scale
    v = rng.uniform(-1, 1, size=(N, 5))
    return u, v


def dot_test(case, seed=11):
    W = smooth_state(case)
    s = prepared(case, W)
    N = case.mesh.n_cells
    u, v = random_dirs(N, W, seed=seed)
    ATv, _ = s.adjoint_product(v)
    Ju = s.tangent_product(u)
    return float(np.sum(v * Ju)), float(np.sum(ATv * u))


@pytest.mark.parametrize("flux", SCHEMES)
@pytest.mark.parametrize("limiter", ["Venkatakrishnan", "OSPRE", "vanLeer", "upwind", "linear"])
def test_adjoint_transposes_tangent(flux, limiter):
    lhs, rhs = dot_test(step_case(flux, limiter))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (flux, limiter, lhs, rhs)


@pytest.mark.parametrize("flux", SCHEMES)
@pytest.mark.parametrize("limiter", ["Venkatakrishnan", "OSPRE", "upwind"])
def test_adjoint_transposes_tangent_far_field(flux, limiter):
    lhs, rhs = dot_test(airfoil(flux=flux, limiter=limiter))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (flux, limiter, lhs, rhs)


@pytest.mark.parametrize("flux,limiter", [("Kurganov", "Venkatakrishnan"), ("HLLC", "OSPRE"), ("AUSM+up", "vanLeer"),
                                          ("HLLCP", "upwind")])
def test_tangent_matches_central_differences(flux, limiter):
    case = step_case(flux, limiter)
    W = smooth_state(case)
    s = prepared(case, W)
    m = case.mesh
    N = m.n_cells
    cells = [int(np.asarray(m.owner)[P.start + P.size // 2]) for P in m.patches
             if P.size > 0 and P.name != "frontAndBack"] + [N // 2]
    Wf = np.concatenate([W[0][:, None], W[1], W[2][:, None]], 1)
    h = 1e-7
    for j in cells:
        for k in (0, 1, 4):
            u = np.zeros((N, 5))
            u[j, k] = max(1.0, abs(Wf[j, k]))
            Ju = s.tangent_product(u)
            fd = (residual_at(s, W, u, h) - residual_at(s, W, u, -h)) / (2 * h)
            s.set_conservative(*W)
            err = np.abs(Ju - fd).max() / np.abs(fd).max()
            assert err <= 1e-5, (flux, limiter, j, k, err)


def test_adjoint_patch_velocity_derivative():
    c = airfoil(flux="AUSM+up", limiter="Venkatakrishnan")
    W = smooth_state(c)
    s = prepared(c, W)
    N = c.mesh.n_cells
    _, v = random_dirs(N, W, seed=5)
    _, dU = s.adjoint_product(v)
    h = 1e-6
    fd = np.zeros(3)
    for k in range(2):           # in-plane components (the case is 2D)
        Rs = []
        for sgn in (1.0, -1.0):
            e = np.zeros(3)
            e[k] = sgn * h
            ck = airfoil(flux="AUSM+up", limiter="Venkatakrishnan", U_scale=lambda U0, e=e: U0 + e)
            sk = prepared(ck, W)
            Rs.append(sk.residual())
        fd[k] = float(np.sum(v * (Rs[0] - Rs[1]) / (2 * h)))
    for k in range(2):
        assert abs(fd[k] - dU[k]) <= 1e-6 * max(abs(fd[k]), abs(dU[k])), (k, fd[k], dU[k])


def converge(c, steps=4000, W0=None, r_ref=None):
    """Steady state of case c: steps until the density residual has dropped
    by 1e-13 relative to r_ref (default: the first step's), or has dropped
    by 1e-11 and stopped falling (the round-off floor).  W0 warm-starts from
    a nearby solution (finite differences), with r_ref of the solve that
    gave it, so both reach the same absolute level.  Returns (solver, drop,
    r_ref)."""
    s = rhodst_b200.solver_for(c)
    if W0 is not None:
        s.set_conservative(*W0)
    r0 = r_ref
    last = np.inf
    for _ in range(steps // 100):
        reps = s.step(100)
        if r0 is None:
            r0 = reps[0]["res_l2"][0]
        r = reps[-1]["res_l2"][0]
        if r < 1e-13 * r0 or (r < 1e-11 * r0 and r > 0.5 * last):
            break
        last = r
    return s, reps[-1]["res_l2"][0] / r0, r0


def converged(c, steps=4000):
    s, drop, _ = converge(c, steps)
    return s, drop


@pytest.mark.parametrize("flux", ["Kurganov", "HLL"])
def test_adjoint_gradient_matches_central_differences(flux):
    alpha = np.radians(2.3)
    drag = (np.cos(alpha), np.sin(alpha), 0.0)
    opts = {}
    base = airfoil(flux=flux, limiter="upwind", **opts)
    s, drop, r0 = converge(base)
    assert drop < 1e-11, drop
    W0 = s.conservative()
    rep, psi = s.adjoint("airfoil", drag, p_ref=1.0, scale=1.0, rel_tol=1e-11, max_cycles=60, n_directions=30,
                         want_psi=True)
    assert rep["residual"] <= 1e-10 * rep["residual0"], rep
    U0 = np.asarray(base.bcs["farfield"]["U"][1], dtype=float)
    uhat = U0 / np.linalg.norm(U0)             # Mach direction: dJ/dM = c dJ/dU . uhat
    grad = float(rep["dJ_dU"] @ uhat)
    h = 1e-6 * np.linalg.norm(U0)
    Js = []
    for sgn in (1.0, -1.0):
        ck = airfoil(flux=flux, limiter="upwind", U_scale=lambda U, sgn=sgn: U + sgn * h * uhat, **opts)
        sk, dk, _ = converge(ck, W0=W0, r_ref=r0)        # warm start from the base solution
        assert dk < 1e-11, dk
        Js.append(sk.objective_gradient("airfoil", drag, p_ref=1.0, scale=1.0)[0])
    fd = (Js[0] - Js[1]) / (2 * h)
    assert abs(grad - fd) <= 1e-5 * abs(fd), (grad, fd, rep)
