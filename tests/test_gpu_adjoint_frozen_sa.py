"""Frozen-turbulence discrete adjoint on the Spalart-Allmaras airfoil, on the
B200: the pressure-drag gradient with respect to the far-field velocity
against central differences of converged states.

The mean flow and SA are first run to a steady state together (first-order
HLL, local time steps ramped to CFL 500); mu_t is then held
(`frozenTurbulence`) and the mean flow alone is converged to round-off at a
fixed CFL of 100, from the SA state.  The adjoint linearizes that frozen
system (convective and viscous terms, muEff = mu(T) + mu_t with mu_t held),
and the finite differences re-converge the same frozen system with the far
field moved by +-h (h = 1e-6 |U_inf|), warm-started from the converged
state.  On the oracle this sequence reaches 1e-12 of the first residual in
about 300 steps per state and the two difference states agree in C_d to
1e-15 whatever the fixed CFL (50 or 150).  Agreement asked: 1e-5 relative.
"""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases

pytestmark = pytest.mark.gpu

ALPHA = np.radians(2.3)
DRAG = (np.cos(ALPHA), np.sin(ALPHA), 0.0)


def sa_case(frozen=False, dU=None):
    c = cases.naca0012_turbulent(ni=97, nj=25, first_cell=5e-3, reynolds=1e5, flux="HLL", limiter="upwind")
    opts = {"timeControls.maxCo": 500.0}
    if frozen:
        opts.update({"frozenTurbulence": True, "timeControls.initialCo": 100.0, "timeControls.maxCo": 100.0})
    c = c.with_options(**opts)
    if dU is not None:
        bcs = {k: dict(v) for k, v in c.bcs.items()}
        kind, U0 = bcs["farfield"]["U"]
        bcs["farfield"]["U"] = (kind, tuple(np.asarray(U0, dtype=float) + dU))
        c.bcs = bcs
    return c


def run_to_floor(s, r_ref, max_steps=3000):
    """Steps until the density residual is below 1e-13 r_ref, or below
    1e-11 r_ref and no longer falling; returns the last relative level."""
    last = np.inf
    for _ in range(max_steps // 100):
        r = s.step(100)[-1]["res_l2"][0] / r_ref
        if r < 1e-13 or (r < 1e-11 and r > 0.5 * last):
            break
        last = r
    return r


def frozen_solver(prim, dU=None, W0=None):
    s = rhodst_b200.Solver(*_mesh_bcs_opts(sa_case(frozen=True, dU=dU)))
    s.set_primitive(*prim)
    if W0 is not None:
        s.set_conservative(*W0)
    return s


def _mesh_bcs_opts(c):
    return c.mesh, c.bcs, c.options


def test_frozen_turbulence_gradient_matches_central_differences():
    base = sa_case()
    s = rhodst_b200.solver_for(base)
    reps = s.step(100)
    r0 = reps[0]["res_l2"][0]
    drop = reps[-1]["res_l2"][0] / r0
    for _ in range(20):
        if drop < 1e-10:
            break
        drop = s.step(100)[-1]["res_l2"][0] / r0
    assert drop < 1e-8, drop
    prim = s.primitive()
    assert np.ptp(prim[3]) > 0                      # a non-uniform nuTilda, so mu_t is not uniform

    sf = frozen_solver(prim)
    assert run_to_floor(sf, r0) < 1e-11
    W0 = sf.conservative()
    rep, _ = sf.adjoint("airfoil", DRAG, p_ref=1.0, rel_tol=1e-11, max_cycles=60)
    assert rep["residual"] <= 1e-10 * rep["residual0"], rep
    U0 = np.asarray(base.bcs["farfield"]["U"][1], dtype=float)
    uhat = U0 / np.linalg.norm(U0)
    grad = float(rep["dJ_dU"] @ uhat)
    h = 1e-6 * np.linalg.norm(U0)
    Js = []
    for sgn in (1.0, -1.0):
        sk = frozen_solver(prim, dU=sgn * h * uhat, W0=W0)
        assert run_to_floor(sk, r0) < 1e-11
        Js.append(sk.objective_gradient("airfoil", DRAG, p_ref=1.0)[0])
    fd = (Js[0] - Js[1]) / (2 * h)
    assert abs(grad - fd) <= 1e-5 * abs(fd), (grad, fd, rep)
