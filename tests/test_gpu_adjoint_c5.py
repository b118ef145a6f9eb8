"""Converged adjoint gradient on the hybrid tetrahedron/prism forward step:
d(step-face pressure force)/dU_inf against central differences of
re-converged states, on the B200.

A 4,416-cell version of the 3D Mach-3 step (30 x 10 x 4 lattice, 25 %
jitter), first-order HLL, local time steps ramped to CFL 50, converged to
round-off; J is the x-force of (p - 1) on the step faces ("obstacle").  The
adjoint's dJ/dU_patch moves the velocity of every patch that carries one
(the inlet's fixed value and the outlet's inflow value); the differences
move both by +-h (h = 1e-6 |U_inf|) and re-converge from the converged
state at a fixed CFL of 50.  On the oracle this sequence reaches 1e-14 of
the first residual in 1,500 steps, each difference state 1e-13 in 400, and
gives dJ/dU_x = 0.9661.  Agreement asked: 1e-5 relative.
"""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases

pytestmark = pytest.mark.gpu


def step_case(dU=0.0, warm=False):
    c = cases.forward_step_3d_hybrid_c5(nx=30, ny=10, nz=4).with_options(**{
        "fluxScheme": "HLL", "interpolationSchemes.reconstruct(rho)": "upwind",
        "interpolationSchemes.reconstruct(U)": "upwind", "interpolationSchemes.reconstruct(T)": "upwind",
        "timeControls.maxCo": 50.0, "precision": "fp64"})
    if warm:
        c = c.with_options(**{"timeControls.initialCo": 50.0})
    bcs = {k: dict(v) for k, v in c.bcs.items()}
    for name in ("inlet", "outlet"):
        kind, U0 = bcs[name]["U"]
        bcs[name]["U"] = (kind, (U0[0] + dU, U0[1], U0[2]))
    c.bcs = bcs
    return c


def converge(c, W0=None, r_ref=None, max_steps=4000):
    s = rhodst_b200.solver_for(c)
    if W0 is not None:
        s.set_conservative(*W0)
    r0, last, r = r_ref, np.inf, np.inf
    for _ in range(max_steps // 100):
        reps = s.step(100)
        if r0 is None:
            r0 = reps[0]["res_l2"][0]
        r = reps[-1]["res_l2"][0] / r0
        if r < 1e-13 or (r < 1e-11 and r > 0.5 * last):
            break
        last = r
    return s, r, r0


def test_step_force_gradient_matches_central_differences():
    s, drop, r0 = converge(step_case())
    assert drop < 1e-11, drop
    W0 = s.conservative()
    rep, _ = s.adjoint("obstacle", (1.0, 0.0, 0.0), p_ref=1.0, rel_tol=1e-11, max_cycles=60)
    assert rep["residual"] <= 1e-10 * rep["residual0"], rep
    h = 3e-6
    Js = []
    for sgn in (1.0, -1.0):
        sk, dk, _ = converge(step_case(sgn * h, warm=True), W0=W0, r_ref=r0)
        assert dk < 1e-11, dk
        Js.append(sk.objective_gradient("obstacle", (1.0, 0.0, 0.0), p_ref=1.0)[0])
    fd = (Js[0] - Js[1]) / (2 * h)
    assert abs(rep["dJ_dU"][0] - fd) <= 1e-5 * abs(fd), (rep["dJ_dU"], fd, rep)
    # the Mach derivative the C5 report quotes: dJ/dM = c_inf dJ/dU_x at fixed T (c_inf = 1 here)
    assert np.isfinite(rep["dJ_dU"]).all()
