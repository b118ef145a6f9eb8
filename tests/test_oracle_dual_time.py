"""Dual-time stepping in the oracle (Dual::iterate, Dual.C:80-124, with the
dual2ndDST ddt, dual2ndDST.C:375-412, and the steadyCheck inner-loop test,
steadyCheck.C:69-98).

(1) Converged inner iterations solve the BDF2 equations: R(W^n+1) +
    a W^n+1 + b W^n + c W^n-1 = 0 with a = 1/dt + 1/(dt + dt0),
    c = dt/(dt0 (dt + dt0)), b = -(a + c); at the first step W^n-1 = W^n
    and dt0 is controlDict's deltaT (foam Time's deltaT0), afterwards the
    previous step's.
(2) The inner loop stops after maxInnerIter + 1 iterations when neither the
    residual level nor the slope test is met.
(3) The physical time step comes from initialCo at initialisation
    (timeDST::initialize calls setTransientDeltaT unconditionally) and stays
    with adjustTimeStep false.
(4) Dual needs dual2ndDST and the reverse.
(5) With Spalart-Allmaras the nuTilda equation takes its own dual2ndDST ddt:
    a steady state is a fixed point of dual steps (either placement of the
    turbulence update), a disturbed nuTilda moves.
(6) SARC1's material derivative of the strain rate takes dual2ndDST's
    fvcDdt(rho, S) over the physical steps (dual2ndDST.C:231-372): its
    coefficients sum to zero (coefft0 = coefft + coefft00), so a steady
    SARC1 state stays a fixed point over the steps where the old times are
    copies (deltaT0 GREAT) and the step where they are distinct.
"""
import functools

import numpy as np
import pytest

from rhodst_b200 import cases
from rhodst_b200._abi import RdstError
from tests.oracle_lib import OracleSolver


def dual_case(**opts):
    base = {"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
            "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.02}
    base.update(opts)
    return cases.forward_step_c1().with_options(**base)


def state(o):
    r, ru, re = o.conservative()
    return np.concatenate([r[:, None], ru, re[:, None]], 1)


def coeffs(dt, dt0):
    a = 1 / dt + 1 / (dt + dt0)
    c = dt / (dt0 * (dt + dt0))
    return a, -(a + c), c


def test_converged_inner_iterations_solve_bdf2():
    c = dual_case(**{"timeIntegration.maxInnerIter": 200, "residualControls.minResudual": 1e-12,
                     "residualControls.magConvergedSlope": 0.0})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    W0 = state(o)
    r1 = o.step(1)[0]
    W1 = state(o)
    R1 = o.residual()
    r2 = o.step(1)[0]
    W2 = state(o)
    R2 = o.residual()
    assert r1["lin_iterations"] < 201 and r2["lin_iterations"] < 201
    a, b, cc = coeffs(r1["deltaT"], 0.02)                 # first step: W^n-1 = W^n, dt0 = controlDict deltaT
    res1 = R1 + a * W1 + b * W0 + cc * W0
    a, b, cc = coeffs(r2["deltaT"], r1["deltaT"])
    res2 = R2 + a * W2 + b * W1 + cc * W0
    for res, Wn1, Wn in ((res1, W1, W0), (res2, W2, W1)):
        scale = np.abs(a * (Wn1 - Wn)).max()
        assert np.abs(res).max() <= 1e-9 * scale, (np.abs(res).max(), scale)


def test_physical_time_step_from_initial_courant():
    c = dual_case()
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    reps = o.step(3)
    dts = [r["deltaT"] for r in reps]
    assert dts[0] != 0.02 and dts[0] == dts[1] == dts[2]
    assert reps[-1]["time"] == pytest.approx(sum(dts))


def test_inner_loop_stops_after_max_inner_iter():
    c = dual_case(**{"timeIntegration.maxInnerIter": 7, "residualControls.minResudual": 0.0,
                     "residualControls.magConvergedSlope": 0.0})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    assert [r["lin_iterations"] for r in o.step(2)] == [8, 8]


def test_slope_test_ends_the_inner_loop():
    """With no residual level the inner loop runs until log(residual)
    flattens (the rounding floor): the scaled slope test ends it before
    maxInnerIter."""
    c = dual_case(**{"timeIntegration.maxInnerIter": 400, "residualControls.minResudual": 0.0})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    for r in o.step(2):
        assert 10 <= r["lin_iterations"] < 401
        assert np.mean(r["lin_initial"]) < 1e-12


@pytest.mark.parametrize("opts", [
    {"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "Euler"},
    {"timeIntegration.timeIntegration": "Single", "ddtSchemes.default": "dual2ndDST"},
])
def test_dual_needs_dual2nd(opts):
    c = cases.forward_step_c1().with_options(**opts)
    with pytest.raises(RdstError):
        OracleSolver(c.mesh, c.bcs, c.options)


def sa_steady(model="SAneg"):
    """A converged first-order SA airfoil state (p, U, T, nuTilda), each
    converged once per model and copied for every test."""
    c, prim = _sa_steady(model)
    return c, tuple(np.array(a) for a in prim)


@functools.lru_cache(maxsize=None)
def _sa_steady(model):
    c = cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL", limiter="upwind",
                                 model=model).with_options(**{"timeControls.maxCo": 500.0})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T, c.nuTilda)
    r0 = None
    for _ in range(20):
        reps = o.step(50)
        r0 = reps[0]["res_l2"][0] if r0 is None else r0
        if reps[-1]["res_l2"][0] < 1e-12 * r0:
            break
    assert reps[-1]["res_l2"][0] < 1e-10 * r0
    return c, o.primitive()


@pytest.mark.parametrize("inner", [False, True])
def test_dual_sa_keeps_a_steady_state(inner):
    """The SA equation with its own dual2ndDST ddt (dual2ndDST.C:456-488,
    turbulence corrected inside the inner loop with innerCorrectTurbulence,
    once after it otherwise): a steady state (W, nuTilda) is a fixed point
    of dual-time steps, since its BDF2 terms vanish and its residuals are
    zero."""
    c, prim = sa_steady()
    d = c.with_options(**{"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
                          "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.05,
                          "timeIntegration.innerCorrectTurbulence": inner, "timeControls.maxCo": 50.0})
    o = OracleSolver(d.mesh, d.bcs, d.options)
    o.set_primitive(*prim)
    reps = o.step(2)
    p2 = o.primitive()
    for a, b in zip(p2, prim):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
    assert all(r["lin_iterations"] >= 1 for r in reps)


@pytest.mark.parametrize("inner", [False, True])
def test_dual_sa_moves_nu_tilda_in_time(inner):
    """From a disturbed nuTilda the dual steps change nuTilda, finite, and
    the two placements of the turbulence update give different paths."""
    c, prim = sa_steady()
    d = c.with_options(**{"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
                          "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.05,
                          "timeIntegration.innerCorrectTurbulence": inner, "timeControls.maxCo": 50.0,
                          "timeIntegration.maxInnerIter": 10})
    nut = prim[3] * (1.0 + 0.5 * np.sin(2.0 * c.mesh.C[:, 0]) ** 2)
    o = OracleSolver(d.mesh, d.bcs, d.options)
    o.set_primitive(prim[0], prim[1], prim[2], nut)
    o.step(2)
    n2 = o.primitive()[3]
    assert np.all(np.isfinite(n2))
    assert np.abs(n2 - nut).max() > 1e-6 * np.abs(nut).max()


def test_adapter_selector_name_selects_dual_time():
    a = dual_case(**{"timeIntegration.maxInnerIter": 3})
    b = a.with_options(**{"timeIntegration.timeIntegration": "GPUDual"})
    ra = OracleSolver(a.mesh, a.bcs, a.options)
    rb = OracleSolver(b.mesh, b.bcs, b.options)
    for o, c in ((ra, a), (rb, b)):
        o.set_primitive(c.p, c.U, c.T)
    x, y = ra.step(1)[0], rb.step(1)[0]
    assert x["lin_iterations"] == y["lin_iterations"] == 4 and x["res_mag"] == y["res_mag"]


@pytest.mark.parametrize("inner", [False, True])
def test_dual_sarc1_keeps_a_steady_state(inner):
    """SARC1 under dual-time stepping: the ddt(rho, S) of its strain-rate
    material derivative vanishes on a steady state at every step: the first
    two, where S.oldTime() and its oldTime() carry one time index (deltaT0
    GREAT, the Euler-like coefficients), and the third, the full BDF2 form."""
    c, prim = sa_steady("SARC1")
    d = c.with_options(**{"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
                          "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.05,
                          "timeIntegration.innerCorrectTurbulence": inner, "timeControls.maxCo": 50.0})
    o = OracleSolver(d.mesh, d.bcs, d.options)
    o.set_primitive(*prim)
    o.step(3)
    for a, b in zip(o.primitive(), prim):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()


def test_dual_sarc1_differs_from_the_model_without_the_multiplier():
    """From a disturbed nuTilda, SARC1's dual steps move nuTilda, finite, and
    away from those of SpalartAllmaras (the same equations without the
    rotation/curvature multiplier)."""
    c, prim = sa_steady("SARC1")
    nut = prim[3] * (1.0 + 0.5 * np.sin(2.0 * c.mesh.C[:, 0]) ** 2)
    out = {}
    for model in ("SARC1", "SpalartAllmaras"):
        d = cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL", limiter="upwind",
                                     model=model).with_options(**{
            "timeControls.maxCo": 50.0, "timeIntegration.timeIntegration": "Dual",
            "ddtSchemes.default": "dual2ndDST", "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.05,
            "timeIntegration.maxInnerIter": 6})
        o = OracleSolver(d.mesh, d.bcs, d.options)
        o.set_primitive(prim[0], prim[1], prim[2], nut)
        o.step(3)
        out[model] = o.primitive()[3]
    n = out["SARC1"]
    assert np.all(np.isfinite(n)) and np.abs(n - nut).max() > 1e-6 * np.abs(nut).max()
    assert np.abs(n - out["SpalartAllmaras"]).max() > 1e-8 * np.abs(n).max()
