"""Shape gradient of the airfoil's pressure drag with respect to 64
Hicks-Henne bump amplitudes, by the discrete adjoint on the B200.

(1) rdst_set_geometry: a context moved onto a mesh of the same topology
    evaluates the residual and objective of a context built on that mesh
    (bit for bit: the per-cell face order does not depend on the geometry);
    a mesh of another topology is rejected and the context is unchanged.
(2) dJ/da at a seeded design point (amplitudes U[-1e-3, 1e-3] chord, seed
    1234) against central differences of the converged J with step 1e-6
    (first-order reconstruction, converged to round-off; the perturbed
    solves warm-start from the design point's solution): the largest
    component, and all 64 along a seeded +-1 direction, 1e-5 relative.
(3) All 64 components against a CPU reference gradient: psi from a sparse
    direct solve with the complex-step Jacobian of the oracle, the explicit
    derivatives by central differences of the oracle's residual and
    objective on the moved meshes; 1e-6 relative to the largest component
    (Kurganov and HLL).
"""
import copy
import ctypes

import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import mesh as M
from rhodst_b200.shape import HicksHenne, shape_gradient
from tests.oracle_lib import ComplexStep, OracleSolver
from tests.test_gpu_adjoint import airfoil, converge, converged, prepared, smooth_state
from tests.test_gpu_adjoint_cs import complex_step_adjoint

pytestmark = pytest.mark.gpu

ALPHA = np.radians(2.3)
DRAG = (np.cos(ALPHA), np.sin(ALPHA), 0.0)


def design_case(flux="Kurganov", limiter="upwind"):
    c = airfoil(flux=flux, limiter=limiter)
    hh = HicksHenne(c.mesh)
    a0 = hh.design_point(hh.n_variables)
    c.mesh = hh.mesh(a0)
    return c, hh, a0


def on_mesh(case, m):
    c = copy.copy(case)
    c.mesh = m
    return c


def test_set_geometry_matches_a_fresh_context():
    c, hh, a0 = design_case(flux="HLLC", limiter="Venkatakrishnan")
    W = smooth_state(c)
    s = prepared(c, W)
    a1 = a0 + np.random.default_rng(3).uniform(-1e-3, 1e-3, a0.size)
    m1 = hh.mesh(a1)
    s.set_geometry(m1)
    s.set_conservative(*W)
    R_moved = s.residual()
    J_moved = s.objective_gradient("airfoil", DRAG, p_ref=1.0)[0]
    fresh = prepared(on_mesh(c, m1), W)
    R_fresh = fresh.residual()
    J_fresh = fresh.objective_gradient("airfoil", DRAG, p_ref=1.0)[0]
    assert np.array_equal(R_moved, R_fresh)
    assert J_moved == J_fresh
    # another topology is refused and leaves the context as it was (the
    # residual without a new state keeps the boundary record, whose in/out
    # and sub/supersonic branches follow the previous evaluation)
    R_before = s.residual()
    other = M.naca_cmesh(97, 23, first_cell=5e-3)
    with pytest.raises(ValueError):
        s.set_geometry(other)
    with pytest.raises(rhodst_b200.RdstError):         # the library's own check
        s._check(s._fn("set_geometry")(s._h, ctypes.byref(s._c_mesh(other))), "set_geometry")
    assert np.array_equal(s.residual(), R_before)


def test_shape_gradient_matches_central_differences():
    c, hh, a0 = design_case(flux="Kurganov")
    s, drop, r0 = converge(c)
    assert drop < 1e-11, drop
    W0 = s.conservative()
    g, rep, _ = shape_gradient(s, hh, a0, "airfoil", DRAG, p_ref=1.0, rel_tol=1e-11)
    assert rep["residual"] <= 1e-10 * rep["residual0"], rep
    h = 1e-6
    k = int(np.argmax(np.abs(g)))
    v = np.random.default_rng(5).choice([-1.0, 1.0], size=g.size)
    # one amplitude, and all 64 at once along a seeded +-1 direction
    # (tolerance relative to sum |g_k v_k|, the scale of the terms)
    for d, expected, scale in ((np.eye(g.size)[k], g[k], abs(g[k])), (v, g @ v, np.abs(g).sum())):
        Js = []
        for sgn in (1.0, -1.0):
            sk, dk, _ = converge(on_mesh(c, hh.mesh(a0 + sgn * h * d)), W0=W0, r_ref=r0)
            assert dk < 1e-11, dk
            Js.append(sk.objective_gradient("airfoil", DRAG, p_ref=1.0)[0])
        fd = (Js[0] - Js[1]) / (2 * h)
        assert abs(expected - fd) <= 1e-5 * scale, (k, expected, fd, scale)


def reference_shape_gradient(case, hh, a0, W, branches, h=1e-6):
    """CPU reference: psi of the complex-step reference of the oracle, the
    explicit derivatives by central differences of the oracle's residual
    and objective on the moved meshes (same branches)."""
    _, Wa, psi = complex_step_adjoint(case, W, branches, "airfoil", DRAG, 1.0, hops=2)
    g = np.zeros(hh.n_variables)
    for k in range(hh.n_variables):
        Rs, Js = [], []
        for sgn in (1.0, -1.0):
            ak = a0.copy()
            ak[k] += sgn * h
            ok = OracleSolver(hh.mesh(ak), case.bcs, case.options)
            ok.set_conservative(*W)
            ck = ComplexStep(ok)
            Rs.append(ck.residual(Wa, None, None, branches=branches)[0])
            Js.append(ck.objective(Wa, "airfoil", DRAG, p_ref=1.0, branches=branches)[0])
        g[k] = (Js[0] - Js[1]) / (2 * h) - float(np.sum(psi * (Rs[0] - Rs[1]))) / (2 * h)
    return g


@pytest.mark.parametrize("flux", ["Kurganov", "HLL"])
def test_shape_gradient_matches_cpu_reference(flux):
    c, hh, a0 = design_case(flux=flux)
    s, drop = converged(c)
    assert drop < 1e-11, drop
    W = s.conservative()
    s.set_conservative(*W)
    s.residual()
    s.set_conservative(*W)
    branches = s.boundary_branches()
    g, rep, _ = shape_gradient(s, hh, a0, "airfoil", DRAG, p_ref=1.0, rel_tol=1e-12)
    assert rep["residual"] <= 1e-11 * rep["residual0"], rep
    ref = reference_shape_gradient(c, hh, a0, W, branches)
    assert np.abs(g - ref).max() <= 1e-6 * np.abs(ref).max(), (np.abs(g - ref).max(), np.abs(ref).max())
