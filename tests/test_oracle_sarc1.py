"""SARC1 (Spalart-Shur rotation/curvature correction with the material
derivative of the strain rate, SARC1.C:125-180) in the oracle: it runs on
the turbulent airfoil, its multiplier is active (the nuTilda field departs
from SARC2's, whose multiplier has no strain-rate history), and a new state
restarts the old-time strain rate (the same state and nuTilda set twice give
the same next step whatever ran before)."""
import numpy as np

from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver


def airfoil(model):
    return cases.naca0012_turbulent(ni=97, nj=25, model=model, first_cell=5e-3)


def run(case, steps):
    o = OracleSolver(case.mesh, case.bcs, case.options)
    o.set_primitive(case.p, case.U, case.T, case.nuTilda)
    reps = o.step(steps)
    return o, reps


def test_sarc1_runs_and_differs_from_sarc2():
    o1, r1 = run(airfoil("SARC1"), 4)
    o2, r2 = run(airfoil("SARC2"), 4)
    n1 = o1.primitive()[3]
    n2 = o2.primitive()[3]
    assert np.all(np.isfinite(n1)) and np.all(n1 >= 0)
    assert all(np.all(np.isfinite(r["res_l2"])) for r in r1)
    assert np.abs(n1 - n2).max() > 1e-6 * np.abs(n2).max()


def test_new_state_restarts_the_old_time_strain_rate():
    case = airfoil("SARC1")
    a, _ = run(case, 3)
    p, U, T, nut = a.primitive()
    W = a.conservative()
    # b: a different history, then the same state as a
    b, _ = run(case, 1)
    for s in (a, b):
        s.set_primitive(p, U, T, nut)
    ra, rb = a.step(1)[0], b.step(1)[0]
    assert np.array_equal(ra["res_l2"], rb["res_l2"])
    assert np.array_equal(a.primitive()[3], b.primitive()[3])
    assert W[0].shape[0] == case.mesh.n_cells


def test_frozen_turbulence_holds_nu_tilda():
    """frozenTurbulence skips the turbulence update: nuTilda stays while the
    mean flow moves."""
    case = airfoil("SAneg").with_options(frozenTurbulence=True)
    o, _ = run(case, 3)
    p, U, T, nut = o.primitive()
    assert np.array_equal(nut, case.nuTilda)
    assert np.abs(p - case.p).max() > 0
