"""Dual-time stepping with Spalart-Allmaras on the B200 against the oracle:
the nuTilda equation with its own dual2ndDST ddt, the turbulence update
inside the inner loop (innerCorrectTurbulence) or once after it.  Three
physical steps from a disturbed nuTilda; inner-iteration counts equal,
states 1e-8 relative (the SA parity tolerance of the other SA tests).
SARC1 takes dual2ndDST's ddt(rho, S) over the physical steps in its
strain-rate material derivative: four steps, so that both the steps whose
old times are copies and the full second-order form are compared."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.mark.parametrize("inner", [False, True])
def test_dual_sa_steps(inner):
    c = cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL", limiter="upwind")
    c = c.with_options(**{"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
                          "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.05,
                          "timeIntegration.innerCorrectTurbulence": inner, "timeControls.maxCo": 50.0,
                          "timeIntegration.maxInnerIter": 8, "ilu.parts": 2})
    part = rhodst_b200.partition_cells(c.mesh.C, 2)
    gpu = rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    ora = OracleSolver(c.mesh, c.bcs, c.options, partition=part)
    nut = c.nuTilda * (1.0 + 0.5 * np.sin(2.0 * c.mesh.C[:, 0]) ** 2)
    for s in (gpu, ora):
        s.set_primitive(c.p, c.U, c.T, nut)
    rg, ro = gpu.step(3), ora.step(3)
    for a, b in zip(rg, ro):
        assert a["lin_iterations"] == b["lin_iterations"]
        assert abs(a["deltaT"] - b["deltaT"]) <= 1e-12 * abs(b["deltaT"])
    for a, b in zip(gpu.primitive(), ora.primitive()):
        assert rel(a, b) < 1e-8


@pytest.mark.parametrize("inner", [False, True])
def test_dual_sarc1_steps(inner):
    """SARC1 with dual-time stepping, four physical steps from a disturbed
    nuTilda on a 65x17 airfoil (Re 1e5, first cell 1e-2).  Mean-flow fields
    at 1e-8; nuTilda at 1e-8 of its maximum beyond 0.1 chord from the wall
    and 1e-4 overall: DS/Dt divides a difference of nearly equal strain
    rates by the time step, which amplifies rounding in the wall layer (the
    single-step SARC1 parity test holds the same bounds for that reason)."""
    c = cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL", limiter="upwind",
                                 model="SARC1")
    c = c.with_options(**{"timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST",
                          "timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.05,
                          "timeIntegration.innerCorrectTurbulence": inner, "timeControls.maxCo": 50.0,
                          "timeIntegration.maxInnerIter": 8, "ilu.parts": 2})
    part = rhodst_b200.partition_cells(c.mesh.C, 2)
    gpu = rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    ora = OracleSolver(c.mesh, c.bcs, c.options, partition=part)
    nut = c.nuTilda * (1.0 + 0.5 * np.sin(2.0 * c.mesh.C[:, 0]) ** 2)
    for s in (gpu, ora):
        s.set_primitive(c.p, c.U, c.T, nut)
    rg, ro = gpu.step(4), ora.step(4)
    for a, b in zip(rg, ro):
        assert a["lin_iterations"] == b["lin_iterations"]
        assert abs(a["deltaT"] - b["deltaT"]) <= 1e-12 * abs(b["deltaT"])
    pg, po = gpu.primitive(), ora.primitive()
    for a, b in zip(pg[:3], po[:3]):
        assert rel(a, b) < 1e-8
    ng, no = pg[3], po[3]
    away = c.mesh.wall_distance >= 0.1
    assert np.abs(ng - no)[away].max() <= 1e-8 * np.abs(no).max()
    assert rel(ng, no) < 1e-4
