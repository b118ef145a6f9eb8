"""Failure detection, made on the host: a NaN or a negative pressure in the
state a caller hands over, and a linear solve cut short by maxIter.

updateFields.H bounds rho, h and p; a state that is still NaN or
non-positive after the bounding ends the step with RDST_ERR_DIVERGED (both
the B200 library and the oracle).  A block solve that stops on maxIter with
neither tolerance nor relTol reached sets bit 3 of the step report's flags
(the solver performance's converged() is false); one that reaches its
tolerance clears it.  The oracle cases run on the CPU; the same cases on the
GPU are marked gpu."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases
from rhodst_b200._abi import RdstError
from tests.oracle_lib import OracleSolver

RDST_ERR_DIVERGED = 4
NOT_CONVERGED = 8


def _solver(kind, case):
    if kind == "gpu":
        return rhodst_b200.Solver(case.mesh, case.bcs, case.options)
    return OracleSolver(case.mesh, case.bcs, case.options)


def _case():
    # density and pressure bounds wide open, so a negative pressure is not
    # clamped away by the bounding
    return cases.forward_step_c1().with_options(**{"fieldBounds.p": "-1e30 1e30", "fieldBounds.rho": "-1e30 1e30"})


def _nan_state(case):
    g = case.options["thermo"]
    rho = case.p / (g["R"] * case.T)
    rhoU = rho[:, None] * case.U
    rhoE = rho * ((g["Cp"] - g["R"]) * case.T + 0.5 * (case.U ** 2).sum(1))
    rho = rho.copy()
    rho[123] = np.nan
    return rho, rhoU, rhoE


def _negative_pressure_state(case):
    p = case.p.copy()
    p[200:210] = -0.5
    return p, case.U, case.T


def _check_nan(kind):
    case = _case()
    s = _solver(kind, case)
    s.set_conservative(*_nan_state(case))
    with pytest.raises(RdstError) as e:
        s.step(1)
    assert e.value.status == RDST_ERR_DIVERGED
    assert "non-physical" in str(e.value)


def _check_negative_pressure(kind):
    case = _case()
    s = _solver(kind, case)
    p, U, T = _negative_pressure_state(case)
    s.set_primitive(p, U, T)
    with pytest.raises(RdstError) as e:
        s.step(1)
    assert e.value.status == RDST_ERR_DIVERGED


def _check_max_iter(kind):
    # one GMRES(2) cycle against an unreachable tolerance: stops on maxIter
    cut = cases.forward_step_c1(n_directions=2, max_iter=1).with_options(
        **{"solvers.W.tolerance": 1e-30, "solvers.W.relTol": 0.0})
    s = _solver(kind, cut)
    s.set_primitive(cut.p, cut.U, cut.T)
    rep = s.step(1)[0]
    assert rep["flags"] & NOT_CONVERGED
    assert rep["lin_iterations"] == 1
    assert max(rep["lin_final"]) > 1e-30
    # a tolerance the first cycle reaches: converged, bit clear
    ok = cases.forward_step_c1(n_directions=20, max_iter=50).with_options(
        **{"solvers.W.tolerance": 1e-3, "solvers.W.relTol": 0.0})
    s = _solver(kind, ok)
    s.set_primitive(ok.p, ok.U, ok.T)
    rep = s.step(1)[0]
    assert not rep["flags"] & NOT_CONVERGED
    assert max(rep["lin_final"]) < 1e-3


def test_oracle_nan_state_diverges():
    _check_nan("oracle")


def test_oracle_negative_pressure_diverges():
    _check_negative_pressure("oracle")


def test_oracle_max_iter_flag():
    _check_max_iter("oracle")


@pytest.mark.gpu
def test_gpu_nan_state_diverges():
    _check_nan("gpu")


@pytest.mark.gpu
def test_gpu_negative_pressure_diverges():
    _check_negative_pressure("gpu")


@pytest.mark.gpu
def test_gpu_max_iter_flag():
    _check_max_iter("gpu")
