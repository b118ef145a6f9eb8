"""B200 library vs. CPU oracle with the RAE2822 tutorial's gradient and
convection schemes (system/fvSchemes): grad(U) cellLimited Gauss linear 1
(the viscous stress, the corrected laplacian and the SA vorticity use the
limited gradient) and div(phi,nuTilda) Gauss linearUpwind grad(nuTilda).
Residuals agree to 1e-11 relative, step trajectories to 1e-8 (the SA
wall-layer rounding amplification of the other SA parity tests).  The
adjoint, which does not linearize the limiter, is refused with
RDST_ERR_UNSUPPORTED."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import _abi, cases
from tests.oracle_lib import OracleSolver
from tests.test_oracle_tutorial_schemes import laminar, sa_case, wavy_state

pytestmark = pytest.mark.gpu

LIMITED = {"gradSchemes.grad(U)": "cellLimited Gauss linear 1"}
LIN_UP = {"divSchemes.div(phi,nuTilda)": "Gauss linearUpwind grad(nuTilda)"}


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("k", ["1", "0.5"])
def test_cell_limited_viscous_residual(k):
    c = laminar(**{"gradSchemes.grad(U)": f"cellLimited Gauss linear {k}"})
    U = wavy_state(c)
    gpu = rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    ora = OracleSolver(c.mesh, c.bcs, c.options)
    for s in (gpu, ora):
        s.set_primitive(c.p, U, c.T)
    assert rel(gpu.residual(), ora.residual()) < 1e-11


def _steps(c, n, parts=4, nut=None):
    c = c.with_options(**{"ilu.parts": parts})
    part = rhodst_b200.partition_cells(c.mesh.C, parts)
    gpu = rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    ora = OracleSolver(c.mesh, c.bcs, c.options, partition=part)
    for s in (gpu, ora):
        s.set_primitive(c.p, c.U, c.T, c.nuTilda if nut is None else nut)
    rg, ro = gpu.step(n), ora.step(n)
    for a, b in zip(rg, ro):
        assert abs(a["res_mag"] - b["res_mag"]) <= 1e-8 * abs(b["res_mag"])
    for a, b in zip(gpu.primitive(), ora.primitive()):
        assert rel(a, b) < 1e-8
    return gpu


def test_sa_steps_with_the_tutorial_schemes():
    c = sa_case(**LIMITED, **LIN_UP)
    nut = c.nuTilda * (1.0 + 0.5 * np.sin(0.3 * c.mesh.C[:, 0]) ** 2)
    _steps(c, 5, nut=nut)


def test_rae2822_tutorial_schemes_steps():
    _steps(cases.rae2822(tutorial_schemes=True), 5, parts=8)


def test_adjoint_of_the_limited_gradient_is_refused():
    c = laminar(**LIMITED)
    s = rhodst_b200.solver_for(c)
    s.step(2)
    with pytest.raises(_abi.RdstError) as e:
        s.adjoint("airfoil", (1.0, 0.0, 0.0), p_ref=1.0)
    assert e.value.status == 6
