"""Hybrid tet/prism mesh (the 3D Mach-3 forward step with jittered
interior nodes) on the B200: residual parity with the FP64 oracle for
HLLC with Venkatakrishnan and OSPRE/OSPREV reconstruction (1e-11 relative
to the field max), a short steady run with subdomain ILU(0) (1e-9 relative
per step; the partition is passed to the oracle), and tangent/adjoint
duality of the discrete adjoint to rounding (1e-10) on the same cells."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver
from tests.test_gpu_adjoint import prepared, random_dirs, smooth_state
from tests.test_gpu_parity import rel

pytestmark = pytest.mark.gpu


def hybrid(limiter="Venkatakrishnan", **opts):
    c = cases.forward_step_3d_hybrid_c5(nx=30, ny=10, nz=6, limiter=limiter, precision="fp64")
    return c.with_options(**opts) if opts else c


@pytest.mark.parametrize("limiter", ["Venkatakrishnan", "OSPRE"])
def test_hybrid_residual_parity(limiter):
    c = hybrid(limiter)
    W = smooth_state(c)
    gpu = rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    ora = OracleSolver(c.mesh, c.bcs, c.options)
    for s in (gpu, ora):
        s.set_conservative(*W)
    Rg, Ro = gpu.residual(), ora.residual()
    assert np.all(np.isfinite(Rg))
    for k in range(5):
        assert rel(Rg[:, k], Ro[:, k]) < 1e-11, (limiter, k)


def test_hybrid_steps_parity():
    c = hybrid(**{"ilu.parts": 4})
    part = rhodst_b200.partition_cells(c.mesh.C, 4)
    gpu = rhodst_b200.solver_for(c)
    ora = OracleSolver(c.mesh, c.bcs, c.options, partition=part)
    ora.set_primitive(c.p, c.U, c.T)
    for k in range(5):
        rg, ro = gpu.step(1)[0], ora.step(1)[0]
        for key in ("res_l2",):
            assert rel(rg[key], ro[key]) < 1e-9, (k, key, rg[key], ro[key])
    for a, b in zip(gpu.conservative(), ora.conservative()):
        assert rel(a, b) < 1e-9


@pytest.mark.parametrize("limiter", ["Venkatakrishnan", "OSPRE", "upwind"])
def test_hybrid_adjoint_transposes_tangent(limiter):
    c = hybrid(limiter)
    W = smooth_state(c)
    s = prepared(c, W)
    u, v = random_dirs(c.mesh.n_cells, W, seed=13)
    ATv, _ = s.adjoint_product(v)
    Ju = s.tangent_product(u)
    lhs, rhs = float(np.sum(v * Ju)), float(np.sum(ATv * u))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (limiter, lhs, rhs)
