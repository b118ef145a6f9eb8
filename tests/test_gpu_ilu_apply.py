"""Subdomain ILU(0) apply on the GPU: the bulk-copy apply (task records
brought into shared memory by one TMA copy per task) against the register
apply, and the breadth-first factorisation order against the oracle.

Tolerances: FP64 trajectories of the two applies agree to 1e-12 relative
per step (they multiply the same factors in a different summation order:
the bulk apply sums each block's product before subtracting it, as the
oracle does); the reduced-precision applies differ in arithmetic (the bulk
apply multiplies FP32 factors in FP32, the register apply in FP64), so
their states agree to 1e-6 after three steps, far below the FP32 factor
rounding.  Breadth-first order: GPU vs oracle 1e-9 per step, as the other
ILU step tests."""
import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _steps(case, n):
    s = rhodst_b200.solver_for(case)
    reps = s.step(n)
    return reps, s.conservative()


def _wing():
    return cases.swept_wing_c3(n_around=48, n_normal=16, n_span=8, n_tip=4, ilu_parts=6)


@pytest.mark.parametrize("order", ["natural", "bfs"])
@pytest.mark.parametrize("which", ["step", "wing"])
def test_bulk_apply_matches_register_apply_fp64(which, order):
    base = (cases.forward_step_c1(preconditioner="ILUC0", n_directions=10).with_options(**{"ilu.parts": 8})
            if which == "step" else _wing())
    out = {}
    for bulk in (True, False):
        out[bulk] = _steps(base.with_options(**{"ilu.bulk": bulk, "ilu.order": order}), 5)
    (ra, Wa), (rb, Wb) = out[True], out[False]
    for a, b in zip(ra, rb):
        assert a["lin_iterations"] == b["lin_iterations"]
        assert abs(a["res_mag"] - b["res_mag"]) <= 1e-12 * abs(b["res_mag"])
    for a, b in zip(Wa, Wb):
        assert rel(a, b) < 1e-12


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_bulk_apply_reduced_precision(prec):
    base = _wing().with_options(precision=prec)
    out = {}
    for bulk in (True, False):
        out[bulk] = _steps(base.with_options(**{"ilu.bulk": bulk}), 3)
    for a, b in zip(out[True][1], out[False][1]):
        assert rel(a, b) < 1e-6


@pytest.mark.parametrize("parts", [1, 8])
def test_bfs_order_steps_match_oracle(parts):
    """ILU(0) factorised in breadth-first order (one part: the whole mesh,
    the renumberMesh analogue; eight parts: each subdomain) on the GPU and
    in the oracle, same partition."""
    case = cases.forward_step_c1(preconditioner="ILUC0", n_directions=10).with_options(
        **{"ilu.parts": parts, "ilu.order": "bfs"})
    part = rhodst_b200.partition_cells(case.mesh.C, parts) if parts > 1 else None
    gpu = rhodst_b200.Solver(case.mesh, case.bcs, case.options)
    ora = OracleSolver(case.mesh, case.bcs, case.options, partition=part)
    for s in (gpu, ora):
        s.set_primitive(case.p, case.U, case.T)
    rg, ro = gpu.step(5), ora.step(5)
    for a, b in zip(rg, ro):
        assert a["lin_iterations"] == b["lin_iterations"]
        assert abs(a["res_mag"] - b["res_mag"]) <= 1e-9 * abs(b["res_mag"])
    for a, b in zip(gpu.conservative(), ora.conservative()):
        assert rel(a, b) < 1e-9
