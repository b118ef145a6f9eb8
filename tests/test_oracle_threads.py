"""The oracle's threaded loops (the CPU baseline runs it on all host cores):
fields, residual histories and linear-solver reports are the same bit for
bit for any thread count, and the RCB partition into processor subdomains
covers every cell with balanced part sizes."""
import numpy as np
import pytest

from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver, set_threads


def run(case, steps, rcb_parts=None):
    o = OracleSolver(case.mesh, case.bcs, case.options, rcb_parts=rcb_parts)
    o.set_primitive(case.p, case.U, case.T, case.nuTilda)
    R = o.residual()
    A = o.assemble()
    reps = o.step(steps)
    return R, A, o.conservative(), [(r["res_l2"], r["lin_final"], r["lin_iterations"]) for r in reps]


@pytest.fixture
def threads():
    yield set_threads
    set_threads(0)


@pytest.mark.parametrize("name", ["c1", "airfoil", "laminar"])
def test_results_do_not_depend_on_the_thread_count(name, threads):
    case = {"c1": lambda: cases.forward_step_c1(),
            "airfoil": lambda: cases.naca0012_inviscid(ni=97, nj=25, first_cell=5e-3),
            "laminar": lambda: cases.naca0012_laminar(ni=97, nj=25, first_cell=5e-3, sutherland=True)}[name]()
    parts = None if name == "c1" else 6
    out = []
    for n in (1, 3):
        assert threads(n) == n
        out.append(run(case, 3, rcb_parts=parts))
    (R1, A1, W1, h1), (R3, A3, W3, h3) = out
    assert np.array_equal(R1, R3)
    for a, b in zip(A1, A3):
        assert np.array_equal(a, b)
    for a, b in zip(W1, W3):
        assert np.array_equal(a, b)
    for (r1, l1, i1), (r3, l3, i3) in zip(h1, h3):
        assert np.array_equal(r1, r3) and np.array_equal(l1, l3) and i1 == i3


def test_rcb_partition_is_balanced():
    case = cases.naca0012_inviscid(ni=97, nj=25, first_cell=5e-3)
    N = case.mesh.n_cells
    for n in (2, 7, 16):
        o = OracleSolver(case.mesh, case.bcs, case.options, rcb_parts=n)
        part = o.partition()
        sizes = np.bincount(part, minlength=n)
        assert sizes.size == n and sizes.sum() == N
        assert sizes.max() - sizes.min() <= 1, sizes
        # the partition only changes the preconditioner: a step still runs
        o.set_primitive(case.p, case.U, case.T)
        assert np.all(np.isfinite(o.step(1)[0]["res_l2"]))
