"""C ABI checks that need no GPU: the library loads, exports every symbol
the header declares, host-only entry points work, and configuration errors
are reported with the reference's selector semantics before any device
work."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import _abi, cases

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "rdst.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rdst_[a-z_]+)\s*\(", text)))


def test_header_symbols_exported(gpulib):
    names = header_functions()
    assert "rdst_step" in names and "rdst_create" in names
    for n in names:
        assert hasattr(gpulib, n), n


def test_version(gpulib):
    assert b"sm_100a" in gpulib.rdst_version()


def test_partition_host_only():
    m = cases.forward_step_c1().mesh
    part = rhodst_b200.partition_cells(m.C, 8)
    counts = np.bincount(part, minlength=8)
    assert counts.sum() == m.n_cells and counts.min() >= m.n_cells // 8 - 1
    part2 = rhodst_b200.partition_cells(m.C, 8)
    assert np.array_equal(part, part2)


@pytest.mark.parametrize("key,value,status", [
    ("fluxScheme", "Roe", 1),                      # unknown selector -> FatalError analogue
    ("Jacobian", "Steger", 1),
    ("solvers.W.preconditioner", "SAMG", 6),       # selectable in foam, not on this path
    ("solvers.W.smoother", "GaussSeidel", 6),       # AMG smoothing is block Jacobi here
    ("amg.omega", "1.5", 1),
    ("solvers.W.nPostSweeps", "-1", 1),
    ("directWaveSpeed", "false", 6),               # latent reference bug rejected
    ("ddtSchemes.default", "dual2ndDST", 6),
    ("timeIntegration.timeIntegration", "Dual", 6),
    ("interpolationSchemes.reconstruct(U)", "OSPRE", 6),
    ("solvers.W.nDirections", "0", 1),
    ("RASModel", "kEpsilon", 1),
    ("timeIntegration.maxInnerIter", "-1", 1),
    ("solvers.W.solver", "CG", 1),                 # symmetric matrices only in foam-extend
    ("solvers.W.preconditioner", "ILUCq", 1),
    ("solvers.W.nSweeps", "0", 1),
    ("solvers.W.fillInLevel", "4", 1),
    ("ilu.partition", "scotch", 1),
    ("device", "gpu0", 1),
    ("gradSchemes.grad(U)", "cellLimited Gauss linear 2", 1),
    ("gradSchemes.grad(U)", "leastSquares", 6),
    ("divSchemes.div(phi,nuTilda)", "Gauss QUICK", 6),
])
def test_config_errors(key, value, status):
    case = cases.forward_step_c1().with_options(**{key: value})
    with pytest.raises(_abi.RdstError) as e:
        rhodst_b200.Solver(case.mesh, case.bcs, case.options)
    assert e.value.status == status


def test_missing_flux_scheme():
    case = cases.forward_step_c1()
    opts = dict(case.options)
    del opts["fluxScheme"]
    with pytest.raises(_abi.RdstError) as e:
        rhodst_b200.Solver(case.mesh, case.bcs, opts)
    assert e.value.status == 1


def test_flatten_options():
    f = _abi.flatten_options({"a": {"b": True, "c": (1.0, 2)}, "d": 1e-3})
    assert f == {"a.b": "true", "a.c": "1.0 2", "d": "0.001"}


def test_valid_options_reach_the_device_check():
    """Options this path takes pass parsing; without a GPU the context
    then fails at the CUDA device check, not earlier."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    for case in (cases.forward_step_c1().with_options(**{"timeIntegration.timeIntegration": "Dual",
                                                         "ddtSchemes.default": "dual2ndDST"}),
                 cases.rae2822(), cases.rae2822(tutorial_schemes=True),
                 cases.naca0012_turbulent(ni=97, nj=25, model="SARC1", first_cell=5e-3),
                 cases.naca0012_turbulent(ni=97, nj=25, model="SARC1", first_cell=5e-3).with_options(**{
                     "timeIntegration.timeIntegration": "Dual", "ddtSchemes.default": "dual2ndDST"}),
                 *[cases.forward_step_c1().with_options(**o) for o in (
                     {"solvers.W.solver": "GaussSeidel", "solvers.W.nSweeps": 2},
                     {"solvers.W.solver": "ILU"},
                     {"solvers.W.preconditioner": "Cholesky"},
                     {"solvers.W.preconditioner": {"preconditioner": "GaussSeidel", "nSweeps": 3}},
                     {"solvers.W.preconditioner": "ILUCp", "solvers.W.fillInLevel": 1},
                     {"solvers.W.preconditioner": "AMG", "solvers.W.nPreSweeps": 1},
                     {"solvers.W.solver": "AMG", "solvers.W.smoother": "Jacobi"},
                     {"device": 0, "ilu.partition": "graph"},
                     {"gradSchemes.grad(U)": "cellLimited Gauss linear 0.5"})]):
        with pytest.raises(_abi.RdstError) as e:
            rhodst_b200.Solver(case.mesh, case.bcs, case.options)
        assert e.value.status == 3, case.name


def test_set_geometry_checks_its_arguments(gpulib):
    gpulib.rdst_set_geometry.restype = ctypes.c_int32
    gpulib.rdst_set_geometry.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert gpulib.rdst_set_geometry(None, None) == 7


def _graph_bisection_reference(m, n_parts):
    """Restatement with scipy: order each set by breadth-first distance from
    the cell farthest from its first cell (then by index), cut at the
    proportional rank, unreached cells last."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import breadth_first_order
    N, Fi = m.n_cells, m.n_internal_faces
    own = np.asarray(m.owner)[:Fi].astype(np.int64)
    nei = np.asarray(m.neighbour)[:Fi].astype(np.int64)
    A = sp.coo_matrix((np.ones(Fi), (own, nei)), shape=(N, N)).tocsr()
    A = (A + A.T).tocsr()

    def dist(G, src):
        order, pred = breadth_first_order(G, src, directed=False, return_predecessors=True)
        d = np.full(G.shape[0], -1, dtype=np.int64)
        d[src] = 0
        for v in order[1:]:
            d[v] = d[pred[v]] + 1
        return d

    out = np.zeros(N, dtype=np.int64)

    def rec(cells, n, p0):
        if n <= 1 or cells.size <= 1:
            out[cells] = p0
            return
        G = A[cells][:, cells]
        d = dist(G, int(np.argmax(dist(G, 0))))
        d[d < 0] = d.max() + 1
        order = np.lexsort((cells, d))
        k = cells.size * (n // 2) // n
        rec(cells[order[:k]], n // 2, p0)
        rec(cells[order[k:]], n - n // 2, p0 + n // 2)

    rec(np.arange(N), n_parts, 0)
    return out


def _level_chains(m, part):
    """Longest wavefront chain (levels) of each part in cell order."""
    Fi = m.n_internal_faces
    own = np.asarray(m.owner)[:Fi]
    nei = np.asarray(m.neighbour)[:Fi]
    level = np.zeros(m.n_cells, dtype=np.int64)
    same = part[own] == part[nei]
    lower = [[] for _ in range(m.n_cells)]
    for a, b in zip(own[same], nei[same]):
        lower[b].append(a)
    for i in range(m.n_cells):
        if lower[i]:
            level[i] = 1 + max(level[k] for k in lower[i])
    mx = np.zeros(part.max() + 1, dtype=np.int64)
    np.maximum.at(mx, part, level)
    return mx + 1


def test_graph_partition_host_only():
    m = cases.naca0012_inviscid(ni=129, nj=33, first_cell=2e-3).mesh
    part = rhodst_b200.partition_graph(m, 16)
    sizes = np.bincount(part, minlength=16)
    assert sizes.sum() == m.n_cells and sizes.max() - sizes.min() <= 1
    assert np.array_equal(part, rhodst_b200.partition_graph(m, 16))
    assert np.array_equal(part, _graph_bisection_reference(m, 16))
    # graph slabs have shorter level chains than coordinate boxes here
    lg = _level_chains(m, part)
    lr = _level_chains(m, rhodst_b200.partition_cells(m.C, 16))
    assert lg.max() <= lr.max() and lg.mean() < lr.mean(), (lg.max(), lr.max(), lg.mean(), lr.mean())
