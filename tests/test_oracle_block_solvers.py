"""Known answers for the oracle's other selectable block preconditioners and
solvers (foam-extend's BlockCholeskyPrecon, BlockGaussSeidelPrecon,
BlockILUCpPrecon, BlockGaussSeidelSolver and BlockILUSolver, instantiated
for the 5x5 block matrix at libraries/vector5/Vector5typedefs/
Vector5typedefs.C:1602-1708), checked against dense algebra on small
assembled systems:

* Cholesky: the diagonal-based incomplete factorisation
  M = (D~ + L) D~^-1 (D~ + U) with D~_i = A_ii - sum_{k<i} A_ik D~_k^-1 A_ki;
  it equals ILUC0 on a mesh whose cell graph has no triangles (quads, and
  the Kuhn tetrahedra of the hybrid step) and differs from it where three
  cells are pairwise neighbours;
* Gauss-Seidel: one application is (D + L)^-1 b, n sweeps are n steps of
  the forward Gauss-Seidel iteration from zero; across partition parts the
  couplings enter only through the residual;
* ILUCp: fillInLevel 0 is ILUC0; level p reproduces A on the pattern of
  cells within p + 1 faces; a level that covers the whole graph is exact LU;
* the stationary solvers converge to numpy.linalg.solve.
"""
import numpy as np
import pytest

from rhodst_b200 import cases, mesh as meshmod
from tests.oracle_lib import OracleSolver
from tests.test_oracle_known_answers import channel_case, dense_system


def oracle_for(c, seed, partition=None):
    o = OracleSolver(c.mesh, c.bcs, c.options, partition=partition)
    rng = np.random.default_rng(seed)
    o.set_primitive(c.p * (1 + 0.1 * rng.random(c.mesh.n_cells)), c.U, c.T)
    return o


def precon_matrix(o, n):
    return np.stack([o.precondition(np.eye(n)[:, k]).ravel() for k in range(n)], axis=1)


def cell_graph(m):
    N = m.n_cells
    adj = [set() for _ in range(N)]
    for f in range(m.n_internal_faces):
        a, b = int(m.owner[f]), int(m.neighbour[f])
        adj[a].add(b)
        adj[b].add(a)
    return adj


def blocks(A, i, j):
    return A[5 * i:5 * i + 5, 5 * j:5 * j + 5]


def dilu_reference(A, N, part=None):
    """(D~ + L) D~^-1 (D~ + U) in cell order, same-part couplings only."""
    same = (lambda a, b: True) if part is None else (lambda a, b: part[a] == part[b])
    Dt = [blocks(A, i, i).copy() for i in range(N)]
    Dinv = [None] * N
    for i in range(N):
        for k in range(i):
            if same(i, k) and np.any(blocks(A, i, k)):
                Dt[i] = Dt[i] - blocks(A, i, k) @ Dinv[k] @ blocks(A, k, i)
        Dinv[i] = np.linalg.inv(Dt[i])
    L = np.zeros_like(A)
    U = np.zeros_like(A)
    Dm = np.zeros_like(A)
    for i in range(N):
        Dm[5 * i:5 * i + 5, 5 * i:5 * i + 5] = Dt[i]
        for j in range(N):
            if i != j and same(i, j):
                (L if j < i else U)[5 * i:5 * i + 5, 5 * j:5 * j + 5] = blocks(A, i, j)
    return (Dm + L) @ np.linalg.inv(Dm) @ (Dm + U)


def split_channel_case(nx=4, ny=3, M=2.0):
    """The channel as prisms: each quad split along a diagonal and each
    triangle at its centroid into three, so the three cells around a
    centroid are pairwise face neighbours (triangles in the cell graph)."""
    X = np.linspace(0, 2.0, nx + 1)
    Y = np.linspace(0, 1.0, ny + 1)
    p2 = np.stack(np.meshgrid(X, Y, indexing="ij"), -1).reshape(-1, 2)
    vid = np.arange((nx + 1) * (ny + 1)).reshape(nx + 1, ny + 1)
    tris = []
    for i in range(nx):
        for j in range(ny):
            a, b, c_, d = vid[i, j], vid[i + 1, j], vid[i + 1, j + 1], vid[i, j + 1]
            tris += [(a, b, c_), (a, c_, d)]
    pts2 = list(p2)
    small = []
    for t in tris:
        g = len(pts2)
        pts2.append(p2[list(t)].mean(axis=0))
        small += [(t[0], t[1], g), (t[1], t[2], g), (t[2], t[0], g)]
    pts2 = np.array(pts2)
    n2 = len(pts2)
    pts = np.concatenate([np.c_[pts2, np.full(n2, -0.05)], np.c_[pts2, np.full(n2, 0.05)]])
    cells = np.array([[a, b, c_, a + n2, b + n2, c_ + n2] for a, b, c_ in small])

    def classify(cc, n):
        out = np.full(cc.shape[0], 2)
        out[np.abs(n[:, 2]) > 0.5] = 3
        out[(out == 2) & (np.abs(cc[:, 0]) < 1e-9)] = 0
        out[(out == 2) & (np.abs(cc[:, 0] - 2.0) < 1e-9)] = 1
        return out

    m = meshmod.build_polymesh(pts, [("prism", cells)], classify,
                               [("inlet", meshmod.PATCH), ("outlet", meshmod.PATCH), ("walls", meshmod.SYMMETRY),
                                ("frontBack", meshmod.EMPTY)])
    ref = channel_case("HLL", nx=2, ny=2, M=M)
    N = m.n_cells
    U0 = (M, 0.0, 0.0)
    return cases.Case("split channel", m, ref.bcs, ref.options, np.ones(N), np.tile(U0, (N, 1)), np.ones(N))


def test_cholesky_equals_iluc0_on_quads():
    c = channel_case("HLLC", nx=8, ny=5)
    b = np.random.default_rng(1).normal(size=5 * c.mesh.n_cells)
    x = {}
    for pc in ("ILUC0", "Cholesky"):
        o = oracle_for(c.with_options(**{"solvers.W.preconditioner": pc}), 2)
        x[pc] = o.precondition(b)
    assert np.array_equal(x["ILUC0"], x["Cholesky"])


def test_cholesky_is_the_diagonal_factorisation_with_cell_triangles():
    c = split_channel_case()
    N = c.mesh.n_cells
    assert N == 6 * 4 * 3
    o = oracle_for(c.with_options(**{"solvers.W.preconditioner": "Cholesky"}), 4)
    A, _ = dense_system(o, c.mesh)
    rng = np.random.default_rng(9)
    b = rng.normal(size=5 * N)
    x = o.precondition(b).ravel()
    M = dilu_reference(A, N)
    assert np.abs(M @ x - b).max() <= 1e-10 * np.abs(b).max()
    # and ILUC0 is a different factorisation here (with triangles in the
    # cell graph ILU(0) also updates off-diagonal blocks)
    o2 = oracle_for(c.with_options(**{"solvers.W.preconditioner": "ILUC0"}), 4)
    x2 = o2.precondition(b).ravel()
    assert np.abs(x2 - x).max() > 1e-8 * np.abs(x).max()


def bfs_rank(mesh, part):
    """Breadth-first factorisation order inside each part, restated from
    its definition: per connected component (by lowest cell), start at a
    pseudo-peripheral cell (two sweeps from the lowest cell, each taking the
    lowest cell of the deepest level), then cells by (level, number)."""
    N, Fi = mesh.n_cells, mesh.n_internal_faces
    adj = [[] for _ in range(N)]
    for f in range(Fi):
        a, b2 = int(mesh.owner[f]), int(mesh.neighbour[f])
        if part[a] == part[b2]:
            adj[a].append(b2)
            adj[b2].append(a)

    def levels(s):
        d = {s: 0}
        front = [s]
        while front:
            nxt = []
            for u in front:
                for v in adj[u]:
                    if v not in d:
                        d[v] = d[u] + 1
                        nxt.append(v)
            front = nxt
        return d

    rank = np.full(N, -1)
    seen = np.zeros(N, bool)
    count = {}
    for s0 in range(N):
        if seen[s0]:
            continue
        comp = sorted(levels(s0))
        seen[comp] = True
        far = lambda d: min(comp, key=lambda i: (-d[i], i))
        start = far(levels(far(levels(comp[0]))))
        d = levels(start)
        p = int(part[s0])
        for i in sorted(comp, key=lambda i: (d[i], i)):
            rank[i] = count.get(p, 0)
            count[p] = rank[i] + 1
    return rank


@pytest.mark.parametrize("parts,order", [(None, "natural"), (3, "natural"), (3, "bfs")])
def test_gauss_seidel_sweeps(parts, order):
    c = channel_case("HLL", nx=8, ny=4).with_options(**{"ilu.order": order})
    N = c.mesh.n_cells
    part = None
    if parts:
        part = (np.arange(N) * parts // N).astype(np.int32)
    rng = np.random.default_rng(12)
    b = rng.normal(size=5 * N)
    o1 = oracle_for(c.with_options(**{"solvers.W.preconditioner": "GaussSeidel"}), 5, partition=part)
    A, _ = dense_system(o1, c.mesh)
    same = np.ones((N, N), bool) if part is None else (part[:, None] == part[None, :])
    key = np.arange(N) if order == "natural" else bfs_rank(c.mesh, np.zeros(N, int) if part is None else part)
    lowmask = np.kron(same & (key[None, :] < key[:, None]), np.ones((5, 5), bool))
    dmask = np.kron(np.eye(N, dtype=bool), np.ones((5, 5), bool))
    DL = np.where(lowmask | dmask, A, 0.0)
    x1 = o1.precondition(b).ravel()
    assert np.allclose(x1, np.linalg.solve(DL, b), rtol=0, atol=1e-11 * np.abs(x1).max())
    # three sweeps: x_{k+1} = x_k + (D + L)^-1 (b - A x_k) from x_0 = 0
    o3 = oracle_for(c.with_options(**{"solvers.W.preconditioner": "GaussSeidel", "solvers.W.nSweeps": 3}), 5,
                    partition=part)
    xr = np.zeros_like(b)
    for _ in range(3):
        xr = xr + np.linalg.solve(DL, b - A @ xr)
    x3 = o3.precondition(b).ravel()
    assert np.allclose(x3, xr, rtol=0, atol=1e-10 * np.abs(xr).max())
    # the nested dictionary form of the preconditioner selects the same
    o3n = oracle_for(c.with_options(**{"solvers.W.preconditioner": {"preconditioner": "GaussSeidel", "nSweeps": 3}}),
                     5, partition=part)
    assert np.array_equal(o3n.precondition(b), x3.reshape(-1, 5))


def test_iluc_p_level_zero_is_iluc0():
    c = channel_case("Kurganov", nx=7, ny=5)
    b = np.random.default_rng(4).normal(size=5 * c.mesh.n_cells)
    o0 = oracle_for(c.with_options(**{"solvers.W.preconditioner": "ILUC0"}), 6)
    op = oracle_for(c.with_options(**{"solvers.W.preconditioner": "ILUCp", "solvers.W.fillInLevel": 0}), 6)
    assert np.array_equal(o0.precondition(b), op.precondition(b))


def extended_pattern(m, level):
    adj = cell_graph(m)
    N = m.n_cells
    pat = np.eye(N, dtype=bool)
    for i in range(N):
        seen = {i}
        front = {i}
        for _ in range(level + 1):
            front = {b for a in front for b in adj[a]} - seen
            seen |= front
        pat[i, list(seen)] = True
    return pat


@pytest.mark.parametrize("level", [1, 2])
def test_iluc_p_reproduces_a_on_the_extended_pattern(level):
    c = channel_case("Kurganov", nx=6, ny=4).with_options(**{"solvers.W.preconditioner": "ILUCp",
                                                             "solvers.W.fillInLevel": level})
    o = oracle_for(c, 7)
    A, _ = dense_system(o, c.mesh)
    n = A.shape[0]
    M = np.linalg.inv(precon_matrix(o, n))
    pat = np.kron(extended_pattern(c.mesh, level), np.ones((5, 5), bool))
    scale = np.abs(A).max()
    assert np.abs((M - A)[pat]).max() < 1e-10 * scale
    assert np.abs((M - A)[~pat]).max() > 1e-8 * scale      # still incomplete
    # a wider pattern is a better approximation of A
    o0 = oracle_for(c.with_options(**{"solvers.W.fillInLevel": level - 1}), 7)
    M0 = np.linalg.inv(precon_matrix(o0, n))
    assert np.linalg.norm(M - A) < np.linalg.norm(M0 - A)


def test_iluc_p_covering_the_graph_is_exact():
    c = channel_case("HLLC", nx=3, ny=2).with_options(**{"solvers.W.preconditioner": "ILUCp",
                                                          "solvers.W.fillInLevel": 3})
    o = oracle_for(c, 8)
    A, _ = dense_system(o, c.mesh)
    b = np.random.default_rng(2).normal(size=A.shape[0])
    x = o.precondition(b).ravel()
    assert np.abs(A @ x - b).max() < 1e-11 * np.abs(b).max()


@pytest.mark.parametrize("solver,opts", [("GaussSeidel", {}), ("GaussSeidel", {"solvers.W.nSweeps": 2}),
                                         ("ILU", {})])
def test_stationary_solvers_vs_dense(solver, opts):
    c = channel_case("HLL", nx=10, ny=5).with_options(**{
        "solvers.W.solver": solver, "solvers.W.tolerance": 1e-13, "solvers.W.relTol": 0.0,
        "solvers.W.maxIter": 3000, "solvers.W.minIter": 1, "ddtSchemes.default": "Euler",
        "timeControls.initialCo": 0.5, "timeControls.minCo": 0.5, "timeControls.maxCo": 0.5, **opts})
    o = oracle_for(c, 8)
    A, s = dense_system(o, c.mesh)
    x_ref = np.linalg.solve(A, s)
    x, rep = o.linear_solve()
    assert 1 < rep["lin_iterations"] < 3000
    assert max(rep["lin_final"]) < 1e-13
    assert np.abs(x.ravel() - x_ref).max() <= 1e-9 * np.abs(x_ref).max()


def test_stationary_solver_iterations_follow_the_sweeps():
    """Two Gauss-Seidel sweeps per iteration take about half the iterations
    of one, and the ILU solver (Cholesky factorisation) fewer still."""
    base = {"solvers.W.tolerance": 1e-12, "solvers.W.relTol": 0.0, "solvers.W.maxIter": 3000,
            "solvers.W.minIter": 1, "ddtSchemes.default": "Euler", "timeControls.initialCo": 0.5,
            "timeControls.minCo": 0.5, "timeControls.maxCo": 0.5}
    c = channel_case("HLL", nx=10, ny=5)
    its = {}
    for name, opts in [("gs1", {"solvers.W.solver": "GaussSeidel"}),
                       ("gs2", {"solvers.W.solver": "GaussSeidel", "solvers.W.nSweeps": 2}),
                       ("ilu", {"solvers.W.solver": "ILU"})]:
        o = oracle_for(c.with_options(**base, **opts), 8)
        its[name] = o.linear_solve()[1]["lin_iterations"]
    assert abs(2 * its["gs2"] - its["gs1"]) <= 2, its
    assert its["ilu"] < its["gs1"], its
