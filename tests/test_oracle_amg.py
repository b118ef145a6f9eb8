"""Known answers for the oracle's block AMG (preconditioner AMG, solver AMG):
plain aggregation of the cell graph, piecewise-constant prolongation,
Galerkin coarse blocks, damped block-Jacobi smoothing, one V-cycle per
application.

* the plan: every node of a level lies in one aggregate, aggregates are
  connected, each level is at most nine tenths of the one above, and the
  hierarchy ends at minCoarseEqns or nMaxLevels;
* one application equals a numpy restatement of the V-cycle built on the
  dense assembled matrix (P^T A P with the aggregation's 0/1 matrices);
* GMRES with AMG and the stationary AMG solver converge to
  numpy.linalg.solve, and AMG makes GMRES need fewer iterations than block
  Jacobi on a larger system.
"""
import numpy as np
import pytest

from tests.oracle_lib import OracleSolver
from tests.test_oracle_known_answers import channel_case, dense_system


def graph(m):
    adj = [set() for _ in range(m.n_cells)]
    for f in range(m.n_internal_faces):
        a, b = int(m.owner[f]), int(m.neighbour[f])
        adj[a].add(b)
        adj[b].add(a)
    return [sorted(s) for s in adj]


def plan(adj, n_coarsest, max_levels):
    """The aggregation passes restated in Python."""
    levels = []
    n = [len(adj)]
    while len(n) < max_levels and n[-1] > n_coarsest:
        agg = [-1] * len(adj)
        na = 0
        for i in range(len(adj)):
            if agg[i] >= 0 or any(agg[j] >= 0 for j in adj[i]):
                continue
            agg[i] = na
            for j in adj[i]:
                agg[j] = na
            na += 1
        first = list(agg)
        for i in range(len(adj)):
            if agg[i] < 0:
                agg[i] = next(first[j] for j in adj[i] if first[j] >= 0)
        if na * 10 > n[-1] * 9:
            break
        cadj = [set() for _ in range(na)]
        for i in range(len(adj)):
            for j in adj[i]:
                if agg[i] != agg[j]:
                    cadj[agg[i]].add(agg[j])
        levels.append(np.array(agg))
        n.append(na)
        adj = [sorted(s) for s in cadj]
    return levels, n


def vcycle_dense(A, b, levels, pre, post, omega, coarsest_sweeps):
    """One V-cycle from zero on dense block matrices."""
    mats = [A]
    Ps = []
    for agg in levels:
        nf = mats[-1].shape[0] // 5
        P = np.zeros((5 * nf, 5 * (agg.max() + 1)))
        for i, I in enumerate(agg):
            P[5 * i:5 * i + 5, 5 * I:5 * I + 5] = np.eye(5)
        Ps.append(P)
        mats.append(P.T @ mats[-1] @ P)

    def dinv(M):
        n = M.shape[0] // 5
        D = np.zeros_like(M)
        for i in range(n):
            D[5 * i:5 * i + 5, 5 * i:5 * i + 5] = np.linalg.inv(M[5 * i:5 * i + 5, 5 * i:5 * i + 5])
        return D

    def cyc(l, bl):
        M = mats[l]
        Di = dinv(M)
        if l == len(mats) - 1:
            x = omega * Di @ bl
            for _ in range(coarsest_sweeps - 1):
                x = x + omega * Di @ (bl - M @ x)
            return x
        x = np.zeros_like(bl)
        for s in range(pre):
            x = omega * Di @ bl if s == 0 else x + omega * Di @ (bl - M @ x)
        xc = cyc(l + 1, Ps[l].T @ (bl - M @ x))
        x = x + Ps[l] @ xc
        for _ in range(post):
            x = x + omega * Di @ (bl - M @ x)
        return x

    return cyc(0, b)


def amg_case(nx=10, ny=6, **opts):
    return channel_case("HLL", nx=nx, ny=ny).with_options(**{"solvers.W.preconditioner": "AMG", **opts})


def test_plan_properties():
    c = channel_case("HLL", nx=40, ny=16)
    adj = graph(c.mesh)
    levels, n = plan(adj, 4, 100)
    assert len(levels) >= 3 and n[-1] <= max(4, int(0.9 * n[-2]) + 1)
    cur = adj
    for agg, nc in zip(levels, n[1:]):
        assert agg.min() == 0 and agg.max() == nc - 1
        assert np.all(np.bincount(agg, minlength=nc) >= 1)
        # each aggregate is connected in its level's graph
        for I in range(nc):
            members = set(np.nonzero(agg == I)[0])
            seen, stack = set(), [next(iter(members))]
            while stack:
                v = stack.pop()
                if v in seen:
                    continue
                seen.add(v)
                stack += [w for w in cur[v] if w in members]
            assert seen == members
        cadj = [set() for _ in range(nc)]
        for i in range(len(cur)):
            for j in cur[i]:
                if agg[i] != agg[j]:
                    cadj[agg[i]].add(agg[j])
        cur = [sorted(s) for s in cadj]
    levels2, n2 = plan(adj, 4, 3)
    assert len(n2) == 3


@pytest.mark.parametrize("opts", [{}, {"solvers.W.nPreSweeps": 1, "solvers.W.nPostSweeps": 1, "amg.omega": 0.8},
                                  {"solvers.W.minCoarseEqns": 20, "amg.coarsestSweeps": 3}])
def test_vcycle_matches_dense_restatement(opts):
    c = amg_case(**opts)
    o = OracleSolver(c.mesh, c.bcs, c.options)
    rng = np.random.default_rng(3)
    o.set_primitive(c.p * (1 + 0.1 * rng.random(c.mesh.n_cells)), c.U, c.T)
    A, _ = dense_system(o, c.mesh)
    pre, post = opts.get("solvers.W.nPreSweeps", 0), opts.get("solvers.W.nPostSweeps", 2)
    levels, n = plan(graph(c.mesh), opts.get("solvers.W.minCoarseEqns", 4), 100)
    assert len(levels) >= 1
    b = rng.normal(size=A.shape[0])
    x_ref = vcycle_dense(A, b, levels, pre, post, opts.get("amg.omega", 0.6), opts.get("amg.coarsestSweeps", 10))
    x = o.precondition(b).ravel()
    assert np.allclose(x, x_ref, rtol=0, atol=1e-11 * np.abs(x_ref).max())


@pytest.mark.parametrize("solver", ["GMRES", "AMG"])
def test_solves_vs_dense(solver):
    c = amg_case(**{"solvers.W.solver": solver, "solvers.W.nDirections": 20, "solvers.W.tolerance": 1e-13,
                    "solvers.W.relTol": 0.0, "solvers.W.maxIter": 2000, "solvers.W.minIter": 1,
                    "ddtSchemes.default": "Euler", "timeControls.initialCo": 0.5, "timeControls.minCo": 0.5,
                    "timeControls.maxCo": 0.5})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    rng = np.random.default_rng(8)
    o.set_primitive(c.p * (1 + 0.2 * rng.random(c.mesh.n_cells)), c.U, c.T)
    A, s = dense_system(o, c.mesh)
    x_ref = np.linalg.solve(A, s)
    x, rep = o.linear_solve()
    assert rep["lin_iterations"] < 2000 and max(rep["lin_final"]) < 1e-13
    assert np.abs(x.ravel() - x_ref).max() <= 1e-9 * np.abs(x_ref).max()


def test_amg_beats_block_jacobi_on_a_larger_system():
    base = {"solvers.W.solver": "GMRES", "solvers.W.nDirections": 60, "solvers.W.tolerance": 1e-10,
            "solvers.W.relTol": 0.0, "solvers.W.maxIter": 50, "solvers.W.minIter": 1,
            "ddtSchemes.default": "Euler", "timeControls.initialCo": 20.0, "timeControls.minCo": 20.0,
            "timeControls.maxCo": 20.0}
    its = {}
    for pc in ("diagonal", "AMG"):
        c = channel_case("HLL", nx=80, ny=24).with_options(**base, **{"solvers.W.preconditioner": pc})
        o = OracleSolver(c.mesh, c.bcs, c.options)
        rng = np.random.default_rng(2)
        o.set_primitive(c.p * (1 + 0.2 * rng.random(c.mesh.n_cells)), c.U, c.T)
        x, rep = o.linear_solve()
        its[pc] = (rep["lin_iterations"], max(rep["lin_final"]))
    assert its["AMG"][1] < 1e-10
    assert its["AMG"][0] <= its["diagonal"][0], its
