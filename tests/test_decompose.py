"""Overlapping domain decomposition (rhodst_b200.decompose) and the
decomposed steady solve (rhodst_b200.distributed) on the CPU.

* Every cell is owned by exactly one subdomain, the halo maps pair up
  (what a rank receives from a peer is what that peer sends, in the same
  order), and with two halo layers the residual of every owned cell equals
  the single-mesh residual exactly (limited reconstruction, HLLCP's
  pressure sensor, viscous terms).
* Two gloo ranks step their subdomains (halo cells held at the exchanged
  states: zero residual, identity rows) with the halo exchange between
  steps and reach the single-mesh steady state: the global owned-cell
  residual falls by 1e-10 and the owned cells' states agree with a
  single-mesh solve to 1e-8.  The per-rank step here is the
  oracle (this tests the decomposition and exchange logic, which are host
  code; the product runs the library's Solver on each rank's GPU).
"""
import os
import tempfile

import numpy as np
import pytest

from rhodst_b200 import cases, decompose
from tests.oracle_lib import OracleSolver


def perturbed(c, seed=1):
    rng = np.random.default_rng(seed)
    N = c.mesh.n_cells
    return (c.p * (1 + 0.05 * rng.random(N)), c.U * (1 + 0.05 * rng.random((N, 1))),
            c.T * (1 + 0.05 * rng.random(N)))


@pytest.mark.parametrize("case_fn,parts,method", [
    (lambda: cases.naca0012_inviscid(ni=97, nj=25, first_cell=5e-3, flux="HLLCP", limiter="Venkatakrishnan"), 3,
     "graph"),
    (lambda: cases.naca0012_laminar(ni=65, nj=17, first_cell=1e-2, flux="AUSM+up", limiter="vanLeer"), 4, "rcb"),
    (lambda: cases.forward_step_3d_hybrid_c5(nx=12, ny=5, nz=2, flux="HLLC", limiter="OSPRE", precision="fp64"), 2,
     "graph"),
])
def test_owned_residuals_are_exact(case_fn, parts, method):
    c = case_fn()
    subs = decompose.decompose(c.mesh, parts, method=method)
    N = c.mesh.n_cells
    count = np.zeros(N, dtype=int)
    for s in subs:
        count[s.cells[s.owned]] += 1
        assert np.all(np.diff(s.cells) > 0)
        for q, ids in s.recv.items():
            peer = subs[q]
            assert np.array_equal(s.cells[ids], peer.cells[peer.send[s.rank]])
            assert not np.any(s.owned[ids]) and np.all(peer.owned[peer.send[s.rank]])
    assert np.all(count == 1)
    p, U, T = perturbed(c)
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(p, U, T)
    R = o.residual()
    bcs = dict(c.bcs)
    bcs[decompose.HALO_PATCH] = {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient"}
    for s in subs:
        os_ = OracleSolver(s.mesh, bcs, c.options)
        os_.set_primitive(p[s.cells], U[s.cells], T[s.cells])
        Rs = os_.residual()
        assert np.abs(Rs[s.owned] - R[s.cells[s.owned]]).max() <= 1e-13 * np.abs(R).max()


def steady_case():
    return cases.naca0012_inviscid(ni=97, nj=25, first_cell=5e-3, flux="HLL", limiter="upwind")


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from rhodst_b200.distributed import DecomposedSolver
    from tests.oracle_lib import OracleSolver as OS
    from tests.oracle_lib import set_threads
    set_threads(2)
    import datetime
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    try:
        d = DecomposedSolver(steady_case(), make_solver=OS)
        hist = [d.residual_l2()[0]]
        for _ in range(8):
            d.step(50)
            hist.append(d.residual_l2()[0])
            if hist[-1] < 1e-12 * hist[0]:
                break
        ids, rho, rhoU, rhoE = d.owned_state()
        np.savez(f"{out}_{rank}.npz", ids=ids, rho=rho, rhoU=rhoU, rhoE=rhoE, hist=np.array(hist))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reach_the_single_mesh_steady_state():
    import socket
    import torch.multiprocessing as mp
    c = steady_case()
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    r0 = None
    for _ in range(40):
        reps = o.step(50)
        r0 = reps[0]["res_l2"][0] if r0 is None else r0
        if reps[-1]["res_l2"][0] < 1e-12 * r0:
            break
    assert reps[-1]["res_l2"][0] < 1e-10 * r0
    W = o.conservative()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "rank")
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        got = [np.load(f"{out}_{r}.npz") for r in range(2)]
    ids = np.concatenate([g["ids"] for g in got])
    assert np.array_equal(np.sort(ids), np.arange(c.mesh.n_cells))
    for g in got:
        assert g["hist"][-1] < 1e-10 * g["hist"][0], g["hist"]
    for k, name in enumerate(("rho", "rhoU", "rhoE")):
        ref = W[k]
        for g in got:
            assert np.abs(g[name] - ref[g["ids"]]).max() <= 1e-8 * np.abs(ref).max(), name


def test_sa_steady_state_is_a_fixed_point_of_the_subdomain_steps():
    """With the Spalart-Allmaras model the halo carries nuTilda too
    (rdst_set_nu_tilda) and held cells keep it in the nuTilda solve: the
    single-mesh steady state (W, nuTilda) loaded into the subdomains is left
    where it is by a step (owned cells, to round-off)."""
    c = cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL",
                                 limiter="upwind").with_options(**{"timeControls.maxCo": 500.0})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T, c.nuTilda)
    r0 = None
    for _ in range(20):
        reps = o.step(50)
        r0 = reps[0]["res_l2"][0] if r0 is None else r0
        if reps[-1]["res_l2"][0] < 1e-12 * r0:
            break
    assert reps[-1]["res_l2"][0] < 1e-10 * r0
    W, prim = o.conservative(), o.primitive()
    bcs = dict(c.bcs)
    bcs[decompose.HALO_PATCH] = {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient",
                                 "nuTilda": "zeroGradient"}
    for s in decompose.decompose(c.mesh, 3):
        cs, own = s.cells, s.owned
        os_ = OracleSolver(s.mesh, bcs, c.options)
        os_.set_primitive(prim[0][cs], prim[1][cs], prim[2][cs], prim[3][cs])
        os_.set_held_cells(~own)
        os_.set_conservative(W[0][cs], W[1][cs], W[2][cs])
        os_.set_nu_tilda(prim[3][cs])
        os_.step(1)
        W2, p2 = os_.conservative(), os_.primitive()
        for a, b in zip(W2, W):
            assert np.abs(a[own] - b[cs][own]).max() <= 1e-12 * np.abs(b).max()
        assert np.abs(p2[3][own] - prim[3][cs][own]).max() <= 1e-12 * np.abs(prim[3]).max()
        # held cells keep their state and nuTilda
        assert np.array_equal(p2[3][~own], prim[3][cs][~own])


@pytest.mark.parametrize("turb", [False, True])
def test_set_cells_is_set_conservative_for_those_cells(turb):
    """Writing a subset of cells with set_cells gives the state that
    set_conservative of the whole field gives (the residual to round-off);
    get_cells reads the six values back."""
    c = (cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5) if turb
         else cases.naca0012_inviscid(ni=65, nj=17, first_cell=1e-2))
    N = c.mesh.n_cells
    rng = np.random.default_rng(4)
    nut0 = c.nuTilda if turb else None
    a = OracleSolver(c.mesh, c.bcs, c.options)
    b = OracleSolver(c.mesh, c.bcs, c.options)
    for s in (a, b):
        s.set_primitive(c.p, c.U, c.T, nut0)
        s.step(2)
    W = a.conservative()
    ids = np.sort(rng.choice(N, size=N // 5, replace=False)).astype(np.int32)
    vals = b.get_cells(ids)
    assert np.array_equal(vals[:, 0], W[0][ids]) and np.array_equal(vals[:, 1:4], W[1][ids])
    vals[:, 0] *= 1.01
    vals[:, 4] *= 1.02
    if turb:
        vals[:, 5] *= 1.3
    b.set_cells(ids, vals)
    rho, rhoU, rhoE = (x.copy() for x in W)
    rho[ids], rhoU[ids], rhoE[ids] = vals[:, 0], vals[:, 1:4], vals[:, 4]
    a.set_conservative(rho, rhoU, rhoE)
    if turb:
        nut = a.primitive()[3].copy()
        nut[ids] = vals[:, 5]
        a.set_nu_tilda(nut)
    for x, y in zip(a.conservative(), b.conservative()):
        assert np.array_equal(x, y)
    # set_conservative re-derives p and T of every cell from W (the last
    # update derived them through the bounded h), set_cells only those it
    # writes: the residuals agree to round-off
    Ra, Rb = a.residual(), b.residual()
    assert np.abs(Ra - Rb).max() <= 1e-12 * np.abs(Ra).max()
    assert np.array_equal(a.primitive()[3], b.primitive()[3])
