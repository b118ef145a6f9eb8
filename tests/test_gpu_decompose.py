"""The decomposed steady solve on the B200 library.

* Held cells (the halo of a subdomain): GPU steps match the oracle's with
  the same held cells on a subdomain mesh, 1e-9.
* Two ranks, each a process with its own context on this GPU, exchange
  halos through gloo between steps (no kernel waits on the other rank) and
  reach the single-context steady state: owned states agree to 1e-8.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import decompose
from tests.oracle_lib import OracleSolver
from tests.test_decompose import steady_case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def sa_case():
    from rhodst_b200 import cases
    return cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL",
                                    limiter="upwind").with_options(**{"timeControls.maxCo": 500.0})


@pytest.mark.parametrize("turb", [False, True], ids=["inviscid", "SA"])
def test_held_cells_steps_parity(turb):
    c = (sa_case() if turb else steady_case()).with_options(**{"ilu.parts": 2})
    sub = decompose.decompose(c.mesh, 3)[1]
    bcs = dict(c.bcs)
    bcs[decompose.HALO_PATCH] = {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient"}
    if turb:
        bcs[decompose.HALO_PATCH]["nuTilda"] = "zeroGradient"
    part = rhodst_b200.partition_cells(sub.mesh.C, 2)
    gpu = rhodst_b200.Solver(sub.mesh, bcs, c.options)
    ora = OracleSolver(sub.mesh, bcs, c.options, partition=part)
    cs = sub.cells
    nut = c.nuTilda[cs] * (1.0 + 0.3 * np.sin(3.0 * c.mesh.C[cs, 0]) ** 2) if turb else None
    for s in (gpu, ora):
        s.set_primitive(c.p[cs], c.U[cs], c.T[cs], nut)
        s.set_held_cells(~sub.owned)
        if turb:
            s.set_nu_tilda(nut)
    W0 = gpu.conservative()
    rg, ro = gpu.step(5), ora.step(5)
    tol = 1e-8 if turb else 1e-9
    for a, b in zip(rg, ro):
        assert abs(a["res_mag"] - b["res_mag"]) <= tol * abs(b["res_mag"])
    Wg, Wo = gpu.conservative(), ora.conservative()
    for a, b, a0 in zip(Wg, Wo, W0):
        assert rel(a, b) < tol
        assert np.array_equal(a[~sub.owned], a0[~sub.owned])          # held cells keep their state
    if turb:
        ng, no = gpu.primitive()[3], ora.primitive()[3]
        assert rel(ng, no) < tol
        assert np.array_equal(ng[~sub.owned], nut[~sub.owned])
    assert np.abs(gpu.residual()[~sub.owned]).max() == 0.0


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from rhodst_b200.distributed import DecomposedSolver
    from tests.test_decompose import steady_case as sc
    import datetime
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    try:
        d = DecomposedSolver(sc())
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


def test_two_ranks_on_one_gpu_reach_the_single_context_steady_state():
    import torch.multiprocessing as mp
    c = steady_case()
    s = rhodst_b200.solver_for(c)
    r0 = None
    for _ in range(12):
        reps = s.step(50)
        r0 = reps[0]["res_l2"][0] if r0 is None else r0
        if reps[-1]["res_l2"][0] < 1e-12 * r0:
            break
    W = s.conservative()
    s.close()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "rank")
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        got = [np.load(f"{out}_{r}.npz") for r in range(2)]
    for g in got:
        assert g["hist"][-1] < 1e-10 * g["hist"][0], g["hist"]
    for k, name in enumerate(("rho", "rhoU", "rhoE")):
        for g in got:
            assert np.abs(g[name] - W[k][g["ids"]]).max() <= 1e-8 * np.abs(W[k]).max(), name


@pytest.mark.parametrize("turb", [False, True], ids=["inviscid", "SA"])
def test_get_and_set_cells_match_the_oracle(turb):
    """rdst_get_cells / rdst_set_cells on the GPU against the oracle's: the
    written cells, the boundary values and mu_t that follow, and the
    residual at the new state (1e-11 relative)."""
    c = sa_case() if turb else steady_case()
    N = c.mesh.n_cells
    gpu = rhodst_b200.Solver(c.mesh, c.bcs, c.options)
    ora = OracleSolver(c.mesh, c.bcs, c.options)
    for s in (gpu, ora):
        s.set_primitive(c.p, c.U, c.T, c.nuTilda if turb else None)
    ids = np.arange(0, N, 7, dtype=np.int32)
    vg, vo = gpu.get_cells(ids), ora.get_cells(ids)
    assert rel(vg, vo) < 1e-14                     # the initial states, each side's own arithmetic
    vals = vo.copy()
    vals[:, 0] *= 1.02
    vals[:, 4] *= 1.03
    if turb:
        vals[:, 5] *= 1.5
    for s in (gpu, ora):
        s.set_cells(ids, vals)
    assert np.array_equal(gpu.get_cells(ids), ora.get_cells(ids))
    assert rel(gpu.residual(), ora.residual()) < 1e-11


@pytest.mark.parametrize("turb", [False, True], ids=["inviscid", "SA"])
def test_device_buffer_halo_roundtrip(turb):
    """rdst_get_cells_device / rdst_set_cells_device (the NCCL halo path of
    the decomposed solver, no host copy) read and write the same values as
    the host-buffer calls: a gather into a torch device buffer equals
    rdst_get_cells, and a scatter from one makes the same state (and the
    same next step) as rdst_set_cells."""
    import torch
    c = sa_case() if turb else steady_case()
    cells = np.arange(0, c.mesh.n_cells, 7, dtype=np.int32)
    a, b = rhodst_b200.solver_for(c), rhodst_b200.solver_for(c)
    a.step(3)
    host = a.get_cells(cells)
    dev = torch.empty((cells.size, 6), dtype=torch.float64, device="cuda")
    a.get_cells_device(cells, dev.data_ptr())
    assert np.array_equal(dev.cpu().numpy(), host)
    # scatter the same values into two fresh contexts: host and device paths
    b.set_cells(cells, host)
    d = rhodst_b200.solver_for(c)
    d.set_cells_device(cells, dev.data_ptr())
    for x, y in zip(b.conservative(), d.conservative()):
        assert np.array_equal(x, y)
    rb, rd = b.step(1)[0], d.step(1)[0]
    assert rb["res_mag"] == rd["res_mag"]
