"""Steady-state solves on several ranks (one GPU each) by overlapping domain
decomposition: each rank steps its own subdomain (owned cells plus two halo
layers, `decompose.py`) with its own context, and after every step the
ranks exchange the states of the halo cells with the owners (point-to-point
through torch.distributed: NCCL between GPUs, gloo on the CPU).

With a Spalart-Allmaras model nuTilda travels with the mean flow and the
halo cells keep it in the segregated nuTilda solve as well.  Within a step
the subdomains are independent (their halos are held at the
values of the last exchange: an overlapping Schwarz iteration in
pseudo-time with Dirichlet data on the halo), so the converged state is
the single-mesh steady state, R = 0 on every owned cell: the owned cells'
residuals are exact once the halos are current.  The reference decomposes
the same way (foam-extend processor patches) but couples the ranks inside
its Krylov iteration; this path trades that coupling for steps with no
collective inside, which suits steady problems only (time-accurate steps
would need the coupling).  The global residual norm is an all-reduce over
the owned cells.
"""
from typing import Callable, Optional

import numpy as np

from . import decompose as _dec


class DecomposedSolver:
    """One overlapping subdomain of `case` per rank of the default (or the
    given) torch.distributed process group.  `make_solver(mesh, bcs,
    options)` builds the per-rank context (default: the B200 library's
    Solver on this rank's GPU)."""

    def __init__(self, case, group=None, method: str = "graph", layers: int = 2,
                 make_solver: Optional[Callable] = None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.turb = case.options.get("RASModel", "laminar") != "laminar"
        td = case.options.get("ddtSchemes", {}).get("default", "Euler")
        if td != "steadyStateDST":
            raise ValueError("the decomposed solver iterates steady states (ddt steadyStateDST)")
        backend = dist.get_backend(group)
        subs = _dec.decompose(case.mesh, self.world, layers=layers, method=method)
        self.sub = subs[self.rank]
        bcs = dict(case.bcs)
        bcs[_dec.HALO_PATCH] = {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient"}
        if self.turb:
            bcs[_dec.HALO_PATCH]["nuTilda"] = "zeroGradient"
        if make_solver is None:
            from . import Solver
            make_solver = Solver
        options = dict(case.options)
        if backend == "nccl":
            # one GPU per rank: the library's context and torch's halo
            # buffers on this rank's device
            import os
            import torch
            options.setdefault("device", int(os.environ.get("LOCAL_RANK", self.rank)))
            torch.cuda.set_device(int(options["device"]))
        self.solver = make_solver(self.sub.mesh, bcs, options)
        c = self.sub.cells
        self.solver.set_primitive(case.p[c], case.U[c], case.T[c], case.nuTilda[c] if self.turb else None)
        # halo cells are held in the steps (zero residual, identity rows):
        # each step solves the owned cells with the halo as Dirichlet data,
        # and the residual norms and the CFL ramp see the owned cells only
        self.solver.set_held_cells(~self.sub.owned)
        self._device = "cuda" if backend == "nccl" else "cpu"

    # -- halo exchange ------------------------------------------------------
    def exchange(self):
        """Owned states -> the peers' halo cells: six values per cell (rho,
        rhoU, rhoE, nuTilda), read and written for the send and halo cells
        only.  Under NCCL the values stay on the GPU: gathered into torch
        device buffers by rdst_get_cells_device, sent and received by NCCL,
        scattered by rdst_set_cells_device; on gloo they go through host
        arrays (rdst_get_cells / rdst_set_cells)."""
        import torch
        device_path = self._device == "cuda" and hasattr(self.solver, "get_cells_device")
        reqs, inbox = [], {}
        for q in sorted(self.sub.recv):
            buf = torch.empty((self.sub.recv[q].size, 6), dtype=torch.float64, device=self._device)
            inbox[q] = buf
            reqs.append(self.dist.irecv(buf, src=q, group=self.group))
        outbox = []
        for q in sorted(self.sub.send):
            if device_path:
                t = torch.empty((self.sub.send[q].size, 6), dtype=torch.float64, device="cuda")
                self.solver.get_cells_device(self.sub.send[q], t.data_ptr())
            else:
                t = torch.from_numpy(self.solver.get_cells(self.sub.send[q])).to(self._device)
            outbox.append(t)
            reqs.append(self.dist.isend(t, dst=q, group=self.group))
        for r in reqs:
            r.wait()
        if inbox:
            ids = np.concatenate([self.sub.recv[q] for q in sorted(inbox)])
            if device_path:
                vals = torch.cat([inbox[q] for q in sorted(inbox)]).contiguous()
                torch.cuda.current_stream().synchronize()
                self.solver.set_cells_device(ids, vals.data_ptr())
            else:
                vals = np.concatenate([inbox[q].cpu().numpy() for q in sorted(inbox)])
                self.solver.set_cells(ids, vals)

    def step(self, n: int = 1):
        """n steps, each followed by the halo exchange; this rank's reports."""
        reps = []
        for _ in range(n):
            reps += self.solver.step(1)
            self.exchange()
        return reps

    # -- global quantities --------------------------------------------------
    def residual_l2(self) -> np.ndarray:
        """||R_k V||_2 over all ranks' owned cells, per component (the
        density residual of the step report, summed over the subdomains)."""
        import torch
        R = self.solver.residual()
        V = np.asarray(self.sub.mesh.V)
        own = self.sub.owned
        s = torch.tensor(((R[own] * V[own, None]) ** 2).sum(axis=0), dtype=torch.float64, device=self._device)
        self.dist.all_reduce(s, group=self.group)
        return np.sqrt(s.cpu().numpy())

    def owned_state(self):
        """(global ids, rho, rhoU, rhoE) of this rank's owned cells."""
        rho, rhoU, rhoE = self.solver.conservative()
        o = self.sub.owned
        return self.sub.cells[o], rho[o], rhoU[o], rhoE[o]
