"""Shape derivatives of the pressure-force objective by the discrete adjoint.

Design variables are Hicks-Henne bump amplitudes on the upper and lower
surfaces of an airfoil mesh: the surface moves normal to the chord by

    dy(x) = sum_k a_k b_k(x),   b_k(x) = sin(pi x^{m_k})^t,   m_k = ln 0.5 / ln h_k,

(Hicks & Henne, J. Aircraft 15(7), 1978), each bump peaking at x = h_k and
vanishing at the leading and trailing edges; the volume mesh follows along
its grid lines (the mesh's `surface_map`), so every design point has the same
topology and the solver context is moved onto it with rdst_set_geometry.

The gradient at a converged state W(a) is

    dJ/da_k = dJ/da_k|_W - psi . dR/da_k|_W,   (dR/dW)^T psi = dJ/dW,

with psi from one adjoint solve (rdst_adjoint) and the explicit derivatives
at fixed W by central differences of the library's own residual and
objective on the moved meshes: two residual evaluations per variable and no
flow solve, so the cost of all n variables is one adjoint solve plus 2n
residual evaluations.  rhoDST itself has no adjoint or shape parametrisation;
R is the residual of rdst_residual (computeFluxDST + calcFields,
baseFluxDST.C:223-255) and J the pressure part of the forceCoeffs objective.
"""
from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np

from . import mesh as _mesh


class HicksHenne:
    """`n_per_side` bumps on each side of the airfoil (lower first, then
    upper), peaks clustered like a cosine spacing in (0, 1), width exponent
    `width`; displacement fields per unit amplitude are precomputed from the
    mesh's surface map."""

    def __init__(self, mesh: _mesh.PolyMesh, n_per_side: int = 32, width: float = 3.0,
                 peaks: Optional[Sequence[float]] = None):
        if mesh.surface_map is None:
            raise ValueError("mesh has no airfoil surface map")
        self.base = mesh
        if peaks is None:
            k = np.arange(1, n_per_side + 1)
            peaks = 0.5 * (1.0 - np.cos(math.pi * k / (n_per_side + 1)))
        self.peaks = np.asarray(peaks, dtype=float)
        if np.any(self.peaks <= 0.0) or np.any(self.peaks >= 1.0):
            raise ValueError("bump peaks must lie inside (0, 1)")
        self.width = float(width)
        self.n_per_side = self.peaks.size
        xs, side, wgt = mesh.surface_map
        B = self.bumps(xs)                                  # (n_per_side, P)
        P = xs.size
        self.D = np.zeros((2 * self.n_per_side, P))         # y displacement per unit amplitude
        for s_idx, sgn in enumerate((-1, 1)):
            sel = side == sgn
            self.D[s_idx * self.n_per_side:(s_idx + 1) * self.n_per_side, sel] = B[:, sel] * wgt[sel]

    @property
    def n_variables(self) -> int:
        return 2 * self.n_per_side

    def bumps(self, x: np.ndarray) -> np.ndarray:
        """b_k(x) for every bump k (rows) at chordwise positions x in [0, 1]."""
        x = np.clip(np.asarray(x, dtype=float), 0.0, 1.0)
        m = math.log(0.5) / np.log(self.peaks)
        return np.sin(math.pi * x[None, :] ** m[:, None]) ** self.width

    def points(self, a: np.ndarray) -> np.ndarray:
        a = np.asarray(a, dtype=float)
        pts = self.base.points.copy()
        pts[:, 1] += a @ self.D
        return pts

    def mesh(self, a: np.ndarray) -> _mesh.PolyMesh:
        """The volume mesh at design point a (base topology)."""
        return _mesh.moved(self.base, self.points(a))

    @staticmethod
    def design_point(n: int, bound: float = 1e-3, seed: int = 1234) -> np.ndarray:
        """Amplitudes drawn uniformly in [-bound, bound] chord from a seeded
        generator."""
        return np.random.default_rng(seed).uniform(-bound, bound, size=n)


def explicit_derivatives(solver, param: HicksHenne, a: np.ndarray, patch: str, direction,
                         p_ref: float = 0.0, scale: float = 1.0, h: float = 1e-6,
                         variables: Optional[Sequence[int]] = None, psi: Optional[np.ndarray] = None):
    """dR/da_k and dJ/da_k at the solver's current state W, by central
    differences in a_k with W held (the solver is moved onto the two meshes
    a +- h e_k and back onto a).  Returns (dR (n, N, 5), dJ (n,)), or with
    `psi` given (psi . dR/da_k (n,), dJ (n,)) without keeping the dR."""
    W = solver.conservative()
    idx = range(param.n_variables) if variables is None else list(variables)
    dR, dJ = [], []
    try:
        for k in idx:
            vals = []
            for sgn in (1.0, -1.0):
                ak = np.array(a, dtype=float)
                ak[k] += sgn * h
                solver.set_geometry(param.mesh(ak))
                solver.set_conservative(*W)
                R = solver.residual()
                J = solver.objective_gradient(patch, direction, p_ref, scale)[0]
                vals.append((R, J))
            dRk = (vals[0][0] - vals[1][0]) / (2 * h)
            dR.append(dRk if psi is None else float(np.sum(psi * dRk)))
            dJ.append((vals[0][1] - vals[1][1]) / (2 * h))
    finally:
        solver.set_geometry(param.mesh(a))
        solver.set_conservative(*W)
        solver.residual()
        solver.set_conservative(*W)
    return np.array(dR), np.array(dJ)


def shape_gradient(solver, param: HicksHenne, a: np.ndarray, patch: str, direction,
                   p_ref: float = 0.0, scale: float = 1.0, h: float = 1e-6, rel_tol: float = 1e-10,
                   max_cycles: int = 60, n_directions: int = 30, variables: Optional[Sequence[int]] = None):
    """dJ/da at the solver's current (converged) state on design point a:
    one adjoint solve plus the explicit derivatives.  Returns (gradient,
    adjoint report, psi)."""
    rep, psi = solver.adjoint(patch, direction, p_ref=p_ref, scale=scale, rel_tol=rel_tol,
                              max_cycles=max_cycles, n_directions=n_directions, want_psi=True)
    psi_dR, dJ = explicit_derivatives(solver, param, a, patch, direction, p_ref, scale, h, variables, psi=psi)
    return dJ - psi_dR, rep, psi


def freestream_derivatives(dJ_dU, force, U_inf, c_inf: float, lift_dir=None):
    """dJ/dMach and dJ/dalpha (per radian) from the adjoint's derivative
    with respect to the free-stream velocity value (rdst_adjoint's dJ_dU)
    and the objective's force vector, for a pressure-force objective whose
    direction turns with the flow angle (drag: d(direction)/dalpha is the
    lift direction).  The free stream U = Mach c (cos alpha, sin alpha, 0)."""
    dJ_dU = np.asarray(dJ_dU, dtype=float)
    U = np.asarray(U_inf, dtype=float)
    speed = float(np.linalg.norm(U))
    alpha = math.atan2(U[1], U[0])
    dU_dM = c_inf * U / speed
    dU_da = speed * np.array([-math.sin(alpha), math.cos(alpha), 0.0])
    if lift_dir is None:
        lift_dir = (-math.sin(alpha), math.cos(alpha), 0.0)
    dJ_dM = float(dJ_dU @ dU_dM)
    dJ_da = float(dJ_dU @ dU_da + np.asarray(force, dtype=float) @ np.asarray(lift_dir, dtype=float))
    return dJ_dM, dJ_da
