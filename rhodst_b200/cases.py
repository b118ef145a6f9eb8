"""Case definitions: mesh + boundary conditions + dictionary entries +
initial fields for the workloads the step is exercised and measured on.

Each builder returns a :class:`Case`; the dictionaries use the reference's
key names (system/rhoDSTDict, fvSchemes, fvSolution, fieldBounds and
constant/thermophysicalProperties of the rhoDST tutorials).
"""
from __future__ import annotations

import copy
import dataclasses
import math
from typing import Any, Dict, Optional

import numpy as np

from . import mesh as _mesh

# normalisedGas of tutorials/forwardStep/constant/thermophysicalProperties:
# "normalisedGas 1 11640.3 2.5 0 0 1" -> molWeight 11640.3, Cp 2.5, mu 0, Pr 1
R_UNIVERSAL = 8314.47
NORMALISED_GAS = {"R": R_UNIVERSAL / 11640.3, "Cp": 2.5}
# air of the RAE2822 tutorial (constant/thermophysicalProperties:
# "specie 1 28.966 1005 0 1.4584e-6 110.33": molWeight, Cp, Hf, As, Ts)
AIR = {"R": R_UNIVERSAL / 28.966, "Cp": 1005.0}
AIR_SUTHERLAND = {"As": 1.4584e-6, "Ts": 110.33}
# foam's sutherlandTransport conducts heat by the modified Eucken relation,
# kappa = mu Cv (1.32 + 1.77 R/Cv): alpha = kappa/Cp = mu/Pr with this Pr
AIR_PR = AIR["Cp"] / (1.32 * (AIR["Cp"] - AIR["R"]) + 1.77 * AIR["R"])


@dataclasses.dataclass
class Case:
    name: str
    mesh: _mesh.PolyMesh
    bcs: Dict[str, Dict[str, Any]]
    options: Dict[str, Any]
    p: np.ndarray
    U: np.ndarray
    T: np.ndarray
    nuTilda: Optional[np.ndarray] = None
    steps: int = 1
    force_patch: Optional[str] = None
    force_dirs: Optional[Dict[str, Any]] = None

    def with_options(self, **updates) -> "Case":
        c = copy.copy(self)
        o = copy.deepcopy(self.options)
        for k, v in updates.items():
            _set_dotted(o, k, v)
        c.options = o
        return c


def _set_dotted(d: dict, key: str, value) -> None:
    parts = key.split(".")
    for p in parts[:-1]:
        d = d.setdefault(p, {})
    d[parts[-1]] = value


def forward_step_c1(refine: int = 1, solver: str = "GMRES", preconditioner: str = "diagonal",
                    n_directions: int = 20, max_iter: int = 1) -> Case:
    """2D inviscid Mach-3 forward-facing step (120x40 minus the step = 4032
    cells at refine=1): Kurganov flux, OSPRE/OSPREV reconstruction, Euler
    implicit step at a fixed global CFL 0.8 (global dt from the
    neighbouring face definition), block-GMRES(20) with block-Jacobi, one
    restart cycle per step.  BCs follow tutorials/forwardStep/0/{p,U,T}."""
    m = _mesh.forward_step_2d(refine)
    U0 = (3.0, 0.0, 0.0)
    bcs = {
        "inlet": {"p": ("fixedValue", 1.0), "U": ("fixedValue", U0), "T": ("fixedValue", 1.0)},
        "outlet": {"p": "zeroGradient", "U": ("inletOutlet", U0), "T": ("inletOutlet", 1.0)},
        "bottom": {"p": "symmetryPlane", "U": "symmetryPlane", "T": "symmetryPlane"},
        "top": {"p": "symmetryPlane", "U": "symmetryPlane", "T": "symmetryPlane"},
        "obstacle": {"p": "zeroGradient", "U": "slip", "T": "zeroGradient"},
    }
    options = {
        "fluxScheme": "Kurganov",
        "Jacobian": "Roe",
        "timeIntegration": {"timeIntegration": "Single"},
        "timeControls": {"adjustTimeStep": True, "neighbouring": True,
                         "initialCo": 0.8, "minCo": 0.8, "maxCo": 0.8},
        "ddtSchemes": {"default": "Euler"},
        "interpolationSchemes": {"reconstruct(rho)": "OSPRE", "reconstruct(U)": "OSPREV",
                                 "reconstruct(T)": "OSPRE"},
        "solvers": {"W": {"solver": solver, "preconditioner": preconditioner,
                          "nDirections": n_directions, "tolerance": 1e-14, "relTol": 0.0,
                          "maxIter": max_iter, "minIter": 1}},
        "fieldBounds": {"rho": (0.001, 10000.0), "p": (0.001, 10000.0), "T": (0.001, 10000.0)},
        "thermo": dict(NORMALISED_GAS),
    }
    N = m.n_cells
    return Case("forwardStep2D", m, bcs, options, np.ones(N), np.tile(U0, (N, 1)), np.ones(N),
                steps=1000)


def _vector_limiter(limiter: str) -> str:
    """Scheme name for reconstruct(U): the TVD limiters take their "V"
    (direction-aware) variant; linear, upwind and Venkatakrishnan are used
    as they are."""
    return limiter if limiter in ("linear", "upwind", "Venkatakrishnan") else limiter + "V"


def farfield_state(mach: float, alpha_deg: float, T_inf: float, p_inf: float, gas: dict):
    g = gas["Cp"] / (gas["Cp"] - gas["R"])
    a = math.sqrt(g * gas["R"] * T_inf)
    al = math.radians(alpha_deg)
    U = (mach * a * math.cos(al), mach * a * math.sin(al), 0.0)
    return U


def naca0012_inviscid(ni: int = 257, nj: int = 65, mach: float = 0.73, alpha: float = 2.3,
                      flux: str = "AUSM+up", limiter: str = "Venkatakrishnan",
                      n_directions: int = 30, preconditioner: str = "ILUC0", first_cell: float = 4e-6) -> Case:
    """NACA0012 C-mesh with characteristic far field, Euler equations,
    local time stepping at CFL 50 (steadyStateDST), block-GMRES(30) with
    block ILU(0).  The inviscid counterpart of the turbulent airfoil case
    (same mesh, flow angle and Mach number)."""
    m = _mesh.naca_cmesh(ni, nj, first_cell=first_cell)
    gas = dict(NORMALISED_GAS)
    U0 = farfield_state(mach, alpha, 1.0, 1.0, gas)
    bcs = {
        "airfoil": {"p": "zeroGradient", "U": "slip", "T": "zeroGradient"},
        "farfield": {"p": ("farField", 1.0), "U": ("farField", U0), "T": ("farField", 1.0)},
    }
    vlim = _vector_limiter(limiter)
    options = {
        "fluxScheme": flux,
        "Jacobian": "Roe",
        "timeControls": {"neighbouring": True, "initialCo": 2.0, "minCo": 0.1, "maxCo": 50.0},
        "ddtSchemes": {"default": "steadyStateDST"},
        "interpolationSchemes": {"reconstruct(rho)": limiter, "reconstruct(U)": vlim,
                                 "reconstruct(T)": limiter},
        "solvers": {"W": {"solver": "GMRES", "preconditioner": preconditioner,
                          "nDirections": n_directions, "tolerance": 1e-12, "relTol": 0.0,
                          "maxIter": 1, "minIter": 1}},
        "fieldBounds": {"rho": (1e-3, 1e4), "p": (1e-3, 1e4), "T": (1e-3, 1e4)},
        "thermo": gas,
    }
    N = m.n_cells
    al = math.radians(alpha)
    return Case("naca0012", m, bcs, options, np.ones(N), np.tile(U0, (N, 1)), np.ones(N), steps=2000,
                force_patch="airfoil",
                force_dirs={"lift": (-math.sin(al), math.cos(al), 0.0), "drag": (math.cos(al), math.sin(al), 0.0)})


def swept_wing_c3(n_around: int = 192, n_normal: int = 64, n_span: int = 64, n_tip: int = 34,
                  precision: str = "fp64", n_directions: int = 20, flux: str = "HLLC",
                  ilu_parts: int = 0) -> Case:
    """Inviscid swept, tapered NACA0012 wing (taper 0.56, LE sweep 30 deg,
    semi-span 1.5 root chords) at Mach 0.84, alpha 3.06 deg, HLLC,
    OSPRE/OSPREV reconstruction, characteristic far field, local time
    stepping (steadyStateDST, CFL ramp to 50), block-GMRES with subdomain
    ILU(0); the Jacobian/ILU factors stored in `precision` (fp64 | fp32 |
    bf16) inside the FP64 defect-correction step.  Default mesh 1.2 M cells."""
    m = _mesh.swept_wing_oh(n_around, n_normal, n_span, n_tip)
    gas = dict(NORMALISED_GAS)
    U0 = farfield_state(0.84, 3.06, 1.0, 1.0, gas)
    bcs = {
        "wing": {"p": "zeroGradient", "U": "slip", "T": "zeroGradient"},
        "farfield": {"p": ("farField", 1.0), "U": ("farField", U0), "T": ("farField", 1.0)},
        "symmetry": {"p": "symmetryPlane", "U": "symmetryPlane", "T": "symmetryPlane"},
    }
    options = {
        "fluxScheme": flux,
        "Jacobian": "Roe",
        "timeControls": {"neighbouring": True, "initialCo": 5.0, "minCo": 0.1, "maxCo": 50.0},
        "ddtSchemes": {"default": "steadyStateDST"},
        "interpolationSchemes": {"reconstruct(rho)": "OSPRE", "reconstruct(U)": "OSPREV",
                                 "reconstruct(T)": "OSPRE"},
        "solvers": {"W": {"solver": "GMRES", "preconditioner": "ILUC0",
                          "nDirections": n_directions, "tolerance": 1e-12, "relTol": 0.0,
                          "maxIter": 1, "minIter": 1}},
        "fieldBounds": {"rho": (1e-3, 1e4), "p": (1e-3, 1e4), "T": (1e-3, 1e4)},
        "thermo": gas,
        "precision": precision,
    }
    if ilu_parts:
        options["ilu"] = {"parts": ilu_parts}
    N = m.n_cells
    al = math.radians(3.06)
    return Case("sweptWing", m, bcs, options, np.ones(N), np.tile(U0, (N, 1)), np.ones(N), steps=2000,
                force_patch="wing",
                force_dirs={"lift": (-math.sin(al), math.cos(al), 0.0), "drag": (math.cos(al), math.sin(al), 0.0)})


def naca0012_laminar(ni: int = 129, nj: int = 33, mach: float = 0.5, alpha: float = 1.0, reynolds: float = 5000.0,
                     flux: str = "AUSM+up", limiter: str = "vanLeer", sutherland: bool = False,
                     first_cell: float = 2e-3) -> Case:
    """Laminar NACA0012 (no-slip adiabatic wall) with the viscous terms of
    calcFields; constant viscosity from the chord Reynolds number, or
    Sutherland's law scaled to the same free-stream viscosity.  Wall spacing
    `first_cell` resolves the Re 5000 boundary layer with ~10 cells."""
    c = naca0012_inviscid(ni, nj, mach=mach, alpha=alpha, flux=flux, limiter=limiter, n_directions=20,
                          first_cell=first_cell)
    gas = c.options["thermo"]
    rho_inf = 1.0 / gas["R"]
    U_inf = mach * math.sqrt(gas["Cp"] / (gas["Cp"] - gas["R"]) * gas["R"])
    mu_inf = rho_inf * U_inf * 1.0 / reynolds
    c.bcs["airfoil"] = {"p": "zeroGradient", "U": ("fixedValue", (0.0, 0.0, 0.0)), "T": "zeroGradient"}
    if sutherland:
        Ts = 0.4
        As = mu_inf * (1.0 + Ts) / 1.0          # mu(T=1) = mu_inf
        c.options["transport"] = {"As": As, "Ts": Ts, "Pr": 0.72}
    else:
        c.options["transport"] = {"mu": mu_inf, "Pr": 0.72}
    c.name = "naca0012_laminar"
    return c


def naca0012_turbulent(ni: int = 257, nj: int = 65, mach: float = 0.73, alpha: float = 2.3,
                       reynolds: float = 6.5e6, model: str = "SAneg", flux: str = "AUSM+up",
                       limiter: str = "Venkatakrishnan", n_directions: int = 30, first_cell: float = 4e-6) -> Case:
    """Steady turbulent NACA0012: C-mesh ni x nj (far field 20 c, wall
    spacing for y+ ~ 1 growing at 1.15), M 0.73, alpha 2.3 deg, chord
    Reynolds 6.5e6 with Sutherland air scaled to the normalised gas,
    Spalart-Allmaras (SAneg default), AUSM+up + Venkatakrishnan, local time
    stepping ramped to CFL 50, block-GMRES(30) + block ILU(0)."""
    from . import mesh as _m
    m = _m.naca_cmesh(ni, nj, first_cell=first_cell)
    m.wall_distance = _m.wall_distance(m, ["airfoil"])
    gas = dict(NORMALISED_GAS)
    U0 = farfield_state(mach, alpha, 1.0, 1.0, gas)
    rho_inf = 1.0 / gas["R"]
    mu_inf = rho_inf * math.hypot(U0[0], U0[1]) / reynolds
    nut_inf = 3.0 * mu_inf / rho_inf                    # nuTilda_inf = 3 nu_inf
    Ts = 110.4 / 255.556                                # Sutherland T_s / T_inf (air at 255.556 K)
    bcs = {
        "airfoil": {"p": "zeroGradient", "U": ("fixedValue", (0.0, 0.0, 0.0)), "T": "zeroGradient",
                    "nuTilda": ("fixedValue", 0.0)},
        "farfield": {"p": ("farField", 1.0), "U": ("farField", U0), "T": ("farField", 1.0),
                     "nuTilda": ("inletOutlet", nut_inf)},
    }
    vlim = _vector_limiter(limiter)
    options = {
        "fluxScheme": flux,
        "Jacobian": "Roe",
        "timeControls": {"neighbouring": True, "initialCo": 2.0, "minCo": 0.1, "maxCo": 50.0},
        "ddtSchemes": {"default": "steadyStateDST"},
        "interpolationSchemes": {"reconstruct(rho)": limiter, "reconstruct(U)": vlim,
                                 "reconstruct(T)": limiter},
        "solvers": {"W": {"solver": "GMRES", "preconditioner": "ILUC0",
                          "nDirections": n_directions, "tolerance": 1e-12, "relTol": 0.0,
                          "maxIter": 1, "minIter": 1},
                    "nuTilda": {"nSweeps": 10}},
        "relaxationFactors": {"nuTilda": 0.5},
        "fieldBounds": {"rho": (1e-3, 1e4), "p": (1e-3, 1e4), "T": (1e-3, 1e4)},
        "thermo": gas,
        "transport": {"As": mu_inf * (1.0 + Ts), "Ts": Ts, "Pr": 0.72},
        "RASModel": model,
    }
    N = m.n_cells
    al = math.radians(alpha)
    return Case("naca0012_SA", m, bcs, options, np.ones(N), np.tile(U0, (N, 1)), np.ones(N),
                nuTilda=np.full(N, nut_inf), steps=4000, force_patch="airfoil",
                force_dirs={"lift": (-math.sin(al), math.cos(al), 0.0), "drag": (math.cos(al), math.sin(al), 0.0)})


def forward_step_3d_hybrid_c5(nx: int = 240, ny: int = 80, nz: int = 56, precision: str = "fp32",
                              limiter: str = "Venkatakrishnan", flux: str = "HLLC", jitter: float = 0.25,
                              seed: int = 20240601) -> Case:
    """3D Mach-3 forward-facing step on a hybrid tet/prism mesh (prisms in
    the lower half, tetrahedra above, conforming; interior nodes jittered by
    up to 25 % of the local spacing from `seed`, less where that would
    flatten a cell): 3.96 M cells at the default size.  HLLC, limited
    reconstruction, steady state by local time stepping (steadyStateDST, CFL
    0.5 ramping to at most 5), block-GMRES(20) with subdomain block ILU(0),
    Jacobian/ILU in `precision` with the FP64 residual.  BCs as the 2D
    step: fixed inflow, supersonic outflow, slip obstacle, symmetry planes
    on the channel walls.  With first-order HLL the steady state is reached
    (1e-10 in about 1,100 steps on a 26 k-cell version); the limited
    second-order iteration stalls near 1e-1, as limiter switching does on
    the other limited cases."""
    m = _mesh.forward_step_3d_hybrid(nx, ny, nz, jitter=jitter, seed=seed)
    U0 = (3.0, 0.0, 0.0)
    bcs = {
        "inlet": {"p": ("fixedValue", 1.0), "U": ("fixedValue", U0), "T": ("fixedValue", 1.0)},
        "outlet": {"p": "zeroGradient", "U": ("inletOutlet", U0), "T": ("inletOutlet", 1.0)},
        "obstacle": {"p": "zeroGradient", "U": "slip", "T": "zeroGradient"},
        "walls": {"p": "symmetryPlane", "U": "symmetryPlane", "T": "symmetryPlane"},
    }
    options = {
        "fluxScheme": flux,
        "Jacobian": "Roe",
        "timeControls": {"neighbouring": True, "initialCo": 0.5, "minCo": 0.1, "maxCo": 5.0},
        "ddtSchemes": {"default": "steadyStateDST"},
        "interpolationSchemes": {"reconstruct(rho)": limiter, "reconstruct(U)": _vector_limiter(limiter),
                                 "reconstruct(T)": limiter},
        "solvers": {"W": {"solver": "GMRES", "preconditioner": "ILUC0", "nDirections": 20,
                          "tolerance": 1e-12, "relTol": 0.0, "maxIter": 1, "minIter": 1}},
        "fieldBounds": {"rho": (1e-3, 1e4), "p": (1e-3, 1e4), "T": (1e-3, 1e4)},
        "thermo": dict(NORMALISED_GAS),
        "precision": precision,
    }
    N = m.n_cells
    return Case("forwardStep3DHybrid", m, bcs, options, np.ones(N), np.tile(U0, (N, 1)), np.ones(N), steps=1000,
                force_patch="obstacle", force_dirs={"lift": (0.0, 1.0, 0.0), "drag": (1.0, 0.0, 0.0)})


def rae2822(model: str = "SpalartAllmaras", flux: str = "Kurganov", limiter: str = "OSPRE",
            tutorial_schemes: bool = False) -> Case:
    """The reference's RAE2822 tutorial (tutorials/RAE2822): its own mesh
    (constant/polyMesh, 23,552 cells, read by rhodst_b200.foam and stored in
    tests/golden/rae2822_mesh.npz), its free stream (0/include/
    freestreamConditions: p 108987.773, U (233.44 9.417 0), T 255.556; nuTilda
    4.4e-5), boundary conditions (far-field p/U/T, no-slip adiabatic airfoil,
    nuTilda inletOutlet / fixedValue 0), Sutherland air, SpalartAllmaras,
    Kurganov with OSPRE/OSPREV, steadyStateDST with the face-based local time
    step at CFL 1 -> 500, BiCGStab + ILUC0 (maxIter 100, tolerance and relTol
    1e-10), nuTilda relaxation 0.5 and the tutorial's field bounds
    (system/*).  With `tutorial_schemes` the tutorial's gradient and
    convection schemes too (system/fvSchemes: grad(U) cellLimited Gauss
    linear 1, div(phi,nuTilda) Gauss linearUpwind grad(nuTilda)); without,
    Gauss linear and upwind."""
    from pathlib import Path
    from . import foam
    fixture = Path(__file__).resolve().parents[1] / "tests" / "golden" / "rae2822_mesh.npz"
    m = foam.load_npz(fixture)
    m.wall_distance = _mesh.wall_distance(m, ["airfoil"])
    p_inf, T_inf, U_inf, nut_inf = 108987.773, 255.556, (233.44, 9.417, 0.0), 4.4e-5
    bcs = {
        "airfoil": {"p": "zeroGradient", "U": ("fixedValue", (0.0, 0.0, 0.0)), "T": "zeroGradient",
                    "nuTilda": ("fixedValue", 0.0)},
        "freestreamBC": {"p": ("farField", p_inf), "U": ("farField", U_inf), "T": ("farField", T_inf),
                         "nuTilda": ("inletOutlet", nut_inf)},
    }
    options = {
        "fluxScheme": flux,
        "Jacobian": "Roe",
        "dependentVariable": "W",
        "timeControls": {"neighbouring": True, "initialCo": 1.0, "minCo": 1.0, "maxCo": 500.0},
        "ddtSchemes": {"default": "steadyStateDST"},
        "interpolationSchemes": {"reconstruct(rho)": limiter, "reconstruct(U)": _vector_limiter(limiter),
                                 "reconstruct(T)": limiter},
        "solvers": {"W": {"solver": "BiCGStab", "preconditioner": "ILUC0", "minIter": 1, "maxIter": 100,
                          "tolerance": 1e-10, "relTol": 1e-10}},
        "relaxationFactors": {"nuTilda": 0.5},
        "fieldBounds": {"rho": (0.01, 10.0), "p": (100.0, 1e6), "T": (10.0, 800.0)},
        "thermo": dict(AIR),
        "transport": dict(AIR_SUTHERLAND, Pr=AIR_PR),
        "RASModel": model,
    }
    if tutorial_schemes:
        options["gradSchemes"] = {"grad(U)": "cellLimited Gauss linear 1"}
        if model != "laminar":
            options["divSchemes"] = {"div(phi,nuTilda)": "Gauss linearUpwind grad(nuTilda)"}
    N = m.n_cells
    al = math.atan2(U_inf[1], U_inf[0])
    return Case("rae2822", m, bcs, options, np.full(N, p_inf), np.tile(np.array(U_inf), (N, 1)),
                np.full(N, T_inf), nuTilda=np.full(N, nut_inf), steps=1000, force_patch="airfoil",
                force_dirs={"lift": (-math.sin(al), math.cos(al), 0.0), "drag": (math.cos(al), math.sin(al), 0.0)})
