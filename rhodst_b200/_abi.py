"""ctypes mirror of include/rdst.h and a thin object wrapper over one
library that exports that ABI.

The wrapper is the Python-side counterpart of the foam-extend host: it
marshals a :class:`rhodst_b200.mesh.PolyMesh`, the boundary conditions and
the dictionary entries into the C structs and calls the library.  Argument
names and meanings follow the reference (rhoDSTDict / fvSchemes /
fvSolution keys, foam patch-field type names).
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int32, c_void_p
from typing import Dict, Mapping, Optional

import numpy as np

RDST_OK = 0
STATUS_NAMES = {0: "RDST_OK", 1: "RDST_ERR_CONFIG", 2: "RDST_ERR_MESH", 3: "RDST_ERR_CUDA",
                4: "RDST_ERR_DIVERGED", 5: "RDST_ERR_TIMEOUT", 6: "RDST_ERR_UNSUPPORTED",
                7: "RDST_ERR_ARG"}

BC_FIXED_VALUE, BC_ZERO_GRADIENT, BC_INLET_OUTLET, BC_SYMMETRY, BC_SLIP, BC_FARFIELD = range(6)
_BC_NAMES = {"fixedValue": BC_FIXED_VALUE, "zeroGradient": BC_ZERO_GRADIENT,
             "inletOutlet": BC_INLET_OUTLET, "symmetryPlane": BC_SYMMETRY, "symmetry": BC_SYMMETRY,
             "slip": BC_SLIP, "noSlip": BC_FIXED_VALUE, "farField": BC_FARFIELD,
             "farFieldPressureDST": BC_FARFIELD, "farFieldVelocityDST": BC_FARFIELD,
             "farFieldTemperatureDST": BC_FARFIELD, "empty": BC_ZERO_GRADIENT,
             "calculated": BC_ZERO_GRADIENT}


class RdstError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class RdstPatch(ctypes.Structure):
    _fields_ = [("start", c_int32), ("size", c_int32), ("type", c_int32),
                ("bc_p", c_int32), ("bc_U", c_int32), ("bc_T", c_int32), ("bc_nuTilda", c_int32),
                ("p_value", c_double), ("U_value", c_double * 3), ("T_value", c_double),
                ("nuTilda_value", c_double)]


class RdstMesh(ctypes.Structure):
    _fields_ = [("n_cells", c_int32), ("n_internal_faces", c_int32), ("n_faces", c_int32),
                ("n_patches", c_int32), ("owner", POINTER(c_int32)), ("neighbour", POINTER(c_int32)),
                ("Sf", POINTER(c_double)), ("Cf", POINTER(c_double)), ("magSf", POINTER(c_double)),
                ("weights", POINTER(c_double)), ("deltaCoeffs", POINTER(c_double)),
                ("C", POINTER(c_double)), ("V", POINTER(c_double)),
                ("patches", POINTER(RdstPatch)), ("wall_distance", POINTER(c_double))]


class RdstObjective(ctypes.Structure):
    _fields_ = [("patch", c_int32), ("direction", c_double * 3), ("p_ref", c_double), ("scale", c_double)]


class RdstAdjointReport(ctypes.Structure):
    _fields_ = [("J", c_double), ("force", c_double * 3), ("dJ_dU", c_double * 3), ("residual0", c_double),
                ("residual", c_double), ("iterations", c_int32), ("cycles", c_int32), ("t_ms", c_double)]


class RdstStepReport(ctypes.Structure):
    _fields_ = [("time", c_double), ("deltaT", c_double), ("courant", c_double),
                ("res_l2", c_double * 5), ("res_mag", c_double),
                ("lin_initial", c_double * 5), ("lin_final", c_double * 5),
                ("lin_iterations", c_int32), ("flags", c_int32),
                ("rdt_min", c_double), ("rdt_max", c_double),
                ("t_flux_ms", c_double), ("t_jacobian_ms", c_double), ("t_precond_ms", c_double),
                ("t_krylov_ms", c_double), ("t_update_ms", c_double)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


def flatten_options(opts: Mapping, prefix: str = "") -> Dict[str, str]:
    """Nested dictionaries (rhoDSTDict / fvSchemes / fvSolution style) to the
    dotted key/value strings the C ABI takes."""
    out: Dict[str, str] = {}
    for k, v in opts.items():
        key = f"{prefix}{k}"
        if isinstance(v, Mapping):
            out.update(flatten_options(v, key + "."))
        elif isinstance(v, bool):
            out[key] = "true" if v else "false"
        elif isinstance(v, (tuple, list)):
            out[key] = " ".join(repr(float(x)) if isinstance(x, float) else str(x) for x in v)
        elif isinstance(v, float):
            out[key] = repr(v)
        else:
            out[key] = str(v)
    return out


def _bc(spec) -> tuple:
    """'zeroGradient' | ('fixedValue', value) | ('inletOutlet', inletValue) |
    ('farField', freestream value) -> (code, value)"""
    if isinstance(spec, str):
        return _BC_NAMES[spec], None
    name, val = spec
    return _BC_NAMES[name], val


def declare(lib: ctypes.CDLL, prefix: str) -> None:
    def f(name, res, args):
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
    vp = c_void_p
    dp = POINTER(c_double)
    f("create", c_int32, [POINTER(RdstMesh), c_int32, POINTER(c_char_p), POINTER(c_char_p), POINTER(vp)])
    f("set_primitive", c_int32, [vp, dp, dp, dp, dp])
    f("set_conservative", c_int32, [vp, dp, dp, dp])
    f("set_held_cells", c_int32, [vp, POINTER(ctypes.c_uint8)])
    f("set_nu_tilda", c_int32, [vp, dp])
    f("get_cells", c_int32, [vp, c_int32, POINTER(c_int32), dp])
    f("set_cells", c_int32, [vp, c_int32, POINTER(c_int32), dp])
    f("get_conservative", c_int32, [vp, dp, dp, dp])
    f("get_primitive", c_int32, [vp, dp, dp, dp, dp])
    f("step", c_int32, [vp, c_int32, POINTER(RdstStepReport)])
    f("residual", c_int32, [vp, dp])
    f("assemble", c_int32, [vp, dp, dp, dp, dp])
    f("forces", c_int32, [vp, c_int32, dp, dp, dp, dp, c_double, c_double, c_double, dp])
    f("last_error", c_char_p, [vp])
    f("destroy", None, [vp])
    f("version", c_char_p, [])
    if hasattr(lib, prefix + "stream"):
        f("stream", c_void_p, [vp])
        f("launch_count", ctypes.c_int64, [vp])
        f("last_step_ms", c_double, [vp])
        f("kernel_stats", c_int32, [vp, c_char_p, POINTER(ctypes.c_int64), POINTER(c_double)])
        f("set_profile", c_int32, [vp, c_int32])
        f("get_cells_device", c_int32, [vp, c_int32, POINTER(c_int32), c_void_p])
        f("set_cells_device", c_int32, [vp, c_int32, POINTER(c_int32), c_void_p])
    if hasattr(lib, prefix + "adjoint"):
        f("objective_gradient", c_int32, [vp, POINTER(RdstObjective), dp, dp, dp, dp])
        f("adjoint_product", c_int32, [vp, dp, dp, dp])
        f("tangent_product", c_int32, [vp, dp, dp])
        f("boundary_branches", c_int32, [vp, dp, dp])
        f("set_geometry", c_int32, [vp, POINTER(RdstMesh)])
        f("adjoint", c_int32, [vp, POINTER(RdstObjective), c_double, c_int32, c_int32, dp,
                               POINTER(RdstAdjointReport)])


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(POINTER(c_double))


class Solver:
    """One context of an rdst-ABI library (the B200 library, or the CPU
    oracle in the test suite).

    ``bcs`` maps patch name -> {"p": spec, "U": spec, "T": spec} with foam
    patch-field type names; ``options`` holds rhoDSTDict / fvSchemes /
    fvSolution / thermo entries (nested dicts or dotted keys).
    """

    def __init__(self, lib: ctypes.CDLL, prefix: str, mesh, bcs: Mapping, options: Mapping):
        self.lib = lib
        self.prefix = prefix
        self.mesh = mesh
        self._h = c_void_p()
        self._keep = []
        m = mesh
        patches = (RdstPatch * len(m.patches))()
        for i, p in enumerate(m.patches):
            P = patches[i]
            P.start, P.size, P.type = p.start, p.size, p.type
            spec = bcs.get(p.name, {})
            if p.type == 3:   # empty
                spec = {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient"}
            elif p.type == 2 and not spec:
                spec = {"p": "symmetryPlane", "U": "symmetryPlane", "T": "symmetryPlane"}
            if not spec:
                raise KeyError(f"no boundary conditions for patch {p.name}")
            P.bc_p, pv = _bc(spec["p"])
            P.bc_U, uv = _bc(spec["U"])
            P.bc_T, tv = _bc(spec["T"])
            P.p_value = float(pv) if pv is not None else 0.0
            uv = uv if uv is not None else (0.0, 0.0, 0.0)
            for k in range(3):
                P.U_value[k] = float(uv[k])
            P.T_value = float(tv) if tv is not None else 0.0
            nv = spec.get("nuTilda", "zeroGradient")
            if isinstance(nv, tuple):
                P.bc_nuTilda = _BC_NAMES[nv[0]]
                P.nuTilda_value = float(nv[1])
            else:
                P.bc_nuTilda = _BC_NAMES[nv]
                P.nuTilda_value = 0.0
            if P.bc_nuTilda == BC_FARFIELD:
                P.bc_nuTilda = BC_INLET_OUTLET
        self._patches = patches
        cm = self._c_mesh(m)
        flat = {}
        for k, v in options.items():
            if isinstance(v, Mapping):
                flat.update(flatten_options({k: v}))
            else:
                flat.update(flatten_options({k: v}))
        keys = (c_char_p * len(flat))(*[k.encode() for k in flat])
        vals = (c_char_p * len(flat))(*[v.encode() for v in flat.values()])
        st = self._fn("create")(ctypes.byref(cm), len(flat), keys, vals, ctypes.byref(self._h))
        if st != RDST_OK:
            raise RdstError(st, f"create failed ({flat.get('fluxScheme')})")
        self.options = flat

    def _c_mesh(self, m):
        """rdst_mesh view of a PolyMesh; the arrays it points to are kept
        alive with the solver."""
        a = dict(
            owner=np.ascontiguousarray(m.owner, dtype=np.int32),
            neighbour=np.ascontiguousarray(m.neighbour, dtype=np.int32),
            Sf=np.ascontiguousarray(m.Sf, dtype=np.float64), Cf=np.ascontiguousarray(m.Cf, dtype=np.float64),
            magSf=np.ascontiguousarray(m.magSf, dtype=np.float64),
            weights=np.ascontiguousarray(m.weights, dtype=np.float64),
            deltaCoeffs=np.ascontiguousarray(m.deltaCoeffs, dtype=np.float64),
            C=np.ascontiguousarray(m.C, dtype=np.float64), V=np.ascontiguousarray(m.V, dtype=np.float64))
        wd = None if m.wall_distance is None else np.ascontiguousarray(m.wall_distance, dtype=np.float64)
        cm = RdstMesh(m.n_cells, m.n_internal_faces, m.n_faces, len(m.patches),
                      a["owner"].ctypes.data_as(POINTER(c_int32)), a["neighbour"].ctypes.data_as(POINTER(c_int32)),
                      _dptr(a["Sf"]), _dptr(a["Cf"]), _dptr(a["magSf"]), _dptr(a["weights"]),
                      _dptr(a["deltaCoeffs"]), _dptr(a["C"]), _dptr(a["V"]), self._patches,
                      _dptr(wd) if wd is not None else None)
        self._arrays = a
        self._keep = [self._patches, cm, wd]
        return cm

    # -- plumbing ---------------------------------------------------------
    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, st: int, what: str):
        if st != RDST_OK:
            msg = self._fn("last_error")(self._h)
            raise RdstError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self._h:
            self._fn("destroy")(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_cells(self) -> int:
        return self.mesh.n_cells

    # -- API --------------------------------------------------------------
    def set_primitive(self, p, U, T, nuTilda=None):
        N = self.n_cells
        p = np.ascontiguousarray(np.broadcast_to(p, (N,)), dtype=np.float64)
        U = np.ascontiguousarray(np.broadcast_to(U, (N, 3)), dtype=np.float64)
        T = np.ascontiguousarray(np.broadcast_to(T, (N,)), dtype=np.float64)
        nt = None if nuTilda is None else np.ascontiguousarray(np.broadcast_to(nuTilda, (N,)), dtype=np.float64)
        self._check(self._fn("set_primitive")(self._h, _dptr(p), _dptr(U), _dptr(T), _dptr(nt)), "set_primitive")

    def set_held_cells(self, mask=None):
        """Cells held at their state in the steps (the halo cells of a
        decomposed run: zero residual, identity rows), or None for none."""
        if mask is None:
            self._check(self._fn("set_held_cells")(self._h, None), "set_held_cells")
            return
        mk = np.ascontiguousarray(np.asarray(mask, dtype=bool), dtype=np.uint8)
        if mk.shape != (self.n_cells,):
            raise ValueError("mask needs one entry per cell")
        self._check(self._fn("set_held_cells")(self._h, mk.ctypes.data_as(POINTER(ctypes.c_uint8))),
                    "set_held_cells")

    def get_cells(self, cells):
        """States of the listed cells: n x 6 (rho, rhoU, rhoE, nuTilda)."""
        ids = np.ascontiguousarray(cells, dtype=np.int32)
        out = np.empty((ids.size, 6))
        self._check(self._fn("get_cells")(self._h, ids.size, ids.ctypes.data_as(POINTER(c_int32)), _dptr(out)),
                    "get_cells")
        return out

    def set_cells(self, cells, values):
        """Write n x 6 states into the listed cells between steps."""
        ids = np.ascontiguousarray(cells, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(ids.size, 6)
        self._check(self._fn("set_cells")(self._h, ids.size, ids.ctypes.data_as(POINTER(c_int32)), _dptr(v)),
                    "set_cells")

    def get_cells_device(self, cells, out_ptr: int):
        """States of the listed cells into a device buffer of the context's
        GPU (n x 6 doubles at out_ptr; B200 library only)."""
        ids = np.ascontiguousarray(cells, dtype=np.int32)
        self._check(self._fn("get_cells_device")(self._h, ids.size, ids.ctypes.data_as(POINTER(c_int32)),
                                                 c_void_p(out_ptr)), "get_cells_device")

    def set_cells_device(self, cells, in_ptr: int):
        """set_cells from a device buffer (n x 6 doubles at in_ptr, ready)."""
        ids = np.ascontiguousarray(cells, dtype=np.int32)
        self._check(self._fn("set_cells_device")(self._h, ids.size, ids.ctypes.data_as(POINTER(c_int32)),
                                                 c_void_p(in_ptr)), "set_cells_device")

    def set_nu_tilda(self, nut):
        """Replace nuTilda between steps (mu_t follows; mean flow and time
        control kept)."""
        nt = np.ascontiguousarray(nut, dtype=np.float64)
        if nt.shape != (self.n_cells,):
            raise ValueError("nuTilda needs one value per cell")
        self._check(self._fn("set_nu_tilda")(self._h, _dptr(nt)), "set_nu_tilda")

    def set_conservative(self, rho, rhoU, rhoE):
        N = self.n_cells
        rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(N)
        rhoU = np.ascontiguousarray(rhoU, dtype=np.float64).reshape(N, 3)
        rhoE = np.ascontiguousarray(rhoE, dtype=np.float64).reshape(N)
        self._check(self._fn("set_conservative")(self._h, _dptr(rho), _dptr(rhoU), _dptr(rhoE)), "set_conservative")

    def conservative(self):
        N = self.n_cells
        rho, rhoU, rhoE = np.empty(N), np.empty((N, 3)), np.empty(N)
        self._check(self._fn("get_conservative")(self._h, _dptr(rho), _dptr(rhoU), _dptr(rhoE)), "get_conservative")
        return rho, rhoU, rhoE

    def primitive(self):
        N = self.n_cells
        p, U, T, nt = np.empty(N), np.empty((N, 3)), np.empty(N), np.empty(N)
        self._check(self._fn("get_primitive")(self._h, _dptr(p), _dptr(U), _dptr(T), _dptr(nt)), "get_primitive")
        return p, U, T, nt

    def step(self, n: int = 1):
        reps = (RdstStepReport * max(n, 1))()
        self._check(self._fn("step")(self._h, n, reps), "step")
        return [reps[i].as_dict() for i in range(n)]

    # -- instrumentation (B200 library only) --------------------------------
    def stream_handle(self) -> int:
        return int(self._fn("stream")(self._h) or 0)

    def launch_count(self) -> int:
        return int(self._fn("launch_count")(self._h))

    def last_step_ms(self) -> float:
        return float(self._fn("last_step_ms")(self._h))

    def set_profile(self, on: bool) -> None:
        self._check(self._fn("set_profile")(self._h, 1 if on else 0), "set_profile")

    def kernel_stats(self, kernel: str):
        n = ctypes.c_int64()
        ms = c_double()
        self._check(self._fn("kernel_stats")(self._h, kernel.encode(), ctypes.byref(n), ctypes.byref(ms)),
                    "kernel_stats")
        return int(n.value), float(ms.value)

    def residual(self) -> np.ndarray:
        out = np.empty((self.n_cells, 5))
        self._check(self._fn("residual")(self._h, _dptr(out)), "residual")
        return out

    def assemble(self):
        N, Fi = self.n_cells, self.mesh.n_internal_faces
        d, u, l, s = np.empty((N, 5, 5)), np.empty((Fi, 5, 5)), np.empty((Fi, 5, 5)), np.empty((N, 5))
        self._check(self._fn("assemble")(self._h, _dptr(d), _dptr(u), _dptr(l), _dptr(s)), "assemble")
        return d, u, l, s

    # ---- discrete adjoint
    def _objective(self, patch: str, direction, p_ref: float, scale: float) -> RdstObjective:
        ob = RdstObjective()
        ob.patch = self.mesh.patch_index(patch)
        for k in range(3):
            ob.direction[k] = float(direction[k])
        ob.p_ref = float(p_ref)
        ob.scale = float(scale)
        return ob

    def objective_gradient(self, patch: str, direction, p_ref: float = 0.0, scale: float = 1.0):
        """J = scale * sum over the patch of (p - p_ref) S . direction, its
        force vector, dJ/dW (N x 5) and the explicit dJ/dU_patch."""
        ob = self._objective(patch, direction, p_ref, scale)
        J, force, dU = c_double(), np.empty(3), np.empty(3)
        dW = np.empty((self.n_cells, 5))
        self._check(self._fn("objective_gradient")(self._h, ctypes.byref(ob), ctypes.byref(J), _dptr(force),
                                                   _dptr(dW), _dptr(dU)), "objective_gradient")
        return float(J.value), force, dW, dU

    def adjoint_product(self, v: np.ndarray):
        """(dR/dW)^T v (N x 5) and (dR/dU_patch)^T v (3)."""
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(self.n_cells, 5)
        u, dU = np.empty((self.n_cells, 5)), np.empty(3)
        self._check(self._fn("adjoint_product")(self._h, _dptr(v), _dptr(u), _dptr(dU)), "adjoint_product")
        return u, dU

    def tangent_product(self, u: np.ndarray) -> np.ndarray:
        """(dR/dW) u (N x 5) by forward-mode linearization."""
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.n_cells, 5)
        Ju = np.empty((self.n_cells, 5))
        self._check(self._fn("tangent_product")(self._h, _dptr(u), _dptr(Ju)), "tangent_product")
        return Ju

    def set_geometry(self, mesh):
        """Move the solver onto `mesh`, which has this solver's topology
        (rdst_set_geometry); state, options and boundary values stay."""
        old = [(p.name, p.start, p.size) for p in self.mesh.patches]
        if [(p.name, p.start, p.size) for p in mesh.patches] != old:
            raise ValueError("set_geometry: the new mesh's patches differ from the solver's")
        cm = self._c_mesh(mesh)
        self._check(self._fn("set_geometry")(self._h, ctypes.byref(cm)), "set_geometry")
        self.mesh = mesh

    def boundary_branches(self):
        """(previous boundary mass flux, far-field Mach) per boundary face
        (face - n_internal_faces): the inputs of the current boundary branches."""
        nb = self.mesh.n_faces - self.mesh.n_internal_faces
        phi, mach = np.empty(nb), np.empty(nb)
        self._check(self._fn("boundary_branches")(self._h, _dptr(phi), _dptr(mach)), "boundary_branches")
        return phi, mach

    def adjoint(self, patch: str, direction, p_ref: float = 0.0, scale: float = 1.0, rel_tol: float = 1e-10,
                max_cycles: int = 50, n_directions: int = 30, want_psi: bool = False):
        """Adjoint solve for the pressure-force objective; returns the report
        as a dict (J, force, dJ_dU, residuals, iterations, t_ms) and psi."""
        ob = self._objective(patch, direction, p_ref, scale)
        rep = RdstAdjointReport()
        psi = np.empty((self.n_cells, 5)) if want_psi else None
        self._check(self._fn("adjoint")(self._h, ctypes.byref(ob), rel_tol, max_cycles, n_directions,
                                        _dptr(psi), ctypes.byref(rep)), "adjoint")
        out = {"J": rep.J, "force": np.array(rep.force[:]), "dJ_dU": np.array(rep.dJ_dU[:]),
               "residual0": rep.residual0, "residual": rep.residual, "iterations": rep.iterations,
               "cycles": rep.cycles, "t_ms": rep.t_ms}
        return out, psi

    def forces(self, patch: str, lift_dir, drag_dir, p_ref: float, q_ref_area: float,
               cofr=(0.25, 0.0, 0.0), pitch_axis=(0.0, 0.0, 1.0), l_ref: float = 1.0):
        out = np.empty(3)
        arr = [np.ascontiguousarray(x, dtype=np.float64) for x in (lift_dir, drag_dir, cofr, pitch_axis)]
        self._check(self._fn("forces")(self._h, self.mesh.patch_index(patch), _dptr(arr[0]), _dptr(arr[1]),
                                       _dptr(arr[2]), _dptr(arr[3]), p_ref, q_ref_area, l_ref, _dptr(out)),
                    "forces")
        return {"Cl": out[0], "Cd": out[1], "Cm": out[2]}
