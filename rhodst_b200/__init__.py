"""rhodst_b200 -- B200 (sm_100a) implementation of rhoDST's fully-coupled
density-based implicit step behind a C ABI (include/rdst.h).

The product is the shared library ``rhodst_b200/librdst.so`` (host C++ +
hand-written CUDA kernels).  This package is its Python host: mesh
generators/geometry (:mod:`rhodst_b200.mesh`), case definitions
(:mod:`rhodst_b200.cases`) and a ctypes wrapper that mirrors the
reference's dictionary-driven interface (:class:`Solver`).  There is no CPU
fallback: without the built library (or without a GPU) construction fails.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Mapping

from . import cases, mesh, shape
from ._abi import RdstError, RdstStepReport, declare, flatten_options
from ._abi import Solver as _AbiSolver

LIB_PATH = Path(__file__).resolve().parent / "librdst.so"
_lib = None


def load_library() -> ctypes.CDLL:
    """Load the in-tree librdst.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m rhodst_b200.build` "
                               "(the B200 path has no CPU fallback)")
        lib = ctypes.CDLL(str(LIB_PATH))
        declare(lib, "rdst_")
        lib.rdst_partition_cells.restype = ctypes.c_int32
        lib.rdst_partition_cells.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double), ctypes.c_int32,
                                             ctypes.POINTER(ctypes.c_int32)]
        i32p = ctypes.POINTER(ctypes.c_int32)
        lib.rdst_partition_graph.restype = ctypes.c_int32
        lib.rdst_partition_graph.argtypes = [ctypes.c_int32, ctypes.c_int32, i32p, i32p, ctypes.c_int32, i32p]
        _lib = lib
    return _lib


class Solver(_AbiSolver):
    """One fully-coupled-step context on the GPU.

    >>> case = cases.forward_step_c1()
    >>> s = Solver(case.mesh, case.bcs, case.options)
    >>> s.set_primitive(case.p, case.U, case.T)
    >>> reports = s.step(10)
    """

    def __init__(self, mesh_, bcs: Mapping, options: Mapping):
        super().__init__(load_library(), "rdst_", mesh_, bcs, options)


def solver_for(case: "cases.Case") -> Solver:
    s = Solver(case.mesh, case.bcs, case.options)
    s.set_primitive(case.p, case.U, case.T, case.nuTilda)
    return s


def partition_cells(C, n_parts: int):
    """Recursive coordinate bisection used by the subdomain ILU(0)."""
    import numpy as np
    lib = load_library()
    C = np.ascontiguousarray(C, dtype=np.float64)
    out = np.empty(C.shape[0], dtype=np.int32)
    st = lib.rdst_partition_cells(C.shape[0], C.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n_parts,
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    if st != 0:
        raise RdstError(st, "partition_cells")
    return out


def partition_graph(mesh, n_parts: int):
    """Recursive graph bisection of the cell graph (the partition of the
    option "ilu.partition" "graph")."""
    import numpy as np
    lib = load_library()
    Fi = int(mesh.n_internal_faces)
    own = np.ascontiguousarray(np.asarray(mesh.owner)[:Fi], dtype=np.int32)
    nei = np.ascontiguousarray(np.asarray(mesh.neighbour)[:Fi], dtype=np.int32)
    out = np.empty(int(mesh.n_cells), dtype=np.int32)
    p = ctypes.POINTER(ctypes.c_int32)
    st = lib.rdst_partition_graph(int(mesh.n_cells), Fi, own.ctypes.data_as(p), nei.ctypes.data_as(p), n_parts,
                                  out.ctypes.data_as(p))
    if st != 0:
        raise RdstError(st, "partition_graph")
    return out


__all__ = ["Solver", "solver_for", "RdstError", "RdstStepReport", "load_library", "partition_cells", "partition_graph",
           "mesh", "cases", "flatten_options"]
