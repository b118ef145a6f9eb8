"""Loader for the CPU FP64 oracle (oracle/rdst_oracle.cpp).

Test infrastructure only: the oracle is the parity checker and the timed
CPU baseline; it is never the thing measured or shipped."""
import ctypes
import subprocess
from pathlib import Path

from rhodst_b200._abi import Solver, declare

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "_build" / "librdst_oracle.so"
_lib = None


def build_oracle() -> Path:
    src = ROOT / "oracle" / "rdst_oracle.cpp"
    deps = [src, ROOT / "include" / "rdst.h", ROOT / "rhodst_b200" / "csrc" / "rdst_options.h"]
    if not ORACLE_SO.exists() or any(p.stat().st_mtime > ORACLE_SO.stat().st_mtime for p in deps):
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return ORACLE_SO


def load_oracle() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(build_oracle()))
        declare(lib, "rdsto_")
        d = ctypes.POINTER(ctypes.c_double)
        lib.rdsto_face_flux.restype = None
        lib.rdsto_face_flux.argtypes = [ctypes.c_int32, d, d, d, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int32, ctypes.c_double, d]
        lib.rdsto_flux_jacobian.restype = None
        lib.rdsto_flux_jacobian.argtypes = [d, d, ctypes.c_double, d]
        lib.rdsto_limiter.restype = ctypes.c_double
        lib.rdsto_limiter.argtypes = [ctypes.c_int32, ctypes.c_double]
        lib.rdsto_set_partition.restype = ctypes.c_int32
        lib.rdsto_set_partition.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]
        lib.rdsto_precondition.restype = ctypes.c_int32
        lib.rdsto_precondition.argtypes = [ctypes.c_void_p, d, d]
        lib.rdsto_linear_solve.restype = ctypes.c_int32
        lib.rdsto_linear_solve.argtypes = [ctypes.c_void_p, d, ctypes.c_void_p]
        _lib = lib
    return _lib


class OracleSolver(Solver):
    def __init__(self, mesh, bcs, options, partition=None):
        super().__init__(load_oracle(), "rdsto_", mesh, bcs, options)
        if partition is not None:
            import numpy as np
            self._part = np.ascontiguousarray(partition, dtype=np.int32)
            self.lib.rdsto_set_partition(self._h, self._part.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))

    def precondition(self, b):
        import numpy as np
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, 5)
        x = np.empty_like(b)
        d = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.rdsto_precondition(self._h, b.ctypes.data_as(d), x.ctypes.data_as(d)), "precondition")
        return x

    def linear_solve(self):
        import numpy as np
        from rhodst_b200._abi import RdstStepReport
        x = np.empty((self.n_cells, 5))
        rep = RdstStepReport()
        self._check(self.lib.rdsto_linear_solve(self._h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                ctypes.byref(rep)), "linear_solve")
        return x, rep.as_dict()
