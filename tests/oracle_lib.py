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
    deps = [src, ROOT / "oracle" / "rdst_cs.inc", ROOT / "include" / "rdst.h", ROOT / "rhodst_b200" / "csrc" / "rdst_options.h"]
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
        lib.rdsto_set_nu_tilda.restype = ctypes.c_int32
        lib.rdsto_set_nu_tilda.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.rdsto_set_held_cells.restype = ctypes.c_int32
        lib.rdsto_set_held_cells.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8)]
        lib.rdsto_grad_U.restype = ctypes.c_int32
        lib.rdsto_grad_U.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.rdsto_precondition.restype = ctypes.c_int32
        lib.rdsto_precondition.argtypes = [ctypes.c_void_p, d, d]
        lib.rdsto_cs_residual.restype = ctypes.c_int32
        lib.rdsto_cs_residual.argtypes = [ctypes.c_void_p, d, d, d, ctypes.c_double, d, d, d, d]
        lib.rdsto_cs_objective.restype = ctypes.c_int32
        lib.rdsto_cs_objective.argtypes = [ctypes.c_void_p, d, d, d, ctypes.c_double, d, d, ctypes.c_int32, d,
                                           ctypes.c_double, ctypes.c_double, d, d, d]
        lib.rdsto_linear_solve.restype = ctypes.c_int32
        lib.rdsto_linear_solve.argtypes = [ctypes.c_void_p, d, ctypes.c_void_p]
        lib.rdsto_set_threads.restype = ctypes.c_int32
        lib.rdsto_set_threads.argtypes = [ctypes.c_int32]
        lib.rdsto_partition_rcb.restype = ctypes.c_int32
        lib.rdsto_partition_rcb.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        lib.rdsto_get_partition.restype = ctypes.c_int32
        lib.rdsto_get_partition.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]
        _lib = lib
    return _lib


def set_threads(n: int = 0) -> int:
    """Threads of the oracle's parallel loops (0: the OpenMP default);
    returns the count in effect.  Results do not depend on it."""
    return int(load_oracle().rdsto_set_threads(n))


class OracleSolver(Solver):
    def __init__(self, mesh, bcs, options, partition=None, rcb_parts=None):
        super().__init__(load_oracle(), "rdsto_", mesh, bcs, options)
        if rcb_parts is not None:
            self._check(self.lib.rdsto_partition_rcb(self._h, int(rcb_parts)), "partition_rcb")
        if partition is not None:
            import numpy as np
            self._part = np.ascontiguousarray(partition, dtype=np.int32)
            self.lib.rdsto_set_partition(self._h, self._part.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))

    def partition(self):
        import numpy as np
        out = np.empty(self.n_cells, dtype=np.int32)
        self._check(self.lib.rdsto_get_partition(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
                    "get_partition")
        return out

    def grad_U(self):
        """grad(U) (N x 3 x 3, [i, a, j] = d U_j / d x_a) as the viscous terms
        use it at the current state (cellLimited when selected)."""
        import numpy as np
        out = np.empty((self.n_cells, 9))
        self._check(self.lib.rdsto_grad_U(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "grad_U")
        return out.reshape(-1, 3, 3)

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


def _dp(a):
    import numpy as np
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a


class ComplexStep:
    """Complex-step derivatives of the oracle's inviscid residual and of the
    pressure-force objective (rdsto_cs_residual / rdsto_cs_objective):
    Im f(x + i h v) / h with h = 1e-30, exact to rounding.  W, u are N x 5
    conservative fields; branches = (phi_prev, mach) per boundary face or
    None for the oracle's own."""
    H = 1e-30

    def __init__(self, oracle: "OracleSolver"):
        self.o = oracle

    def residual(self, W, u=None, dU=None, branches=None):
        import numpy as np
        N = self.o.n_cells
        keep = []
        def p(a):
            if a is None:
                return None
            q, arr = _dp(a)
            keep.append(arr)
            return q
        R, dR = np.empty((N, 5)), np.empty((N, 5))
        ph, mc = branches if branches is not None else (None, None)
        st = self.o.lib.rdsto_cs_residual(self.o._h, p(W), p(u), p(dU), self.H, p(ph), p(mc), p(R), p(dR))
        self.o._check(st, "cs_residual")
        return R, dR

    def objective(self, W, patch: str, direction, p_ref=0.0, scale=1.0, u=None, dU=None, branches=None,
                  per_cell=False):
        import numpy as np
        keep = []
        def p(a):
            if a is None:
                return None
            q, arr = _dp(a)
            keep.append(arr)
            return q
        J, dJ = ctypes.c_double(), ctypes.c_double()
        ph, mc = branches if branches is not None else (None, None)
        cells = np.zeros(self.o.n_cells) if per_cell else None
        st = self.o.lib.rdsto_cs_objective(self.o._h, p(W), p(u), p(dU), self.H, p(ph), p(mc),
                                           self.o.mesh.patch_index(patch), p(list(direction)), p_ref, scale,
                                           ctypes.byref(J), ctypes.byref(dJ),
                                           cells.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if per_cell else None)
        self.o._check(st, "cs_objective")
        return (J.value, dJ.value, cells) if per_cell else (J.value, dJ.value)


def conservative_array(W):
    """(rho, rhoU, rhoE) -> N x 5."""
    import numpy as np
    rho, rhoU, rhoE = W
    return np.ascontiguousarray(np.concatenate([rho[:, None], rhoU, rhoE[:, None]], 1))


def distance2_colors(mesh, hops: int = 2):
    """Greedy colouring of the cells such that two cells of one colour are
    more than `hops` face-hops apart (hops = 2 for a residual whose rows
    depend on face neighbours only, 4 when they depend on neighbours of
    neighbours)."""
    import numpy as np
    N = mesh.n_cells
    own = np.asarray(mesh.owner[:mesh.n_internal_faces])
    nei = np.asarray(mesh.neighbour)
    adj = [[] for _ in range(N)]
    for a, b in zip(own, nei):
        adj[a].append(int(b))
        adj[b].append(int(a))
    color = -np.ones(N, dtype=np.int64)
    for i in range(N):
        seen = {i}
        front = [i]
        for _ in range(hops):
            nxt = []
            for x in front:
                for y in adj[x]:
                    if y not in seen:
                        seen.add(y)
                        nxt.append(y)
            front = nxt
        used = {int(color[j]) for j in seen if color[j] >= 0}
        k = 0
        while k in used:
            k += 1
        color[i] = k
    return color, adj
