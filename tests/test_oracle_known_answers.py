"""Known-answer tests that pin the CPU oracle.

The reference (rhoDST on foam-extend 4.1) cannot be built here and ships no
tests or golden outputs, so the oracle is pinned by properties the
restated algorithms must satisfy exactly or to round-off:

* every flux scheme is consistent: F(W, W) = physical Euler flux;
* conservation/orientation: F(W_L, W_R, S) = -F(W_R, W_L, -S);
* supersonic upwinding: for M_n > 1 on both sides, F = F(W_L) (all schemes);
* the Roe block is the exact Euler flux Jacobian: A(W).n W = F(W).n
  (homogeneity) and A matches central differences of F;
* free-stream preservation: R(W) = 0 for a uniform flow on the channel;
* ILU(0) is exact LU on a mesh whose graph has no fill (a 1D chain);
* ILU(0) reproduces A on its sparsity pattern (LU)_ij = A_ij;
* GMRES and BiCGStab converge to numpy.linalg.solve on the assembled system.
"""
import ctypes
import math

import numpy as np
import pytest

from rhodst_b200 import cases, mesh as meshmod
from tests.oracle_lib import OracleSolver, load_oracle

G = 1.4
SCHEMES = {"Kurganov": 0, "HLL": 1, "HLLC": 2, "HLLCP": 3, "AUSM+": 4, "AUSM+up": 5, "AUSM": 6}
D = ctypes.POINTER(ctypes.c_double)


def side(rho, U, p, scheme):
    """(rho, rhoU, rPsi, e, s) as the reconstruction hands it to a scheme."""
    U = np.asarray(U, dtype=float)
    rPsi = p / rho
    e = rPsi / (G - 1.0)                 # h - p/rho with h = gamma e
    if scheme in ("Kurganov", "AUSM"):
        s = math.sqrt(G * rPsi)
    else:
        H = e + 0.5 * U @ U + p / rho
        s = math.sqrt(2 * (G - 1) / (G + 1) * H)
    return np.array([rho, *(rho * U), rPsi, e, s])


def face_flux(lib, scheme, so, sn, S, f=1.0):
    out = np.empty(8)
    so = np.ascontiguousarray(so, dtype=float)
    sn = np.ascontiguousarray(sn, dtype=float)
    S = np.ascontiguousarray(S, dtype=float)
    lib.rdsto_face_flux(SCHEMES[scheme], so.ctypes.data_as(D), sn.ctypes.data_as(D), S.ctypes.data_as(D),
                        G, f, 0, 0.5, out.ctypes.data_as(D))
    return out[:5]


def euler_flux(rho, U, p, S):
    U = np.asarray(U, dtype=float)
    S = np.asarray(S, dtype=float)
    un = U @ S
    E = p / (rho * (G - 1)) + 0.5 * U @ U
    return np.array([rho * un, *(rho * U * un + p * S), (rho * E + p) * un])


STATES = [(1.0, (0.3, 0.1, 0.0), 1.0 / 1.4), (1.4, (3.0, 0.0, 0.0), 1.0), (0.5, (-0.2, 0.4, 0.1), 0.3),
          (2.0, (0.0, 0.0, 0.0), 2.0)]
NORMALS = [(1.0, 0.0, 0.0), (0.3, -0.7, 0.2), (0.0, 0.05, 0.0)]


@pytest.mark.parametrize("scheme", list(SCHEMES))
@pytest.mark.parametrize("state", STATES)
@pytest.mark.parametrize("S", NORMALS)
def test_flux_consistency(oracle, scheme, state, S):
    rho, U, p = state
    s = side(rho, U, p, scheme)
    F = face_flux(oracle, scheme, s, s, S)
    Fe = euler_flux(rho, U, p, S)
    scale = np.abs(Fe).max() + p * np.linalg.norm(S)
    if scheme == "AUSM+up":
        # AUSM+up's interface speed a_1/2 = min(a*^2/max(a*, Un), ...) differs
        # between the two sides even for equal states; consistency holds for
        # |Un| < a* (the subsonic branch) only.
        a_star = s[6]
        if abs(np.asarray(U) @ (np.asarray(S) / np.linalg.norm(S))) >= a_star:
            pytest.skip("AUSM+up interface speed is side-dependent in the supersonic branch")
    assert np.abs(F - Fe).max() <= 1e-12 * scale


@pytest.mark.parametrize("scheme", list(SCHEMES))
def test_flux_orientation(oracle, scheme):
    rng = np.random.default_rng(3)
    for _ in range(20):
        a = side(rng.uniform(0.5, 2), rng.uniform(-0.5, 0.5, 3), rng.uniform(0.5, 2), scheme)
        b = side(rng.uniform(0.5, 2), rng.uniform(-0.5, 0.5, 3), rng.uniform(0.5, 2), scheme)
        S = rng.normal(size=3)
        F1 = face_flux(oracle, scheme, a, b, S)
        F2 = face_flux(oracle, scheme, b, a, -S)
        assert np.abs(F1 + F2).max() <= 1e-12 * (np.abs(F1).max() + 1)


@pytest.mark.parametrize("scheme", [s for s in SCHEMES if s != "Kurganov"])
def test_supersonic_upwinding(oracle, scheme):
    # both states supersonic along +n: the upwind (owner) flux is returned
    L = (1.0, (3.0, 0.2, 0.0), 1.0 / 1.4)
    R = (1.3, (2.8, -0.1, 0.0), 1.2 / 1.4)
    S = np.array([0.1, 0.0, 0.0])
    F = face_flux(oracle, scheme, side(*L, scheme), side(*R, scheme), S)
    FL = euler_flux(*L, S)
    assert np.abs(F - FL).max() <= 1e-12 * np.abs(FL).max()


def test_kurganov_supersonic_upwinding(oracle):
    # KNP: a- = 0 when both sides are supersonic along +n -> owner flux
    L = (1.0, (3.0, 0.2, 0.0), 1.0 / 1.4)
    R = (1.3, (2.8, -0.1, 0.0), 1.2 / 1.4)
    S = np.array([0.1, 0.0, 0.0])
    F = face_flux(oracle, "Kurganov", side(*L, "Kurganov"), side(*R, "Kurganov"), S)
    assert np.abs(F - euler_flux(*L, S)).max() <= 1e-12 * np.abs(euler_flux(*L, S)).max()


def roe_jacobian(lib, W, n):
    out = np.empty(25)
    W = np.ascontiguousarray(W, dtype=float)
    n = np.ascontiguousarray(n, dtype=float)
    lib.rdsto_flux_jacobian(W.ctypes.data_as(D), n.ctypes.data_as(D), G, out.ctypes.data_as(D))
    return out.reshape(5, 5)


def flux_of_W(W, n):
    rho = W[0]
    U = W[1:4] / rho
    p = (G - 1) * (W[4] - 0.5 * rho * U @ U)
    return euler_flux(rho, U, p, n)


@pytest.mark.parametrize("state", STATES[:3])
def test_roe_block_is_euler_jacobian(oracle, state):
    rho, U, p = state
    U = np.asarray(U)
    W = np.array([rho, *(rho * U), p / (G - 1) + 0.5 * rho * U @ U])
    n = np.array([0.6, -0.64, 0.48])
    A = roe_jacobian(oracle, W, n)
    # homogeneity of degree one: F(W) = A(W) W
    assert np.allclose(A @ W, flux_of_W(W, n), rtol=0, atol=1e-13 * np.abs(flux_of_W(W, n)).max())
    # central differences
    J = np.empty((5, 5))
    for k in range(5):
        h = 1e-6 * max(abs(W[k]), 1.0)
        e = np.zeros(5)
        e[k] = h
        J[:, k] = (flux_of_W(W + e, n) - flux_of_W(W - e, n)) / (2 * h)
    assert np.abs(A - J).max() < 1e-7 * np.abs(J).max()


def test_limiters(oracle):
    # OSPRE (Waterson-Deconinck): psi(1) = 1, psi(r<=0) = 0, psi -> 1.5
    assert abs(oracle.rdsto_limiter(2, 1.0) - 1.0) < 1e-15
    assert oracle.rdsto_limiter(2, -0.5) == 0.0
    assert abs(oracle.rdsto_limiter(2, 1e6) - 1.5) < 1e-5
    assert abs(oracle.rdsto_limiter(3, 1.0) - 1.0) < 1e-15       # vanLeer
    assert oracle.rdsto_limiter(3, -2.0) == 0.0
    assert oracle.rdsto_limiter(4, 3.0) == 1.0                   # Minmod


def channel_case(flux, nx=16, ny=6, lim=("OSPRE", "OSPREV"), M=2.0):
    """Uniform flow through a straight channel: inlet fixedValue, outlet
    zeroGradient, symmetry walls, empty front/back."""
    X = np.linspace(0, 2.0, nx + 1)
    Y = np.linspace(0, 1.0, ny + 1)
    Z = np.array([-0.05, 0.05])
    pts = np.stack(np.meshgrid(X, Y, Z, indexing="ij"), -1).reshape(-1, 3)
    # mildly skewed interior (so gradients are non-trivial geometry)
    idx = np.arange(pts.shape[0]).reshape(nx + 1, ny + 1, 2)
    pts = pts.copy()
    inner = np.zeros((nx + 1, ny + 1, 2), bool)
    inner[1:-1, 1:-1, :] = True
    rng = np.random.default_rng(11)
    shift = rng.uniform(-0.2, 0.2, size=(nx + 1, ny + 1, 1, 2)) * np.array([2.0 / nx, 1.0 / ny])
    shift = np.repeat(shift, 2, axis=2)
    pts[:, :2] += (shift * inner[..., None]).reshape(-1, 2)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    cells = meshmod._hex_from_lattice(idx, ii.ravel(), jj.ravel(), np.zeros(nx * ny, dtype=int))

    def classify(c, n):
        out = np.full(c.shape[0], 2)
        out[np.abs(n[:, 2]) > 0.5] = 3
        out[(out == 2) & (np.abs(c[:, 0]) < 1e-9)] = 0
        out[(out == 2) & (np.abs(c[:, 0] - 2.0) < 1e-9)] = 1
        return out

    m = meshmod.build_polymesh(pts, [("hex", cells)], classify,
                               [("inlet", meshmod.PATCH), ("outlet", meshmod.PATCH), ("walls", meshmod.SYMMETRY),
                                ("frontBack", meshmod.EMPTY)])
    U0 = (M, 0.0, 0.0)
    bcs = {"inlet": {"p": ("fixedValue", 1.0), "U": ("fixedValue", U0), "T": ("fixedValue", 1.0)},
           "outlet": {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient"}}
    base = cases.forward_step_c1()
    opts = dict(base.options)
    opts["fluxScheme"] = flux
    opts["interpolationSchemes"] = {"reconstruct(rho)": lim[0], "reconstruct(U)": lim[1], "reconstruct(T)": lim[0]}
    N = m.n_cells
    return cases.Case("channel", m, bcs, opts, np.ones(N), np.tile(U0, (N, 1)), np.ones(N))


@pytest.mark.parametrize("scheme", list(SCHEMES))
@pytest.mark.parametrize("lim", [("OSPRE", "OSPREV"), ("linear", "linear"), ("Venkatakrishnan", "Venkatakrishnan")])
def test_freestream_preservation(scheme, lim):
    c = channel_case(scheme, lim=lim, M=0.5 if scheme == "AUSM+up" else 2.0)
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    R = o.residual()
    assert np.abs(R).max() < 1e-10


def dense_system(o, m):
    d, u, l, s = o.assemble()
    N = m.n_cells
    A = np.zeros((5 * N, 5 * N))
    for i in range(N):
        A[5 * i:5 * i + 5, 5 * i:5 * i + 5] = d[i]
    for f in range(m.n_internal_faces):
        a, b = m.owner[f], m.neighbour[f]
        A[5 * a:5 * a + 5, 5 * b:5 * b + 5] = u[f]
        A[5 * b:5 * b + 5, 5 * a:5 * a + 5] = l[f]
    return A, s.ravel()


def test_ilu_exact_on_chain():
    c = channel_case("HLLC", nx=24, ny=1)
    c = c.with_options(**{"solvers.W.preconditioner": "ILUC0"})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    rng = np.random.default_rng(5)
    W = np.ones((c.mesh.n_cells, 1))
    o.set_primitive(c.p * (1 + 0.1 * rng.random(c.mesh.n_cells)), c.U, c.T)
    A, s = dense_system(o, c.mesh)
    b = rng.normal(size=5 * c.mesh.n_cells)
    x = o.precondition(b).ravel()
    assert np.allclose(A @ x, b, rtol=0, atol=1e-10 * np.abs(b).max())


def test_ilu_pattern_property():
    c = channel_case("Kurganov", nx=6, ny=4).with_options(**{"solvers.W.preconditioner": "ILUC0"})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    rng = np.random.default_rng(6)
    o.set_primitive(c.p * (1 + 0.1 * rng.random(c.mesh.n_cells)), c.U, c.T)
    A, _ = dense_system(o, c.mesh)
    n = A.shape[0]
    Minv = np.stack([o.precondition(np.eye(n)[:, k]).ravel() for k in range(n)], axis=1)
    M = np.linalg.inv(Minv)
    pattern = np.abs(A) > 0
    blockpat = np.zeros_like(pattern)
    N = c.mesh.n_cells
    for i in range(N):
        blockpat[5 * i:5 * i + 5, 5 * i:5 * i + 5] = True
    for f in range(c.mesh.n_internal_faces):
        a, b = c.mesh.owner[f], c.mesh.neighbour[f]
        blockpat[5 * a:5 * a + 5, 5 * b:5 * b + 5] = True
        blockpat[5 * b:5 * b + 5, 5 * a:5 * a + 5] = True
    err = np.abs((M - A)[blockpat]).max() / np.abs(A).max()
    assert err < 1e-10
    # and it is not the exact inverse (there is fill outside the pattern)
    assert np.abs((M - A)[~blockpat]).max() > 1e-8 * np.abs(A).max()


@pytest.mark.parametrize("solver,precon", [("GMRES", "ILUC0"), ("GMRES", "diagonal"), ("BiCGStab", "ILUC0"),
                                           ("BiCGStab", "diagonal"), ("GMRES", "none")])
def test_krylov_vs_dense(solver, precon):
    c = channel_case("HLL", nx=10, ny=5).with_options(**{
        "solvers.W.solver": solver, "solvers.W.preconditioner": precon, "solvers.W.nDirections": 10,
        "solvers.W.tolerance": 1e-14, "solvers.W.relTol": 0.0, "solvers.W.maxIter": 400,
        "solvers.W.minIter": 1, "ddtSchemes.default": "Euler", "timeControls.initialCo": 5.0,
        "timeControls.minCo": 5.0, "timeControls.maxCo": 5.0})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    rng = np.random.default_rng(8)
    o.set_primitive(c.p * (1 + 0.2 * rng.random(c.mesh.n_cells)), c.U, c.T)
    A, s = dense_system(o, c.mesh)
    x_ref = np.linalg.solve(A, s)
    x, rep = o.linear_solve()
    assert np.abs(x.ravel() - x_ref).max() <= 1e-9 * np.abs(x_ref).max(), rep


def test_viscous_linear_field_interior():
    """A linear velocity field on a uniform (unjittered) mesh: the Gauss
    gradient is exact and the stresses are constant, so the viscous momentum
    terms (laplacian(muEff, U) + div(tauMC)) vanish in interior cells."""
    nx, ny = 12, 8
    X = np.linspace(0, 2.0, nx + 1)
    Y = np.linspace(0, 1.0, ny + 1)
    Z = np.array([-0.05, 0.05])
    pts = np.stack(np.meshgrid(X, Y, Z, indexing="ij"), -1).reshape(-1, 3)
    idx = np.arange(pts.shape[0]).reshape(nx + 1, ny + 1, 2)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    cells = meshmod._hex_from_lattice(idx, ii.ravel(), jj.ravel(), np.zeros(nx * ny, dtype=int))

    def classify(c, n):
        out = np.full(c.shape[0], 0)
        out[np.abs(n[:, 2]) > 0.5] = 1
        return out

    m = meshmod.build_polymesh(pts, [("hex", cells)], classify, [("walls", meshmod.PATCH), ("fb", meshmod.EMPTY)])
    base = channel_case("Kurganov", nx=4, ny=2)
    opts = dict(base.options)
    opts["interpolationSchemes"] = {"reconstruct(rho)": "linear", "reconstruct(U)": "linear", "reconstruct(T)": "linear"}
    N = m.n_cells
    U = np.zeros((N, 3))
    U[:, 0] = 0.3 + 0.2 * m.C[:, 1] + 0.1 * m.C[:, 0]
    U[:, 1] = 0.05 * m.C[:, 0] - 0.1 * m.C[:, 1]
    bcs = {"walls": {"p": "zeroGradient", "U": "zeroGradient", "T": "zeroGradient"}}
    R = {}
    for mu in (0.0, 0.01):
        o2 = dict(opts)
        o2["transport"] = {"mu": mu, "Pr": 0.72}
        o = OracleSolver(m, bcs, o2)
        o.set_primitive(np.ones(N), U, np.ones(N))
        R[mu] = o.residual()
    # cells whose neighbours' gradients are all exact (two layers in from the
    # zero-gradient boundary)
    interior = (m.C[:, 0] > 2.0 / nx * 2.5) & (m.C[:, 0] < 2.0 - 2.0 / nx * 2.5) & \
               (m.C[:, 1] > 1.0 / ny * 2.5) & (m.C[:, 1] < 1.0 - 1.0 / ny * 2.5)
    assert interior.sum() >= 15
    dR = R[0.01][interior, 1:4] - R[0.0][interior, 1:4]
    assert np.abs(dR).max() < 1e-11


def test_cell_centre_local_time_step_keeps_the_initial_courant():
    """setSteadyStateDeltaT with neighbouring false divides by the scalar
    courant (timeDST.C:221-227), which a steady run never changes: maxCo has
    no effect there, while the face-based definition ramps per cell."""
    from rhodst_b200 import cases
    from tests.oracle_lib import OracleSolver

    def run(nb, max_co):
        c = cases.naca0012_inviscid(ni=97, nj=25, flux="HLL", limiter="upwind", first_cell=5e-3)
        c = c.with_options(**{"timeControls.neighbouring": nb, "timeControls.maxCo": max_co})
        o = OracleSolver(c.mesh, c.bcs, c.options)
        o.set_primitive(c.p, c.U, c.T)
        reps = o.step(12)
        return [r["rdt_max"] for r in reps], o.conservative()[0]

    a, Wa = run(False, 50.0)
    b, Wb = run(False, 500.0)
    assert a == b and np.array_equal(Wa, Wb)
    c, _ = run(True, 50.0)
    d, _ = run(True, 500.0)
    assert c != d


def test_transient_initial_time_step_comes_from_initial_courant():
    """timeDST::initialize calls setTransientDeltaT for every unsteady run
    (timeDST.C:196-205): with adjustTimeStep false the physical time step is
    the initialCo one, not controlDict's deltaT, and it stays."""
    from rhodst_b200 import cases
    from tests.oracle_lib import OracleSolver
    c = cases.forward_step_c1().with_options(**{"timeControls.adjustTimeStep": False, "controlDict.deltaT": 0.5})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    dts = [r["deltaT"] for r in o.step(3)]
    assert dts[0] < 0.5 and dts[0] == dts[1] == dts[2]
    c2 = c.with_options(**{"timeControls.initialCo": 2 * c.options["timeControls"]["initialCo"]})
    o2 = OracleSolver(c2.mesh, c2.bcs, c2.options)
    o2.set_primitive(c2.p, c2.U, c2.T)
    assert o2.step(1)[0]["deltaT"] == pytest.approx(2 * dts[0], rel=1e-12)
