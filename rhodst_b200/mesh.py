"""Mesh layer: polyMesh-style connectivity, finite-volume geometry and the
generators for the forward-step, airfoil, swept-wing and hybrid-step cases.

foam-extend is not available, so this module supplies the arrays an
``fvMesh`` would hand to the drop-in (owner/neighbour addressing, Sf, Cf,
magSf, C, V, weights, deltaCoeffs and the patch table).  The geometry follows
foam-extend's primitiveMesh/surfaceInterpolation definitions:

* face centre/area: triangle fan about the face's point average
  (``primitiveMeshFaceCentresAndAreas``), triangles closed-form;
* cell centre/volume: pyramid decomposition about the average of the cell's
  face centres (``primitiveMeshCellCentresAndVols``);
* weights  w = |Sf.(C_N - Cf)| / (|Sf.(Cf - C_P)| + |Sf.(C_N - Cf)|), 1 on
  boundary faces;
* deltaCoeffs = 1/max(n.d, 0.05|d|) (the stabilised form quoted in
  libraries/rhoDST/timeDST/timeDST.C:244 of rhoDST).

Face ordering is foam's upper-triangular order: internal faces sorted by
owner then neighbour, boundary faces grouped by patch.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

# patch geometric types (mirror include/rdst.h RDST_PATCH_*)
PATCH = 0
WALL = 1
SYMMETRY = 2
EMPTY = 3

# local outward faces per cell shape (vertex orderings follow foam's cell models)
_HEX_FACES = np.array([[0, 4, 7, 3], [1, 2, 6, 5], [0, 1, 5, 4],
                       [3, 7, 6, 2], [0, 3, 2, 1], [4, 5, 6, 7]], dtype=np.int64)
_PRISM_FACES = [[0, 2, 1, -1], [3, 4, 5, -1], [0, 1, 4, 3], [1, 2, 5, 4], [2, 0, 3, 5]]
_TET_FACES = [[0, 2, 1, -1], [0, 1, 3, -1], [1, 2, 3, -1], [0, 3, 2, -1]]


@dataclasses.dataclass
class Patch:
    name: str
    type: int          # PATCH / WALL / SYMMETRY / EMPTY
    start: int
    size: int


@dataclasses.dataclass
class PolyMesh:
    points: np.ndarray          # (P,3)
    faces: np.ndarray           # (F,4) vertex ids, -1 padded for triangles
    owner: np.ndarray           # (F,)  int32
    neighbour: np.ndarray       # (Fi,) int32
    patches: List[Patch]
    n_cells: int
    # geometry (filled by compute_geometry)
    Sf: np.ndarray = None
    Cf: np.ndarray = None
    magSf: np.ndarray = None
    C: np.ndarray = None
    V: np.ndarray = None
    weights: np.ndarray = None
    deltaCoeffs: np.ndarray = None
    wall_distance: Optional[np.ndarray] = None
    # airfoil meshes: per point, the chordwise position x_s of the surface
    # point its grid line starts from, the side (+1 upper, -1 lower, 0 not
    # on an airfoil grid line) and the weight with which a normal
    # displacement of that surface point carries over to it
    surface_map: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])

    @property
    def n_internal_faces(self) -> int:
        return int(self.neighbour.shape[0])

    def patch(self, name: str) -> Patch:
        for p in self.patches:
            if p.name == name:
                return p
        raise KeyError(name)

    def patch_index(self, name: str) -> int:
        for i, p in enumerate(self.patches):
            if p.name == name:
                return i
        raise KeyError(name)


# --------------------------------------------------------------------------
# connectivity
# --------------------------------------------------------------------------

def _cell_faces(cells: np.ndarray, table) -> np.ndarray:
    table = np.asarray(table, dtype=np.int64)
    nc = cells.shape[0]
    nf = table.shape[0]
    out = np.full((nc, nf, 4), -1, dtype=np.int64)
    for k in range(nf):
        for m in range(4):
            if table[k, m] >= 0:
                out[:, k, m] = cells[:, table[k, m]]
    return out.reshape(nc * nf, 4)


def build_polymesh(points: np.ndarray,
                   cell_blocks: Sequence[Tuple[str, np.ndarray]],
                   classify: Callable[[np.ndarray, np.ndarray], np.ndarray],
                   patch_defs: Sequence[Tuple[str, int]]) -> PolyMesh:
    """Build foam-ordered polyMesh connectivity from cell vertex lists.

    ``cell_blocks`` is a sequence of (shape, cells) with shape in
    {"hex","prism","tet"}; cells are numbered in the order given.
    ``classify(face_centres, face_normals)`` returns a patch index per
    boundary face (indices into ``patch_defs`` = [(name, type), ...]).
    """
    faces_all = []
    fcell_all = []
    base = 0
    for shape, cells in cell_blocks:
        cells = np.asarray(cells, dtype=np.int64)
        table = {"hex": _HEX_FACES, "prism": _PRISM_FACES, "tet": _TET_FACES}[shape]
        f = _cell_faces(cells, table)
        nf = len(table)
        faces_all.append(f)
        fcell_all.append(np.repeat(np.arange(base, base + cells.shape[0], dtype=np.int64), nf))
        base += cells.shape[0]
    n_cells = base
    faces = np.concatenate(faces_all)
    fcell = np.concatenate(fcell_all)

    key = np.sort(faces, axis=1)
    order = np.lexsort((key[:, 3], key[:, 2], key[:, 1], key[:, 0]))
    ks = key[order]
    same = np.all(ks[1:] == ks[:-1], axis=1)
    first = np.zeros(len(order), dtype=bool)
    second = np.zeros(len(order), dtype=bool)
    first[:-1] = same
    second[1:] = same
    if np.any(first & second):
        raise ValueError("non-manifold mesh: a face is shared by more than two cells")
    ia = order[:-1][same]
    ib = order[1:][same]
    ca, cb = fcell[ia], fcell[ib]
    own_is_a = ca < cb
    own_face = np.where(own_is_a, ia, ib)
    owner_i = np.minimum(ca, cb)
    neigh_i = np.maximum(ca, cb)
    srt = np.lexsort((neigh_i, owner_i))
    int_faces = faces[own_face[srt]]
    owner_i = owner_i[srt]
    neigh_i = neigh_i[srt]

    single = ~(first | second)
    bidx = order[single]
    bfaces = faces[bidx]
    bowner = fcell[bidx]
    bc, bn = _face_centres_normals(points, bfaces)
    pid = np.asarray(classify(bc, bn), dtype=np.int64)
    if np.any(pid < 0) or np.any(pid >= len(patch_defs)):
        raise ValueError("boundary face left unclassified")
    bsrt = np.lexsort((bidx, pid))
    bfaces = bfaces[bsrt]
    bowner = bowner[bsrt]
    pid = pid[bsrt]

    patches = []
    start = int_faces.shape[0]
    for k, (name, ptype) in enumerate(patch_defs):
        sz = int(np.count_nonzero(pid == k))
        patches.append(Patch(name, ptype, start, sz))
        start += sz
    mesh = PolyMesh(points=np.ascontiguousarray(points, dtype=np.float64),
                    faces=np.concatenate([int_faces, bfaces]).astype(np.int64),
                    owner=np.concatenate([owner_i, bowner]).astype(np.int32),
                    neighbour=neigh_i.astype(np.int32),
                    patches=patches, n_cells=n_cells)
    compute_geometry(mesh)
    return mesh


def _face_centres_normals(points, faces):
    Cf, Sf = face_centres_areas(points, faces)
    return Cf, Sf / np.linalg.norm(Sf, axis=1)[:, None]


# --------------------------------------------------------------------------
# geometry (foam-extend primitiveMesh / surfaceInterpolation definitions)
# --------------------------------------------------------------------------

def face_centres_areas(points: np.ndarray, faces: np.ndarray):
    tri = faces[:, 3] < 0
    P = points
    Cf = np.empty((faces.shape[0], 3))
    Sf = np.empty((faces.shape[0], 3))
    if np.any(tri):
        f = faces[tri]
        p0, p1, p2 = P[f[:, 0]], P[f[:, 1]], P[f[:, 2]]
        Cf[tri] = (p0 + p1 + p2) / 3.0
        Sf[tri] = 0.5 * np.cross(p1 - p0, p2 - p0)
    q = ~tri
    if np.any(q):
        f = faces[q]
        pts = [P[f[:, m]] for m in range(4)]
        fc = (pts[0] + pts[1] + pts[2] + pts[3]) / 4.0
        sumN = np.zeros_like(fc)
        sumA = np.zeros(fc.shape[0])
        sumAc = np.zeros_like(fc)
        for m in range(4):
            a, b = pts[m], pts[(m + 1) % 4]
            c = a + b + fc
            n = np.cross(b - a, fc - a)
            ar = np.linalg.norm(n, axis=1)
            sumN += n
            sumA += ar
            sumAc += ar[:, None] * c
        Cf[q] = (1.0 / 3.0) * sumAc / sumA[:, None]
        Sf[q] = 0.5 * sumN
    return Cf, Sf


def compute_geometry(mesh: PolyMesh) -> None:
    Cf, Sf = face_centres_areas(mesh.points, mesh.faces)
    own = mesh.owner.astype(np.int64)
    nei = mesh.neighbour.astype(np.int64)
    Fi = nei.shape[0]
    N = mesh.n_cells
    # estimated cell centre = average of the cell's face centres
    cEst = np.zeros((N, 3))
    nf = np.zeros(N)
    np.add.at(cEst, own, Cf)
    np.add.at(nf, own, 1.0)
    np.add.at(cEst, nei, Cf[:Fi])
    np.add.at(nf, nei, 1.0)
    cEst /= nf[:, None]
    VSMALL = 1e-300
    pv_o = np.maximum(np.einsum("ij,ij->i", Sf, Cf - cEst[own]), VSMALL)
    pc_o = 0.75 * Cf + 0.25 * cEst[own]
    pv_n = np.maximum(np.einsum("ij,ij->i", Sf[:Fi], cEst[nei] - Cf[:Fi]), VSMALL)
    pc_n = 0.75 * Cf[:Fi] + 0.25 * cEst[nei]
    ctr = np.zeros((N, 3))
    vol = np.zeros(N)
    np.add.at(ctr, own, pv_o[:, None] * pc_o)
    np.add.at(vol, own, pv_o)
    np.add.at(ctr, nei, pv_n[:, None] * pc_n)
    np.add.at(vol, nei, pv_n)
    C = ctr / vol[:, None]
    V = vol / 3.0
    magSf = np.linalg.norm(Sf, axis=1)
    w = np.ones(Sf.shape[0])
    SfdOwn = np.abs(np.einsum("ij,ij->i", Sf[:Fi], Cf[:Fi] - C[own[:Fi]]))
    SfdNei = np.abs(np.einsum("ij,ij->i", Sf[:Fi], C[nei] - Cf[:Fi]))
    w[:Fi] = SfdNei / (SfdOwn + SfdNei)
    d = np.empty_like(Cf)
    d[:Fi] = C[nei] - C[own[:Fi]]
    d[Fi:] = Cf[Fi:] - C[own[Fi:]]
    nrm = Sf / magSf[:, None]
    dc = 1.0 / np.maximum(np.einsum("ij,ij->i", nrm, d), 0.05 * np.linalg.norm(d, axis=1))
    mesh.Sf, mesh.Cf, mesh.magSf = Sf, Cf, magSf
    mesh.C, mesh.V, mesh.weights, mesh.deltaCoeffs = C, V, w, dc


def wall_distance(mesh: PolyMesh, wall_patches: Sequence[str]) -> np.ndarray:
    """Nearest distance from each cell centre to the wall faces (exact
    point-to-face-centre search refined by the face plane), used by SA."""
    from scipy.spatial import cKDTree
    idx = []
    for name in wall_patches:
        p = mesh.patch(name)
        idx.append(np.arange(p.start, p.start + p.size))
    idx = np.concatenate(idx)
    tree = cKDTree(mesh.Cf[idx])
    _, j = tree.query(mesh.C, k=1)
    f = idx[j]
    n = mesh.Sf[f] / mesh.magSf[f][:, None]
    dplane = np.abs(np.einsum("ij,ij->i", mesh.C - mesh.Cf[f], n))
    dcent = np.linalg.norm(mesh.C - mesh.Cf[f], axis=1)
    return np.minimum(dplane, dcent) if False else dplane


# --------------------------------------------------------------------------
# generators
# --------------------------------------------------------------------------

def _hex_from_lattice(idx: np.ndarray, ii: np.ndarray, jj: np.ndarray, kk: np.ndarray) -> np.ndarray:
    """Hex cells (i..i+1, j..j+1, k..k+1) from a lattice point-id array."""
    return np.stack([idx[ii, jj, kk], idx[ii + 1, jj, kk], idx[ii + 1, jj + 1, kk], idx[ii, jj + 1, kk],
                     idx[ii, jj, kk + 1], idx[ii + 1, jj, kk + 1], idx[ii + 1, jj + 1, kk + 1],
                     idx[ii, jj + 1, kk + 1]], axis=1)


def forward_step_2d(refine: int = 1) -> PolyMesh:
    """2D Mach-3 forward-facing step: channel 3.0 x 1.0, step 0.2 high at
    x = 0.6, uniform spacing 1/(40*refine), one cell thick (z in [-0.05,0.05]).

    Block layout and numbering follow tutorials/forwardStep/constant/polyMesh/
    blockMeshDict (three blocks, x fastest within a block) at 1/3 of its
    resolution for refine=1: 24x8 + 24x32 + 96x32 = 4032 cells.
    """
    nx, ny = 120 * refine, 40 * refine
    sx, sy = 24 * refine, 8 * refine
    h = 1.0 / (40 * refine)
    X = np.arange(nx + 1) * h
    Y = np.arange(ny + 1) * h
    Z = np.array([-0.05, 0.05])
    idx = np.arange((nx + 1) * (ny + 1) * 2).reshape(nx + 1, ny + 1, 2)
    pts = np.stack(np.meshgrid(X, Y, Z, indexing="ij"), axis=-1).reshape(-1, 3)
    blocks = [(0, sx, 0, sy), (0, sx, sy, ny), (sx, nx, sy, ny)]
    cells = []
    for (i0, i1, j0, j1) in blocks:
        jj, ii = np.meshgrid(np.arange(j0, j1), np.arange(i0, i1), indexing="ij")
        ii, jj = ii.ravel(), jj.ravel()
        cells.append(_hex_from_lattice(idx, ii, jj, np.zeros_like(ii)))
    cells = np.concatenate(cells)
    used = np.unique(cells)
    remap = -np.ones(pts.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    pts = pts[used]
    cells = remap[cells]
    xs, ys = sx * h, sy * h
    tol = 1e-9

    def classify(c, n):
        out = np.full(c.shape[0], -1)
        out[np.abs(n[:, 2]) > 0.5] = 5
        m = out < 0
        out[m & (np.abs(c[:, 0]) < tol)] = 0
        out[m & (np.abs(c[:, 0] - nx * h) < tol)] = 1
        out[m & (np.abs(c[:, 1]) < tol)] = 2
        out[m & (np.abs(c[:, 1] - ny * h) < tol)] = 3
        ob = m & (out < 0) & (((np.abs(c[:, 0] - xs) < tol) & (c[:, 1] < ys + tol)) |
                              ((np.abs(c[:, 1] - ys) < tol) & (c[:, 0] > xs - tol)))
        out[ob] = 4
        return out

    return build_polymesh(pts, [("hex", cells)], classify,
                          [("inlet", PATCH), ("outlet", PATCH), ("bottom", SYMMETRY),
                           ("top", SYMMETRY), ("obstacle", PATCH), ("defaultFaces", EMPTY)])


def naca00xx(x: np.ndarray, t: float = 0.12, closed_te: bool = True) -> np.ndarray:
    """Half thickness of the NACA 4-digit symmetric section (chord 1); the
    closed trailing-edge variant uses -0.1036 for the x^4 coefficient."""
    a4 = -0.1036 if closed_te else -0.1015
    return 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 + a4 * x ** 4)


def _stretch(n: int, first: float, length: float) -> np.ndarray:
    """n+1 monotone coordinates in [0,length] with a geometric first spacing
    `first` (ratio solved by bisection), used for wall-normal grading."""
    if n * first >= length:
        return np.linspace(0.0, length, n + 1)
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        L = first * (r ** n - 1.0) / (r - 1.0)
        if L > length:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    s = first * (r ** np.arange(n + 1) - 1.0) / (r - 1.0)
    s *= length / s[-1]
    return s


def naca_cmesh(ni: int = 257, nj: int = 65, farfield: float = 20.0, first_cell: float = 4e-6,
               ratio: float = 1.15,
               wake_points: Optional[int] = None, span: float = 0.1) -> PolyMesh:
    """NACA0012 C-mesh with ni x nj hex cells (one thick), far field at
    `farfield` chords, wall-normal geometric spacing starting at
    `first_cell` growing by `ratio` (the rest of the cells stretch faster
    where `ratio` alone would not reach the far field).  The wake cut is
    an internal face set (cells on both sides are connected).

    Patches: airfoil (wall), farfield (patch), frontAndBack (empty).
    """
    if wake_points is None:
        wake_points = max(8, ni // 6)
    nw = wake_points
    nair = ni - 2 * nw            # cells around the airfoil
    if nair < 16:
        raise ValueError("ni too small for the wake/airfoil split")
    # airfoil surface: cosine clustering, TE lower -> LE -> TE upper
    beta = np.linspace(0.0, 2.0 * math.pi, nair + 1)
    xs = 0.5 * (1.0 + np.cos(beta))
    ys = np.where(beta <= math.pi, -1.0, 1.0) * naca00xx(xs)
    # wake line from TE to the far field, clustered at the TE
    ds_te = math.hypot(xs[1] - xs[0], ys[1] - ys[0])
    wx = 1.0 + _stretch(nw, ds_te, farfield - 1.0)
    # inner line (j = 0): lower wake (reversed), airfoil, upper wake
    x0 = np.concatenate([wx[::-1], xs[1:-1], wx])
    y0 = np.zeros_like(x0)
    y0[nw + 1:nw + nair] = ys[1:-1]
    # outer boundary: wake lines map straight across to the C's straight
    # edges, the airfoil maps onto the semicircle by surface arc fraction
    n_i = x0.size               # ni + 1 points
    R = farfield
    xo = np.empty(n_i)
    yo = np.empty(n_i)
    xo[:nw + 1] = x0[:nw + 1]
    yo[:nw + 1] = -R
    xo[nw + nair:] = x0[nw + nair:]
    yo[nw + nair:] = R
    sa = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(xs), np.diff(ys)))])
    th = math.pi * sa / sa[-1]
    xo[nw:nw + nair + 1] = 1.0 - R * np.sin(th)
    yo[nw:nw + nair + 1] = -R * np.cos(th)
    eta = _two_stage(nj, first_cell / R, ratio)
    P = np.empty((n_i, nj + 1, 2))
    for j, e in enumerate(eta):
        P[:, j, 0] = x0 + e * (xo - x0)
        P[:, j, 1] = y0 + e * (yo - y0)
    # lattice -> 3D points; merge the two wake-cut lines (i and ni-i at j=0)
    nip = n_i
    Z = np.array([-0.5 * span, 0.5 * span])
    pts = np.zeros((nip, nj + 1, 2, 3))
    pts[:, :, :, 0] = P[:, :, None, 0]
    pts[:, :, :, 1] = P[:, :, None, 1]
    pts[:, :, :, 2] = Z[None, None, :]
    idx = np.arange(nip * (nj + 1) * 2).reshape(nip, nj + 1, 2)
    # points on the lower wake cut (i <= nw, j = 0) are merged with upper ones
    for i in range(nw + 1):
        idx[i, 0, :] = idx[nip - 1 - i, 0, :]
    jj, ii = np.meshgrid(np.arange(nj), np.arange(nip - 1), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    cells = _hex_from_lattice(idx, ii, jj, np.zeros_like(ii))
    # orient: make volumes positive
    ptsf = pts.reshape(-1, 3)
    used = np.unique(cells)
    remap = -np.ones(ptsf.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    ptsf = ptsf[used]
    cells = remap[cells]
    v = _hex_signed_volume(ptsf, cells)
    flip = v < 0
    if np.any(flip):
        cells[flip] = cells[flip][:, [0, 3, 2, 1, 4, 7, 6, 5]]

    def classify(c, n):
        out = np.full(c.shape[0], 1)
        out[np.abs(n[:, 2]) > 0.5] = 2
        r = np.hypot(c[:, 0] - 0.5, c[:, 1])
        out[(out == 1) & (r < 0.6)] = 0
        return out

    mesh = build_polymesh(ptsf, [("hex", cells)], classify,
                          [("airfoil", WALL), ("farfield", PATCH), ("frontAndBack", EMPTY)])
    # surface map: every point of grid line i moves with the surface point
    # i at weight 1 - eta_j (the interpolation above is linear in y0 and the
    # outer boundary does not depend on the surface's y)
    i_lat = np.broadcast_to(np.arange(nip)[:, None, None], pts.shape[:3]).reshape(-1)[used]
    e_lat = np.broadcast_to(eta[None, :, None], pts.shape[:3]).reshape(-1)[used]
    on_air = (i_lat >= nw + 1) & (i_lat <= nw + nair - 1)
    si = np.clip(i_lat - nw, 0, nair)
    side = np.where(on_air, np.where(beta[si] <= math.pi, -1, 1), 0).astype(np.int8)
    mesh.surface_map = (np.where(on_air, xs[si], 0.0), side, np.where(on_air, 1.0 - e_lat, 0.0))
    return mesh


def moved(mesh: PolyMesh, points: np.ndarray) -> PolyMesh:
    """The mesh with its points replaced (same faces, cells, patches and
    numbering) and its geometry recomputed; the wall distance is recomputed
    from the wall patches when the mesh carries one."""
    out = dataclasses.replace(mesh, points=np.ascontiguousarray(points, dtype=np.float64))
    compute_geometry(out)
    if mesh.wall_distance is not None:
        out.wall_distance = wall_distance(out, [p.name for p in mesh.patches if p.type == WALL])
    return out


def _two_stage(n: int, first: float, ratio: float) -> np.ndarray:
    """n+1 points in [0,1]: geometric growth `ratio` from `first`; if that
    does not reach 1 within n cells, the outer part of the distribution
    switches to the geometric ratio that closes it (continuous spacing)."""
    s = first * (ratio ** np.arange(n + 1) - 1.0) / (ratio - 1.0)
    if s[-1] >= 1.0:
        return s / s[-1]
    m = int(0.6 * n)
    inner = s[:m + 1]
    rest = _stretch(n - m, first * ratio ** m, 1.0 - inner[-1])
    return np.concatenate([inner, inner[-1] + rest[1:]])


def _hex_signed_volume(pts, cells):
    """Signed volume of hexes by the divergence theorem over the six faces
    of the local vertex ordering (robust to collinear corner vertices)."""
    p = pts[cells]
    vol = np.zeros(cells.shape[0])
    for f in _HEX_FACES:
        a, b, c, d = (p[:, f[k]] for k in range(4))
        S = 0.5 * np.cross(c - a, d - b)
        C = 0.25 * (a + b + c + d)
        vol += np.einsum("ij,ij->i", C, S)
    return vol / 3.0


def swept_wing_oh(n_around: int = 192, n_normal: int = 64, n_span: int = 64, n_tip: int = 34,
                  taper: float = 0.56, sweep_deg: float = 30.0, semi_span: float = 1.5,
                  farfield: float = 10.0, first_cell: float = 2e-3) -> PolyMesh:
    """Extruded NACA0012 swept, tapered wing (root chord 1) in an O-H hex mesh.

    Each spanwise station carries an O-grid (n_around x n_normal) around the
    local section, with a circular far field of radius `farfield` about the
    section's mid-chord; n_span cell layers span the wing (z in
    [0, semi_span]) and n_tip layers continue to the far-field side plane.
    Beyond the tip the O-grid's inner ring is collapsed onto the tip chord
    line and its upper/lower points are merged, so that slit is internal;
    the first layer past the tip closes the wing with a tip cap.
    Patches: wing (wall), farfield (patch), symmetry (symmetryPlane, z = 0).
    Cell count = n_around * n_normal * (n_span + n_tip); defaults give
    192 * 64 * 98 = 1,204,224.
    """
    if n_around % 2:
        raise ValueError("n_around must be even")
    sw = math.tan(math.radians(sweep_deg))
    nprof = n_around
    beta = 2.0 * math.pi * np.arange(nprof) / nprof
    xa = 0.5 * (1.0 + np.cos(beta))             # TE(1) -> upper -> LE(0) -> lower -> TE
    ya = np.where(beta <= math.pi, 1.0, -1.0) * naca00xx(xa)
    eta = _stretch(n_normal, first_cell / farfield, 1.0)
    zs_w = semi_span * np.linspace(0.0, 1.0, n_span + 1)
    ztip = _stretch(n_tip, semi_span / n_span, farfield - semi_span)
    zs = np.concatenate([zs_w, semi_span + ztip[1:]])
    nk = zs.size
    pts = np.zeros((nprof, n_normal + 1, nk, 3))
    thf = np.arctan2(ya, xa - 0.5)
    for k, z in enumerate(zs):
        zw = min(z, semi_span)
        chord = 1.0 - (1.0 - taper) * zw / semi_span
        xle = sw * zw
        thick = 1.0 if k <= n_span else 0.0
        sx = xle + chord * xa
        sy = chord * ya * thick
        cx = xle + 0.5 * chord
        ox = cx + farfield * np.cos(thf)
        oy = farfield * np.sin(thf)
        for j, e in enumerate(eta):
            pts[:, j, k, 0] = sx + e * (ox - sx)
            pts[:, j, k, 1] = sy + e * (oy - sy)
            pts[:, j, k, 2] = z
    idx = np.arange(pts.shape[0] * pts.shape[1] * pts.shape[2]).reshape(pts.shape[:3])
    for k in range(n_span + 1, nk):          # collapsed ring: merge upper/lower points
        for i in range(1, nprof // 2):
            idx[nprof - i, 0, k] = idx[i, 0, k]
    ii, jj, kk = np.meshgrid(np.arange(nprof), np.arange(n_normal), np.arange(nk - 1), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    ip = (ii + 1) % nprof
    cells = np.stack([idx[ii, jj, kk], idx[ip, jj, kk], idx[ip, jj + 1, kk], idx[ii, jj + 1, kk],
                      idx[ii, jj, kk + 1], idx[ip, jj, kk + 1], idx[ip, jj + 1, kk + 1],
                      idx[ii, jj + 1, kk + 1]], axis=1)
    o = np.lexsort((ii, jj, kk))             # section by section, ring by ring
    cells = cells[o]
    ptsf = pts.reshape(-1, 3)
    used = np.unique(cells)
    remap = -np.ones(ptsf.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    ptsf = ptsf[used]
    cells = remap[cells]
    v = _hex_signed_volume(ptsf, cells)
    if np.any(v < 0):
        cells[v < 0] = cells[v < 0][:, [0, 3, 2, 1, 4, 7, 6, 5]]
    zmax = zs[-1]

    def classify(c, n):
        out = np.full(c.shape[0], 1)
        out[(np.abs(c[:, 2]) < 1e-9) & (np.abs(n[:, 2]) > 0.9)] = 2
        zc = np.minimum(c[:, 2], semi_span)
        chord = 1.0 - (1.0 - taper) * zc / semi_span
        r = np.hypot(c[:, 0] - (sw * zc + 0.5 * chord), c[:, 1])
        side = np.abs(c[:, 2] - zmax) < 1e-9
        out[(out == 1) & (r < 0.5 * farfield) & ~side] = 0
        return out

    return build_polymesh(ptsf, [("hex", cells)], classify,
                          [("wing", WALL), ("farfield", PATCH), ("symmetry", SYMMETRY)])


def forward_step_3d_hybrid(nx: int = 240, ny: int = 80, nz: int = 40, jitter: float = 0.25,
                           seed: int = 20240601, prism_fraction: float = 0.5) -> PolyMesh:
    """3D Mach-3 forward-facing step on a hybrid tet/prism mesh.

    Channel 3.0 x 1.0 x 0.5, step 0.2 high at x = 0.6.  The structured
    lattice (nx, ny, nz) minus the step is split into prisms (two per hex,
    y-extruded triangles) for y < prism_fraction and tetrahedra (six per
    hex, Kuhn split) above; the prisms' triangles use the tetrahedra's face
    diagonal, so the two layers are conforming.  Interior nodes are jittered by up to
    `jitter` x the local spacing, uniformly, from `seed`.
    Patches: inlet, outlet, obstacle (patch), walls (symmetryPlane: bottom,
    top, sides).
    """
    Lx, Ly, Lz = 3.0, 1.0, 0.5
    hx, hy, hz = Lx / nx, Ly / ny, Lz / nz
    sx = int(round(0.6 / hx))
    sy = int(round(0.2 / hy))
    X = np.arange(nx + 1) * hx
    Y = np.arange(ny + 1) * hy
    Zc = np.arange(nz + 1) * hz
    pts = np.stack(np.meshgrid(X, Y, Zc, indexing="ij"), axis=-1)
    rng = np.random.default_rng(seed)
    interior = np.ones((nx + 1, ny + 1, nz + 1), dtype=bool)
    interior[0, :, :] = interior[-1, :, :] = False
    interior[:, 0, :] = interior[:, -1, :] = False
    interior[:, :, 0] = interior[:, :, -1] = False
    interior[sx:, :sy + 1, :] = False        # step surface and inside
    jit = rng.uniform(-jitter, jitter, size=pts.shape) * np.array([hx, hy, hz]) * interior[..., None]
    idx = np.arange(pts.shape[0] * pts.shape[1] * pts.shape[2]).reshape(pts.shape[:3])
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    keep = ~((ii >= sx) & (jj < sy))
    ii, jj, kk = ii[keep], jj[keep], kk[keep]
    o = np.lexsort((ii, jj, kk))
    ii, jj, kk = ii[o], jj[o], kk[o]
    hexes = _hex_from_lattice(idx, ii, jj, kk)
    pr = (jj * hy) < prism_fraction * Ly
    hp = hexes[pr]
    ht = hexes[~pr]
    # prisms: the x-z quad split along its (i,k)-(i+1,k+1) diagonal and
    # extruded in y, the diagonal the Kuhn tetrahedra below use on their
    # y-faces, so prism and tetrahedron layers share their triangles
    p1 = np.stack([hp[:, 0], hp[:, 1], hp[:, 5], hp[:, 3], hp[:, 2], hp[:, 6]], axis=1)
    p2 = np.stack([hp[:, 0], hp[:, 5], hp[:, 4], hp[:, 3], hp[:, 6], hp[:, 7]], axis=1)
    prisms = np.stack([p1, p2], axis=1).reshape(-1, 6)
    # Kuhn split of a hex into 6 tets along the 0-6 diagonal
    kuhn = [[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]]
    tets = np.stack([ht[:, k] for k in kuhn], axis=1).reshape(-1, 4)
    ptsf = pts.reshape(-1, 3)

    def tet_vol(P, t):
        p = P[t]
        return np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    # orient on the lattice: tets positively, prisms with the first triangle
    # counter-clockwise seen along the extrusion
    neg = tet_vol(ptsf, tets) < 0
    tets[neg] = tets[neg][:, [0, 2, 1, 3]]
    neg = tet_vol(ptsf, prisms[:, :4]) < 0
    prisms[neg] = prisms[neg][:, [0, 2, 1, 3, 5, 4]]
    # jitter, halved at the corners of any cell it would flatten below a
    # fifth of its lattice volume (a Kuhn tetrahedron is a sixth of a cube:
    # a quarter-spacing move of its corners can invert it); prisms checked
    # by their three tetrahedra
    pr_tets = np.concatenate([prisms[:, [0, 1, 2, 3]], prisms[:, [1, 2, 3, 4]], prisms[:, [2, 3, 4, 5]]])
    checks = np.concatenate([tets, pr_tets])
    v0 = np.abs(tet_vol(ptsf, checks))
    jf = jit.reshape(-1, 3).copy()
    for _ in range(40):
        bad = tet_vol(ptsf + jf, checks) < 0.2 * v0
        if not np.any(bad):
            break
        jf[np.unique(checks[bad])] *= 0.5
    ptsf = ptsf + jf
    used = np.unique(np.concatenate([prisms.ravel(), tets.ravel()]))
    remap = -np.ones(ptsf.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    ptsf = ptsf[used]
    prisms = remap[prisms]
    tets = remap[tets]
    tol = 1e-9
    xs, ys = sx * hx, sy * hy

    def classify(c, n):
        out = np.full(c.shape[0], 3)
        out[np.abs(c[:, 0]) < tol] = 0
        out[np.abs(c[:, 0] - Lx) < tol] = 1
        ob = (((np.abs(c[:, 0] - xs) < tol) & (c[:, 1] < ys + tol)) |
              ((np.abs(c[:, 1] - ys) < tol) & (c[:, 0] > xs - tol)))
        out[ob] = 2
        return out

    return build_polymesh(ptsf, [("prism", prisms), ("tet", tets)], classify,
                          [("inlet", PATCH), ("outlet", PATCH), ("obstacle", PATCH), ("walls", SYMMETRY)])
