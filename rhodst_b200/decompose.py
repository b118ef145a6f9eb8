"""Domain decomposition of a cell mesh into overlapping subdomains, one per
rank (the role of foam-extend's decomposePar and processor patches in the
reference's only parallel mode).

Each rank's subdomain is its owned cells (graph or coordinate bisection of
the cell graph) plus `layers` layers of halo cells around them.  Two layers
make the residual of every owned cell exact: its faces need the
reconstructed states of its face neighbours, whose limited gradients need
their own neighbours.  The subdomain is an ordinary mesh in the library's
sense: its cells in ascending global order (so foam's face ordering, owner
< neighbour sorted by owner, carries over), the original boundary faces of
its cells in their patches, and the faces cut by the halo's edge in one
extra patch `halo` (zero-gradient conditions; only outer halo cells see
it, and their residuals are not used).  `send`/`recv` list, per peer rank,
the local cells whose state goes to / comes from that peer, in the same
(ascending global) order on both sides.
"""
import dataclasses
from typing import Dict, List

import numpy as np

from . import mesh as _mesh

HALO_PATCH = "halo"


@dataclasses.dataclass
class Subdomain:
    rank: int
    cells: np.ndarray                  # global ids of the subdomain's cells, ascending
    owned: np.ndarray                  # bool over `cells`: owned by this rank (not halo)
    mesh: "_mesh.PolyMesh"             # the subdomain mesh (local id = position in `cells`)
    send: Dict[int, np.ndarray]        # peer -> local ids of owned cells the peer holds as halo
    recv: Dict[int, np.ndarray]        # peer -> local ids of halo cells the peer owns


def _adjacency(m):
    Fi = m.n_internal_faces
    own = np.asarray(m.owner[:Fi], dtype=np.int64)
    nei = np.asarray(m.neighbour, dtype=np.int64)
    a = np.concatenate([own, nei])
    b = np.concatenate([nei, own])
    order = np.argsort(a, kind="stable")
    start = np.zeros(m.n_cells + 1, dtype=np.int64)
    np.add.at(start, a + 1, 1)
    return np.cumsum(start), b[order]


def partition(m, n_parts: int, method: str = "graph") -> np.ndarray:
    from . import partition_cells, partition_graph
    if n_parts == 1:
        return np.zeros(m.n_cells, dtype=np.int32)
    if method == "graph":
        return partition_graph(m, n_parts)
    if method == "rcb":
        return partition_cells(m.C, n_parts)
    raise ValueError("method must be graph or rcb")


def _submesh(m, cells: np.ndarray) -> "_mesh.PolyMesh":
    N, Fi, F = m.n_cells, m.n_internal_faces, m.n_faces
    local = np.full(N, -1, dtype=np.int64)
    local[cells] = np.arange(cells.size)
    own = np.asarray(m.owner, dtype=np.int64)
    nei = np.asarray(m.neighbour, dtype=np.int64)
    lo, ln = local[own[:Fi]], local[nei]
    keep = (lo >= 0) & (ln >= 0)
    cut = (lo >= 0) ^ (ln >= 0)
    fi = np.nonzero(keep)[0]
    fc = np.nonzero(cut)[0]
    flip = ln[fc] >= 0                                     # the inside cell is the original neighbour
    Sf, Cf, magSf = np.asarray(m.Sf), np.asarray(m.Cf), np.asarray(m.magSf)
    C = np.asarray(m.C)[cells]
    parts_faces, parts_owner, patches = [fi], [lo[fi]], []
    start = fi.size
    for P in m.patches:
        f = np.arange(P.start, P.start + P.size)
        f = f[local[own[f]] >= 0]
        parts_faces.append(f)
        parts_owner.append(local[own[f]])
        patches.append(_mesh.Patch(P.name, P.type, start, f.size))
        start += f.size
    co = np.where(flip, ln[fc], lo[fc])
    patches.append(_mesh.Patch(HALO_PATCH, _mesh.PATCH, start, fc.size))
    faces_g = np.concatenate(parts_faces + [fc])
    owner = np.concatenate(parts_owner + [co]).astype(np.int32)
    sgn = np.ones(faces_g.size)
    sgn[faces_g.size - fc.size:][flip] = -1.0
    faces = np.asarray(m.faces)[faces_g].copy()
    # a flipped face lists its vertices the other way round (v0 v3 v2 v1, or
    # v0 v2 v1 for a triangle, whose -1 pad stays last)
    fv = faces[faces_g.size - fc.size:]
    f_flip = fv[flip]
    tri = f_flip[:, 3] < 0
    f_new = np.where(tri[:, None], f_flip[:, [0, 2, 1, 3]], f_flip[:, [0, 3, 2, 1]])
    fv[flip] = f_new
    faces[faces_g.size - fc.size:] = fv
    sub = _mesh.PolyMesh(points=m.points, faces=faces, owner=owner, neighbour=ln[fi].astype(np.int32),
                         patches=patches, n_cells=int(cells.size))
    sub.Sf = Sf[faces_g] * sgn[:, None]
    sub.Cf = Cf[faces_g].copy()
    sub.magSf = magSf[faces_g].copy()
    sub.C = C
    sub.V = np.asarray(m.V)[cells].copy()
    w = np.ones(faces_g.size)
    w[:fi.size] = np.asarray(m.weights)[fi]
    dc = np.asarray(m.deltaCoeffs)[faces_g].copy()
    # cut faces become boundary faces of the inside cell: foam's boundary
    # weight 1 and delta coefficient from the inside centre to the face
    b0 = faces_g.size - fc.size
    d = sub.Cf[b0:] - C[owner[b0:]]
    nrm = sub.Sf[b0:] / sub.magSf[b0:, None]
    dc[b0:] = 1.0 / np.maximum(np.einsum("ij,ij->i", nrm, d), 0.05 * np.linalg.norm(d, axis=1))
    sub.weights, sub.deltaCoeffs = w, dc
    if m.wall_distance is not None:
        sub.wall_distance = np.asarray(m.wall_distance)[cells].copy()
    return sub


def decompose(m, n_parts: int, layers: int = 2, method: str = "graph", part=None) -> List[Subdomain]:
    """Overlapping subdomains of mesh `m`, one per part."""
    if layers < 2:
        raise ValueError("two halo layers are needed for exact residuals of the owned cells")
    part = partition(m, n_parts, method) if part is None else np.asarray(part, dtype=np.int32)
    start, adj = _adjacency(m)
    subs = []
    for p in range(n_parts):
        ext = part == p
        for _ in range(layers):
            idx = np.nonzero(ext)[0]
            nb = np.concatenate([adj[start[i]:start[i + 1]] for i in idx]) if idx.size else np.zeros(0, int)
            ext = ext.copy()
            ext[nb] = True
        cells = np.nonzero(ext)[0]
        subs.append(Subdomain(p, cells, part[cells] == p, _submesh(m, cells), {}, {}))
    for s in subs:
        halo = s.cells[~s.owned]
        owners = part[halo]
        for q in np.unique(owners):
            g = halo[owners == q]                           # ascending global ids
            s.recv[int(q)] = np.searchsorted(s.cells, g)
            subs[int(q)].send[s.rank] = np.searchsorted(subs[int(q)].cells, g)
    return subs
