"""foam polyMesh input: the mesh of an existing rhoDST case.

`read_polymesh(dir)` reads an ASCII `constant/polyMesh` (points, faces,
owner, neighbour, boundary) into a PolyMesh with the library's geometry
(face centres and area vectors, cell centres and volumes, weights, delta
coefficients), keeping foam's face numbering: internal faces in upper
triangular order, then the patches by startFace.  Faces of three or four
vertices (the hex, prism and tet meshes this path runs); patch types
patch, wall, symmetryPlane/symmetry and empty.

`save_npz` / `load_npz` store the topology compactly (a mesh read once can
travel without the case directory).
"""
from __future__ import annotations

import re
from pathlib import Path
from typing import List, Tuple

import numpy as np

from . import mesh as _mesh

_PATCH_TYPES = {"patch": _mesh.PATCH, "wall": _mesh.WALL, "symmetryPlane": _mesh.SYMMETRY,
                "symmetry": _mesh.SYMMETRY, "empty": _mesh.EMPTY}


def _strip(text: str) -> str:
    """Text after the FoamFile header with comments removed."""
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    m = re.search(r"FoamFile\s*\{.*?\}", text, flags=re.S)
    if m:
        text = text[m.end():]
    return text


def _header(text: str) -> dict:
    m = re.search(r"FoamFile\s*\{(.*?)\}", text, flags=re.S)
    out = {}
    if m:
        for k, v in re.findall(r"(\w+)\s+([^;]+);", m.group(1)):
            out[k] = v.strip().strip('"')
    return out


def _list_body(text: str) -> Tuple[int, str]:
    """The count and the parenthesised body of the file's top-level list."""
    m = re.search(r"(\d+)\s*\(", text)
    if not m:
        raise ValueError("no list in file")
    n = int(m.group(1))
    start = m.end()
    end = text.rindex(")")
    return n, text[start:end]


def _read(path: Path) -> Tuple[dict, str]:
    raw = path.read_text()
    hdr = _header(raw)
    if hdr.get("format", "ascii") != "ascii":
        raise ValueError(f"{path}: only ascii polyMesh files are read")
    return hdr, _strip(raw)


def read_points(path: Path) -> np.ndarray:
    _, t = _read(path)
    n, body = _list_body(t)
    vals = np.array(re.findall(r"[-+0-9.eE]+", body), dtype=float)
    if vals.size != 3 * n:
        raise ValueError(f"{path}: {vals.size} numbers for {n} points")
    return vals.reshape(n, 3)


def read_labels(path: Path) -> np.ndarray:
    _, t = _read(path)
    n, body = _list_body(t)
    vals = np.array(body.split(), dtype=np.int64)
    if vals.size != n:
        raise ValueError(f"{path}: {vals.size} labels for {n}")
    return vals


def read_faces(path: Path) -> np.ndarray:
    """faceList 'k(v0 .. vk-1)' per face -> (F, 4), -1 padded for triangles."""
    _, t = _read(path)
    n, body = _list_body(t)
    items = re.findall(r"(\d+)\s*\(([^)]*)\)", body)
    if len(items) != n:
        raise ValueError(f"{path}: {len(items)} faces for {n}")
    out = np.full((n, 4), -1, dtype=np.int64)
    for i, (k, verts) in enumerate(items):
        v = verts.split()
        if int(k) != len(v) or len(v) not in (3, 4):
            raise ValueError(f"{path}: face {i} has {len(v)} vertices (3 or 4 are read)")
        out[i, :len(v)] = [int(x) for x in v]
    return out


def read_boundary(path: Path) -> List[Tuple[str, str, int, int]]:
    """(name, type, startFace, nFaces) per patch, in file order."""
    _, t = _read(path)
    n, body = _list_body(t)
    out = []
    for name, block in re.findall(r"(\w+)\s*\{(.*?)\}", body, flags=re.S):
        fields = dict(re.findall(r"(\w+)\s+([^;]+);", block))
        out.append((name, fields["type"].strip(), int(fields["startFace"]), int(fields["nFaces"])))
    if len(out) != n:
        raise ValueError(f"{path}: {len(out)} patches for {n}")
    return out


def read_polymesh(directory) -> _mesh.PolyMesh:
    d = Path(directory)
    points = read_points(d / "points")
    faces = read_faces(d / "faces")
    owner = read_labels(d / "owner")
    neighbour = read_labels(d / "neighbour")
    bnd = read_boundary(d / "boundary")
    return assemble(points, faces, owner, neighbour, bnd)


def assemble(points, faces, owner, neighbour, bnd) -> _mesh.PolyMesh:
    """PolyMesh from foam's arrays (checked for foam's ordering rules)."""
    F, Fi = faces.shape[0], neighbour.shape[0]
    if owner.shape[0] != F:
        raise ValueError("owner list does not cover the faces")
    if np.any(owner[:Fi] >= neighbour):
        raise ValueError("internal faces must have owner < neighbour")
    patches = []
    pos = Fi
    for name, ptype, start, size in bnd:
        if start != pos:
            raise ValueError(f"patch {name} does not follow the previous faces")
        if ptype not in _PATCH_TYPES:
            raise ValueError(f"patch {name}: type {ptype} is not read")
        patches.append(_mesh.Patch(name, _PATCH_TYPES[ptype], start, size))
        pos += size
    if pos != F:
        raise ValueError("patches do not end at the last face")
    m = _mesh.PolyMesh(points=np.ascontiguousarray(points, dtype=np.float64), faces=faces.astype(np.int64),
                       owner=owner.astype(np.int32), neighbour=neighbour.astype(np.int32), patches=patches,
                       n_cells=int(owner.max()) + 1)
    _mesh.compute_geometry(m)
    return m


def save_npz(m: _mesh.PolyMesh, path) -> None:
    np.savez_compressed(path, points=m.points, faces=m.faces.astype(np.int32), owner=m.owner,
                        neighbour=m.neighbour,
                        patch_names=np.array([p.name for p in m.patches]),
                        patch_types=np.array([p.type for p in m.patches], dtype=np.int32),
                        patch_start=np.array([p.start for p in m.patches], dtype=np.int64),
                        patch_size=np.array([p.size for p in m.patches], dtype=np.int64))


def load_npz(path) -> _mesh.PolyMesh:
    z = np.load(path)
    names = {v: k for k, v in _PATCH_TYPES.items() if k != "symmetry"}
    bnd = [(str(n), names[int(t)], int(s), int(k)) for n, t, s, k in
           zip(z["patch_names"], z["patch_types"], z["patch_start"], z["patch_size"])]
    return assemble(z["points"], z["faces"].astype(np.int64), z["owner"].astype(np.int64),
                    z["neighbour"].astype(np.int64), bnd)
