"""foam case input and output: the mesh and fields of an existing rhoDST case.

`read_polymesh(dir)` reads a `constant/polyMesh` (points, faces, owner,
neighbour, boundary) in foam's ascii or binary format, gzipped (`name.gz`)
or not, faces as a faceList or a binary faceCompactList, into a PolyMesh with the library's geometry
(face centres and area vectors, cell centres and volumes, weights, delta
coefficients), keeping foam's face numbering: internal faces in upper
triangular order, then the patches by startFace.  Faces of three or four
vertices (the hex, prism and tet meshes this path runs); patch types
patch, wall, symmetryPlane/symmetry and empty.

`write_polymesh` writes a mesh back in either format (the meshes the
library generates become foam cases); `save_npz` / `load_npz` store the
topology compactly (a mesh read once can
travel without the case directory).

`read_field` reads a vol field, ascii or binary (uniform or nonuniform
internal field, per-patch entries, '#include' and '$' macros as the
tutorials use them); `write_state` / `read_state` write (in either format)
and read p, U, T and nuTilda as a time directory a foam case restarts
from.

`block_mesh(dict)` builds the meshes tutorials define by blockMeshDict
(hex blocks, simpleGrading, straight edges).

`read_case(dir)` turns a whole rhoDST case directory into a Case: mesh,
fields and boundary conditions, and the options of rhoDSTDict, fvSchemes,
fvSolution, controlDict, thermophysicalProperties and RASProperties under
their own names; `case.notes` lists the entries this path does not take.
"""
from __future__ import annotations

import gzip
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
        for k, v in re.findall(r'(\w+)\s+("[^"]*"|[^;]+);', m.group(1)):   # arch is quoted and holds ';'
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


def _load(path: Path) -> bytes:
    """The file's bytes; `name.gz` (foam's writeCompression) when `name`
    itself is absent, gzip content decompressed either way."""
    path = Path(path)
    if not path.exists() and path.with_name(path.name + ".gz").exists():
        path = path.with_name(path.name + ".gz")
    data = path.read_bytes()
    if data[:2] == b"\x1f\x8b":
        data = gzip.decompress(data)
    return data


class _Binary:
    """Reader of foam's binary list files.  A binary file keeps the text
    FoamFile header; each list is its count in text, then '(' and the raw
    items, then ')' (foam writes no parentheses for an empty list).  The
    header's arch entry gives the byte order and the label and scalar
    widths ("LSB;label=32;scalar=64" when absent)."""

    def __init__(self, path: Path, data: bytes, hdr: dict):
        self.path, self.data = path, data
        arch = hdr.get("arch", "")
        order = ">" if "MSB" in arch else "<"
        lw = re.search(r"label\s*=\s*(\d+)", arch)
        sw = re.search(r"scalar\s*=\s*(\d+)", arch)
        self.label = np.dtype(f"{order}i{int(lw.group(1)) // 8 if lw else 4}")
        self.scalar = np.dtype(f"{order}f{int(sw.group(1)) // 8 if sw else 8}")
        m = re.search(rb"FoamFile\s*\{.*?\}", data, flags=re.S)
        self.pos = m.end() if m else 0

    def _skip(self):
        d, n = self.data, len(self.data)
        while self.pos < n:
            c = d[self.pos:self.pos + 1]
            if c.isspace():
                self.pos += 1
            elif d.startswith(b"//", self.pos):
                e = d.find(b"\n", self.pos)
                self.pos = n if e < 0 else e + 1
            elif d.startswith(b"/*", self.pos):
                e = d.find(b"*/", self.pos + 2)
                if e < 0:
                    raise ValueError(f"{self.path}: unterminated comment")
                self.pos = e + 2
            else:
                return

    def count(self) -> int:
        self._skip()
        m = re.compile(rb"\d+").match(self.data, self.pos)
        if not m:
            raise ValueError(f"{self.path}: expected a list count at byte {self.pos}")
        self.pos = m.end()
        return int(m.group(0))

    def _expect(self, ch: bytes):
        if self.data[self.pos:self.pos + 1] != ch:
            raise ValueError(f"{self.path}: expected {ch!r} at byte {self.pos}")
        self.pos += 1

    def items(self, n: int, dtype: np.dtype, per: int = 1) -> np.ndarray:
        """The raw block of a list whose count n was just read (`per`
        components an item: 3 for a vector)."""
        self._skip()
        if n == 0:
            if self.data.startswith(b"()", self.pos):
                self.pos += 2
            return np.zeros(0, dtype=dtype.newbyteorder("="))
        self._expect(b"(")
        end = self.pos + n * per * dtype.itemsize
        if end + 1 > len(self.data):
            raise ValueError(f"{self.path}: list of {n} items runs past the end of the file")
        out = np.frombuffer(self.data, dtype=dtype, count=n * per, offset=self.pos)
        self.pos = end
        self._expect(b")")
        return out.astype(dtype.newbyteorder("="))

    def list(self, dtype: np.dtype) -> np.ndarray:
        return self.items(self.count(), dtype)


def _open(path: Path):
    """(header, text) of an ascii file or (header, _Binary) of a binary one."""
    data = _load(path)
    m = re.search(rb"FoamFile\s*\{.*?\}", data, flags=re.S)     # the header precedes any binary data
    hdr = _header(m.group(0).decode("latin-1")) if m else {}
    if hdr.get("format", "ascii") == "binary":
        return hdr, _Binary(path, data, hdr)
    if hdr.get("format", "ascii") != "ascii":
        raise ValueError(f"{path}: format {hdr.get('format')} is neither ascii nor binary")
    return hdr, _strip(data.decode("latin-1"))


def read_points(path: Path) -> np.ndarray:
    _, t = _open(path)
    if isinstance(t, _Binary):
        n = t.count()
        return t.items(n, t.scalar, per=3).astype(np.float64).reshape(n, 3)
    n, body = _list_body(t)
    vals = np.array(re.findall(r"[-+0-9.eE]+", body), dtype=float)
    if vals.size != 3 * n:
        raise ValueError(f"{path}: {vals.size} numbers for {n} points")
    return vals.reshape(n, 3)


def read_labels(path: Path) -> np.ndarray:
    _, t = _open(path)
    if isinstance(t, _Binary):
        return t.list(t.label).astype(np.int64)
    n, body = _list_body(t)
    vals = np.array(body.split(), dtype=np.int64)
    if vals.size != n:
        raise ValueError(f"{path}: {vals.size} labels for {n}")
    return vals


def _pad_faces(path, sizes: np.ndarray, flat: np.ndarray) -> np.ndarray:
    """(F, 4) vertex table, -1 padded for triangles, from per-face sizes and
    the faces' vertices back to back."""
    bad = np.flatnonzero((sizes < 3) | (sizes > 4))
    if bad.size:
        raise ValueError(f"{path}: face {bad[0]} has {sizes[bad[0]]} vertices (3 or 4 are read)")
    out = np.full((sizes.size, 4), -1, dtype=np.int64)
    start = np.concatenate(([0], np.cumsum(sizes)[:-1]))
    for k in range(4):
        has = sizes > k
        out[has, k] = flat[start[has] + k]
    return out


def read_faces(path: Path) -> np.ndarray:
    """faceList 'k(v0 .. vk-1)' per face, or a binary faceList or
    faceCompactList (offsets, then the vertices back to back) -> (F, 4),
    -1 padded for triangles."""
    hdr, t = _open(path)
    if isinstance(t, _Binary):
        if hdr.get("class") == "faceCompactList":
            offsets = t.list(t.label).astype(np.int64)
            flat = t.list(t.label).astype(np.int64)
            if offsets.size == 0 or offsets[0] != 0 or offsets[-1] != flat.size or np.any(np.diff(offsets) < 0):
                raise ValueError(f"{path}: compact face offsets do not cover the vertex list")
            return _pad_faces(path, np.diff(offsets), flat)
        n = t.count()
        t._skip()
        t._expect(b"(")
        sizes = np.zeros(n, dtype=np.int64)
        parts = []
        for i in range(n):
            v = t.list(t.label)
            sizes[i] = v.size
            parts.append(v)
        t._skip()
        t._expect(b")")
        flat = np.concatenate(parts).astype(np.int64) if parts else np.zeros(0, np.int64)
        return _pad_faces(path, sizes, flat)
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
    """(name, type, startFace, nFaces) per patch, in file order (the
    boundary file is text in a binary case too)."""
    t = _strip(_load(path).decode("latin-1"))
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


def write_polymesh(directory, m: _mesh.PolyMesh, fmt: str = "ascii", compact: bool = False,
                   compress: bool = False, label_bits: int = 32) -> None:
    """Writes m as a foam `constant/polyMesh` (points, faces, owner,
    neighbour, boundary) in foam's ascii or binary format: faces as a
    faceList, or with `compact` (binary only) as a faceCompactList of
    offsets and vertices back to back, the form foam's binary output uses;
    `compress` writes each list file gzipped as `name.gz`, as foam does
    under writeCompression.  The boundary file stays text."""
    if fmt not in ("ascii", "binary"):
        raise ValueError("fmt is ascii or binary")
    if compact and fmt != "binary":
        raise ValueError("faceCompactList is written in binary only")
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    lab = np.dtype(f"<i{label_bits // 8}")
    arch = f"LSB;label={label_bits};scalar=64"

    def head(cls, obj, binary):
        return ("FoamFile\n{\n    version     2.0;\n    format      " + ("binary" if binary else "ascii") +
                ";\n" + (f'    arch        "{arch}";\n' if binary else "") +
                f"    class       {cls};\n    location    \"constant/polyMesh\";\n    object      {obj};\n}}\n\n")

    def blist(values: np.ndarray) -> bytes:
        n = values.shape[0]
        if n == 0:
            return b"\n0\n"
        return f"\n{n}\n(".encode() + np.ascontiguousarray(values).tobytes() + b")"

    def put(name, payload: bytes):
        if compress:
            (d / (name + ".gz")).write_bytes(gzip.compress(payload))
        else:
            (d / name).write_bytes(payload)

    binary = fmt == "binary"
    sizes = (m.faces >= 0).sum(axis=1)
    if binary:
        put("points", head("vectorField", "points", True).encode() +
            blist(np.asarray(m.points, dtype="<f8").reshape(-1, 3)) + b"\n")
        if compact:
            offsets = np.concatenate(([0], np.cumsum(sizes))).astype(lab)
            flat = m.faces[m.faces >= 0].astype(lab)
            put("faces", head("faceCompactList", "faces", True).encode() + blist(offsets) + blist(flat) + b"\n")
        else:
            body = b"".join(blist(f[:k].astype(lab)) for f, k in zip(m.faces, sizes))
            put("faces", head("faceList", "faces", True).encode() + f"\n{len(sizes)}\n(".encode() + body +
                b"\n)\n")
        put("owner", head("labelList", "owner", True).encode() + blist(m.owner.astype(lab)) + b"\n")
        put("neighbour", head("labelList", "neighbour", True).encode() + blist(m.neighbour.astype(lab)) + b"\n")
    else:
        pts = "\n".join("(%.17g %.17g %.17g)" % tuple(p) for p in m.points)
        put("points", (head("vectorField", "points", False) + f"{len(m.points)}\n(\n{pts}\n)\n").encode())
        fcs = "\n".join(f"{k}(" + " ".join(str(int(v)) for v in f[:k]) + ")" for f, k in zip(m.faces, sizes))
        put("faces", (head("faceList", "faces", False) + f"{len(sizes)}\n(\n{fcs}\n)\n").encode())
        for name, arr in (("owner", m.owner), ("neighbour", m.neighbour)):
            body = "\n".join(str(int(v)) for v in arr)
            put(name, (head("labelList", name, False) + f"{len(arr)}\n(\n{body}\n)\n").encode())
    names = {v: k for k, v in _PATCH_TYPES.items() if k != "symmetry"}
    ents = "".join(f"    {p.name}\n    {{\n        type            {names[p.type]};\n"
                   f"        nFaces          {p.size};\n        startFace       {p.start};\n    }}\n"
                   for p in m.patches)
    (d / "boundary").write_text(head("polyBoundaryMesh", "boundary", binary) + f"{len(m.patches)}\n(\n{ents})\n")


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


# ---------------------------------------------------------------- fields
# ASCII volScalarField / volVectorField files: read the internal field
# (uniform or nonuniform), the boundary patches' types and values, with
# '#include' files and '$name' substitutions resolved the way the tutorials
# use them; write the state as fields a foam case restarts from.

_LIST_WIDTH = {"scalar": 1, "vector": 3, "symmTensor": 6, "tensor": 9}


def _binary_lists(path: Path, blocks: list) -> str:
    """The file as text.  In a binary file each 'nonuniform List<T> n (raw)'
    is replaced by a placeholder '@@BINk@@' whose values go to blocks[k]
    (the raw items can hold any byte, so the text parser never sees them);
    the header's arch gives the scalar width and byte order."""
    data = _load(path)
    m = re.search(rb"FoamFile\s*\{.*?\}", data, flags=re.S)
    hdr = _header(m.group(0).decode("latin-1")) if m else {}
    if hdr.get("format", "ascii") != "binary":
        return data.decode("latin-1")
    b = _Binary(path, data, hdr)
    pat = re.compile(rb"nonuniform\s+List<(\w+)>\s*(\d+)")
    out, pos = [], 0
    while True:
        m = pat.search(data, pos)
        if not m:
            break
        kind = m.group(1).decode()
        if kind not in _LIST_WIDTH:
            raise ValueError(f"{path}: List<{kind}> is not read")
        n, per = int(m.group(2)), _LIST_WIDTH[kind]
        b.pos = m.end()
        vals = b.items(n, b.scalar, per=per).astype(np.float64)
        blocks.append(vals.reshape(n, per) if per > 1 else vals)
        out.append(data[pos:m.start()].decode("latin-1") + f"@@BIN{len(blocks) - 1}@@")
        pos = b.pos
    out.append(data[pos:].decode("latin-1"))
    return "".join(out)


def _resolve(path: Path, chain=(), blocks=None) -> str:
    """File text with '#include "f"' replaced by the included text
    (relative to the including file) and comments removed; binary lists
    of a binary file go to `blocks` (placeholders in the text)."""
    path = Path(path)
    if path in chain:
        raise ValueError(f"#include loop at {path}")
    text = _binary_lists(path, [] if blocks is None else blocks)
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)

    def inc(m):
        return _resolve(path.parent / m.group(1), chain + (path,), blocks)
    return re.sub(r'#include\s+"([^"]+)"', inc, text)


def _top_entries(text: str) -> dict:
    """Top-level 'name value;' entries (values as strings)."""
    out = {}
    depth = 0
    for m in re.finditer(r"[{}]|(\w+)\s+([^;{}]+);", text):
        if m.group(0) == "{":
            depth += 1
        elif m.group(0) == "}":
            depth -= 1
        elif depth == 0 and m.group(1):
            out[m.group(1)] = m.group(2).strip()
    return out


def _value(s: str, macros: dict, blocks=()):
    """'uniform x' | 'uniform (a b c)' | 'nonuniform List<...> n (...)' |
    '$name' | a binary list's placeholder -> float, tuple or array."""
    s = s.strip()
    for _ in range(8):
        m = re.search(r"\$(\w+)", s)
        if not m:
            break
        s = s[:m.start()] + macros[m.group(1)] + s[m.end():]
    m = re.fullmatch(r"@@BIN(\d+)@@", s)
    if m:
        return blocks[int(m.group(1))]
    if s.startswith("uniform"):
        s = s[len("uniform"):].strip()
    if s.startswith("nonuniform"):
        m = re.match(r"nonuniform\s+List<(\w+)>\s+(\d+)\s*\((.*)\)\s*$", s, flags=re.S)
        if not m:
            raise ValueError("nonuniform list not understood")
        kind, n = m.group(1), int(m.group(2))
        nums = np.array(re.findall(r"[-+0-9.eE]+", m.group(3)), dtype=float)
        return nums.reshape(n, 3) if kind == "vector" else nums.reshape(n)
    if s.startswith("("):
        return tuple(float(x) for x in s.strip("()").split())
    return float(s)


def read_field(path):
    """(internal, boundary): the internal field (float, 3-tuple or array)
    and per patch a dict of its entries (type, value, ... as parsed)."""
    blocks = []
    text = _resolve(Path(path), blocks=blocks)
    hdr = re.search(r"FoamFile\s*\{.*?\}", text, flags=re.S)
    body = text[hdr.end():] if hdr else text
    macros = {k: v for k, v in _top_entries(body).items()}
    m = re.search(r"internalField\s+(.*?);\s*\n", body, flags=re.S)
    internal = _value(m.group(1), macros, blocks)
    bm = re.search(r"boundaryField\s*\{(.*)\}", body, flags=re.S)
    boundary = {}
    if bm:
        for name, block in re.findall(r"(\w+)\s*\{(.*?)\}", bm.group(1), flags=re.S):
            entries = {k: v.strip() for k, v in re.findall(r"(\w+)\s+([^;]+);", block)}
            for k in ("value", "inletValue", "freestreamValue"):
                if k in entries:
                    entries[k] = _value(entries[k], macros, blocks)
            boundary[name] = entries
    return internal, boundary


def _fmt_list(values: np.ndarray) -> str:
    if values.ndim == 1:
        kind = "scalar"
        rows = "\n".join(repr(float(x)) for x in values)
    else:
        kind = "vector"
        rows = "\n".join("(%r %r %r)" % (float(a), float(b), float(c)) for a, b, c in values)
    return f"nonuniform List<{kind}> {values.shape[0]}\n(\n{rows}\n)"


def _fmt_list_binary(values: np.ndarray) -> bytes:
    kind = "scalar" if values.ndim == 1 else "vector"
    n = values.shape[0]
    head = f"nonuniform List<{kind}> {n}\n".encode()
    return head + (b"(" + np.ascontiguousarray(values, dtype="<f8").tobytes() + b")" if n else b"")


def write_field(path, name: str, values, mesh: _mesh.PolyMesh, boundary_values=None, dimensions="[0 0 0 0 0 0 0]",
                fmt: str = "ascii"):
    """A vol field in foam's ascii or binary format with the cell values
    and, per non-empty patch, 'calculated' boundary values
    (boundary_values[patch] arrays, or the adjacent cells' values)."""
    if fmt not in ("ascii", "binary"):
        raise ValueError("fmt is ascii or binary")
    binary = fmt == "binary"
    lists: List[bytes] = []

    def fmt_list(v):
        if not binary:
            return _fmt_list(v)
        lists.append(_fmt_list_binary(v))
        return f"@@BIN{len(lists) - 1}@@"

    values = np.asarray(values, dtype=float)
    cls = "volScalarField" if values.ndim == 1 else "volVectorField"
    own = np.asarray(mesh.owner)
    lines = ["FoamFile", "{", "    version     2.0;", f"    format      {fmt};",
             *(['    arch        "LSB;label=32;scalar=64";'] if binary else []), f"    class       {cls};",
             f"    object      {name};", "}", "", f"dimensions      {dimensions};", "",
             f"internalField   {fmt_list(values)};", "", "boundaryField", "{"]
    for p in mesh.patches:
        lines.append(f"    {p.name}")
        lines.append("    {")
        if p.type == _mesh.EMPTY:
            lines.append("        type            empty;")
        else:
            bv = None if boundary_values is None else boundary_values.get(p.name)
            if bv is None:
                bv = values[own[p.start:p.start + p.size]]
            lines.append("        type            calculated;")
            lines.append(f"        value           {fmt_list(np.asarray(bv, dtype=float))};")
        lines.append("    }")
    lines += ["}", ""]
    text = "\n".join(lines).encode()
    for k, raw in enumerate(lists):
        text = text.replace(f"@@BIN{k}@@".encode(), raw, 1)
    Path(path).write_bytes(text)


def write_state(directory, mesh: _mesh.PolyMesh, p, U, T, nuTilda=None, fmt: str = "ascii"):
    """p, U, T (and nuTilda) of a solver state as a foam time directory,
    in foam's ascii or binary format."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    write_field(d / "p", "p", p, mesh, dimensions="[1 -1 -2 0 0 0 0]", fmt=fmt)
    write_field(d / "U", "U", U, mesh, dimensions="[0 1 -1 0 0 0 0]", fmt=fmt)
    write_field(d / "T", "T", T, mesh, dimensions="[0 0 0 1 0 0 0]", fmt=fmt)
    if nuTilda is not None:
        write_field(d / "nuTilda", "nuTilda", nuTilda, mesh, dimensions="[0 2 -1 0 0 0 0]", fmt=fmt)


def read_state(directory, mesh: _mesh.PolyMesh):
    """p, U, T, nuTilda (None when absent) as cell arrays from a time
    directory (uniform fields expanded)."""
    d = Path(directory)
    N = mesh.n_cells

    def cells(name, vec):
        if not (d / name).exists() and not (d / (name + ".gz")).exists():
            return None
        v, _ = read_field(d / name)
        if isinstance(v, np.ndarray):
            return v
        return np.tile(np.asarray(v, dtype=float), (N, 1)) if vec else np.full(N, float(v))
    return cells("p", False), cells("U", True), cells("T", False), cells("nuTilda", False)


# ---------------------------------------------------------------- case
# A whole rhoDST case directory as a Case: the mesh, the 0/ fields and their
# boundary conditions, and the options this path takes from system/ and
# constant/ (rhoDSTDict, fvSchemes, fvSolution, controlDict,
# thermophysicalProperties, RASProperties), with foam's own key names.

def parse_dict(text: str) -> dict:
    """A foam dictionary as nested dicts of strings (comments removed,
    '#include' already resolved by the caller)."""
    tokens = re.findall(r'"[^"]*"|[{};]|[^\s{};]+', text)
    pos = 0

    def block():
        nonlocal pos
        out = {}
        while pos < len(tokens):
            t = tokens[pos]
            if t == "}":
                pos += 1
                return out
            if t == ";":
                pos += 1
                continue
            key = t
            pos += 1
            if pos < len(tokens) and tokens[pos] == "{":
                pos += 1
                out[key] = block()
                continue
            vals = []
            depth = 0
            while pos < len(tokens) and not (tokens[pos] == ";" and depth == 0):
                if tokens[pos] == "{":
                    depth += 1
                elif tokens[pos] == "}":
                    if depth == 0:
                        break
                    depth -= 1
                vals.append(tokens[pos])
                pos += 1
            if pos < len(tokens) and tokens[pos] == ";":
                pos += 1
            out[key] = " ".join(vals)
        return out
    return block()


def read_dict(path) -> dict:
    text = _resolve(Path(path))
    d = parse_dict(text)
    d.pop("FoamFile", None)
    return d


def _bool(v: str) -> bool:
    return v.strip().lower() in ("true", "yes", "on", "1")


def _thermo(d: dict):
    """(thermo, transport) options from thermophysicalProperties."""
    ttype = d["thermoType"]
    mix = d["mixture"].split()
    # specie: name nMoles molWeight; hConstThermo: Cp Hf; transport: As Ts | mu Pr
    mol_w, Cp = float(mix[2]), float(mix[3])
    R = 8314.47 / mol_w
    thermo = {"R": R, "Cp": Cp}
    if "sutherlandTransport" in ttype:
        As, Ts = float(mix[5]), float(mix[6])
        Cv = Cp - R
        return thermo, {"As": As, "Ts": Ts, "Pr": Cp / (1.32 * Cv + 1.77 * R)}   # Eucken conductivity
    if "constTransport" in ttype:
        mu, Pr = float(mix[5]), float(mix[6])
        return thermo, ({"mu": mu, "Pr": Pr} if mu > 0 else None)
    raise ValueError(f"thermoType {ttype} is not read")


_FARFIELD_KEY = {"p": "pInf", "U": "UInf", "T": "TInf"}


def _bc_spec(field: str, e: dict):
    t = e["type"]
    if t.startswith("farField"):
        v = e[_FARFIELD_KEY[field]]
        return ("farField", _value(v, {}) if not isinstance(v, (float, tuple)) else v)
    if t == "fixedValue":
        return ("fixedValue", e["value"])
    if t == "inletOutlet":
        return ("inletOutlet", e["inletValue"])
    if t in ("zeroGradient", "slip", "symmetryPlane", "symmetry", "calculated"):
        return t
    raise ValueError(f"boundary condition {t} of {field} is not read")


def read_case(directory, time: str = "0"):
    """The case at `directory` (mesh, `time` fields, options) as a Case;
    `case.notes` lists the entries this path does not take."""
    from .cases import Case, _vector_limiter  # noqa: F401  (Case type)
    d = Path(directory)
    poly = d / "constant" / "polyMesh"
    if (poly / "points").exists() or (poly / "points.gz").exists():
        m = read_polymesh(poly)
    elif (poly / "blockMeshDict").exists():
        m = block_mesh(read_dict(poly / "blockMeshDict"))
    else:
        raise FileNotFoundError(f"{poly}: no polyMesh and no blockMeshDict")
    notes = []
    rho = read_dict(d / "system" / "rhoDSTDict")
    schemes = read_dict(d / "system" / "fvSchemes")
    sol = read_dict(d / "system" / "fvSolution")
    ctrl = read_dict(d / "system" / "controlDict")
    thermo, transport = _thermo(read_dict(d / "constant" / "thermophysicalProperties"))
    ras_path = d / "constant" / "RASProperties"
    model = "laminar"
    if ras_path.exists():
        ras = read_dict(ras_path)
        if _bool(ras.get("turbulence", "off")):
            model = ras["RASModel"]
    opts = {}
    for k in ("fluxScheme", "Jacobian", "dependentVariable", "lowMach", "Mainf", "directWaveSpeed"):
        if k in rho:
            opts[k] = rho[k]
    for sub in ("timeIntegration", "timeControls", "residualControls"):
        if sub in rho:
            opts[sub] = dict(rho[sub])
    opts["ddtSchemes"] = {"default": schemes["ddtSchemes"]["default"]}
    interp = schemes.get("interpolationSchemes", {})
    opts["interpolationSchemes"] = {k: v for k, v in interp.items() if k.startswith("reconstruct(")}
    # the gradient and convection schemes this path selects by name: grad(U)
    # (Gauss linear or cellLimited) and div(phi,nuTilda) (upwind or
    # linearUpwind); the entries of equations this path does not solve
    # (k, epsilon, e) are not read
    grads = {k: " ".join(v.split()) for k, v in schemes.get("gradSchemes", {}).items()}
    divs = {k: " ".join(v.split()) for k, v in schemes.get("divSchemes", {}).items()}
    taken = {}
    if grads.get("grad(U)", "Gauss linear") != "Gauss linear":
        taken.setdefault("gradSchemes", {})["grad(U)"] = grads["grad(U)"]
    for k, v in grads.items():
        if k not in ("default", "grad(U)") and v != "Gauss linear":
            notes.append(f"gradSchemes {k} {v}: Gauss linear here")
    if grads.get("default", "Gauss linear") != "Gauss linear":
        notes.append(f"gradSchemes default {grads['default']}: Gauss linear here")
    if model != "laminar" and "div(phi,nuTilda)" in divs and divs["div(phi,nuTilda)"] != "Gauss upwind":
        taken.setdefault("divSchemes", {})["div(phi,nuTilda)"] = divs["div(phi,nuTilda)"]
    opts.update(taken)
    dep = opts.get("dependentVariable", "W")
    W = sol["solvers"].get(dep, sol["solvers"].get("W"))
    opts["solvers"] = {"W": {k: W[k] for k in ("solver", "preconditioner", "nDirections", "tolerance", "relTol",
                                                "maxIter", "minIter", "nSweeps", "fillInLevel") if k in W}}
    if "relaxationFactors" in sol and "nuTilda" in sol["relaxationFactors"]:
        opts["relaxationFactors"] = {"nuTilda": sol["relaxationFactors"]["nuTilda"]}
    if "fieldBounds" in sol:
        opts["fieldBounds"] = dict(sol["fieldBounds"])
    opts["controlDict"] = {"deltaT": ctrl["deltaT"]}
    if "startTime" in ctrl:
        opts["controlDict"]["startTime"] = ctrl["startTime"]
    opts["thermo"] = thermo
    if transport:
        opts["transport"] = transport
    if model != "laminar":
        opts["RASModel"] = model
    # fields and boundary conditions
    td = d / time
    N = m.n_cells
    fields, bfields = {}, {}
    for f in ("p", "U", "T", "nuTilda"):
        if (td / f).exists():
            fields[f], bfields[f] = read_field(td / f)
    bcs = {}
    for p in m.patches:
        if p.type == _mesh.EMPTY:
            continue
        spec = {}
        for f in ("p", "U", "T", "nuTilda"):
            if f in bfields and p.name in bfields[f]:
                spec[f] = _bc_spec(f, bfields[f][p.name])
        bcs[p.name] = spec

    def cells(v, vec):
        if isinstance(v, np.ndarray):
            return v
        return np.tile(np.asarray(v, dtype=float), (N, 1)) if vec else np.full(N, float(v))
    if model != "laminar":
        m.wall_distance = _mesh.wall_distance(m, [p.name for p in m.patches if p.type == _mesh.WALL])
    case = Case(d.name, m, bcs, opts, cells(fields["p"], False), cells(fields["U"], True), cells(fields["T"], False),
                nuTilda=cells(fields["nuTilda"], False) if "nuTilda" in fields else None)
    case.notes = notes
    return case


# ---------------------------------------------------------------- blockMesh
# Meshes that tutorials define by constant/polyMesh/blockMeshDict: hex
# blocks with simpleGrading, straight edges, patches by block faces and the
# unlisted boundary faces in 'defaultFaces' (empty), as blockMesh builds
# them.  Cells are numbered block by block, the block's first direction
# fastest; coincident points of neighbouring blocks are merged.

def _graded(n: int, ratio: float) -> np.ndarray:
    """n+1 coordinates in [0,1], last cell / first cell = ratio."""
    if n < 1:
        raise ValueError("a block needs at least one cell per direction")
    if abs(ratio - 1.0) < 1e-14:
        return np.linspace(0.0, 1.0, n + 1)
    r = ratio ** (1.0 / (n - 1)) if n > 1 else 1.0
    if n == 1 or abs(r - 1.0) < 1e-14:
        return np.linspace(0.0, 1.0, n + 1)
    x = (r ** np.arange(n + 1) - 1.0) / (r ** n - 1.0)
    return x


def _tuples(s: str):
    return [tuple(float(x) for x in t.split()) for t in re.findall(r"\(([^()]*)\)", s)]


def block_mesh(d: dict) -> _mesh.PolyMesh:
    scale = float(d.get("convertToMeters", d.get("scale", "1")))
    verts = np.array(_tuples(d["vertices"]), dtype=float) * scale
    if re.search(r"\w", d.get("edges", "()").strip("() ")):
        raise ValueError("curved block edges are not generated")
    if re.search(r"\w", d.get("mergePatchPairs", "()").strip("() ")):
        raise ValueError("mergePatchPairs is not generated")
    blocks = re.findall(r"hex\s*\(([^)]*)\)\s*\(([^)]*)\)\s*simpleGrading\s*\(([^)]*)\)", d["blocks"])
    if not blocks:
        raise ValueError("no hex blocks")
    corner = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    pts_all, cells_all = [], []
    base = 0
    for vs, ns, gs in blocks:
        v = verts[[int(x) for x in vs.split()]]
        n = [int(x) for x in ns.split()]
        g = [float(x) for x in gs.split()]
        if len(g) != 3:
            raise ValueError("simpleGrading with three ratios is generated")
        s, t, u = (_graded(n[k], g[k]) for k in range(3))
        S, T, Uu = np.meshgrid(s, t, u, indexing="ij")          # (nx+1, ny+1, nz+1)
        w = [(1 - S) * (1 - T) * (1 - Uu), S * (1 - T) * (1 - Uu), S * T * (1 - Uu), (1 - S) * T * (1 - Uu),
             (1 - S) * (1 - T) * Uu, S * (1 - T) * Uu, S * T * Uu, (1 - S) * T * Uu]
        P = sum(w[k][..., None] * v[k] for k in range(8))       # trilinear in the block's corners
        pid = base + np.arange(P[..., 0].size).reshape(P.shape[:3])
        pts_all.append(P.reshape(-1, 3, order="C"))
        # cells: i fastest, then j, then k; hex vertex order as foam's
        k_, j_, i_ = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
        i_, j_, k_ = i_.ravel(), j_.ravel(), k_.ravel()
        c = np.stack([pid[i_, j_, k_], pid[i_ + 1, j_, k_], pid[i_ + 1, j_ + 1, k_], pid[i_, j_ + 1, k_],
                      pid[i_, j_, k_ + 1], pid[i_ + 1, j_, k_ + 1], pid[i_ + 1, j_ + 1, k_ + 1],
                      pid[i_, j_ + 1, k_ + 1]], axis=1)
        cells_all.append(c)
        base += P[..., 0].size
    pts = np.concatenate(pts_all)
    cells = np.concatenate(cells_all)
    # merge coincident points (neighbouring blocks share their face points)
    tol = 1e-9 * max(1.0, float(np.abs(pts).max()))
    key = np.round(pts / tol).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    pts = pts[first[order]]
    cells = rank[inv.ravel()][cells]
    # patches from block faces
    bnd = d.get("boundary", {})
    if isinstance(bnd, str):            # boundary ( name { type ..; faces (..); } ... )
        body = bnd.strip()
        if not (body.startswith("(") and body.endswith(")")):
            raise ValueError("boundary must be a list of named patch dictionaries")
        bnd = parse_dict(body[1:-1])
    defs, quads = [], []
    for name, pd in bnd.items():
        defs.append((name, _PATCH_TYPES[pd["type"].strip()]))
        quads.append([verts[[int(x) for x in q]] for q in
                      [t.split() for t in re.findall(r"\(([^()]*)\)", pd.get("faces", ""))]])
    defs.append(("defaultFaces", _mesh.EMPTY))

    def classify(centres, normals):
        out = np.full(centres.shape[0], len(defs) - 1)
        for pi, qs in enumerate(quads):
            for q in qs:
                nq = np.cross(q[2] - q[0], q[3] - q[1])
                nq /= np.linalg.norm(nq)
                on = np.abs((centres - q[0]) @ nq) < 1e-9 * max(1.0, np.abs(q).max())
                lo, hi = q.min(0) - 1e-12, q.max(0) + 1e-12
                inside = np.all((centres >= lo) & (centres <= hi), axis=1)
                out[on & inside] = pi
        return out
    return _mesh.build_polymesh(pts, [("hex", cells)], classify, defs)
