"""foam polyMesh input (rhodst_b200.foam) and the reference's RAE2822
tutorial case: the reader against the tutorial's own files (when the
reference tree is given by RHODST_REFERENCE, the root of a rhoDST checkout),
the stored mesh's geometry, foam's ordering checks, and the oracle running
the case."""
import os
from pathlib import Path

import numpy as np
import pytest

from rhodst_b200 import cases, foam
from rhodst_b200 import mesh as M

FIXTURE = Path(__file__).resolve().parent / "golden" / "rae2822_mesh.npz"
# the reference tree (a rhoDST checkout) when RHODST_REFERENCE names one;
# the tests that read its tutorial files skip without it
_REF = Path(os.environ["RHODST_REFERENCE"]) if os.environ.get("RHODST_REFERENCE") else Path("/nonexistent")
TUTORIAL = _REF / "tutorials/RAE2822/constant/polyMesh"


@pytest.mark.skipif(not TUTORIAL.exists(), reason="RHODST_REFERENCE does not name a reference tree")
def test_reader_matches_the_stored_tutorial_mesh():
    a = foam.read_polymesh(TUTORIAL)
    b = foam.load_npz(FIXTURE)
    assert np.array_equal(a.points, b.points) and np.array_equal(a.faces, b.faces)
    assert np.array_equal(a.owner, b.owner) and np.array_equal(a.neighbour, b.neighbour)
    assert [(p.name, p.type, p.start, p.size) for p in a.patches] == \
           [(p.name, p.type, p.start, p.size) for p in b.patches]


def test_tutorial_mesh_geometry():
    m = foam.load_npz(FIXTURE)
    assert (m.n_cells, m.n_faces, m.n_internal_faces) == (23552, 94608, 46704)
    assert [(p.name, p.type) for p in m.patches] == [("frontAndBackPlanes", M.EMPTY), ("freestreamBC", M.PATCH),
                                                     ("airfoil", M.WALL)]
    assert m.V.min() > 0
    S = np.zeros((m.n_cells, 3))
    Fi = m.n_internal_faces
    np.add.at(S, m.owner, m.Sf)
    np.add.at(S, m.neighbour, -m.Sf[:Fi])
    assert np.abs(S).max() <= 1e-12 * np.abs(m.Sf).max()          # closed cells
    d = m.C[m.neighbour] - m.C[m.owner[:Fi]]
    assert np.all(np.einsum("ij,ij->i", d, m.Sf[:Fi]) > 0)        # owner -> neighbour normals
    air = m.patch("airfoil")
    x = m.Cf[air.start:air.start + air.size, 0]
    assert 0 < x.min() and x.max() < 1                             # unit chord


def _write(d: Path, name: str, cls: str, body: str):
    (d / name).write_text("FoamFile\n{\n    version 2.0;\n    format ascii;\n    class " + cls +
                          ";\n    object " + name + ";\n}\n// comment\n" + body)


def _two_cells(d: Path, owner_first=True):
    pts = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0),
           (0, 0, 1), (1, 0, 1), (2, 0, 1), (0, 1, 1), (1, 1, 1), (2, 1, 1)]
    _write(d, "points", "vectorField", f"{len(pts)}\n(\n" + "\n".join(f"({a} {b} {c})" for a, b, c in pts) + "\n)\n")
    faces = [(1, 4, 10, 7),                                      # internal x = 1, normal +x
             (0, 6, 9, 3), (2, 5, 11, 8),                        # x = 0, x = 2
             (0, 1, 7, 6), (1, 2, 8, 7), (3, 9, 10, 4), (4, 10, 11, 5),
             (0, 3, 4, 1), (1, 4, 5, 2), (6, 7, 10, 9), (7, 8, 11, 10)]
    _write(d, "faces", "faceList", f"{len(faces)}\n(\n" + "\n".join("4(%d %d %d %d)" % f for f in faces) + "\n)\n")
    own = [0, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1]
    nei = [1] if owner_first else [0]
    if not owner_first:
        own[0] = 1
    _write(d, "owner", "labelList", f"{len(own)}\n(\n" + "\n".join(map(str, own)) + "\n)\n")
    _write(d, "neighbour", "labelList", f"{len(nei)}\n(\n" + "\n".join(map(str, nei)) + "\n)\n")
    _write(d, "boundary", "polyBoundaryMesh", """3
(
    inlet { type patch; nFaces 1; startFace 1; }
    outlet { type patch; nFaces 1; startFace 2; }
    walls { type wall; inGroups 1(wall); nFaces 8; startFace 3; }
)
""")


def test_reader_on_a_two_cell_mesh(tmp_path):
    _two_cells(tmp_path)
    m = foam.read_polymesh(tmp_path)
    assert m.n_cells == 2 and m.n_internal_faces == 1
    assert np.allclose(m.V, 1.0) and np.allclose(m.Sf[0], (1, 0, 0))
    assert np.allclose(m.C, [(0.5, 0.5, 0.5), (1.5, 0.5, 0.5)])
    assert [p.name for p in m.patches] == ["inlet", "outlet", "walls"] and m.patches[2].type == M.WALL


def test_reader_checks_foam_ordering(tmp_path):
    _two_cells(tmp_path, owner_first=False)
    with pytest.raises(ValueError):
        foam.read_polymesh(tmp_path)


def test_tutorial_case_runs_on_the_oracle():
    from tests.oracle_lib import OracleSolver
    c = cases.rae2822()
    o = OracleSolver(c.mesh, c.bcs, c.options, rcb_parts=4)
    o.set_primitive(c.p, c.U, c.T, c.nuTilda)
    reps = o.step(20)
    r = [x["res_l2"][0] for x in reps]
    assert np.all(np.isfinite(r)) and r[-1] < 0.5 * r[0]
    nut = o.primitive()[3]
    assert nut.min() >= 0 and np.isfinite(nut).all()


FIELDS = _REF / "tutorials/RAE2822/0"


@pytest.mark.skipif(not FIELDS.exists(), reason="RHODST_REFERENCE does not name a reference tree")
def test_tutorial_fields_match_the_case():
    """The tutorial's 0/ fields (with their #include and $ macros) give the
    free stream and boundary conditions cases.rae2822 sets."""
    c = cases.rae2822()
    p, bp = foam.read_field(FIELDS / "p")
    U, bU = foam.read_field(FIELDS / "U")
    T, bT = foam.read_field(FIELDS / "T")
    nut, bn = foam.read_field(FIELDS / "nuTilda")
    assert p == c.bcs["freestreamBC"]["p"][1] == c.p[0]
    assert U == tuple(c.bcs["freestreamBC"]["U"][1]) and np.array_equal(c.U[0], U)
    assert T == c.bcs["freestreamBC"]["T"][1] == c.T[0]
    assert nut == c.bcs["freestreamBC"]["nuTilda"][1] == c.nuTilda[0]
    assert bp["freestreamBC"]["type"] == "farFieldPressureDST" and bp["airfoil"]["type"] == "zeroGradient"
    assert bU["airfoil"]["type"] == "fixedValue" and bU["airfoil"]["value"] == (0.0, 0.0, 0.0)
    assert bn["freestreamBC"]["type"] == "inletOutlet" and bn["airfoil"]["value"] == 0.0
    # the far-field conditions carry the free stream from the included file
    assert float(bp["freestreamBC"]["pInf"]) == p


def test_state_round_trip_through_foam_fields(tmp_path):
    from tests.oracle_lib import OracleSolver
    c = cases.rae2822()
    o = OracleSolver(c.mesh, c.bcs, c.options, rcb_parts=4)
    o.set_primitive(c.p, c.U, c.T, c.nuTilda)
    o.step(2)
    p, U, T, nut = o.primitive()
    foam.write_state(tmp_path / "2", c.mesh, p, U, T, nut)
    p2, U2, T2, n2 = foam.read_state(tmp_path / "2", c.mesh)
    assert np.array_equal(p, p2) and np.array_equal(U, U2) and np.array_equal(T, T2) and np.array_equal(nut, n2)
    # a restart from the written fields evaluates the same residual
    r = OracleSolver(c.mesh, c.bcs, c.options, rcb_parts=4)
    r.set_primitive(p2, U2, T2, n2)
    o.set_primitive(p, U, T, nut)
    assert np.array_equal(r.residual(), o.residual())
    # uniform fields expand to every cell
    q, _, _, _ = foam.read_state(tmp_path / "missing", c.mesh)
    assert q is None


CASE = _REF / "tutorials/RAE2822"


@pytest.mark.skipif(not CASE.exists(), reason="RHODST_REFERENCE does not name a reference tree")
def test_case_reader_gives_the_tutorial_case():
    """read_case on the tutorial directory yields the options, boundary
    conditions and initial fields cases.rae2822 sets (numerically), names
    what this path does not take, and runs the same steps."""
    from rhodst_b200._abi import flatten_options
    from tests.oracle_lib import OracleSolver
    a = foam.read_case(CASE)
    b = cases.rae2822(tutorial_schemes=True)
    fa, fb = flatten_options(a.options), flatten_options(b.options)
    fa.pop("controlDict.deltaT"); fa.pop("controlDict.startTime"); fa.pop("dependentVariable"); fb.pop("dependentVariable")
    fa.pop("timeIntegration.timeIntegration")
    assert fa.keys() == fb.keys()
    for k in fa:
        try:
            va = [float(x) for x in fa[k].split()]
            vb = [float(x) for x in fb[k].split()]
            assert va == pytest.approx(vb, rel=1e-15), k
        except ValueError:
            assert fa[k].lower() == fb[k].lower(), k
    assert a.bcs == b.bcs
    assert np.array_equal(a.p, b.p) and np.array_equal(a.U, b.U) and np.array_equal(a.T, b.T)
    assert np.array_equal(a.nuTilda, b.nuTilda)
    assert a.options["gradSchemes"]["grad(U)"] == "cellLimited Gauss linear 1"
    assert a.options["divSchemes"]["div(phi,nuTilda)"] == "Gauss linearUpwind grad(nuTilda)"
    ra, rb = [], []
    for c, out in ((a, ra), (b, rb)):
        o = OracleSolver(c.mesh, c.bcs, c.options, rcb_parts=4)
        o.set_primitive(c.p, c.U, c.T, c.nuTilda)
        out += [r["res_l2"][0] for r in o.step(2)]
    assert ra == rb


def test_dictionary_parser():
    d = foam.parse_dict("""
        a 1;   b  (1 2 3);
        sub { x yes; y "q w"; inner { z 1e-5; } }
        c uniform (0 0 0);
    """)
    assert d["a"] == "1" and d["c"].split() == ["uniform", "(0", "0", "0)"]
    assert d["b"].split() == ["(1", "2", "3)"]
    assert d["sub"] == {"x": "yes", "y": '"q w"', "inner": {"z": "1e-5"}}


STEP = _REF / "tutorials/forwardStep"
STEP_DUAL = _REF / "tutorials/forwardStepDual"


@pytest.mark.skipif(not STEP.exists(), reason="RHODST_REFERENCE does not name a reference tree")
def test_block_mesh_tutorial_is_the_forward_step():
    """The forwardStep tutorial's blockMeshDict gives the built-in generator's
    mesh at full resolution (same cells, numbering and patches)."""
    c = foam.read_case(STEP)
    r = M.forward_step_2d(3)
    assert np.abs(c.mesh.C - r.C).max() < 1e-12
    assert np.array_equal(c.mesh.owner, r.owner) and np.array_equal(c.mesh.neighbour, r.neighbour)
    assert [(p.name, p.type, p.start, p.size) for p in c.mesh.patches] == \
           [(p.name, p.type, p.start, p.size) for p in r.patches]
    assert c.bcs["obstacle"] == {"p": "zeroGradient", "U": "slip", "T": "zeroGradient"}
    assert c.bcs["inlet"]["U"] == ("fixedValue", (3.0, 0.0, 0.0))
    assert c.options["ddtSchemes"]["default"] == "Euler" and "transport" not in c.options
    from tests.oracle_lib import OracleSolver
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    assert np.isfinite(o.step(1)[0]["res_mag"])


@pytest.mark.skipif(not STEP_DUAL.exists(), reason="RHODST_REFERENCE does not name a reference tree")
def test_dual_time_tutorial_reads_and_runs():
    from tests.oracle_lib import OracleSolver
    c = foam.read_case(STEP_DUAL)
    assert c.options["timeIntegration"]["timeIntegration"] == "Dual"
    assert c.options["ddtSchemes"]["default"] == "dual2ndDST"
    c = c.with_options(**{"timeIntegration.maxInnerIter": 2})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, c.U, c.T)
    r = o.step(1)[0]
    assert r["lin_iterations"] == 3 and np.isfinite(r["res_mag"])


def test_block_mesh_grading_and_merging():
    d = foam.parse_dict("""
        vertices ((0 0 0) (1 0 0) (2 0 0) (0 1 0) (1 1 0) (2 1 0)
                  (0 0 1) (1 0 1) (2 0 1) (0 1 1) (1 1 1) (2 1 1));
        blocks (hex (0 1 4 3 6 7 10 9) (4 2 1) simpleGrading (2 1 1)
                hex (1 2 5 4 7 8 11 10) (3 2 1) simpleGrading (1 1 1));
        edges ();
        boundary ( left { type patch; faces ((0 6 9 3)); }
                   walls { type wall; faces ((0 1 7 6) (1 2 8 7) (3 9 10 4) (4 10 11 5)); } );
    """)
    m = foam.block_mesh(d)
    assert m.n_cells == 14 and m.points.shape[0] == (5 + 3) * 3 * 2    # the shared x = 1 points merged
    assert m.n_internal_faces == (3 * 2 + 4 * 1) + (2 * 2 + 3 * 1) + 2  # block 0, block 1, shared faces
    xs = np.unique(np.round(m.points[:, 0], 12))
    dx = np.diff(xs[xs <= 1 + 1e-12])
    assert dx[-1] / dx[0] == pytest.approx(2.0)                         # last/first cell of block 0
    names = [(p.name, p.type, p.size) for p in m.patches]
    assert names == [("left", M.PATCH, 2), ("walls", M.WALL, 14), ("defaultFaces", M.EMPTY, 28 + 2)]
    assert np.isclose(m.V.sum(), 2.0)


def _same_mesh(a, b):
    assert np.array_equal(a.points, b.points) and np.array_equal(a.faces, b.faces)
    assert np.array_equal(a.owner, b.owner) and np.array_equal(a.neighbour, b.neighbour)
    assert [(p.name, p.type, p.start, p.size) for p in a.patches] == \
           [(p.name, p.type, p.start, p.size) for p in b.patches]
    assert np.array_equal(a.V, b.V) and np.array_equal(a.Sf, b.Sf)


@pytest.mark.parametrize("fmt,compact,compress", [("ascii", False, False), ("binary", False, False),
                                                   ("binary", True, False), ("binary", True, True),
                                                   ("ascii", False, True)])
def test_polymesh_round_trip(tmp_path, fmt, compact, compress):
    """A hybrid tet/prism mesh (triangles and quads) written in each of
    foam's forms and read back: topology, points and geometry bit for bit."""
    m = M.forward_step_3d_hybrid(nx=12, ny=4, nz=3, jitter=0.25)
    assert set((m.faces >= 0).sum(axis=1)) == {3, 4}
    foam.write_polymesh(tmp_path, m, fmt=fmt, compact=compact, compress=compress)
    if compress:
        assert (tmp_path / "points.gz").exists() and not (tmp_path / "points").exists()
    _same_mesh(foam.read_polymesh(tmp_path), m)


def test_binary_rae2822_tutorial_mesh(tmp_path):
    """The tutorial's mesh as a binary faceCompactList case reads back as
    the stored ascii one."""
    m = foam.load_npz(FIXTURE)
    foam.write_polymesh(tmp_path, m, fmt="binary", compact=True)
    assert b"faceCompactList" in (tmp_path / "faces").read_bytes()[:400]
    _same_mesh(foam.read_polymesh(tmp_path), m)


def _binary_file(path, cls, arch, payload: bytes):
    path.write_bytes(("FoamFile\n{\n    version 2.0;\n    format binary;\n" +
                      (f'    arch "{arch}";\n' if arch else "") +
                      f"    class {cls};\n    object {path.name};\n}}\n// a comment\n/* and a block one */\n")
                     .encode() + payload)


def test_binary_arch_widths_and_byte_order(tmp_path):
    """The header's arch names the byte order and the label and scalar widths."""
    lab = np.array([3, 0, 7, 2**33], dtype=">i8")
    _binary_file(tmp_path / "owner", "labelList", "MSB;label=64;scalar=64",
                 b"\n4\n(" + lab.tobytes() + b")\n")
    assert foam.read_labels(tmp_path / "owner").tolist() == [3, 0, 7, 2**33]
    pts = np.array([[0.5, -1.25, 3.0], [1e-300, 2.0, -0.0]], dtype="<f4")
    _binary_file(tmp_path / "points", "vectorField", "LSB;label=32;scalar=32",
                 b"\n2\n(" + pts.tobytes() + b")\n")
    assert np.array_equal(foam.read_points(tmp_path / "points"), pts.astype(np.float64))
    # no arch entry: 32-bit little-endian labels
    _binary_file(tmp_path / "neighbour", "labelList", None, b"\n3\n(" + np.array([1, 2, 5], "<i4").tobytes() + b")")
    assert foam.read_labels(tmp_path / "neighbour").tolist() == [1, 2, 5]


def test_binary_empty_lists(tmp_path):
    """foam writes an empty binary list as its count alone; '0()' reads too."""
    _binary_file(tmp_path / "a", "labelList", "LSB;label=32;scalar=64", b"\n0\n")
    _binary_file(tmp_path / "b", "labelList", "LSB;label=32;scalar=64", b"\n0()\n")
    assert foam.read_labels(tmp_path / "a").size == 0 and foam.read_labels(tmp_path / "b").size == 0


def test_binary_malformed_files_are_rejected(tmp_path):
    vals = np.arange(5, dtype="<i4")
    _binary_file(tmp_path / "short", "labelList", "LSB;label=32;scalar=64", b"\n6\n(" + vals.tobytes() + b")")
    with pytest.raises(ValueError, match="past the end"):
        foam.read_labels(tmp_path / "short")
    _binary_file(tmp_path / "noparen", "labelList", "LSB;label=32;scalar=64", b"\n5\n" + vals.tobytes())
    with pytest.raises(ValueError, match="expected"):
        foam.read_labels(tmp_path / "noparen")
    # compact faces whose offsets do not reach the end of the vertex list
    off = np.array([0, 3, 6], "<i4")
    flat = np.arange(7, dtype="<i4")
    _binary_file(tmp_path / "faces", "faceCompactList", "LSB;label=32;scalar=64",
                 b"\n3\n(" + off.tobytes() + b")\n7\n(" + flat.tobytes() + b")")
    with pytest.raises(ValueError, match="offsets"):
        foam.read_faces(tmp_path / "faces")
    # a pentagon is refused as in ascii
    off = np.array([0, 5], "<i4")
    _binary_file(tmp_path / "faces", "faceCompactList", "LSB;label=32;scalar=64",
                 b"\n2\n(" + off.tobytes() + b")\n5\n(" + np.arange(5, dtype="<i4").tobytes() + b")")
    with pytest.raises(ValueError, match="5 vertices"):
        foam.read_faces(tmp_path / "faces")


def test_binary_state_round_trip(tmp_path):
    """p, U, T, nuTilda written as binary foam fields (internal and patch
    value lists raw) read back bit for bit, gzipped files too, with the
    patch entries parsed around the raw blocks."""
    m = M.forward_step_3d_hybrid(nx=12, ny=4, nz=3, jitter=0.25)
    rng = np.random.default_rng(7)
    N = m.n_cells
    # values whose bytes include ';', '{', '}' and ')' exercise the raw blocks
    p = rng.uniform(0.5, 2.0, N)
    p[:4] = np.frombuffer(b";;;;;;;;{{{{}}}}))))))((((((;{}(" , dtype="<f8")
    U = rng.normal(size=(N, 3))
    T = rng.uniform(0.8, 1.2, N)
    nut = rng.uniform(0, 1e-3, N)
    foam.write_state(tmp_path / "1", m, p, U, T, nut, fmt="binary")
    assert b"format      binary" in (tmp_path / "1" / "p").read_bytes()[:300]
    p2, U2, T2, n2 = foam.read_state(tmp_path / "1", m)
    assert np.array_equal(p, p2, equal_nan=True) and np.array_equal(U, U2)
    assert np.array_equal(T, T2) and np.array_equal(nut, n2)
    _, bnd = foam.read_field(tmp_path / "1" / "U")
    for patch in m.patches:
        e = bnd[patch.name]
        if patch.type == M.EMPTY:
            assert e["type"] == "empty"
        else:
            assert e["type"] == "calculated"
            assert np.array_equal(e["value"], U[m.owner[patch.start:patch.start + patch.size]])
    # gzipped, as foam writes under writeCompression
    import gzip
    for name in ("p", "U", "T", "nuTilda"):
        f = tmp_path / "1" / name
        (tmp_path / "1" / (name + ".gz")).write_bytes(gzip.compress(f.read_bytes()))
        f.unlink()
    p3, U3, _, _ = foam.read_state(tmp_path / "1", m)
    assert np.array_equal(p, p3, equal_nan=True) and np.array_equal(U, U3)


def test_binary_field_with_an_empty_patch_list(tmp_path):
    """foam writes an empty binary list as its count alone."""
    vals = np.array([1.5, -2.0, 3.25])
    body = (b"FoamFile\n{\n    version 2.0;\n    format binary;\n    arch \"LSB;label=32;scalar=64\";\n"
            b"    class volScalarField;\n    object p;\n}\ndimensions [1 -1 -2 0 0 0 0];\n\n"
            b"internalField   nonuniform List<scalar> 3\n(" + vals.astype("<f8").tobytes() + b");\n\n"
            b"boundaryField\n{\n    a\n    {\n        type calculated;\n        value nonuniform List<scalar> 0\n;\n"
            b"    }\n    b\n    {\n        type fixedValue;\n        value uniform 2;\n    }\n}\n")
    (tmp_path / "p").write_bytes(body)
    internal, bnd = foam.read_field(tmp_path / "p")
    assert np.array_equal(internal, vals)
    assert bnd["a"]["value"].size == 0 and bnd["b"]["value"] == 2.0


@pytest.mark.skipif(not CASE.exists(), reason="RHODST_REFERENCE does not name a reference tree")
def test_case_reader_on_a_binary_copy_of_the_tutorial(tmp_path):
    """The tutorial case with its polyMesh rewritten in foam's binary,
    compact and gzipped form reads as the ascii case does."""
    import shutil
    d = tmp_path / "RAE2822"
    shutil.copytree(CASE, d, ignore=shutil.ignore_patterns("sets", "*Zones"))
    m = foam.read_polymesh(d / "constant/polyMesh")
    for f in ("points", "faces", "owner", "neighbour", "boundary"):
        (d / "constant/polyMesh" / f).unlink()
    foam.write_polymesh(d / "constant/polyMesh", m, fmt="binary", compact=True, compress=True)
    a, b = foam.read_case(CASE), foam.read_case(d)
    _same_mesh(a.mesh, b.mesh)
    assert a.bcs == b.bcs and a.options == b.options
    assert np.array_equal(a.p, b.p) and np.array_equal(a.U, b.U) and np.array_equal(a.nuTilda, b.nuTilda)
