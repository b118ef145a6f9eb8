"""Writes tests/golden/rae2822_mesh.npz: the mesh of the reference's RAE2822
tutorial (tutorials/RAE2822/constant/polyMesh, ascii) read with
rhodst_b200.foam, stored compactly so that tests and cases run without the
reference tree.  Run from the repository root:

    python tests/golden/make_rae2822.py <rhoDST checkout>

(or with RHODST_REFERENCE naming the checkout)."""
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from rhodst_b200 import foam  # noqa: E402



def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RHODST_REFERENCE")
    if not ref:
        raise SystemExit("usage: make_rae2822.py <rhoDST checkout> (or set RHODST_REFERENCE)")
    m = foam.read_polymesh(Path(ref) / "tutorials/RAE2822/constant/polyMesh")
    out = Path(__file__).resolve().parent / "rae2822_mesh.npz"
    foam.save_npz(m, out)
    print(f"{out}: {m.n_cells} cells, {m.n_faces} faces, patches "
          f"{[(p.name, p.type, p.start, p.size) for p in m.patches]}")


if __name__ == "__main__":
    main()
