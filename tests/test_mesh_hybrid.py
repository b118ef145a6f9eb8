"""The hybrid tet/prism forward-step mesh: conforming (the prism layers'
triangles meet the Kuhn tetrahedra's faces, no internal boundary faces),
untangled after the jitter (every cell closed, owner-to-neighbour vectors
along the face normals), the domain's volume, and a first-order steady
state the oracle reaches on it."""
import numpy as np
import pytest

from rhodst_b200 import cases
from rhodst_b200 import mesh as M


@pytest.mark.parametrize("jitter", [0.0, 0.25])
def test_hybrid_mesh_is_valid(jitter):
    m = M.forward_step_3d_hybrid(30, 10, 4, jitter=jitter)
    Fi = m.n_internal_faces
    S = np.zeros((m.n_cells, 3))
    np.add.at(S, m.owner, m.Sf)
    np.add.at(S, m.neighbour, -m.Sf[:Fi])
    assert np.abs(S).max() <= 1e-14 * np.abs(m.Sf).max()          # closed cells
    d = m.C[m.neighbour] - m.C[m.owner[:Fi]]
    assert np.all(np.einsum("ij,ij->i", d, m.Sf[:Fi]) > 0)         # no tangled cells
    assert m.V.min() > 0 and m.V.sum() == pytest.approx(3.0 * 1.0 * 0.5 - 2.4 * 0.2 * 0.5, rel=1e-12)
    walls = m.patch("walls")
    c = m.Cf[walls.start:walls.start + walls.size]
    outer = (np.abs(c[:, 1]) < 1e-9) | (np.abs(c[:, 1] - 1.0) < 1e-9) | (np.abs(c[:, 2]) < 1e-9) | \
            (np.abs(c[:, 2] - 0.5) < 1e-9)
    assert outer.all()                                             # no internal "walls" faces
    # two prisms per hex below y = 0.5, six tets above
    n_hex = 30 * 10 * 4 - 24 * 2 * 4          # the step (x >= 0.6, y < 0.2) removed
    n_pr_hex = 30 * 5 * 4 - 24 * 2 * 4
    assert m.n_cells == 2 * n_pr_hex + 6 * (n_hex - n_pr_hex)


def test_hybrid_step_reaches_a_first_order_steady_state():
    from tests.oracle_lib import OracleSolver
    c = cases.forward_step_3d_hybrid_c5(nx=30, ny=10, nz=4).with_options(**{
        "fluxScheme": "HLL", "interpolationSchemes.reconstruct(rho)": "upwind",
        "interpolationSchemes.reconstruct(U)": "upwind", "interpolationSchemes.reconstruct(T)": "upwind",
        "timeControls.maxCo": 50.0, "precision": "fp64"})
    o = OracleSolver(c.mesh, c.bcs, c.options, rcb_parts=4)
    o.set_primitive(c.p, c.U, c.T)
    r0, r = None, None
    for _ in range(20):
        reps = o.step(50)
        r0 = reps[0]["res_l2"][0] if r0 is None else r0
        r = reps[-1]["res_l2"][0] / r0
        if r < 1e-8:
            break
    assert r < 1e-8, r
