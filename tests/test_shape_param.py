"""Hicks-Henne shape parametrisation of the airfoil mesh (host side, no GPU):
bump shapes, the surface displacement, linearity of the point motion in the
amplitudes, and the moved mesh's topology and geometry."""
import numpy as np
import pytest

from rhodst_b200 import mesh as M
from rhodst_b200.shape import HicksHenne


@pytest.fixture(scope="module")
def base():
    return M.naca_cmesh(97, 25, first_cell=5e-3)


def test_bumps_peak_at_their_centres_and_vanish_at_the_edges(base):
    hh = HicksHenne(base)
    assert hh.n_variables == 64
    B = hh.bumps(hh.peaks)
    assert np.allclose(np.diag(B), 1.0, atol=1e-14)
    edges = hh.bumps(np.array([0.0, 1.0]))
    assert np.abs(edges).max() <= 1e-12
    x = np.linspace(0, 1, 1001)
    Bx = hh.bumps(x)
    assert Bx.min() >= 0.0 and Bx.max() <= 1.0 + 1e-15
    assert np.all(np.argmax(Bx, axis=1) == np.round(hh.peaks * 1000).astype(int))


def test_design_point_is_seeded_and_bounded():
    a = HicksHenne.design_point(64)
    assert np.array_equal(a, np.random.default_rng(1234).uniform(-1e-3, 1e-3, 64))
    assert np.abs(a).max() <= 1e-3


def test_surface_moves_by_the_bumps(base):
    hh = HicksHenne(base)
    a = hh.design_point(64)
    pts = hh.points(a)
    x, side, w = base.surface_map
    on = (side != 0) & (w == 1.0)
    lo, up = side == -1, side == 1
    dy = np.zeros(pts.shape[0])
    Bx = hh.bumps(x)
    dy[lo] = (a[:32] @ Bx)[lo]
    dy[up] = (a[32:] @ Bx)[up]
    assert np.allclose(pts[on, 1], side[on] * M.naca00xx(x[on]) + dy[on], rtol=0, atol=1e-15)
    assert np.array_equal(pts[:, 0], base.points[:, 0]) and np.array_equal(pts[:, 2], base.points[:, 2])
    # leading and trailing edge points, the wake and the far field stay
    fixed = side == 0
    assert np.array_equal(pts[fixed], base.points[fixed])


def test_point_motion_is_linear_in_the_amplitudes(base):
    hh = HicksHenne(base)
    rng = np.random.default_rng(7)
    a, b = rng.uniform(-1e-3, 1e-3, (2, 64))
    lhs = hh.points(a + b) - base.points
    rhs = (hh.points(a) - base.points) + (hh.points(b) - base.points)
    assert np.abs(lhs - rhs).max() <= 4 * np.finfo(float).eps * np.abs(base.points).max()


def test_moved_mesh_keeps_topology_and_recomputes_geometry(base):
    hh = HicksHenne(base)
    m = hh.mesh(hh.design_point(64))
    assert np.array_equal(m.owner, base.owner) and np.array_equal(m.neighbour, base.neighbour)
    assert [(p.name, p.start, p.size) for p in m.patches] == [(p.name, p.start, p.size) for p in base.patches]
    assert m.V.min() > 0
    ref = M.PolyMesh(points=m.points, faces=m.faces, owner=m.owner, neighbour=m.neighbour,
                     patches=m.patches, n_cells=m.n_cells)
    M.compute_geometry(ref)
    for name in ("Sf", "Cf", "magSf", "C", "V", "weights", "deltaCoeffs"):
        assert np.array_equal(getattr(m, name), getattr(ref, name)), name
    # the volume change is of the order of the displacement
    assert 0 < np.abs(m.V - base.V).max() < 1e-2 * base.V.max()


def test_freestream_derivatives_chain_rule():
    """For J = a . U(M, alpha) + b . d(alpha), d = (cos, sin, 0) the drag
    direction, the adjoint quantities dJ/dU = a and force = b give dJ/dMach
    and dJ/dalpha; checked against central differences of J."""
    import math
    from rhodst_b200.shape import freestream_derivatives
    a = np.array([0.3, -1.2, 0.7])
    b = np.array([2.0, 0.5, -0.4])
    c_inf, M0, al0 = 1.3, 0.73, math.radians(2.3)

    def J(M, al):
        U = M * c_inf * np.array([math.cos(al), math.sin(al), 0.0])
        return a @ U + b @ np.array([math.cos(al), math.sin(al), 0.0])
    U0 = M0 * c_inf * np.array([math.cos(al0), math.sin(al0), 0.0])
    dM, da = freestream_derivatives(a, b, U0, c_inf)
    h = 1e-6
    assert dM == pytest.approx((J(M0 + h, al0) - J(M0 - h, al0)) / (2 * h), rel=1e-8)
    assert da == pytest.approx((J(M0, al0 + h) - J(M0, al0 - h)) / (2 * h), rel=1e-8)
