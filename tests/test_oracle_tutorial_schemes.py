"""Known answers for the RAE2822 tutorial's gradient and convection schemes
in the oracle (system/fvSchemes: grad(U) cellLimited Gauss linear 1,
div(phi,nuTilda) Gauss linearUpwind grad(nuTilda)):

* cellLimited: on cells whose faces are all internal the limited gradient
  equals a numpy restatement of foam-extend's cellLimitedGrad for a vector
  field applied to the Gauss gradient; every extrapolation (Cf - C).grad U_j
  to those faces then stays inside the spread of U_j over the neighbours;
  k < 1 widens the spread (limits less); a linear field on a uniform mesh
  is not limited away from the boundary;
* linearUpwind: with a uniform nuTilda (zero gradient) the steps equal the
  upwind ones to round-off, and with a varying one they differ;
* the options parse as the tutorial writes them.
"""
import numpy as np
import pytest

from rhodst_b200 import cases
from tests.oracle_lib import OracleSolver


def laminar(**opts):
    c = cases.naca0012_laminar(ni=65, nj=17, first_cell=1e-2)
    return c.with_options(**opts) if opts else c


def wavy_state(c, seed=3):
    rng = np.random.default_rng(seed)
    C = c.mesh.C
    k = rng.uniform(1.0, 3.0, size=(3, 3))
    U = c.U.copy()
    for j in range(2):
        U[:, j] += 0.2 * np.abs(c.U[:, 0]).max() * np.sin(C @ k[j] + j)
    return U


def interior_cells(m):
    """Cells with no boundary face other than the empty front and back."""
    from rhodst_b200 import mesh as meshmod
    own = np.asarray(m.owner)
    nb = np.zeros(m.n_cells, dtype=int)
    for P in m.patches:
        if P.type != meshmod.EMPTY:
            np.add.at(nb, own[P.start:P.start + P.size], 1)
    return np.nonzero(nb == 0)[0]


def cell_faces(m):
    faces = [[] for _ in range(m.n_cells)]
    for f in range(m.n_internal_faces):
        faces[m.owner[f]].append(f)
        faces[m.neighbour[f]].append(f)
    return faces


def limited_reference(m, U, g, cells, k):
    """foam-extend cellLimitedGrad<vector> on interior cells: per velocity
    component the spread over the face neighbours, widened for k < 1, and
    the limiter min over faces of maxD/d or minD/d."""
    faces = cell_faces(m)
    out = g.copy()
    Cf = np.asarray(m.Cf)
    for i in cells:
        nb = [m.neighbour[f] if m.owner[f] == i else m.owner[f] for f in faces[i]]
        mx = np.maximum(U[i], U[nb].max(axis=0)) - U[i]
        mn = np.minimum(U[i], U[nb].min(axis=0)) - U[i]
        if k < 1.0:
            w = (1.0 / k - 1.0) * (mx - mn)
            mx, mn = mx + w, mn - w
        lim = np.ones(3)
        for f in faces[i]:
            d = Cf[f] - m.C[i]
            e = d[0] * g[i, 0] + d[1] * g[i, 1] + d[2] * g[i, 2]
            for j in range(3):
                if e[j] > mx[j] + 1e-300:
                    lim[j] = min(lim[j], mx[j] / e[j])
                elif e[j] < mn[j] - 1e-300:
                    lim[j] = min(lim[j], mn[j] / e[j])
        out[i] = g[i] * lim[None, :]
    return out


@pytest.mark.parametrize("k", [1.0, 0.5])
def test_cell_limited_gradient_matches_a_restatement(k):
    base = laminar()
    U = wavy_state(base)
    o0 = OracleSolver(base.mesh, base.bcs, base.options)
    o0.set_primitive(base.p, U, base.T)
    g0 = o0.grad_U()
    c = laminar(**{"gradSchemes.grad(U)": f"cellLimited Gauss linear {k:g}"})
    o = OracleSolver(c.mesh, c.bcs, c.options)
    o.set_primitive(c.p, U, c.T)
    g = o.grad_U()
    cells = interior_cells(c.mesh)
    assert cells.size > 500
    ref = limited_reference(c.mesh, U, g0, cells, k)
    assert np.allclose(g[cells], ref[cells], rtol=1e-13, atol=1e-13 * np.abs(g0).max())
    if k == 1.0:
        assert np.abs(g[cells] - g0[cells]).max() > 1e-3 * np.abs(g0).max()    # it does limit here
        # extrapolations to the faces stay inside the neighbours' spread
        faces = cell_faces(c.mesh)
        Cf = np.asarray(c.mesh.Cf)
        for i in cells[::7]:
            nb = [c.mesh.neighbour[f] if c.mesh.owner[f] == i else c.mesh.owner[f] for f in faces[i]]
            hi = np.maximum(U[i], U[nb].max(axis=0))
            lo = np.minimum(U[i], U[nb].min(axis=0))
            for f in faces[i]:
                Uf = U[i] + (Cf[f] - c.mesh.C[i]) @ g[i]
                span = hi - lo + 1e-14
                assert np.all(Uf <= hi + 1e-12 * span) and np.all(Uf >= lo - 1e-12 * span)


def test_widening_limits_less():
    base = laminar()
    U = wavy_state(base, seed=5)
    gs = {}
    for k in (1.0, 0.5):
        c = laminar(**{"gradSchemes.grad(U)": f"cellLimited Gauss linear {k:g}"})
        o = OracleSolver(c.mesh, c.bcs, c.options)
        o.set_primitive(c.p, U, c.T)
        gs[k] = o.grad_U()
    assert np.all(np.abs(gs[0.5]) >= np.abs(gs[1.0]) * (1 - 1e-14) - 1e-300)
    assert np.abs(gs[0.5]).sum() > np.abs(gs[1.0]).sum()


def test_linear_field_is_not_limited_inside():
    """A linear velocity field on a uniform lattice: face extrapolations lie
    between the neighbours, so the limiter is one away from the boundary."""
    from tests.test_oracle_known_answers import channel_case
    c = channel_case("HLL", nx=12, ny=8)
    m = c.mesh
    # the unjittered lattice of the channel (uniform spacing)
    X, Y = m.C[:, 0], m.C[:, 1]
    U = np.stack([1.0 + 0.3 * X - 0.2 * Y, 0.1 + 0.05 * X + 0.4 * Y, np.zeros_like(X)], axis=1)
    o0 = OracleSolver(m, c.bcs, c.options)
    o0.set_primitive(c.p, U, c.T)
    o1 = OracleSolver(m, c.bcs, c.with_options(**{"gradSchemes.grad(U)": "cellLimited Gauss linear 1"}).options)
    o1.set_primitive(c.p, U, c.T)
    cells = interior_cells(m)
    g0, g1 = o0.grad_U()[cells], o1.grad_U()[cells]
    ref = limited_reference(m, U, o0.grad_U(), cells, 1.0)[cells]
    assert np.allclose(g1, ref, rtol=1e-13, atol=1e-15)


def sa_case(**opts):
    c = cases.naca0012_turbulent(ni=65, nj=17, first_cell=1e-2, reynolds=1e5, flux="HLL", limiter="upwind")
    return c.with_options(**opts) if opts else c


def test_linear_upwind_nu_tilda():
    lu = {"divSchemes.div(phi,nuTilda)": "Gauss linearUpwind grad(nuTilda)"}
    out = {}
    for name, opts in (("upwind", {}), ("linearUpwind", lu)):
        c = sa_case(**opts)
        o = OracleSolver(c.mesh, c.bcs, c.options)
        # uniform nuTilda: its gradient is zero inside, the correction too
        o.set_primitive(c.p, c.U, c.T, c.nuTilda)
        o.step(1)
        out[name] = o.primitive()[3]
    # the first update starts from a uniform field: only boundary-adjacent
    # gradients are non-zero, so compare a second step from a varying field
    assert np.isfinite(out["linearUpwind"]).all()
    nut_var = None
    res = {}
    for name, opts in (("upwind", {}), ("linearUpwind", lu)):
        c = sa_case(**opts)
        o = OracleSolver(c.mesh, c.bcs, c.options)
        C = c.mesh.C
        nut_var = c.nuTilda * (1.0 + 0.5 * np.sin(0.3 * C[:, 0]) ** 2)
        o.set_primitive(c.p, c.U, c.T, nut_var)
        o.step(1)
        res[name] = o.primitive()[3]
    assert np.abs(res["linearUpwind"] - res["upwind"]).max() > 1e-6 * np.abs(res["upwind"]).max()


def test_linear_upwind_is_exact_for_uniform_nu_tilda_away_from_walls():
    """With nuTilda uniform and held at the far-field value on every
    boundary, grad nuTilda is zero everywhere (to the round-off of the
    closed-cell face sums) and linearUpwind adds nothing: the steps are
    those of upwind to round-off."""
    out = {}
    for name, opts in (("upwind", {}), ("linearUpwind", {"divSchemes.div(phi,nuTilda)":
                                                          "Gauss linearUpwind grad(nuTilda)"})):
        c = sa_case(**opts)
        bcs = {k: dict(v) for k, v in c.bcs.items()}
        nut_inf = float(c.nuTilda[0])
        bcs["airfoil"]["nuTilda"] = ("fixedValue", nut_inf)
        c.bcs = bcs
        o = OracleSolver(c.mesh, c.bcs, c.options)
        o.set_primitive(c.p, c.U, c.T, c.nuTilda)
        o.step(1)
        out[name] = o.primitive()[3]
    scale = np.abs(out["upwind"]).max()
    assert np.abs(out["upwind"] - out["linearUpwind"]).max() <= 1e-12 * scale


def test_scheme_entries_parse_as_written():
    """Dictionary entries with runs of blanks select the same schemes."""
    U = wavy_state(laminar(), seed=2)
    gs = []
    for entry in ("cellLimited Gauss linear 1", "cellLimited   Gauss  linear\t1"):
        c = laminar(**{"gradSchemes.grad(U)": entry, "gradSchemes.default": "Gauss  linear"})
        o = OracleSolver(c.mesh, c.bcs, c.options)
        o.set_primitive(c.p, U, c.T)
        gs.append(o.grad_U())
    assert np.array_equal(gs[0], gs[1])
