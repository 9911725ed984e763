"""The CPU restatement of SOL 101 output recovery (oracle_recover) against
closed-form answers: rigid-body motion recovers nothing, uniform membrane
strain and uniform curvature give N = h D eps and M = -br D kappa h^3/12, the
linear parts are linear in u, the pressure-deck moment scale, bar end forces
of a pure stretch, and the section-point stress formula.

The reference cannot run here (no Julia); these pin the restatement to the
mechanics it encodes, not to the reference's own outputs."""
import dataclasses

import numpy as np
import pytest

import oracle as O
from jf_2026_05_19_b200 import decks
from jf_2026_05_19_b200.decks import ModelArrays, N_SHELL_PROP

# record columns that are linear in u (everything but the blended CQUAD4
# shear, the principal stress, von Mises and the status)
LINEAR = [c for c in range(48) if c not in (6, 7, 20, 21, 46, 47)]


def _rigid(m: ModelArrays, t, w):
    """Rigid-body field u = t + w x X, theta = w, in each node's CD frame."""
    t, w = np.asarray(t, float), np.asarray(w, float)
    u = np.zeros(m.ndof)
    for i in range(m.n_nodes):
        ut, ur = t + np.cross(w, m.coords[i]), w
        if m.node_R is not None:
            ut, ur = m.node_R[i].T @ ut, m.node_R[i].T @ ur
        u[6 * i:6 * i + 3], u[6 * i + 3:6 * i + 6] = ut, ur
    return u


def _tri_plate(n=2, size=100.0, h=2.0, E=70000.0, nu=0.3):
    """Flat plate of n x n squares, each split into two CTRIA3."""
    p = decks.plate_c1(n=n, size=size, h=h, E=E, nu=nu)
    q = p.q4_nodes
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]]).astype(np.int32)
    return dataclasses.replace(p, q4_nodes=np.zeros((0, 4), np.int32), q4_prop=np.zeros((0, N_SHELL_PROP)),
                               t3_nodes=tri, t3_prop=np.tile(p.q4_prop[0], (tri.shape[0], 1)))


def _normal_sign(m, nodes):
    """+1 when the element normal of the first element is +z."""
    p = m.coords[nodes]
    n = np.cross(p[1] - p[0], p[2] - p[0])
    return 1.0 if n[2] > 0 else -1.0


def test_rigid_body_motion_recovers_nothing():
    m = decks.barrel_small(seed=2, n_circ=48, n_axial=12)
    sh_d, bar_d = O.recover(m, decks.smooth_displacement(m, seed=3))
    sh, bar = O.recover(m, _rigid(m, [0.3, -0.2, 0.1], [1e-3, -2e-3, 5e-4]))
    assert (sh[:, 21] == 1).all() and (bar[:, 17] == 1).all()
    for cols in (slice(0, 3), slice(3, 6), slice(6, 8), slice(8, 14), slice(22, 34), slice(34, 46)):
        assert np.abs(sh[:, cols]).max() <= 1e-9 * np.abs(sh_d[:, cols]).max()
    assert np.abs(bar[:, :17]).max() <= 1e-9 * np.abs(bar_d[:, :17]).max()


@pytest.mark.parametrize("kind", ["quad4", "tria3"])
def test_uniform_membrane_strain(kind):
    """u = e0 (x, y): an equi-biaxial strain, the same in every in-plane frame."""
    m = decks.plate_c1(n=4, size=100.0) if kind == "quad4" else _tri_plate(n=3)
    prop = m.q4_prop if kind == "quad4" else m.t3_prop
    E, nu, h = prop[0, 1], prop[0, 2], prop[0, 0]
    e0 = 1e-4
    u = np.zeros(m.ndof)
    u[0::6], u[1::6] = e0 * m.coords[:, 0], e0 * m.coords[:, 1]
    sh, _ = O.recover(m, u)
    n_exp = h * E / (1 - nu) * e0
    tol = 1e-10 * n_exp
    assert np.abs(sh[:, 0] - n_exp).max() < tol and np.abs(sh[:, 1] - n_exp).max() < tol
    assert np.abs(sh[:, 2]).max() < tol and np.abs(sh[:, 3:6]).max() < tol
    for c in (14, 15, 17, 18):
        assert np.abs(sh[:, c] - e0).max() < 1e-10 * e0
    if kind == "quad4":
        corners = sh[:, 22:34].reshape(-1, 4, 3)
        assert np.abs(corners[:, :, 0] - n_exp).max() < tol and np.abs(corners[:, :, 2]).max() < tol


def test_uniform_curvature_quad4():
    """theta = k (-y, x), w = 0: kappa = (k, k, 0) in every in-plane frame."""
    m = decks.plate_c1(n=4, size=100.0)
    E, nu, h, br = m.q4_prop[0, 1], m.q4_prop[0, 2], m.q4_prop[0, 0], m.q4_prop[0, 4]
    k = 1e-5
    u = np.zeros(m.ndof)
    u[3::6], u[4::6] = -k * m.coords[:, 1], k * m.coords[:, 0]
    sh, _ = O.recover(m, u)
    s = _normal_sign(m, m.q4_nodes[0])
    m_exp = -br * E / (1 - nu) * k * s * h ** 3 / 12
    assert np.abs(sh[:, 3] - m_exp).max() < 1e-10 * abs(m_exp)
    assert np.abs(sh[:, 4] - m_exp).max() < 1e-10 * abs(m_exp)
    assert np.abs(sh[:, 5]).max() < 1e-10 * abs(m_exp)
    # fibre strains: eps = z kappa
    assert np.abs(sh[:, 14] - (-h / 2) * k * s).max() < 1e-10 * k * h


def test_uniform_curvature_isolated_tria3():
    """A lone CTRIA3 has no shared edge (macro weight 0): M is the CST curvature's."""
    full = _tri_plate(n=1)
    m = dataclasses.replace(full, t3_nodes=full.t3_nodes[:1], t3_prop=full.t3_prop[:1])
    E, nu, h, br = m.t3_prop[0, 1], m.t3_prop[0, 2], m.t3_prop[0, 0], m.t3_prop[0, 4]
    k = 1e-5
    u = np.zeros(m.ndof)
    u[3::6], u[4::6] = -k * m.coords[:, 1], k * m.coords[:, 0]
    sh, _ = O.recover(m, u)
    s = _normal_sign(m, m.t3_nodes[0])
    m_exp = -br * E / (1 - nu) * k * s * h ** 3 / 12
    assert abs(sh[0, 3] - m_exp) < 1e-10 * abs(m_exp) and abs(sh[0, 4] - m_exp) < 1e-10 * abs(m_exp)
    # the plate macro gives a transverse shear (theta is not the gradient of w)
    assert np.abs(sh[0, 6:8]).max() > 0


def test_macro_blend_changes_interior_triangles_only():
    """Triangles with two or more shared edges get weight >= 1/2 and a blended M;
    the lone triangle of a one-square plate has one shared edge (weight 0)."""
    m = _tri_plate(n=3)
    u = decks.smooth_displacement(m, seed=4)
    sh, _ = O.recover(m, u)
    lone = dataclasses.replace(m, t3_nodes=m.t3_nodes[:1], t3_prop=m.t3_prop[:1])
    sh1, _ = O.recover(lone, u)
    # an interior triangle (three shared edges) differs from the same triangle alone
    interior = 4  # square (1, 1), first half: all edges shared in a 3 x 3 split plate
    solo = dataclasses.replace(m, t3_nodes=m.t3_nodes[interior:interior + 1], t3_prop=m.t3_prop[:1])
    sh_solo, _ = O.recover(solo, u)
    assert np.allclose(sh[interior, 0:3], sh_solo[0, 0:3], rtol=1e-12, atol=0)   # N unaffected
    assert not np.allclose(sh[interior, 3:6], sh_solo[0, 3:6], rtol=1e-6, atol=0)  # M blended
    assert sh1[0, 21] == 1


def test_linear_parts_are_linear():
    m = decks.barrel_small(seed=2, n_circ=48, n_axial=12)
    a = decks.smooth_displacement(m, seed=5)
    b = decks.smooth_displacement(m, seed=6)
    sa, ba = O.recover(m, a)
    sb, bb = O.recover(m, b)
    sc, bc = O.recover(m, a + 2.0 * b)
    lin = sa[:, LINEAR] + 2.0 * sb[:, LINEAR]
    scale = np.abs(lin).max(axis=0) + 1e-300
    assert (np.abs(sc[:, LINEAR] - lin) / scale).max() < 1e-9
    blin = ba[:, :17] + 2.0 * bb[:, :17]
    assert (np.abs(bc[:, :17] - blin) / (np.abs(blin).max(axis=0) + 1e-300)).max() < 1e-9
    # CTRIA3 shear is linear too (area-weighted macro shears)
    nq = m.q4_nodes.shape[0]
    tq = sa[nq:, 6:8] + 2.0 * sb[nq:, 6:8]
    assert np.abs(sc[nq:, 6:8] - tq).max() < 1e-9 * np.abs(tq).max()


def test_pressure_deck_scales_bending_dominated_rectangles():
    m = decks.plate_c1(n=6, size=120.0)
    x, y = m.coords[:, 0] / 120.0, m.coords[:, 1] / 120.0
    u = np.zeros(m.ndof)
    u[2::6] = np.sin(np.pi * x) * np.sin(np.pi * y)            # a bending mode, no membrane
    u[3::6] = np.pi / 120.0 * np.sin(np.pi * x) * np.cos(np.pi * y)
    u[4::6] = -np.pi / 120.0 * np.cos(np.pi * x) * np.sin(np.pi * y)
    plain, _ = O.recover(m, u)
    scaled, _ = O.recover(m, u, flags=O.RECOVER_PRESSURE_DECK)
    mq = np.abs(plain[:, 6:8]).max(axis=1)
    mn = np.abs(plain[:, 0:3]).max(axis=1)
    hit = (mq > 1e-8) & ~(mn > np.maximum(1e-6, 1e-4 * mq))
    assert hit.any()
    assert np.allclose(scaled[hit, 3:6], 0.99 * plain[hit, 3:6], rtol=1e-14, atol=0)
    assert np.array_equal(scaled[~hit, 3:6], plain[~hit, 3:6])
    assert np.array_equal(scaled[:, 0:3], plain[:, 0:3]) and np.array_equal(scaled[:, 8:20], plain[:, 8:20])
    # the twisting moment stays constant across the corner rows
    assert np.array_equal(scaled[:, [36, 39, 42, 45]], np.repeat(scaled[:, 5:6], 4, axis=1))
    # a deck with bars never scales (the library adds the no-bar condition)
    b = decks.barrel_small(seed=1, n_circ=24, n_axial=6)
    ub = decks.smooth_displacement(b, seed=2)
    assert np.array_equal(O.recover(b, ub, flags=O.RECOVER_PRESSURE_DECK)[0], O.recover(b, ub)[0])


def _bar_deck(L=500.0, E=70000.0, G=26000.0):
    coords = np.array([[0.0, 0.0, 0.0], [L, 0.0, 0.0]])
    sec = decks.pbarl_section("BAR", [20.0, 40.0])
    prop = np.array([decks.bar_prop_row(sec, E, G, (0.0, 0.0, 1.0))])
    e = np.zeros((0,), np.int32)
    return ModelArrays(coords=coords, q4_nodes=np.zeros((0, 4), np.int32), q4_prop=np.zeros((0, N_SHELL_PROP)),
                       t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, N_SHELL_PROP)),
                       bar_nodes=np.array([[0, 1]], np.int32), bar_prop=prop, bar_pin=np.zeros((1, 2), np.int32),
                       rbe2_master=e, rbe2_cm=e, rbe2_slave_ptr=np.zeros(1, np.int64), rbe2_slaves=e)


def test_bar_stretch_and_section_points():
    m = _bar_deck()
    A, E, L = m.bar_prop[0, 0], m.bar_prop[0, 7], 500.0
    u = np.zeros(m.ndof)
    u[6] = 0.25
    _, bar = O.recover(m, u)
    assert abs(bar[0, 0] - E * A * 0.25 / L) < 1e-10 * E * A * 0.25 / L
    assert abs(bar[0, 8] - E * 0.25 / L) < 1e-12 * E
    assert np.abs(bar[0, 1:8]).max() < 1e-9 * abs(bar[0, 0]) and bar[0, 17] == 1
    # a bend: the section-point stresses follow the reference's formula from the end moments
    u = np.zeros(m.ndof)
    u[6 + 1], u[6 + 5] = 0.5, 1e-3
    pts = np.array([[10.0, 20.0, -10.0, 20.0, -10.0, -20.0, 10.0, -20.0, -1.0]])
    _, bar = O.recover(m, u, bar_points=pts)
    Iz, Iy, I12 = m.bar_prop[0, 1], m.bar_prop[0, 2], m.bar_prop[0, 3]
    den = Iz * Iy - I12 ** 2
    for end, (m1, m2) in enumerate(((bar[0, 4], bar[0, 5]), (bar[0, 6], bar[0, 7]))):
        for j in range(4):
            yj, zj = pts[0, 2 * j], pts[0, 2 * j + 1]
            want = -((m1 * Iy - m2 * I12) * yj + (m2 * Iz - m1 * I12) * zj) / den
            assert abs(bar[0, 9 + 4 * end + j] - want) <= 1e-12 * max(abs(want), 1.0)
    assert np.abs(bar[0, 9:17]).max() > 0
    # zero-length bar: skipped
    z = dataclasses.replace(m, coords=np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.0]]))
    assert O.recover(z, u)[1][0, 17] == 0
