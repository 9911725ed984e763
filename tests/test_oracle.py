"""CPU tests of the oracle: golden fixtures, physics known-answers, error behaviour."""
import os

import numpy as np
import pytest

import oracle as O
from helpers import LAMBDA_TOL, ROW_TOL, load_factors, rowmax_rel_err, static_solution, to_csc
from jf_2026_05_19_b200 import decks

GOLD = os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.npz")


def test_golden_fixtures_reproduce():
    import golden.make_golden as mg
    g = np.load(GOLD)
    for name, m in mg.golden_decks().items():
        cp, rv, nz, mx, dg = O.assemble_k(m)
        assert np.array_equal(cp, g[f"{name}__colptr"]) and np.array_equal(rv, g[f"{name}__rowval"])
        assert rowmax_rel_err(cp, g[f"{name}__k"], nz) <= ROW_TOL
        _, _, nzg = O.assemble_kg(m, g[f"{name}__u"])
        assert rowmax_rel_err(cp, g[f"{name}__kg"], nzg) <= ROW_TOL
        assert abs(mx - g[f"{name}__max"][0]) <= 1e-12 * mx
    lc_q4, lc_t3, prop = mg.element_cases()
    assert np.allclose(O.q4_local(lc_q4, prop), g["q4_local"], rtol=0, atol=1e-12 * np.abs(g["q4_local"]).max())
    assert np.allclose(O.t3_local(lc_t3, prop), g["t3_local"], rtol=0, atol=1e-12 * np.abs(g["t3_local"]).max())


def _rigid_modes(lc, nn):
    X = np.hstack([lc, np.zeros((nn, 1))])
    modes = []
    for d in range(3):
        v = np.zeros(6 * nn); v[d::6] = 1; modes.append(v)
    v = np.zeros(6 * nn); v[0::6] = -X[:, 1]; v[1::6] = X[:, 0]; v[5::6] = 1; modes.append(v)
    v = np.zeros(6 * nn); v[2::6] = X[:, 1]; v[3::6] = 1; modes.append(v)
    v = np.zeros(6 * nn); v[2::6] = -X[:, 0]; v[4::6] = 1; modes.append(v)
    return modes


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_quad4_symmetric_and_rigid_body(seed):
    rng = np.random.default_rng(seed)
    lc = np.array([[-5.0, -4.0], [5.0, -4.0], [5.0, 4.0], [-5.0, 4.0]]) + rng.uniform(-1, 1, (4, 2))
    lc -= lc.mean(0)
    prop = decks.shell_prop_row(rng.uniform(1, 3), 70000.0, 0.33)
    K = O.q4_local(lc, prop)
    s = np.abs(K).max()
    assert np.abs(K - K.T).max() <= 1e-13 * s
    for v in _rigid_modes(lc, 4):
        assert np.abs(K @ v).max() <= 1e-11 * s
    ev = np.linalg.eigvalsh(0.5 * (K + K.T))
    assert (ev > 1e-9 * s).sum() == 18   # exactly the six rigid-body modes are free


def test_tria3_rigid_body():
    lc = np.array([[-5.0, -3.0], [6.0, -2.0], [-1.0, 5.0]])
    lc -= lc.mean(0)
    K = O.t3_local(lc, decks.shell_prop_row(2.0, 70000.0, 0.33))
    s = np.abs(K).max()
    for v in _rigid_modes(lc, 3):
        assert np.abs(K @ v).max() <= 1e-11 * s


def test_plate_buckling_coefficient():
    """Simply supported square plate: lambda_1 ~ 4 pi^2 D / b^2 (k = 4), mesh error < 1%."""
    m = decks.plate_c1()
    cp, rv, nz, mx, dg = O.assemble_k(m)
    K = to_csc(cp, rv, nz, m.ndof)
    u, free = static_solution(m, K, O.constraint_map(m))
    cpg, rvg, nzg = O.assemble_kg(m, u)
    assert np.array_equal(cp, cpg) and np.array_equal(rv, rvg)
    lam = load_factors(K, to_csc(cpg, rvg, nzg, m.ndof), free, k=3)
    D = 70000 * 2.0 ** 3 / (12 * (1 - 0.33 ** 2))
    classical = 4 * np.pi ** 2 * D / 400.0 ** 2
    assert abs(lam[0] - classical) / classical < 0.01


def test_kg_linear_in_displacement():
    m = decks.barrel_small(n_circ=24, n_axial=6)
    u = decks.smooth_displacement(m, seed=2)
    cp, rv, a = O.assemble_kg(m, u)
    _, _, b = O.assemble_kg(m, 2.5 * u)
    assert rowmax_rel_err(cp, 2.5 * a, b) <= 1e-12


def test_orig_diag_and_max():
    m = decks.stiffened_panel_c2(lx=60.0, ly=40.0, stringer_every=2)
    cp, rv, nz, mx, dg = O.assemble_k(m)
    K = to_csc(cp, rv, nz, m.ndof)
    assert np.allclose(K.diagonal(), dg, rtol=1e-12, atol=0)   # no constraints: K diag == orig_diag
    assert mx >= np.abs(nz).max() * (1 - 1e-12) or mx > 0


def test_rbe2_constraint_map_and_empty_dependent_rows():
    m = decks.barrel_small(n_circ=24, n_axial=4)
    dep, ptr, ind, coef = O.constraint_map(m)
    assert len(dep) == 24 * 6
    cp, rv, nz, mx, dg = O.assemble_k(m)
    lens = np.diff(cp)
    assert np.all(lens[dep - 1] == 0)          # dependent dofs leave no structural entries
    # rigid rotation coefficients: translation of a slave depends on master translation + rotations
    assert np.all(np.abs(coef) > 1e-15)


def test_kg_offset_bars_raise_like_reference():
    m = decks.stiffened_panel_c2(lx=60.0, ly=40.0, stringer_every=2, stringer_offset=12.0)
    with pytest.raises(O.OracleError) as e:
        O.assemble_kg(m, np.zeros(m.ndof))
    assert e.value.status == 7
    O.assemble_k(m)   # K with offsets is fine


def test_unsupported_branches_are_refused():
    import dataclasses
    from decks_extra import skewed_plane, warped
    m = skewed_plane()
    with pytest.raises(O.OracleError) as e:
        O.assemble_k(warped(m))
    assert e.value.status == 2
    pin = m.bar_pin.copy(); pin[0, 0] = 45
    with pytest.raises(O.OracleError):
        O.assemble_k(dataclasses.replace(m, bar_pin=pin))
    with pytest.raises(O.OracleError):
        O.assemble_k(dataclasses.replace(m, param_snorm=20.0))


def _bars_only_barrel():
    import dataclasses
    m = decks.barrel_small(seed=2, n_circ=72, n_axial=24)
    return dataclasses.replace(m, q4_nodes=np.zeros((0, 4), np.int32), q4_prop=np.zeros((0, decks.N_SHELL_PROP)),
                               t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, decks.N_SHELL_PROP)))


def _reordered(m, seed):
    import dataclasses
    r = np.random.default_rng(seed)
    pq, pt, pb = (r.permutation(a.shape[0]) for a in (m.q4_nodes, m.t3_nodes, m.bar_nodes))
    return dataclasses.replace(m, q4_nodes=m.q4_nodes[pq], q4_prop=m.q4_prop[pq], t3_nodes=m.t3_nodes[pt],
                               t3_prop=m.t3_prop[pt], bar_nodes=m.bar_nodes[pb], bar_prop=m.bar_prop[pb],
                               bar_pin=m.bar_pin[pb])


def test_element_order_rounding_sets_the_parity_bound():
    """The reference sums each matrix entry in its element Dict order, which is
    arbitrary.  On the bars-only barrel the RBE2 centre node's rows sum terms up
    to ~3e4 times their row max, so reordering the elements moves the oracle's
    own K past 1e-12 of the row max -- the bound cannot hold there for any
    implementation -- while every entry stays within SUM_TOL * eps * sum|terms|."""
    from helpers import EPS, SUM_TOL, parity_ratio
    m = _bars_only_barrel()
    cp, rv, nz, _, _, det = O.assemble_k(m, detail=True, abs_sums=True)
    u = decks.smooth_displacement(m, seed=7)
    _, _, kg, detg = O.assemble_kg(m, u, detail=True, abs_sums=True)
    worst_row = 0.0
    for seed in range(3):
        mp = _reordered(m, seed)
        cp2, rv2, nz2, _, _ = O.assemble_k(mp)
        _, _, kg2 = O.assemble_kg(mp, u)
        assert np.array_equal(cp, cp2) and np.array_equal(rv, rv2)
        worst_row = max(worst_row, rowmax_rel_err(cp, nz, nz2))
        assert np.abs(nz2 - nz).max() > 0.0
        assert parity_ratio(cp, nz, nz2, det["abs_sums"]) <= 1.0
        assert parity_ratio(cp, kg, kg2, detg["abs_sums"]) <= 1.0
        assert np.all(np.abs(nz2 - nz) <= SUM_TOL * EPS * det["abs_sums"])
    assert worst_row > ROW_TOL


def test_abs_sums_bound_the_values():
    m = decks.barrel_small(seed=2, n_circ=24, n_axial=12)
    cp, rv, nz, _, _, det = O.assemble_k(m, detail=True, abs_sums=True)
    a = det["abs_sums"]
    assert a.shape == nz.shape and np.all(a >= np.abs(nz) * (1 - 1e-15))
    assert det["t_elements"] >= 0.0 and det["t_sparse"] >= 0.0


def test_kg_rounding_scale_covers_the_equibiaxial_conditioning():
    """At an equibiaxial membrane stress the principal-transverse KG depends on a
    principal angle set by rounding noise: one-ulp perturbations of u move the
    oracle's own KG by a large fraction of the row max.  The rounding scale the
    parity bound uses must cover that (and stay tight in a generic state)."""
    from helpers import parity_ratio, rowmax_rel_err
    m = decks.plate_c1(n=6)
    x, y = m.coords[:, 0], m.coords[:, 1]
    rng = np.random.default_rng(0)
    for d, sensitive in ((0.0, True), (1e-9, True), (None, False)):
        u = np.zeros(6 * m.n_nodes)
        if d is None:                                   # uniaxial: a well-defined direction
            u[0::6] = 1e-3 * x
        else:
            u[0::6], u[1::6] = 1e-3 * x, 1e-3 * (1.0 + d) * y
        cp, rv, nz, det = O.assemble_kg(m, u, detail=True, abs_sums=True)
        worst_err = worst_ratio = 0.0
        for _ in range(3):
            up = u * (1.0 + 2.2e-16 * rng.standard_normal(u.size))
            nz2 = O.assemble_kg(m, up)[2]
            worst_err = max(worst_err, rowmax_rel_err(cp, nz, nz2))
            worst_ratio = max(worst_ratio, parity_ratio(cp, nz, nz2, det["abs_sums"]))
        if sensitive:
            assert worst_err > 1e-10, (d, worst_err)    # the reference formula is ill-conditioned here
        else:
            assert worst_err < 1e-12, worst_err
        assert worst_ratio <= 1.0, (d, worst_ratio)
