"""Oracle checks of the shell-thickness sensitivity element (CPU, not reference-pinned).

The oracle's dK/dh of stiffness_quad4_generic is the closed form of what the
reference's forward-mode AD returns (dKdx.jl:218-230); here it is pinned
against central differences of the oracle's own K(h) on both branches of the
phi2 shear factor.  The CTRIA3 derivative is forward-mode differentiation
(dual numbers) of the oracle's stiffness_tria3_generic, as the reference's
forward AD is; it is pinned the same way.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
from jf_2026_05_19_b200 import decks


def _quad(seed, size=20.0):
    rng = np.random.default_rng(seed)
    base = np.array([[-1.0, -1.0], [1.0, -1.0], [1.0, 1.0], [-1.0, 1.0]]) * (size / 2)
    lc = base + rng.uniform(-0.15, 0.15, (4, 2)) * size
    return lc - lc.mean(0)


def _tri(seed, size=20.0):
    rng = np.random.default_rng(seed)
    lc = np.array([[0.0, 0.0], [size, 0.0], [0.3 * size, 0.8 * size]]) + rng.uniform(-0.1, 0.1, (3, 2)) * size
    return lc - lc.mean(0)


def _richardson(fun, h, d):
    D1 = (fun(h + d) - fun(h - d)) / (2 * d)
    D2 = (fun(h + d / 2) - fun(h - d / 2)) / d
    return (4 * D2 - D1) / 3


@pytest.mark.parametrize("h", [1.5, 9.0])  # phi2 = 10 h^2 / (4 |det Jc|): < 1 at 1.5, saturated at 9
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_q4_generic_dkdh_matches_central_difference(h, seed):
    lc, E, nu = _quad(seed), 70000.0, 0.33
    K, dK = O.q4_generic_local(lc, E, nu, h)
    fd = _richardson(lambda x: O.q4_generic_local(lc, E, nu, x)[0], h, h / 200)
    assert np.abs(K - K.T).max() <= 1e-9 * np.abs(K).max()
    assert np.abs(dK - fd).max() <= 1e-7 * np.abs(dK).max()


@pytest.mark.parametrize("h", [0.5, 2.0, 6.0])
@pytest.mark.parametrize("seed", [0, 3])
def test_t3_generic_dkdh_matches_central_difference(h, seed):
    lc, E, nu = _tri(seed), 70000.0, 0.3
    _, dK = O.t3_generic_local(lc, E, nu, h)
    fd = _richardson(lambda x: O.t3_generic_local(lc, E, nu, x)[0], h, h / 256)
    assert np.abs(dK - fd).max() <= 1e-9 * np.abs(dK).max()


def test_t3_generic_is_the_assembly_tria_at_default_properties():
    """stiffness_tria3_generic is stiffness_tria3_matrices_generic with bend ratio 1,
    TS/T 5/6, G = E / 2(1 + nu) and K6ROT 100, i.e. the assembly's CTRIA3 for such a deck."""
    lc, E, nu, h = _tri(5), 70000.0, 0.33, 2.5
    K, _ = O.t3_generic_local(lc, E, nu, h)
    Ka = O.t3_local(lc, decks.shell_prop_row(h, E, nu), 100.0)
    assert np.allclose(K, Ka, rtol=1e-13, atol=1e-13 * np.abs(K).max())


def test_model_contraction_and_pseudo_load_agree():
    """u' (dK/dh u over all elements) equals the sum of the per-element u' dK_e/dh u."""
    m = decks.barrel_small(seed=2, n_circ=24, n_axial=8)
    assert m.t3_nodes.shape[0] > 0
    u = decks.smooth_displacement(m, seed=4)
    cq, ct, load = O.dkdh(m, a=u, b=u, u=u)
    total = cq.sum() + ct.sum()
    assert abs(u @ load - total) <= 1e-11 * (np.abs(cq).sum() + np.abs(ct).sum())
    v = decks.smooth_displacement(m, seed=5)
    cq2, ct2, _ = O.dkdh(m, a=u, b=v)
    cq3, ct3, _ = O.dkdh(m, a=v, b=u)
    assert np.allclose(cq2, cq3, rtol=1e-9, atol=1e-12 * np.abs(cq2).max())
    assert np.allclose(ct2, ct3, rtol=1e-7, atol=1e-9 * np.abs(ct2).max())


def test_pseudo_load_is_local_to_the_mask():
    m = decks.plate_c1(n=6)
    u = decks.smooth_displacement(m, seed=1)
    mask = np.zeros(m.q4_nodes.shape[0], np.uint8)
    mask[7] = 1
    _, _, load = O.dkdh(m, u=u, mask_q4=mask, mask_t3=np.zeros(0, np.uint8))
    touched = np.zeros(load.size, bool)
    for n in m.q4_nodes[7]:
        touched[6 * n:6 * n + 6] = True
    assert np.abs(load[~touched]).max() == 0.0 and np.abs(load[touched]).max() > 0.0


def test_membrane_field_sensitivity_does_not_depend_on_thickness():
    """With in-plane displacements only the membrane and drilling terms act; both are
    linear in h, so u' dK/dh u is the same at h and 2h."""
    m = decks.plate_c1(n=4)
    rng = np.random.default_rng(0)
    u = np.zeros(6 * m.coords.shape[0])
    u[0::6] = rng.normal(size=m.coords.shape[0]) * 1e-3
    u[1::6] = rng.normal(size=m.coords.shape[0]) * 1e-3
    c1, _, _ = O.dkdh(m, a=u, b=u)
    m2 = dataclasses.replace(m, q4_prop=m.q4_prop.copy())
    m2.q4_prop[:, 0] *= 2.0
    c2, _, _ = O.dkdh(m2, a=u, b=u)
    assert np.allclose(c2, c1, rtol=1e-10)


def test_kg_contractions_sum_to_assembled_quadratic_form():
    """sum_e phi' KG_e phi equals phi' KG phi of the assembled KG on a shell deck
    without RBE2 (no constraint redistribution, no bars); KG_e is linear in the thickness at fixed u,
    so c_e / h_e is phi' dKG_e/dh phi."""
    import dataclasses
    from decks_extra import skewed_plane
    m = skewed_plane(seed=4)
    m = dataclasses.replace(m, rbe2_master=m.rbe2_master[:0], rbe2_cm=m.rbe2_cm[:0],
                            rbe2_slave_ptr=m.rbe2_slave_ptr[:1], rbe2_slaves=m.rbe2_slaves[:0],
                            bar_nodes=m.bar_nodes[:0], bar_prop=m.bar_prop[:0], bar_pin=m.bar_pin[:0])
    u = decks.smooth_displacement(m, seed=5)
    phi = decks.smooth_displacement(m, seed=6)
    cq, ct = O.kg_contract(m, u, phi, phi)
    colptr, rowval, nz = O.assemble_kg(m, u)
    K = O.to_scipy(colptr, rowval, nz, m.ndof)
    total = phi @ (K @ phi)
    assert abs(cq.sum() + ct.sum() - total) <= 1e-10 * (np.abs(cq).sum() + np.abs(ct).sum())
    m2 = m.with_thickness(2.0 * m.q4_prop[:, 0], 2.0 * m.t3_prop[:, 0])
    cq2, ct2 = O.kg_contract(m2, u, phi, phi)
    assert np.allclose(cq2, 2.0 * cq, rtol=1e-11, atol=1e-14 * np.abs(cq).max())
    assert np.allclose(ct2, 2.0 * ct, rtol=1e-11, atol=1e-14 * np.abs(ct).max())
