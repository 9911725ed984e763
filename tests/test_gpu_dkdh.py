"""GPU shell-thickness sensitivities (dK/dh contractions and pseudo-load) against the oracle.

CQUAD4: both sides evaluate the closed-form derivative.  CTRIA3: the oracle
differentiates forward-mode (dual numbers) and the GPU kernel evaluates the
closed form of the same derivative.  Both agree to rounding: 1e-10 of the
largest value.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu

Q4_TOL, T3_TOL = 1e-10, 1e-10


def _decks():
    from decks_extra import skewed_plane
    thick = decks.plate_c1(n=8)
    thick = dataclasses.replace(thick, q4_prop=thick.q4_prop.copy())
    thick.q4_prop[:, 0] = 40.0  # phi2 saturated: shear term linear in h
    return {
        "barrel_small": decks.barrel_small(seed=2, n_circ=48, n_axial=12),
        "skewed_cd_frames": skewed_plane(seed=3),
        "thick_plate": thick,
    }


DECKS = _decks()


def _close(got, ref, tol):
    if ref.size == 0:
        return got.size == 0
    return np.abs(got - ref).max() <= tol * max(np.abs(ref).max(), 1e-300)


@pytest.mark.parametrize("name", sorted(DECKS))
def test_contractions_match_oracle(name, cuda_device):
    m = DECKS[name]
    a = decks.smooth_displacement(m, seed=11)
    b = decks.smooth_displacement(m, seed=12)
    oq, ot, _ = O.dkdh(m, a=a, b=b)
    with native.GpuModel(m) as g:
        cq, ct = g.dkdh_contract(a, b)
    assert _close(cq, oq, Q4_TOL), np.abs(cq - oq).max()
    assert _close(ct, ot, T3_TOL), np.abs(ct - ot).max()


@pytest.mark.parametrize("name", sorted(DECKS))
def test_pseudo_load_matches_oracle(name, cuda_device):
    m = DECKS[name]
    u = decks.smooth_displacement(m, seed=13)
    rng = np.random.default_rng(7)
    nq, nt = m.q4_nodes.shape[0], m.t3_nodes.shape[0]
    mq = (rng.random(nq) < 0.4).astype(np.uint8)
    mt = (rng.random(nt) < 0.6).astype(np.uint8)
    with native.GpuModel(m) as g:
        # CQUAD4 group only: closed form on both sides
        _, _, ol = O.dkdh(m, u=u, mask_q4=mq, mask_t3=np.zeros(nt, np.uint8))
        gl = g.dkdh_load(u, mq, np.zeros(nt, np.uint8))
        assert _close(gl, ol, Q4_TOL)
        # mixed group, and every element (null masks)
        _, _, ol = O.dkdh(m, u=u, mask_q4=mq, mask_t3=mt)
        assert _close(g.dkdh_load(u, mq, mt), ol, T3_TOL)
        _, _, ol = O.dkdh(m, u=u)
        assert _close(g.dkdh_load(u), ol, T3_TOL)


def test_load_and_contraction_agree_and_device_forms_match(cuda_device):
    """u' (dK/dh u) equals the summed contractions u' dK_e/dh u; the device entry
    points give the host entry points' bits; repeated calls are bitwise repeatable."""
    import torch
    m = DECKS["barrel_small"]
    u = decks.smooth_displacement(m, seed=14)
    with native.GpuModel(m) as g:
        cq, ct = g.dkdh_contract(u, u)
        load = g.dkdh_load(u)
        total = cq.sum() + ct.sum()
        assert abs(u @ load - total) <= 1e-10 * (np.abs(cq).sum() + np.abs(ct).sum())
        assert np.array_equal(load, g.dkdh_load(u))
        du = torch.from_numpy(u).cuda()
        dcq = torch.empty(cq.size, dtype=torch.float64, device="cuda")
        dct = torch.empty(ct.size, dtype=torch.float64, device="cuda")
        dl = torch.empty(u.size, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g.dkdh_contract_device(du.data_ptr(), du.data_ptr(), dcq.data_ptr(), dct.data_ptr())
        g.dkdh_load_device(du.data_ptr(), None, None, dl.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(dcq.cpu().numpy(), cq) and np.array_equal(dct.cpu().numpy(), ct)
        assert np.array_equal(dl.cpu().numpy(), load)


def test_sensitivities_follow_thickness_updates(cuda_device):
    """After jfg_update_properties (the optimiser's thickness step) the contractions use the
    new thicknesses, as a handle built from the updated deck does."""
    m = DECKS["barrel_small"]
    rng = np.random.default_rng(21)
    hq = rng.uniform(0.8, 3.0, m.q4_nodes.shape[0])
    ht = rng.uniform(0.8, 3.0, m.t3_nodes.shape[0])
    u = decks.smooth_displacement(m, seed=22)
    oq, ot, _ = O.dkdh(m.with_thickness(hq, ht), a=u, b=u)
    with native.GpuModel(m) as g:
        g.dkdh_contract(u, u)
        g.update_thickness(hq, ht)
        cq, ct = g.dkdh_contract(u, u)
    assert _close(cq, oq, Q4_TOL) and _close(ct, ot, T3_TOL)


@pytest.mark.parametrize("name", sorted(DECKS))
def test_kg_contractions_match_oracle(name, cuda_device):
    """Per-element phi' KG_e phi (jfg_kg_contract) against the oracle's element
    KG triplets; the call does not count as a KG assembly in the timing."""
    m = DECKS[name]
    u = decks.smooth_displacement(m, seed=31)
    phi = decks.smooth_displacement(m, seed=32)
    oq, ot = O.kg_contract(m, u, phi, phi)
    with native.GpuModel(m) as g:
        cq, ct = g.kg_contract(u, phi, phi)
        _, n_kg = g.timing_accumulated("kg")
    assert n_kg == 0
    assert _close(cq, oq, 1e-10), np.abs(cq - oq).max()
    assert _close(ct, ot, 1e-10), np.abs(ct - ot).max()
