"""GPU SOL 101 output recovery (jfg_recover_stresses) against the oracle.

Each record column group (forces, moments, shears, fibre stresses, strains,
principal stress, corner forces and moments, von Mises; bar forces and section
stresses) must agree to 1e-9 of the group's largest oracle value, and the
status columns exactly.  Both sides solve the same small systems (K_bb, the
CTRIA3 macro condensation) in different orders, so agreement is to rounding,
not bitwise.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
from jf_2026_05_19_b200 import decks, native, solver

pytestmark = pytest.mark.gpu

TOL = 1e-9
SHELL_GROUPS = {"N": slice(0, 3), "M": slice(3, 6), "Q": slice(6, 8), "stress": slice(8, 14), "strain": slice(14, 20),
                "principal": slice(20, 21), "corner_N": slice(22, 34), "corner_M": slice(34, 46), "vm": slice(46, 48)}


def _tri_plate(n=4):
    """Flat plate: the first half of the squares CQUAD4, the rest split into CTRIA3."""
    p = decks.plate_c1(n=n, size=200.0)
    q = p.q4_nodes
    nh = q.shape[0] // 2
    rest = q[nh:]
    tri = np.concatenate([rest[:, [0, 1, 2]], rest[:, [0, 2, 3]]]).astype(np.int32)
    return dataclasses.replace(p, q4_nodes=q[:nh], q4_prop=p.q4_prop[:nh], t3_nodes=tri,
                               t3_prop=np.tile(p.q4_prop[0], (tri.shape[0], 1)))


def _decks():
    from decks_extra import skewed_plane
    thick = decks.plate_c1(n=8)
    thick = dataclasses.replace(thick, q4_prop=thick.q4_prop.copy())
    thick.q4_prop[:, 0] = 40.0  # phi2 saturated
    return {
        "barrel_small": decks.barrel_small(seed=2, n_circ=48, n_axial=12),
        "skewed_cd_frames": skewed_plane(seed=3),
        "thick_plate": thick,
        "mixed_plate": _tri_plate(),
    }


DECKS = _decks()


def _bar_points(m, seed=0):
    rng = np.random.default_rng(seed)
    nb = m.bar_nodes.shape[0]
    pts = rng.uniform(-30.0, 30.0, (nb, 9))
    pts[:, 8] = np.where(rng.random(nb) < 0.3, 1.0, -1.0)
    return pts


def _assert_records(sg, so, bg=None, bo=None):
    assert np.array_equal(sg[:, 21], so[:, 21])
    for name, cols in SHELL_GROUPS.items():
        ref = so[:, cols]
        if ref.size == 0:
            continue
        err = np.abs(sg[:, cols] - ref).max()
        assert err <= TOL * max(np.abs(ref).max(), 1e-300), (name, err, np.abs(ref).max())
    if bg is not None and bo.size:
        assert np.array_equal(bg[:, 17], bo[:, 17])
        for cols in (slice(0, 8), slice(8, 9), slice(9, 17)):
            ref = bo[:, cols]
            assert np.abs(bg[:, cols] - ref).max() <= TOL * max(np.abs(ref).max(), 1e-300)


@pytest.mark.parametrize("name", sorted(DECKS))
def test_records_match_oracle(name, cuda_device):
    m = DECKS[name]
    u = decks.smooth_displacement(m, seed=21)
    pts = _bar_points(m) if m.bar_nodes.shape[0] else None
    so, bo = O.recover(m, u, bar_points=pts)
    with native.GpuModel(m) as g:
        sg, bg = g.recover_stresses(u, pts)
    _assert_records(sg, so, bg, bo)


def test_pressure_deck_flag(cuda_device):
    m = decks.plate_c1(n=10, size=200.0)
    x, y = m.coords[:, 0] / 200.0, m.coords[:, 1] / 200.0
    u = np.zeros(m.ndof)
    u[2::6] = np.sin(np.pi * x) * np.sin(np.pi * y)
    u[3::6] = np.pi / 200.0 * np.sin(np.pi * x) * np.cos(np.pi * y)
    u[4::6] = -np.pi / 200.0 * np.cos(np.pi * x) * np.sin(np.pi * y)
    so, _ = O.recover(m, u, flags=O.RECOVER_PRESSURE_DECK)
    plain, _ = O.recover(m, u)
    assert not np.array_equal(so[:, 3:6], plain[:, 3:6])
    with native.GpuModel(m) as g:
        sg, _ = g.recover_stresses(u, pressure_deck=True)
    _assert_records(sg, so)


def test_device_form_and_thickness_update(cuda_device):
    """The device entry point gives the host entry point's bits; after a
    thickness update the records follow the new PSHELL thicknesses."""
    import torch
    m = DECKS["barrel_small"]
    u = decks.smooth_displacement(m, seed=22)
    pts = _bar_points(m, seed=3)
    nq, nt, nb = m.q4_nodes.shape[0], m.t3_nodes.shape[0], m.bar_nodes.shape[0]
    with native.GpuModel(m) as g:
        sh, bar = g.recover_stresses(u, pts)
        du = torch.from_numpy(u).cuda()
        dp = torch.from_numpy(pts).cuda()
        dsh = torch.empty((nq + nt, 48), dtype=torch.float64, device="cuda")
        dbar = torch.empty((nb, 18), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g.recover_stresses_device(du.data_ptr(), dp.data_ptr(), 0, dsh.data_ptr(), dbar.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(dsh.cpu().numpy(), sh) and np.array_equal(dbar.cpu().numpy(), bar)
        rng = np.random.default_rng(5)
        hq, ht = rng.uniform(0.8, 3.0, nq), rng.uniform(0.8, 3.0, nt)
        g.update_thickness(hq, ht)
        sg, _ = g.recover_stresses(u)
    so, _ = O.recover(m.with_thickness(hq, ht), u)
    _assert_records(sg, so)


def test_reference_style_results(cuda_device):
    """solver.recover_shell_stresses / recover_bar_stresses fill the reference's
    results dictionary from the records, keyed by element ID."""
    m = DECKS["barrel_small"]
    model = solver.model_dict_from_arrays(m)
    m2, id_map, X, node_R = solver.model_arrays_from_dict(model)
    u = decks.smooth_displacement(m2, seed=23)
    stresses, results = {}, {}
    solver.recover_shell_stresses(model, id_map, X, node_R, u, {}, stresses, results)
    solver.recover_bar_stresses(model, id_map, X, node_R, u, stresses, results)
    so, bo = O.recover(m2, u, bar_points=m2.bar_points)
    nq, nt, nb = m2.q4_nodes.shape[0], m2.t3_nodes.shape[0], m2.bar_nodes.shape[0]
    assert len(results["forces"]["quad4"]) == nq and len(results["forces"]["tria3"]) == nt
    assert len(results["forces_bilin"]["quad4"]) == 5 * nq and len(results["forces"]["cbar"]) == nb
    assert len(results["stresses"]["quad4"]) == nq and len(results["strains"]["tria3"]) == nt
    row = results["forces"]["quad4"][3]
    j = int(np.nonzero(m2.q4_eid == row["eid"])[0][0])
    scale = np.abs(so[:, 0:3]).max()
    assert abs(row["fx"] - so[j, 0]) <= TOL * scale
    assert abs(stresses[row["eid"]] - so[j, 20]) <= TOL * np.abs(so[:, 20]).max()
    st = results["stresses"]["tria3"][2]
    jt = nq + int(np.nonzero(m2.t3_eid == st["eid"])[0][0])
    assert st["z1"]["fiber_dist"] == -m2.t3_prop[jt - nq, 0] / 2
    assert abs(st["z2"]["von_mises"] - so[jt, 47]) <= TOL * np.abs(so[:, 47]).max()
    b = results["stresses"]["cbar"][1]
    jb = int(np.nonzero(m2.bar_eid == b["eid"])[0][0])
    assert abs(b["axial"] - bo[jb, 8]) <= TOL * np.abs(bo[:, 8]).max()
    assert stresses[b["eid"]] == abs(b["axial"])


def test_edge_cases(cuda_device):
    """A zero-length bar (skipped, status 0), a deck with shells only and one
    with bars only: records and status columns as the oracle's."""
    from decks_extra import skewed_plane
    m = DECKS["barrel_small"]
    z = DECKS["skewed_cd_frames"]  # carries one zero-length bar
    u = decks.smooth_displacement(z, seed=41)
    so, bo = O.recover(z, u)
    with native.GpuModel(z) as g:
        sg, bg = g.recover_stresses(u)
    assert (bo[:, 17] == 0).sum() == 1 and np.array_equal(bg[:, 17], bo[:, 17])
    _assert_records(sg, so, bg, bo)
    shells = dataclasses.replace(skewed_plane(seed=5), bar_nodes=np.zeros((0, 2), np.int32),
                                 bar_prop=np.zeros((0, 18)), bar_pin=np.zeros((0, 2), np.int32))
    u = decks.smooth_displacement(shells, seed=42)
    so, bo = O.recover(shells, u)
    with native.GpuModel(shells) as g:
        sg, bg = g.recover_stresses(u)
    assert bg.shape == (0, 18)
    _assert_records(sg, so)
    bars = dataclasses.replace(m, q4_nodes=np.zeros((0, 4), np.int32), q4_prop=np.zeros((0, 7)),
                               t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, 7)))
    u = decks.smooth_displacement(bars, seed=43)
    so, bo = O.recover(bars, u, bar_points=_bar_points(bars))
    with native.GpuModel(bars) as g:
        sg, bg = g.recover_stresses(u, _bar_points(bars))
    assert sg.shape == (0, 48)
    _assert_records(sg, so, bg, bo)
