"""GPU parity: the CUDA C-ABI path against the CPU oracle on the same inputs.

Bars: CSC pattern (colptr/rowval) bit-exact; every K and KG nonzero within
ROW_TOL = 1e-12 of its row's max magnitude, or within SUM_TOL * eps times the
sum of the magnitudes of the terms it adds up where that is larger (rows of an
RBE2 master, see tests/helpers.py); max_elem_stiff and orig_diag within 1e-12
relative; the first buckling load factors within 1e-9.
"""
import dataclasses
import os

import numpy as np
import pytest

import oracle as O
from helpers import LAMBDA_TOL, ROW_TOL, load_factors, parity_ratio, rowmax_rel_err, static_solution, to_csc
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.npz")


def _decks():
    from decks_extra import (bars_only_barrel, plate_axis_rbe2, single_cell_tria3, single_quad4, skewed_plane,
                             with_unused_nodes)
    return {
        "bars_only_barrel": bars_only_barrel(),
        "single_quad4": single_quad4(),
        "single_cell_tria3": single_cell_tria3(),
        # full-size stiffened panel (18k CQUAD4, 4k CTRIA3, 2k CBAR) without
        # stringer offsets, so KG is defined (test_full_size_panel covers offsets)
        "panel_c2_no_offset": decks.stiffened_panel_c2(seed=0, stringer_offset=0.0),
        # the 480 x 96 barrel (64.6k elements) with the bench barrel's element mix
        "barrel_480x96": decks.barrel_c4(seed=0, n_circ=480, n_axial=96, ring_every=8, longeron_every=7,
                                         name="barrel_480x96"),
        # partial-CM RBE2 with an axis offset: the master's rows hold different
        # columns, which the block path avoids by treating masters as special
        "plate_axis_rbe2": plate_axis_rbe2(),
        "plate_40x40": decks.plate_c1(),
        "panel_no_offset": decks.stiffened_panel_c2(seed=1, lx=300.0, ly=200.0, stringer_every=4, stringer_offset=0.0),
        "barrel_small": decks.barrel_small(seed=2, n_circ=72, n_axial=24),
        "skewed_cd_frames": skewed_plane(seed=3),
        "skewed_unused_nodes": with_unused_nodes(skewed_plane(seed=4, cd_frames=False)),
        "membrane_only": dataclasses.replace(decks.plate_c1(n=10), q4_prop=np.tile(
            decks.shell_prop_row(1.5, 70000.0, 0.3, br=0.0), (100, 1))),
        "k6rot_tria_only": dataclasses.replace(skewed_plane(seed=5, tri_frac=1.0), k6rot=0.0),
    }


DECKS = _decks()


def _check_k(g, m):
    cp, rv = g.pattern()
    ocp, orv, onz, omx, odg, det = O.assemble_k(m, detail=True, abs_sums=True)
    assert np.array_equal(cp, ocp), "colptr differs"
    assert np.array_equal(rv, orv), "rowval differs"
    nz, mx, dg = g.assemble_k()
    assert parity_ratio(cp, onz, nz, det["abs_sums"]) <= 1.0, rowmax_rel_err(cp, onz, nz)
    assert abs(mx - omx) <= 1e-12 * abs(omx)
    scale = max(np.abs(odg).max(), 1.0)
    assert np.abs(dg - odg).max() <= 1e-12 * scale
    return cp, nz


def _check_model(m, cuda_device, seed=7):
    g = native.GpuModel(m)
    try:
        cp, nz = _check_k(g, m)
        u = decks.smooth_displacement(m, seed=seed)
        _, _, ognz, det = O.assemble_kg(m, u, detail=True, abs_sums=True)
        gnz = g.assemble_kg(u)
        assert parity_ratio(cp, ognz, gnz, det["abs_sums"]) <= 1.0, rowmax_rel_err(cp, ognz, gnz)
        return g, nz, gnz, u
    except Exception:
        g.close()
        raise


@pytest.mark.parametrize("name", sorted(DECKS))
def test_k_kg_match_oracle(name, cuda_device):
    g, *_ = _check_model(DECKS[name], cuda_device)
    g.close()


def test_full_size_panel_with_offsets(cuda_device):
    """The full stiffened panel as specified (12 mm stringer offsets): K matches,
    and KG raises like the reference does for offset bars."""
    m = decks.stiffened_panel_c2(seed=0)
    with native.GpuModel(m) as g:
        _check_k(g, m)
        with pytest.raises(native.JfgError) as e:
            g.assemble_kg(np.zeros(g.ndof))
        assert e.value.status == 7


def test_golden_fixtures(cuda_device):
    import golden.make_golden as mg
    gold = np.load(GOLD)
    for name, m in mg.golden_decks().items():
        with native.GpuModel(m) as g:
            cp, rv = g.pattern()
            assert np.array_equal(cp, gold[f"{name}__colptr"]) and np.array_equal(rv, gold[f"{name}__rowval"])
            nz, mx, dg = g.assemble_k()
            assert rowmax_rel_err(cp, gold[f"{name}__k"], nz) <= ROW_TOL
            assert rowmax_rel_err(cp, gold[f"{name}__kg"], g.assemble_kg(gold[f"{name}__u"])) <= ROW_TOL


def test_constraint_map_matches(cuda_device):
    m = DECKS["barrel_small"]
    with native.GpuModel(m) as g:
        a = g.constraint_map()
        b = O.constraint_map(m)
        for x, y in zip(a[:3], b[:3]):
            assert np.array_equal(x, y)
        assert np.array_equal(a[3], b[3])


def test_bitwise_repeatable(cuda_device):
    m = DECKS["barrel_small"]
    u = decks.smooth_displacement(m, seed=1)
    with native.GpuModel(m) as g:
        k1, _, _ = g.assemble_k()
        kg1 = g.assemble_kg(u)
        k2, _, _ = g.assemble_k()
        kg2 = g.assemble_kg(u)
        assert np.array_equal(k1, k2) and np.array_equal(kg1, kg2)
    with native.GpuModel(m) as g2:    # a fresh handle gives the same bits
        assert np.array_equal(g2.assemble_k()[0], k1)


def test_device_api_matches_host_api(cuda_device):
    import torch
    m = DECKS["panel_no_offset"]
    u = decks.smooth_displacement(m, seed=4)
    with native.GpuModel(m) as g:
        nz, mx, dg = g.assemble_k()
        kg = g.assemble_kg(u)
        dnz = torch.empty(g.nnz, dtype=torch.float64, device="cuda")
        dkg = torch.empty(g.nnz, dtype=torch.float64, device="cuda")
        ddg = torch.empty(g.ndof, dtype=torch.float64, device="cuda")
        dmx = torch.zeros(1, dtype=torch.float64, device="cuda")
        du = torch.from_numpy(u).cuda()
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        g.set_stream(s.cuda_stream)
        g.assemble_k_device(dnz.data_ptr(), dmx.data_ptr(), ddg.data_ptr())
        g.assemble_kg_device(du.data_ptr(), dkg.data_ptr())
        s.synchronize()
        assert np.array_equal(dnz.cpu().numpy(), nz)
        assert np.array_equal(dkg.cpu().numpy(), kg)
        assert np.array_equal(ddg.cpu().numpy(), dg) and float(dmx.item()) == mx
        g.set_stream(0)


def test_thickness_update_equals_fresh_model(cuda_device):
    m = DECKS["panel_no_offset"]
    rng = np.random.default_rng(9)
    hq = rng.uniform(1.0, 4.0, m.q4_nodes.shape[0])
    ht = rng.uniform(1.0, 4.0, m.t3_nodes.shape[0])
    m2 = m.with_thickness(hq, ht)
    u = decks.smooth_displacement(m, seed=2)
    with native.GpuModel(m) as g, native.GpuModel(m2) as g2:
        g.update_thickness(hq, ht)
        assert np.array_equal(g.assemble_k()[0], g2.assemble_k()[0])
        assert np.array_equal(g.assemble_kg(u), g2.assemble_kg(u))


def test_kg_offset_bars_raise_like_reference(cuda_device):
    m = decks.stiffened_panel_c2(lx=100.0, ly=60.0, stringer_every=2, stringer_offset=12.0)
    with native.GpuModel(m) as g:
        cp, rv = g.pattern()
        ocp, orv, onz, _, _ = O.assemble_k(m)
        assert np.array_equal(rv, orv)
        assert rowmax_rel_err(cp, onz, g.assemble_k()[0]) <= ROW_TOL   # K with offsets matches
        with pytest.raises(native.JfgError) as e:
            g.assemble_kg(np.zeros(g.ndof))
        assert e.value.status == 7


def test_unsupported_and_invalid_inputs(cuda_device):
    from decks_extra import skewed_plane, warped
    m = skewed_plane(seed=6)
    for bad, status in [(warped(m), 2), (dataclasses.replace(m, param_snorm=10.0), 2)]:
        with pytest.raises(native.JfgError) as e:
            native.GpuModel(bad)
        assert e.value.status == status
    q = m.q4_nodes.copy(); q[0, 0] = m.n_nodes + 5
    with pytest.raises(native.JfgError) as e:
        native.GpuModel(dataclasses.replace(m, q4_nodes=q))
    assert e.value.status == 1
    with native.GpuModel(m) as g:
        with pytest.raises(ValueError):
            g.assemble_kg(np.zeros(3))


def test_plate_load_factors_match(cuda_device):
    """SOL 105 consumer fed oracle vs GPU matrices: first 10 load factors within 1e-9."""
    m = decks.plate_c1()
    ocp, orv, onz, _, _ = O.assemble_k(m)
    Ko = to_csc(ocp, orv, onz, m.ndof)
    u, free = static_solution(m, Ko, O.constraint_map(m))
    _, _, ognz = O.assemble_kg(m, u)
    lam_o = load_factors(Ko, to_csc(ocp, orv, ognz, m.ndof), free, k=10)
    with native.GpuModel(m) as g:
        cp, rv = g.pattern()
        Kg_ = to_csc(cp, rv, g.assemble_k()[0], m.ndof)
        lam_g = load_factors(Kg_, to_csc(cp, rv, g.assemble_kg(u), m.ndof), free, k=10)
    assert lam_o.size == 10 and lam_g.size == 10
    assert np.all(np.abs(lam_g - lam_o) <= LAMBDA_TOL * np.abs(lam_o))
    D = 70000 * 8 / (12 * (1 - 0.33 ** 2))
    assert abs(lam_g[0] / (4 * np.pi ** 2 * D / 400.0 ** 2) - 1) < 0.01


def test_barrel_load_factors_match(cuda_device):
    """The barrel with bars and the RBE2 end ring: first 10 load factors within 1e-9."""
    m = decks.barrel_small(seed=1, n_circ=48, n_axial=12)
    ocp, orv, onz, _, _ = O.assemble_k(m)
    Ko = to_csc(ocp, orv, onz, m.ndof)
    cmap = O.constraint_map(m)
    u, free = static_solution(m, Ko, cmap)
    _, _, ognz = O.assemble_kg(m, u)
    lam_o = load_factors(Ko, to_csc(ocp, orv, ognz, m.ndof), free, k=10, sigma=0.0)
    with native.GpuModel(m) as g:
        cp, rv = g.pattern()
        Kg_ = to_csc(cp, rv, g.assemble_k()[0], m.ndof)
        lam_g = load_factors(Kg_, to_csc(cp, rv, g.assemble_kg(u), m.ndof), free, k=10, sigma=0.0)
    assert lam_o.size == 10 and lam_g.size == 10
    assert np.all(np.abs(lam_g - lam_o) <= LAMBDA_TOL * np.abs(lam_o))


def test_reference_interface_mirror(cuda_device):
    """assemble_stiffness / assemble_geometric_stiffness on a reference-style model dictionary."""
    from jf_2026_05_19_b200 import solver
    m = DECKS["barrel_small"]
    model = solver.model_dict_from_arrays(m)
    K, id_map, X, ndof, node_R, mx, rbe3_map, snorm, diag = solver.assemble_stiffness(model, membrane_incomp=False)
    ocp, orv, onz, omx, odg = O.assemble_k(m)
    Kc = K.tocsc()
    assert np.array_equal(Kc.indptr + 1, ocp) and np.array_equal(Kc.indices + 1, orv)
    assert rowmax_rel_err(ocp, onz, Kc.data) <= ROW_TOL and abs(mx - omx) <= 1e-12 * omx
    assert ndof == m.ndof and snorm == {} and len(rbe3_map) == 72 * 6
    u = decks.smooth_displacement(m, seed=5)
    Kg = solver.assemble_geometric_stiffness(model, id_map, X, node_R, ndof, u, snorm, rbe3_map).tocsc()
    _, _, ognz = O.assemble_kg(m, u)
    assert rowmax_rel_err(ocp, ognz, Kg.data) <= ROW_TOL
    # a thickness update in the dictionary is picked up (handle reused, properties updated)
    for p in model["PSHELLs"].values():
        p["T"] *= 1.5
    K2 = solver.assemble_stiffness(model)[0].tocsc()
    m2 = m.with_thickness(m.q4_prop[:, 0] * 1.5, m.t3_prop[:, 0] * 1.5)
    _, _, onz2, _, _ = O.assemble_k(m2)
    assert rowmax_rel_err(ocp, onz2, K2.data) <= ROW_TOL
    with pytest.raises(NotImplementedError):
        solver.assemble_stiffness(model, shear_center_only=True)
    solver.release()
