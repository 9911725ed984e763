"""CPU tests of the host-side mirror of the reference interface and helpers."""
import numpy as np

from jf_2026_05_19_b200 import decks, roofline, solver


def test_model_dict_round_trip():
    from decks_extra import skewed_plane
    m = skewed_plane(seed=2)
    model = solver.model_dict_from_arrays(m)
    m2, id_map, coords, node_R = solver.model_arrays_from_dict(model)
    assert np.allclose(m2.coords, m.coords) and np.array_equal(m2.q4_nodes, m.q4_nodes)
    assert np.array_equal(m2.t3_nodes, m.t3_nodes) and np.array_equal(m2.bar_nodes, m.bar_nodes)
    assert np.allclose(m2.q4_prop, m.q4_prop, rtol=1e-15) and np.allclose(m2.t3_prop, m.t3_prop, rtol=1e-15)
    assert np.allclose(m2.bar_prop, m.bar_prop, rtol=1e-15)
    assert np.array_equal(m2.rbe2_slaves, m.rbe2_slaves) and np.array_equal(m2.rbe2_cm, m.rbe2_cm)
    assert np.allclose(m2.node_R, m.node_R)
    assert id_map[int(m.node_ids[0])] == 1 and len(node_R) == m.n_nodes


def test_unsupported_cards_refused():
    model = solver.model_dict_from_arrays(decks.plate_c1(n=2))
    model["RBE3s"] = {"1": {}}
    try:
        solver.model_arrays_from_dict(model)
    except NotImplementedError:
        return
    raise AssertionError("RBE3 must be refused")


def test_roofline_constants():
    c = {"quad4": 1, "tria3": 0, "bar": 0}
    assert roofline.flops_per_step(c) == 2 * (30_603 + 31_216)
    assert roofline.bytes_per_step(c, 0) == 4 * (24 + 48 + 4) + 64 + 2 * 576 * 4


def test_barrel_generator_counts():
    m = decks.barrel_c4(n_circ=72, n_axial=24, ring_every=6, longeron_every=6)
    c = m.counts()
    assert c["quad4"] + c["tria3"] // 2 == 72 * 24
    assert c["rbe2_slaves"] == 72


def test_build_hash_covers_every_included_file():
    """The stale-library guard hashes every file the library is compiled from:
    each csrc header and the public header are reached through #include."""
    import glob
    import os
    from jf_2026_05_19_b200 import build
    d = set(build.deps())
    for p in glob.glob(os.path.join(build.CSRC, "*.cuh")) + glob.glob(os.path.join(build.CSRC, "*.cu")):
        assert os.path.normpath(p) in d, p
    assert os.path.join(build.ROOT, "include", "jfem_gpu.h") in d
