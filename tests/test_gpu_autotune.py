"""Launch-shape autotuner: every candidate shape gives the same bits, the
tuner keeps a legal shape, and its stored choice is read back per size class."""
import numpy as np
import pytest

from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu

SHAPES = [dict(quad4_warps=q, tria3_k_warps=t, tria3_kg_threads=n, bar_k_threads=n, bar_kg_threads=n)
          for q, t, n in ((4, 4, 128), (8, 2, 32), (8, 4, 64), (4, 2, 64))]


def test_every_launch_shape_gives_the_same_bits(cuda_device):
    m = decks.barrel_small(seed=6, n_circ=48, n_axial=16)   # CQUAD4 + CTRIA3 + bars + RBE2
    u = decks.smooth_displacement(m, seed=2)
    with native.GpuModel(m) as g:
        ref = None
        for cfg in SHAPES:
            assert g.launch_config(cfg) == cfg
            k, mx, dg = g.assemble_k()
            kg = g.assemble_kg(u)
            if ref is None:
                ref = (k, mx, dg, kg)
            else:
                assert np.array_equal(k, ref[0]) and mx == ref[1] and np.array_equal(dg, ref[2]), cfg
                assert np.array_equal(kg, ref[3]), cfg
        with pytest.raises(native.JfgError):
            g.launch_config(dict(SHAPES[0], quad4_warps=5))


def test_autotune_choice_is_stored_and_read_back(cuda_device, tmp_path, monkeypatch):
    monkeypatch.setenv("JFG_TUNE_FILE", str(tmp_path / "tune.txt"))
    m = decks.barrel_small(seed=6, n_circ=48, n_axial=16)
    u = decks.smooth_displacement(m, seed=2)
    with native.GpuModel(m) as g:
        k0 = g.assemble_k()[0]
        cfg = g.autotune(read=False, write=True)
        assert cfg["quad4_warps"] in (4, 8) and cfg["tria3_k_warps"] in (2, 4)
        assert all(cfg[k] in (32, 64, 128) for k in ("tria3_kg_threads", "bar_k_threads", "bar_kg_threads"))
        assert np.array_equal(g.assemble_k()[0], k0)           # tuned shape, same bits
    lines = (tmp_path / "tune.txt").read_text().split("\n")
    assert sum(1 for x in lines if x.strip()) == 5
    with native.GpuModel(m) as g2:
        g2.launch_config(SHAPES[3] if cfg != SHAPES[3] else SHAPES[1])
        assert g2.autotune(read=True, write=False) == cfg    # read back, no timing
        assert np.array_equal(g2.assemble_kg(u), g2.assemble_kg(u))
