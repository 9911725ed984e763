"""The persistent CQUAD4 + block-reduction kernel (jfg_persistent_config).

It computes the same slots as the separate kernels and sums every block in
the same slot order, so K, max |K_e|, orig_diag and KG must equal the
separate path's bit for bit, for any chunk size (several chunks per mesh,
blocks spanning chunks) and either CQUAD4 CTA width.  The separate path's
values are the ones the parity tests compare with the oracle.
"""
import dataclasses

import numpy as np
import pytest

from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu


def _decks():
    from decks_extra import skewed_plane
    return [
        decks.barrel_small(seed=4, n_circ=48, n_axial=16),                   # CQUAD4 + CTRIA3 + bars + RBE2
        dataclasses.replace(skewed_plane(seed=7), k6rot=100.0),              # CD frames, membrane-only PSHELLs
        decks.stiffened_panel_c2(seed=2, lx=200.0, ly=120.0, stringer_every=4, stringer_offset=0.0),
        decks.plate_c1(n=12),
    ]


def _assemble(g, m, u):
    k, mx, dg = g.assemble_k()
    kg = g.assemble_kg(u)
    return k, mx, dg, kg


@pytest.mark.parametrize("deck", range(4))
def test_persistent_equals_separate_bitwise(cuda_device, deck):
    m = _decks()[deck]
    u = decks.smooth_displacement(m, seed=40 + deck)
    with native.GpuModel(m) as g:
        assert g.persistent()["persistent"] == 0            # off by default
        ref = _assemble(g, m, u)
        for warps in (4, 8):
            cfg = dict(g.launch_config(), quad4_warps=warps)
            g.launch_config(cfg)
            for chunk in (24, 96, 9600):
                s = g.persistent(True, chunk)
                assert s == {"persistent": 1, "chunk_quad4": chunk}
                for call in range(2):                       # the second call reuses the task list
                    got = _assemble(g, m, u)
                    tag = f"deck {deck} warps {warps} chunk {chunk} call {call}"
                    assert np.array_equal(got[0], ref[0]), "K " + tag
                    assert got[1] == ref[1], "max " + tag
                    assert np.array_equal(got[2], ref[2]), "orig_diag " + tag
                    assert np.array_equal(got[3], ref[3]), "KG " + tag
                g.persistent(False)
                assert np.array_equal(_assemble(g, m, u)[0], ref[0])


def test_persistent_device_calls_replay_from_a_cuda_graph(cuda_device):
    """Once a first call has built the task list, device K and KG calls on the
    persistent kernel capture into a CUDA graph and replay to the same bits."""
    import torch
    m = decks.barrel_small(seed=5, n_circ=48, n_axial=12)
    u = decks.smooth_displacement(m, seed=3)
    with native.GpuModel(m) as g:
        ref = _assemble(g, m, u)
        g.persistent(True, 48)
        du = torch.from_numpy(u).cuda()
        nzk, nzg = (torch.full((g.nnz,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2))
        mx = torch.zeros(1, dtype=torch.float64, device="cuda")
        dg = torch.zeros(g.ndof, dtype=torch.float64, device="cuda")
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        g.set_stream(s.cuda_stream)
        g.assemble_k_device(nzk.data_ptr(), mx.data_ptr(), dg.data_ptr())    # builds the task list
        g.assemble_kg_device(du.data_ptr(), nzg.data_ptr())
        s.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            g.assemble_k_device(nzk.data_ptr(), mx.data_ptr(), dg.data_ptr())
            g.assemble_kg_device(du.data_ptr(), nzg.data_ptr())
        for _ in range(2):
            nzk.fill_(float("nan")); nzg.fill_(float("nan")); dg.fill_(float("nan"))
            graph.replay()
            torch.cuda.synchronize()
            assert np.array_equal(nzk.cpu().numpy(), ref[0])
            assert float(mx.item()) == ref[1]
            assert np.array_equal(dg.cpu().numpy(), ref[2])
            assert np.array_equal(nzg.cpu().numpy(), ref[3])
        g.set_stream(0)
        del graph


def test_persistent_settings_and_fallbacks(cuda_device):
    from decks_extra import bars_only_barrel
    m = decks.plate_c1(n=6)
    with native.GpuModel(m) as g:
        with pytest.raises(native.JfgError) as e:
            g.persistent(True, 25)                          # not a multiple of 24
        assert e.value.status == 1
        assert g.persistent() == {"persistent": 0, "chunk_quad4": 9600}
    b = bars_only_barrel()                                   # no CQUAD4: the separate path serves it
    ub = decks.smooth_displacement(b, seed=1)
    with native.GpuModel(b) as g:
        ref = _assemble(g, b, ub)
        g.persistent(True, 24)
        got = _assemble(g, b, ub)
        for x, y in zip(ref, got):
            assert np.array_equal(np.asarray(x), np.asarray(y))
