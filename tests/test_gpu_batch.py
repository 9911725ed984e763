"""Batched variants: one launch per kernel over several property sets of one mesh.

Each variant of a batch must equal, bit for bit, a single-model assembly of
that variant (its own model handle), for K, max_elem_stiff, orig_diag and KG;
the single-model path itself is checked against the oracle in
test_gpu_parity.py.
"""
import dataclasses

import numpy as np
import pytest

from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu


def _variants(m, n_var, seed=5):
    """n_var (model, u) pairs: new shell thicknesses, scaled bar sections, own u."""
    rng = np.random.default_rng(seed)
    out = []
    for v in range(n_var):
        hq = rng.uniform(0.8, 3.0, m.q4_nodes.shape[0])
        ht = rng.uniform(0.8, 3.0, m.t3_nodes.shape[0])
        mv = m.with_thickness(hq, ht)
        bp = mv.bar_prop.copy()
        f = rng.uniform(0.7, 1.4)
        bp[:, [0, 1, 2, 4]] *= [f, f ** 3, f, f ** 3]   # A, I1, I2, J of a taller section
        mv = dataclasses.replace(mv, bar_prop=bp)
        out.append((mv, hq, ht, decks.smooth_displacement(m, seed=100 + v)))
    return out


def _single(mv, u):
    with native.GpuModel(mv) as g:
        k, mx, dg = g.assemble_k()
        kg = g.assemble_kg(u)
    return k, mx, dg, kg


def test_batch_variants_equal_single_calls(cuda_device):
    import torch
    m = decks.barrel_small(seed=3, n_circ=48, n_axial=16)   # CQUAD4 + CTRIA3 + bars + RBE2
    assert m.t3_nodes.shape[0] and m.bar_nodes.shape[0] and m.rbe2_master.shape[0]
    n_var = 3
    vs = _variants(m, n_var)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    with native.GpuModel(m) as g:
        g.batch_reserve(n_var)
        h = t(np.stack([np.concatenate([hq, ht]) for _, hq, ht, _ in vs]))
        bp = t(np.stack([mv.bar_prop for mv, *_ in vs]))
        u = t(np.stack([uv for *_, uv in vs]))
        nzk = torch.empty(n_var, g.nnz, dtype=torch.float64, device="cuda")
        nzg = torch.empty_like(nzk)
        mx = torch.zeros(n_var, dtype=torch.float64, device="cuda")
        dg = torch.empty(n_var, g.ndof, dtype=torch.float64, device="cuda")
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        g.set_stream(s.cuda_stream)
        g.assemble_batch_device(n_var, h.data_ptr(), bp.data_ptr(), u.data_ptr(), None, nzk.data_ptr(), mx.data_ptr(),
                                dg.data_ptr(), nzg.data_ptr())
        s.synchronize()
        g.set_stream(0)
        for v, (mv, _, _, uv) in enumerate(vs):
            k1, mx1, dg1, kg1 = _single(mv, uv)
            assert np.array_equal(nzk[v].cpu().numpy(), k1), f"K variant {v}"
            assert np.array_equal(nzg[v].cpu().numpy(), kg1), f"KG variant {v}"
            assert float(mx[v].item()) == mx1
            assert np.array_equal(dg[v].cpu().numpy(), dg1)


def test_batch_shared_displacement_and_defaults(cuda_device):
    """u_stride 0 shares one field; null thickness / bar pointers use the handle's own."""
    import torch
    m = decks.stiffened_panel_c2(seed=1, lx=300.0, ly=200.0, stringer_every=4, stringer_offset=0.0)
    u = decks.smooth_displacement(m, seed=3)
    k1, _, _, kg1 = _single(m, u)
    n_var = 4
    with native.GpuModel(m) as g:
        g.batch_reserve(n_var)
        du = torch.from_numpy(u).cuda()
        nzk = torch.empty(n_var, g.nnz, dtype=torch.float64, device="cuda")
        nzg = torch.empty_like(nzk)
        torch.cuda.synchronize()
        g.assemble_batch_device(n_var, u_ptr=du.data_ptr(), u_stride=0, nzk_ptr=nzk.data_ptr(), nzkg_ptr=nzg.data_ptr())
        torch.cuda.synchronize()
        for v in range(n_var):
            assert np.array_equal(nzk[v].cpu().numpy(), k1)
            assert np.array_equal(nzg[v].cpu().numpy(), kg1)


def test_batch_argument_errors(cuda_device):
    import torch
    m = decks.plate_c1(n=6)
    with native.GpuModel(m) as g:
        g.batch_reserve(2)
        nz = torch.empty(3, g.nnz, dtype=torch.float64, device="cuda")
        with pytest.raises(native.JfgError):
            g.assemble_batch_device(3, nzk_ptr=nz.data_ptr())          # more variants than reserved
        with pytest.raises(native.JfgError):
            g.assemble_batch_device(1, nzkg_ptr=nz.data_ptr())         # KG without u
        du = torch.zeros(g.ndof, dtype=torch.float64, device="cuda")
        with pytest.raises(native.JfgError):
            g.assemble_batch_device(1, u_ptr=du.data_ptr(), u_stride=5, nzkg_ptr=nz.data_ptr())
        assert g.batch_workspace_bytes(4) == 4 * g.batch_workspace_bytes(1) > 0


def test_batch_call_replays_from_a_cuda_graph(cuda_device):
    """The batched device call, captured once into a CUDA graph and replayed,
    gives the same bits as the direct call (the library times nothing and
    waits on nothing while its stream is being captured)."""
    import torch
    m = decks.barrel_small(seed=4, n_circ=48, n_axial=16)
    n_var = 4
    vs = _variants(m, n_var, seed=8)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    with native.GpuModel(m) as g:
        g.batch_reserve(n_var)
        h = t(np.stack([np.concatenate([hq, ht]) for _, hq, ht, _ in vs]))
        bp = t(np.stack([mv.bar_prop for mv, *_ in vs]))
        u = t(np.stack([uv for *_, uv in vs]))
        outs = [torch.full((n_var, g.nnz), float("nan"), dtype=torch.float64, device="cuda") for _ in range(4)]
        mx = [torch.zeros(n_var, dtype=torch.float64, device="cuda") for _ in range(2)]
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        g.set_stream(s.cuda_stream)
        g.assemble_batch_device(n_var, h.data_ptr(), bp.data_ptr(), u.data_ptr(), None, outs[0].data_ptr(),
                                mx[0].data_ptr(), 0, outs[1].data_ptr())
        s.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            g.assemble_batch_device(n_var, h.data_ptr(), bp.data_ptr(), u.data_ptr(), None, outs[2].data_ptr(),
                                    mx[1].data_ptr(), 0, outs[3].data_ptr())
        for _ in range(2):
            outs[2].fill_(float("nan")); outs[3].fill_(float("nan"))
            graph.replay()
            torch.cuda.synchronize()
            assert torch.equal(outs[0], outs[2]) and torch.equal(outs[1], outs[3])
            assert torch.equal(mx[0], mx[1])
        g.set_stream(0)
        del graph
