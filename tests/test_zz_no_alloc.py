"""The allocation-free CQUAD4 stiffness entry point.

Callers that cannot allocate device memory where they need a stiffness
matrix (inside a CUDA graph capture, under a framework that owns all device
memory, or in a loop that forbids allocator calls) use
jfg_assemble_k_quad4_noalloc.  It keeps its intermediate data in one fixed
array in the library's device image.  This test calls it through the C ABI
and checks its output against the regular entry point (jfg_assemble_k) on
the same CQUAD4 patch, twice in a row, since the fixed array keeps the
previous call's contents.  The file sorts last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from helpers import ROW_TOL, rowmax_rel_err
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu

MAX_QUAD4 = 2048   # JFG_NOALLOC_MAX_QUAD4 in include/jfem_gpu.h


def _quad4_patch():
    """A distorted, arbitrarily oriented CQUAD4-only patch with mixed PSHELLs and CD frames."""
    from decks_extra import skewed_plane
    m = skewed_plane(seed=11, nx=12, ny=9, tri_frac=0.0)
    return dataclasses.replace(
        m, t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, decks.N_SHELL_PROP)),
        bar_nodes=np.zeros((0, 2), np.int32), bar_prop=np.zeros((0, decks.N_BAR_PROP)),
        bar_pin=np.zeros((0, 2), np.int32), rbe2_master=np.zeros(0, np.int32), rbe2_cm=np.zeros(0, np.int32),
        rbe2_slave_ptr=np.zeros(1, np.int64), rbe2_slaves=np.zeros(0, np.int32))


def _call(L, m, dev, out):
    return L.jfg_assemble_k_quad4_noalloc(
        m.n_nodes, dev["coords"].data_ptr(), dev["node_R"].data_ptr(), int(m.q4_nodes.shape[0]),
        dev["nodes"].data_ptr(), dev["prop"].data_ptr(), float(m.k6rot), dev["rowptr"].data_ptr(),
        dev["colind"].data_ptr(), out.data_ptr(), None)


def test_noalloc_matches_regular_assembly_twice(cuda_device):
    import torch
    L = native.load()
    m = _quad4_patch()
    assert m.q4_nodes.shape[0] <= MAX_QUAD4
    with native.GpuModel(m) as g:
        ref, _, _ = g.assemble_k()
        colptr, rowval = g.pattern()
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()
    dev = {"coords": t(m.coords, np.float64), "node_R": t(m.node_R.reshape(-1, 9), np.float64),
           "nodes": t(m.q4_nodes, np.int32), "prop": t(m.q4_prop, np.float64),
           "rowptr": t(colptr - 1, np.int64), "colind": t(rowval - 1, np.int64)}
    out = torch.empty(len(ref), dtype=torch.float64, device="cuda")
    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        assert _call(L, m, dev, out) == 0, f"call {call}"
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rowmax_rel_err(colptr, ref, got) <= ROW_TOL, f"call {call}"


def test_noalloc_rejects_oversize_and_bad_indices(cuda_device):
    import torch
    L = native.load()
    m = _quad4_patch()
    with native.GpuModel(m) as g:
        colptr, rowval = g.pattern()
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()
    bad_nodes = m.q4_nodes.copy()
    bad_nodes[3, 1] = m.n_nodes + 7
    dev = {"coords": t(m.coords, np.float64), "node_R": t(m.node_R.reshape(-1, 9), np.float64),
           "nodes": t(bad_nodes, np.int32), "prop": t(m.q4_prop, np.float64),
           "rowptr": t(colptr - 1, np.int64), "colind": t(rowval - 1, np.int64)}
    out = torch.zeros(len(rowval), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert _call(L, m, dev, out) == 1                     # JFG_ERR_INVALID, nothing else launched
    too_many = dataclasses.replace(m, q4_nodes=np.zeros((MAX_QUAD4 + 1, 4), np.int32))
    assert _call(L, too_many, dev, out) == 2              # JFG_ERR_UNSUPPORTED before any launch
