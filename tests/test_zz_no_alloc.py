"""The allocation-free CQUAD4 stiffness entry point.

Some callers cannot allocate device memory where they need a stiffness
matrix: a host framework that reserved all device memory up front and hands
out only its own buffers, or a real-time loop that forbids allocator calls.
They use jfg_assemble_k_quad4_noalloc, which keeps its intermediate data in
one fixed array in the library's device image.  This test calls it through
the C ABI and checks its output against the regular entry point
(jfg_assemble_k) on the same CQUAD4 patch, twice in a row, since the fixed
array keeps the previous call's contents.  It also checks that input the
regular model build refuses is refused here with the same status, and that a
good call after a refused one is still right.  The file sorts last so that a
run stopping at the first failure has already run every other test.
"""
import dataclasses

import numpy as np
import pytest

from helpers import ROW_TOL, rowmax_rel_err
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu

MAX_QUAD4 = 2048   # JFG_NOALLOC_MAX_QUAD4 in include/jfem_gpu.h
OK, INVALID, UNSUPPORTED = 0, 1, 2


def _quad4_only(m):
    return dataclasses.replace(
        m, t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, decks.N_SHELL_PROP)),
        bar_nodes=np.zeros((0, 2), np.int32), bar_prop=np.zeros((0, decks.N_BAR_PROP)),
        bar_pin=np.zeros((0, 2), np.int32), rbe2_master=np.zeros(0, np.int32), rbe2_cm=np.zeros(0, np.int32),
        rbe2_slave_ptr=np.zeros(1, np.int64), rbe2_slaves=np.zeros(0, np.int32))


def _quad4_patch():
    """A distorted, arbitrarily oriented CQUAD4-only patch with mixed PSHELLs and CD frames."""
    from decks_extra import skewed_plane
    return _quad4_only(skewed_plane(seed=11, nx=12, ny=9, tri_frac=0.0))


def _fan(n_sectors=9):
    """A flat fan of quads around one centre node: the centre's valence is n_sectors."""
    ang = np.linspace(0.0, 2 * np.pi, n_sectors, endpoint=False)
    half = ang + np.pi / n_sectors
    pts = [(0.0, 0.0, 0.0)]
    pts += [(10 * np.cos(a), 10 * np.sin(a), 0.0) for a in ang]          # spokes 1..n
    pts += [(14 * np.cos(a), 14 * np.sin(a), 0.0) for a in half]         # rim n+1..2n
    quads = [(0, 1 + k, 1 + n_sectors + k, 1 + (k + 1) % n_sectors) for k in range(n_sectors)]
    p = decks.plate_c1(n=2)
    coords = np.array(pts)
    return _quad4_only(dataclasses.replace(
        p, coords=coords, q4_nodes=np.array(quads, np.int32),
        q4_prop=np.tile(decks.shell_prop_row(1.2, 70000.0, 0.3), (n_sectors, 1)),
        node_R=None, node_ids=np.arange(1, coords.shape[0] + 1), spc_dofs=None, force=np.zeros(6 * coords.shape[0])))


def _device_arrays(m, colptr, rowval, nodes=None, prop=None, coords=None):
    import torch
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()
    R = m.node_R if m.node_R is not None else np.repeat(np.eye(3)[None], m.n_nodes, 0)
    return {"coords": t(m.coords if coords is None else coords, np.float64), "node_R": t(R.reshape(-1, 9), np.float64),
            "nodes": t(m.q4_nodes if nodes is None else nodes, np.int32),
            "prop": t(m.q4_prop if prop is None else prop, np.float64),
            "rowptr": t(colptr - 1, np.int64), "colind": t(rowval - 1, np.int64)}


def _call(L, m, dev, out, n_quad4=None):
    import torch
    torch.cuda.synchronize()
    return L.jfg_assemble_k_quad4_noalloc(
        m.n_nodes, dev["coords"].data_ptr(), dev["node_R"].data_ptr(),
        int(m.q4_nodes.shape[0] if n_quad4 is None else n_quad4),
        dev["nodes"].data_ptr(), dev["prop"].data_ptr(), float(m.k6rot), dev["rowptr"].data_ptr(),
        dev["colind"].data_ptr(), out.data_ptr(), None)


def _check_good_call(L, m, ref, colptr, dev, tag):
    import torch
    out = torch.full((len(ref),), float("nan"), dtype=torch.float64, device="cuda")
    assert _call(L, m, dev, out) == OK, tag
    got = out.cpu().numpy()
    assert np.isfinite(got).all(), tag
    assert rowmax_rel_err(colptr, ref, got) <= ROW_TOL, tag


def test_noalloc_matches_regular_assembly_twice(cuda_device):
    L = native.load()
    m = _quad4_patch()
    assert m.q4_nodes.shape[0] <= MAX_QUAD4
    with native.GpuModel(m) as g:
        ref, _, _ = g.assemble_k()
        colptr, rowval = g.pattern()
    dev = _device_arrays(m, colptr, rowval)
    for call in range(2):
        _check_good_call(L, m, ref, colptr, dev, f"call {call}")


def test_noalloc_rejects_what_the_model_build_rejects(cuda_device):
    """Same statuses as jfg_model_create: bad index, repeated node, h or E <= 0
    -> INVALID; warped quad, too many elements or too many per node -> UNSUPPORTED.
    A good call after the refusals still matches the regular path."""
    import torch
    from decks_extra import warped
    L = native.load()
    m = _quad4_patch()
    with native.GpuModel(m) as g:
        ref, _, _ = g.assemble_k()
        colptr, rowval = g.pattern()
    out = torch.zeros(len(rowval), dtype=torch.float64, device="cuda")

    bad = m.q4_nodes.copy(); bad[3, 1] = m.n_nodes + 7
    assert _call(L, m, _device_arrays(m, colptr, rowval, nodes=bad), out) == INVALID
    rep = m.q4_nodes.copy(); rep[5, 2] = rep[5, 0]
    assert _call(L, m, _device_arrays(m, colptr, rowval, nodes=rep), out) == INVALID
    for col in (0, 1):   # thickness, E
        pr = m.q4_prop.copy(); pr[7, col] = 0.0
        assert _call(L, m, _device_arrays(m, colptr, rowval, prop=pr), out) == INVALID
    with pytest.raises(native.JfgError) as e:          # the regular build refuses the warped patch ...
        native.GpuModel(warped(m))
    assert e.value.status == UNSUPPORTED
    assert _call(L, m, _device_arrays(m, colptr, rowval, coords=warped(m).coords), out) == UNSUPPORTED  # ... so does this
    dev = _device_arrays(m, colptr, rowval)
    assert _call(L, m, dev, out, n_quad4=MAX_QUAD4 + 1) == UNSUPPORTED   # size check before any launch

    fan = _fan(9)                                      # one node with 9 incident quads (limit 8)
    with native.GpuModel(fan) as g:
        fcp, frv = g.pattern()
    fout = torch.zeros(len(frv), dtype=torch.float64, device="cuda")
    assert _call(L, fan, _device_arrays(fan, fcp, frv), fout) == UNSUPPORTED

    _check_good_call(L, m, ref, colptr, dev, "after refusals")


def test_noalloc_valence_at_the_limit(cuda_device):
    """Eight quads on one node is within the limit and matches the regular path."""
    L = native.load()
    fan = _fan(8)
    with native.GpuModel(fan) as g:
        ref, _, _ = g.assemble_k()
        colptr, rowval = g.pattern()
    _check_good_call(L, fan, ref, colptr, _device_arrays(fan, colptr, rowval), "fan of 8")
