"""Group handles: several models of uneven size and mixed element types in one
handle, so every launch takes bins from all of them.

Each member's slice of the group's K, KG, orig_diag and pattern must equal,
bit for bit, the member assembled on its own handle (whose values the parity
tests compare with the oracle); batched design variants of the group must
equal each member's variant assembled alone.
"""
import dataclasses

import numpy as np
import pytest

from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu


def _members():
    from decks_extra import skewed_plane
    return [
        decks.plate_c1(n=12),                                              # CQUAD4 only
        decks.barrel_small(seed=4, n_circ=48, n_axial=12),                 # CQUAD4 + CTRIA3 + bars + RBE2
        decks.stiffened_panel_c2(seed=2, lx=200.0, ly=120.0, stringer_every=4, stringer_offset=0.0),
        dataclasses.replace(skewed_plane(seed=7), k6rot=100.0),            # CD frames, membrane-only PSHELLs, zero-length bar
        decks.plate_c1(n=3),                                               # tiny
    ]


def _alone(m, u):
    with native.GpuModel(m) as g:
        cp, rv = g.pattern()
        k, mx, dg = g.assemble_k()
        kg = g.assemble_kg(u)
    return cp, rv, k, mx, dg, kg


def test_group_members_equal_their_own_handles(cuda_device):
    ms = _members()
    us = [decks.smooth_displacement(m, seed=30 + i) for i, m in enumerate(ms)]
    with native.GpuGroup(ms) as g:
        assert g.ndof == sum(m.ndof for m in ms)
        k, mx, dg = g.assemble_k()
        kg = g.assemble_kg(np.concatenate(us))
        maxes = []
        for i, (m, u) in enumerate(zip(ms, us)):
            cp, rv, k1, mx1, dg1, kg1 = _alone(m, u)
            gcp, grv = g.member_pattern(i)
            assert np.array_equal(gcp, cp) and np.array_equal(grv, rv), f"pattern of member {i}"
            assert np.array_equal(g.member_values(k, i), k1), f"K of member {i}"
            assert np.array_equal(g.member_values(kg, i), kg1), f"KG of member {i}"
            assert np.array_equal(g.member_dofs(dg, i), dg1), f"orig_diag of member {i}"
            maxes.append(mx1)
        assert mx == max(maxes)
        assert g.nnz == sum(g.member(i)["nnz"] for i in range(len(ms)))


def test_group_variants_in_one_launch(cuda_device):
    """Design variants of every member in the same launches (own thickness per element)."""
    import torch
    ms = _members()[:3]
    n_var = 3
    rng = np.random.default_rng(11)
    hs = [[rng.uniform(0.8, 3.0, m.q4_nodes.shape[0] + m.t3_nodes.shape[0]) for m in ms] for _ in range(n_var)]
    us = [decks.smooth_displacement(m, seed=50 + i) for i, m in enumerate(ms)]
    with native.GpuGroup(ms) as g:
        # group order: all CQUAD4s (member by member), then all CTRIA3s
        nq = [m.q4_nodes.shape[0] for m in ms]
        h_rows = []
        for v in range(n_var):
            q = np.concatenate([hs[v][i][:nq[i]] for i in range(len(ms))])
            t = np.concatenate([hs[v][i][nq[i]:] for i in range(len(ms))])
            h_rows.append(np.concatenate([q, t]))
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        h = dev(np.stack(h_rows))
        u = dev(np.concatenate(us))
        g.batch_reserve(n_var)
        nzk = torch.empty(n_var, g.nnz, dtype=torch.float64, device="cuda")
        nzg = torch.empty_like(nzk)
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        g.set_stream(s.cuda_stream)
        g.assemble_batch_device(n_var, h.data_ptr(), 0, u.data_ptr(), 0, nzk.data_ptr(), 0, 0, nzg.data_ptr())
        s.synchronize()
        g.set_stream(0)
        K, KG = nzk.cpu().numpy(), nzg.cpu().numpy()
        for v in range(n_var):
            for i, m in enumerate(ms):
                mv = m.with_thickness(hs[v][i][:nq[i]], hs[v][i][nq[i]:])
                _, _, k1, _, _, kg1 = _alone(mv, us[i])
                assert np.array_equal(g.member_values(K[v], i), k1), f"K variant {v} member {i}"
                assert np.array_equal(g.member_values(KG[v], i), kg1), f"KG variant {v} member {i}"


def test_group_rejects_a_bad_member(cuda_device):
    ms = _members()[:2]
    q = ms[1].q4_nodes.copy()
    q[0, 0] = ms[1].n_nodes + 3          # in range of the merged mesh, not of the member
    bad = dataclasses.replace(ms[1], q4_nodes=q)
    with pytest.raises(native.JfgError) as e:
        native.GpuGroup([ms[0], bad])
    assert e.value.status == 1 and "member 1" in e.value.msg
    with pytest.raises(native.JfgError) as e:
        native.GpuGroup([ms[0], dataclasses.replace(ms[1], k6rot=50.0)])
    assert e.value.status == 1
