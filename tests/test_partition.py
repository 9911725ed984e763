"""Row-block partition of one mesh (CPU; the oracle assembles each part).

Every rank's owned CSC columns, joined in rank order, must equal the whole
model's matrix bit for bit, for K and KG, including the rows of an RBE2
master whose slaves another rank owns; and the gather over a world-size-2
gloo process group must give the same.
"""
import os
import socket
import sys

import numpy as np
import pytest

import oracle as O
from jf_2026_05_19_b200 import decks, partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _model():
    # barrel with CBEAM rings, CBAR longerons and the RBE2 end ring; its master
    # (the centre node) is the last node, its slaves the last ring
    return decks.barrel_small(seed=3, n_circ=48, n_axial=12)


def _parts_join(m, parts, fn):
    blocks = []
    for r in range(parts):
        p = partition.part_of(m, r, parts)
        cp, rv, nz = fn(p.model)[:3]
        blocks.append(partition.owned_columns(p, cp, rv, nz))
    return partition.join_columns(blocks)


@pytest.mark.parametrize("parts", [1, 2, 3, 5])
def test_owned_columns_join_to_the_whole_matrix(parts):
    m = _model()
    u = decks.smooth_displacement(m, seed=4)
    cp, rv, nz, _, _ = O.assemble_k(m)
    jcp, jrv, jnz = _parts_join(m, parts, O.assemble_k)
    assert np.array_equal(jcp, cp) and np.array_equal(jrv, rv) and np.array_equal(jnz, nz)
    _, _, kg = O.assemble_kg(m, u)
    _, _, jkg = _parts_join(m, parts, lambda mm: O.assemble_kg(mm, u))
    assert np.array_equal(jkg, kg)


def test_ranges_cover_the_nodes_and_halo_is_small():
    m = decks.barrel_c4(seed=3, n_circ=240, n_axial=96, ring_every=8, longeron_every=10)
    for parts in (2, 4, 8):
        rg = partition.node_ranges(m, parts)
        assert rg[0][0] == 0 and rg[-1][1] == m.n_nodes
        assert all(a[1] == b[0] for a, b in zip(rg, rg[1:]))
        h = partition.halo_elements(m, parts)
        assert 0.0 <= h["overhead"] < 0.1, h


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import oracle as Ow
    from jf_2026_05_19_b200 import partition as P
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m = _model()
        p = P.part_of(m, rank, world)
        cp, rv, nz, _, _ = Ow.assemble_k(p.model)
        jcp, jrv, jnz = P.gather_columns(dist, p, P.owned_columns(p, cp, rv, nz))
        fcp, frv, fnz, _, _ = Ow.assemble_k(m)
        out[rank] = bool(np.array_equal(jcp, fcp) and np.array_equal(jrv, frv) and np.array_equal(jnz, fnz))
    finally:
        dist.destroy_process_group()


def test_gather_over_gloo_world_2():
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_gloo_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0] and out[1]
