"""Row-block partition on the GPU: the parts' owned columns, each assembled on
its own handle (one GPU here, the parts in turn), join to the whole model's
K and KG bit for bit."""
import numpy as np
import pytest

from jf_2026_05_19_b200 import decks, native, partition

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("parts", [2, 4])
def test_gpu_parts_join_to_the_whole_matrix(parts, cuda_device):
    m = decks.barrel_small(seed=5, n_circ=72, n_axial=24)
    u = decks.smooth_displacement(m, seed=9)
    with native.GpuModel(m) as g:
        cp, rv = g.pattern()
        k, _, _ = g.assemble_k()
        kg = g.assemble_kg(u)
    bk, bkg = [], []
    for r in range(parts):
        p = partition.part_of(m, r, parts)
        with native.GpuModel(p.model) as gp:
            pcp, prv = gp.pattern()
            bk.append(partition.owned_columns(p, pcp, prv, gp.assemble_k()[0]))
            bkg.append(partition.owned_columns(p, pcp, prv, gp.assemble_kg(u)))
    jcp, jrv, jk = partition.join_columns(bk)
    _, _, jkg = partition.join_columns(bkg)
    assert np.array_equal(jcp, cp) and np.array_equal(jrv, rv)
    assert np.array_equal(jk, k) and np.array_equal(jkg, kg)
