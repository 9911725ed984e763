"""GPU parity on the benchmarked barrel itself (1440 x 696 cells: 902,016
CQUAD4, 200,448 CTRIA3, 68,832 CBEAM/CBAR, RBE2 end ring; 6.02M dof, 317M
nonzeros): the same bars as tests/test_gpu_parity.py, K and KG against the
oracle at full size.  The oracle needs about a minute on 16 host threads and
~40 GB of host memory."""
import numpy as np
import pytest

import oracle as O
from helpers import parity_ratio, rowmax_rel_err
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu


def test_benchmark_barrel_k_kg_match_oracle(cuda_device):
    m = decks.barrel_c4(seed=0)
    u = decks.smooth_displacement(m, seed=1)
    with native.GpuModel(m) as g:
        cp, rv = g.pattern()
        nz, mx, dg = g.assemble_k()
        gnz = g.assemble_kg(u)
    ocp, orv, onz, omx, odg, det = O.assemble_k(m, detail=True, abs_sums=True)
    assert np.array_equal(cp, ocp) and np.array_equal(rv, orv)
    del orv, ocp
    assert parity_ratio(cp, onz, nz, det["abs_sums"]) <= 1.0, rowmax_rel_err(cp, onz, nz)
    assert abs(mx - omx) <= 1e-12 * abs(omx)
    assert np.abs(dg - odg).max() <= 1e-12 * max(np.abs(odg).max(), 1.0)
    del onz, nz, det
    _, _, ognz, detg = O.assemble_kg(m, u, detail=True, abs_sums=True)
    assert parity_ratio(cp, ognz, gnz, detg["abs_sums"]) <= 1.0, rowmax_rel_err(cp, ognz, gnz)
