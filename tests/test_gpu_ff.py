"""Free-dof submatrices on the device: 0.5 (A_ff + A_ff') of K and KG.

Checked against scipy on the same values: A[free][:, free], then A_ff +
A_ff' with exact zeros removed (as Julia's sparse + stores only nonzero
sums) and halved; the CSC arrays must match exactly, and so must max|A_ff|
and max|A_ff - A_ff'| (the reference's Kg asymmetry diagnostic).
"""
import numpy as np
import pytest

from helpers import free_dofs, to_csc
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu


def _scipy_ff(A, free):
    Aff = A[free][:, free].tocsc()
    S = (Aff + Aff.T).tocsc()
    S.eliminate_zeros()
    S = S * 0.5
    S.sort_indices()
    return S, abs(Aff).max(), abs(Aff - Aff.T).max()


@pytest.mark.parametrize("deck", ["barrel_small", "plate"])
def test_free_dof_submatrices_match_scipy(deck, cuda_device):
    import torch
    m = decks.barrel_small(seed=2, n_circ=72, n_axial=24) if deck == "barrel_small" else decks.plate_c1(n=20)
    u = decks.smooth_displacement(m, seed=5)
    with native.GpuModel(m) as g:
        colptr, rowval = g.pattern()
        K, _, _ = g.assemble_k()
        KG = g.assemble_kg(u)
        dep = g.constraint_map()[0]
        Kc = to_csc(colptr, rowval, K, m.ndof)
        free = free_dofs(m, dep, Kc)
        g.ff_set_free(free)
        for vals in (K, KG):
            d = torch.from_numpy(vals).cuda()
            cp, rv, v, amax, asym = g.ff_extract(d.data_ptr())
            S, smax, sasym = _scipy_ff(to_csc(colptr, rowval, vals, m.ndof), free)
            assert np.array_equal(cp - 1, S.indptr) and np.array_equal(rv - 1, S.indices)
            assert np.array_equal(v, S.data)
            assert amax == smax and asym == sasym
        # Kg's zeroed drill rows leave its pattern, so it is smaller than K's
        assert g.ff_extract(torch.from_numpy(KG).cuda().data_ptr())[0][-1] < \
            g.ff_extract(torch.from_numpy(K).cuda().data_ptr())[0][-1]


def test_free_dof_list_is_checked(cuda_device):
    m = decks.plate_c1(n=4)
    with native.GpuModel(m) as g:
        with pytest.raises(native.JfgError):
            g.ff_set_free(np.array([3, 2, 5]))            # not increasing
        with pytest.raises(native.JfgError):
            g.ff_set_free(np.array([0, m.ndof]))          # out of range
