"""CQUAD4 KG in stress states where the principal directions are degenerate
or nearly so.

The reference takes the principal angle as 0.5 atan2(2 txy, sxx - syy) and
its cos/sin (FEMKernels.jl:6891-6902); the GPU kernel uses the half-angle
identities instead.  At equal principal stresses the angle is undefined and
the principal-transverse KG does not depend on it; near that point the two
forms must still agree within the parity bound.  Membrane states from linear
displacement fields on a flat plate: equibiaxial, nearly equibiaxial (relative
differences 1e-12, 1e-9, 1e-6), pure shear (45 degrees), uniaxial.
"""
import numpy as np
import pytest

import oracle as O
from helpers import parity_ratio, rowmax_rel_err
from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu

EPS = 1e-3


def _field(m, kind):
    x, y = m.coords[:, 0], m.coords[:, 1]
    u = np.zeros(6 * m.n_nodes)
    if kind == "equibiaxial":
        u[0::6], u[1::6] = EPS * x, EPS * y
    elif kind.startswith("near"):
        d = float(kind.split("_")[1])
        u[0::6], u[1::6] = EPS * x, EPS * (1.0 + d) * y
    elif kind == "shear":
        u[0::6], u[1::6] = 0.5 * EPS * y, 0.5 * EPS * x
    elif kind == "uniaxial":
        u[0::6] = EPS * x
    return u


@pytest.mark.parametrize("kind", ["equibiaxial", "near_1e-12", "near_1e-9", "near_1e-6", "shear", "uniaxial"])
def test_kg_matches_oracle_in_degenerate_stress_states(cuda_device, kind):
    m = decks.plate_c1(n=10)
    u = _field(m, kind)
    with native.GpuModel(m) as g:
        cp, _ = g.pattern()
        _, _, ognz, det = O.assemble_kg(m, u, detail=True, abs_sums=True)
        gnz = g.assemble_kg(u)
    assert np.abs(ognz).max() > 0.0
    assert parity_ratio(cp, ognz, gnz, det["abs_sums"]) <= 1.0, (kind, rowmax_rel_err(cp, ognz, gnz))
