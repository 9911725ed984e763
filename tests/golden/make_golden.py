"""Generate the golden fixtures in tests/golden/ from the CPU oracle.

The reference (Julia) cannot run in this environment and ships no golden
vectors, so these fixtures pin the oracle's own outputs on small seeded decks
(regression fixtures; parity with the reference itself stays unpinned).  The
GPU parity tests compare against them as well.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from jf_2026_05_19_b200 import decks  # noqa: E402


def golden_decks():
    return {
        "plate_6x6": decks.plate_c1(n=6, size=60.0),
        "panel_small": decks.stiffened_panel_c2(seed=3, lx=80.0, ly=40.0, esize=10.0, stringer_every=2,
                                                stringer_offset=0.0, name="panel_small"),
        "barrel_tiny": decks.barrel_small(seed=5, n_circ=24, n_axial=4),
    }


def element_cases():
    lc_q4 = np.array([[-5.0, -4.0], [5.5, -4.2], [4.8, 5.0], [-5.2, 4.3]])
    lc_t3 = np.array([[-5.0, -3.0], [6.0, -2.0], [-1.0, 5.0]])
    prop = decks.shell_prop_row(2.0, 70000.0, 0.33)
    return lc_q4, lc_t3, prop


def main():
    out = {}
    for name, m in golden_decks().items():
        cp, rv, nz, mx, dg = O.assemble_k(m)
        u = decks.smooth_displacement(m, seed=11)
        _, _, nzg = O.assemble_kg(m, u)
        out[f"{name}__colptr"] = cp
        out[f"{name}__rowval"] = rv
        out[f"{name}__k"] = nz
        out[f"{name}__kg"] = nzg
        out[f"{name}__max"] = np.array([mx])
        out[f"{name}__diag"] = dg
        out[f"{name}__u"] = u
    lc_q4, lc_t3, prop = element_cases()
    out["q4_local"] = O.q4_local(lc_q4, prop)
    out["t3_local"] = O.t3_local(lc_t3, prop)
    np.savez_compressed(os.path.join(HERE, "oracle_fixtures.npz"), **out)
    print("wrote", os.path.join(HERE, "oracle_fixtures.npz"))


if __name__ == "__main__":
    main()
