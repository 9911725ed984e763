"""Frozen algorithmic work constants of the element hot path.

Canonical FP64 flop counts per element (1 FMA = 2 flops), counted as the
dense block products written in the reference's element kernels with the
block-diagonal node transformation exploited and redundant recomputation
removed (src/FEMKernels.jl stiffness_quad4_matrices :3185-4034, MacNeal shear
:4715-4978, geometric_stiffness_quad4 :7554-7985, tria3 :7157-7385,
frame3d :140-229 and :7441-7471; transforms src/solver/assembly.jl).

Canonical bytes per element: nodal coordinates (24 B) and displacements
(48 B) per node, 4 B connectivity per node, 64 B of property record, and the
scatter-map index reads (4 B per n_dof^2 entry) for K and KG; plus 8 B per
nonzero for each of the two CSR value writes.  The pattern is built once per
model and excluded.
"""
from __future__ import annotations

FLOPS = {
    "quad4_k": 2 * 30_603,
    "quad4_kg": 2 * 31_216,
    "tria3_k": 2 * 30_871,
    "tria3_kg": 2 * 2_088,
    "bar_k": 2 * 1_300,
    "bar_kg": 2 * 1_550,
}

# FP64 flops the closed-form kernels actually execute per element (2 DFMA +
# DADD + DMUL thread instructions, from ncu counters of one launch of each
# kernel on a 240 x 96 barrel; the capture is summarised under profiles/).
# They divide the same launch time as FLOPS to give the hardware fraction of
# the FP64 peak beside the canonical-work rate.
EXECUTED_FLOPS = {
    "quad4_k": 13_127,
    "quad4_kg": 9_733,
    "tria3_k": 18_835,
}

NODES = {"quad4": 4, "tria3": 3, "bar": 2}
NDOF = {"quad4": 24, "tria3": 18, "bar": 12}


def flops_per_step(counts: dict) -> float:
    """FP64 flops of one K + KG pass over a model with the given element counts."""
    return sum(counts[t] * (FLOPS[f"{t}_k"] + FLOPS[f"{t}_kg"]) for t in ("quad4", "tria3", "bar"))


def bytes_per_step(counts: dict, nnz: int) -> float:
    b = 0.0
    for t in ("quad4", "tria3", "bar"):
        n = counts[t]
        b += n * (NODES[t] * (24 + 48 + 4) + 64) + 2 * n * NDOF[t] ** 2 * 4
    return b + 2 * nnz * 8


def kernel_flops(kernel: str, count: int) -> float:
    """Algorithmic flops of one launch of an element kernel over `count` elements."""
    return FLOPS[kernel] * count


def kernel_executed_flops(kernel: str, count: int):
    """Executed FP64 flops of one launch, or None where no counter capture exists."""
    f = EXECUTED_FLOPS.get(kernel)
    return None if f is None else f * count
