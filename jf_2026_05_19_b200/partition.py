"""Row-block partition of one mesh over several GPUs (one process per GPU).

The reference assembles a model in one process, its CQUAD4 loop threaded
(src/solver/assembly.jl:2657) and the KG shell loop threaded (:4772).  Here
rank r of P owns a contiguous range of nodes, i.e. the rows -- and, K and KG
being symmetric, the CSC columns -- of those nodes' dofs.  Its sub-model keeps
the whole node set and the RBE2 list, and the elements that can contribute to
an owned column:

  * every element with a node in the owned range, and
  * every element touching a slave node of an RBE2 whose master is owned
    (the redistribution turns a slave's entries into the master's;
    constraints.jl:329-361).

Elements keep their relative order, so every owned column is assembled from
the same contributions in the same order as on one GPU: bit for bit the same
values.  Elements touching two ranges are computed by both (halo elements).
The only exchange is one gather of the column blocks; there is no collective
inside the assembly.
"""
from __future__ import annotations

import dataclasses
from typing import List, Tuple

import numpy as np

from .decks import ModelArrays


@dataclasses.dataclass
class Part:
    rank: int
    node_lo: int          # owned nodes [node_lo, node_hi)
    node_hi: int
    model: ModelArrays    # sub-model: all nodes, the elements this rank assembles
    q4: np.ndarray        # indices of its elements in the full model, per type
    t3: np.ndarray
    bar: np.ndarray

    @property
    def dof_lo(self) -> int:
        return 6 * self.node_lo

    @property
    def dof_hi(self) -> int:
        return 6 * self.node_hi


def node_ranges(m: ModelArrays, parts: int) -> List[Tuple[int, int]]:
    """Contiguous node ranges with about equal element work: each element is
    charged to its lowest node, weighted by its type's share of the flops."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    w = np.zeros(m.n_nodes)
    for nodes, cost in ((m.q4_nodes, 4.0), (m.t3_nodes, 2.0), (m.bar_nodes, 0.2)):
        if nodes.shape[0]:
            np.add.at(w, nodes.min(axis=1), cost)
    c = np.cumsum(w)
    total = c[-1] if c.size else 0.0
    cuts = [0]
    for r in range(1, parts):
        cuts.append(int(np.searchsorted(c, total * r / parts, side="left")) + 1)
    cuts.append(m.n_nodes)
    cuts = np.maximum.accumulate(np.clip(cuts, 0, m.n_nodes))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(parts)]


def _touching(nodes: np.ndarray, mark: np.ndarray) -> np.ndarray:
    if nodes.shape[0] == 0:
        return np.zeros(0, np.int64)
    return np.nonzero(mark[nodes].any(axis=1))[0]


def part_of(m: ModelArrays, rank: int, parts: int, ranges=None) -> Part:
    """The sub-model rank `rank` of `parts` assembles."""
    ranges = ranges or node_ranges(m, parts)
    lo, hi = ranges[rank]
    owned = np.zeros(m.n_nodes, bool)
    owned[lo:hi] = True
    need = owned.copy()
    for r in range(m.rbe2_master.shape[0]):                   # slaves of owned masters
        if owned[m.rbe2_master[r]]:
            need[m.rbe2_slaves[m.rbe2_slave_ptr[r]:m.rbe2_slave_ptr[r + 1]]] = True
    q4 = _touching(m.q4_nodes, need)
    t3 = _touching(m.t3_nodes, need)
    bar = _touching(m.bar_nodes, need)
    sub = dataclasses.replace(m, q4_nodes=m.q4_nodes[q4], q4_prop=m.q4_prop[q4], t3_nodes=m.t3_nodes[t3],
                              t3_prop=m.t3_prop[t3], bar_nodes=m.bar_nodes[bar], bar_prop=m.bar_prop[bar],
                              bar_pin=m.bar_pin[bar], name=f"{m.name} rows {rank}/{parts}")
    return Part(rank, lo, hi, sub, q4, t3, bar)


def owned_columns(part: Part, colptr: np.ndarray, rowval: np.ndarray, nzval: np.ndarray):
    """The owned CSC columns of a part's matrix: (colptr slice rebased to 1,
    rowval, nzval).  colptr/rowval are 1-based, as jfg_pattern_fill gives them."""
    a, b = colptr[part.dof_lo] - 1, colptr[part.dof_hi] - 1
    return colptr[part.dof_lo:part.dof_hi + 1] - a, rowval[a:b], nzval[a:b]


def join_columns(blocks) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The whole CSC from the ranks' owned column blocks, in rank order."""
    colptr, rowval, nzval = [np.array([1], np.int64)], [], []
    off = 0
    for cp, rv, nz in blocks:
        colptr.append(cp[1:] + off)
        off += int(cp[-1] - 1)
        rowval.append(rv)
        nzval.append(nz)
    return np.concatenate(colptr), np.concatenate(rowval), np.concatenate(nzval)


def halo_elements(m: ModelArrays, parts: int) -> dict:
    """How much element work the partition repeats: elements assembled over all
    ranks against the model's own count."""
    ranges = node_ranges(m, parts)
    tot = sum(part_of(m, r, parts, ranges).model.n_elements for r in range(parts))
    return {"elements": int(m.n_elements), "assembled": int(tot), "overhead": tot / max(m.n_elements, 1) - 1.0}


def gather_columns(dist, part: Part, block, device=None):
    """All ranks' owned column blocks on every rank (torch.distributed
    all_gather of the sizes, then of the padded blocks); returns the joined CSC.
    Every rank takes the same collective steps."""
    import torch
    cp, rv, nz = block
    dev = device if device is not None else torch.device("cpu")
    sizes = torch.tensor([cp.shape[0], rv.shape[0]], dtype=torch.int64, device=dev)
    all_sizes = [torch.zeros_like(sizes) for _ in range(dist.get_world_size())]
    dist.all_gather(all_sizes, sizes)
    ncp = max(int(s[0]) for s in all_sizes)
    nnz = max(int(s[1]) for s in all_sizes)

    def pad(a, n, dt):
        t = torch.zeros(n, dtype=dt, device=dev)
        t[:a.shape[0]] = torch.as_tensor(a, dtype=dt, device=dev)
        return t

    out = []
    for a, n, dt in ((cp, ncp, torch.int64), (rv, nnz, torch.int64), (nz, nnz, torch.float64)):
        mine = pad(a, n, dt)
        got = [torch.zeros_like(mine) for _ in range(dist.get_world_size())]
        dist.all_gather(got, mine)
        out.append(got)
    blocks = []
    for r, s in enumerate(all_sizes):
        c, k = int(s[0]), int(s[1])
        blocks.append((out[0][r][:c].cpu().numpy(), out[1][r][:k].cpu().numpy(), out[2][r][:k].cpu().numpy()))
    return join_columns(blocks)
