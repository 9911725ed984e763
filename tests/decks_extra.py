"""Extra seeded decks that exercise the edge cases of the default branch."""
import dataclasses

import numpy as np

from jf_2026_05_19_b200 import decks as D


def rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def skewed_plane(seed=0, nx=7, ny=5, cd_frames=True, membrane_only_frac=0.2, tri_frac=0.3):
    """Distorted, arbitrarily oriented flat mesh: mixed PSHELLs, CD frames, bars."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0, 70.0, nx + 1); ys = np.linspace(0, 40.0, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    X = X + rng.uniform(-2.5, 2.5, X.shape); Y = Y + rng.uniform(-2.5, 2.5, Y.shape)
    P = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    R = rotation(rng)
    coords = P @ R.T + rng.uniform(-100, 100, 3)
    idx = lambda i, j: j * (nx + 1) + i
    quads = D._grid_quads(nx, ny, idx)
    keep, tris, pick = D._split_quads(quads, tri_frac, rng)

    def props(n):
        rows = []
        for _ in range(n):
            br = 0.0 if rng.random() < membrane_only_frac else rng.uniform(0.5, 1.5)
            row = D.shell_prop_row(rng.uniform(0.8, 3.0), rng.uniform(50e3, 200e3), rng.uniform(0.2, 0.4),
                                   br=br, tst=rng.uniform(0.7, 1.0))
            row[6] = row[3] * rng.uniform(0.5, 1.5)   # MID3 with a different G
            rows.append(row)
        return np.array(rows).reshape(-1, D.N_SHELL_PROP)

    # bars along the first grid row (varied sections), one zero-length bar
    bars, rows = [], []
    E, G, _ = D.mat1_complete(70000.0, None, 0.33)
    for i in range(nx):
        a, b = idx(i, 0), idx(i + 1, 0)
        sec = D.pbarl_section("BAR", (rng.uniform(5, 20), rng.uniform(2, 6)))
        if i % 3 == 1:
            sec = (sec[0], sec[1], sec[2], sec[3], 0.0, 0.0)       # K1 = K2 = 0: Euler-Bernoulli
        v = (0.0, 0.0, 0.0) if i % 4 == 2 else tuple(R @ np.array([0.0, 0.3, 1.0]))
        rows.append(D.bar_prop_row(sec, E, G, v, I12=(rng.uniform(-50, 50) if i % 2 else 0.0)))
        bars.append((a, b))
    bars.append((idx(nx, ny), idx(nx, ny)))
    rows.append(D.bar_prop_row(D.pbarl_section("BAR", (10.0, 3.0)), E, G, (0.0, 0.0, 1.0)))
    node_R = None
    if cd_frames:
        node_R = np.stack([rotation(rng) if rng.random() < 0.5 else np.eye(3) for _ in range(coords.shape[0])])
    m = D.ModelArrays(coords=coords, q4_nodes=keep, q4_prop=props(keep.shape[0]), t3_nodes=tris,
                      t3_prop=props(tris.shape[0]), bar_nodes=np.array(bars, np.int32),
                      bar_prop=np.array(rows), bar_pin=np.zeros((len(bars), 2), np.int32),
                      rbe2_master=np.array([idx(0, ny)], np.int32), rbe2_cm=np.array([D.cm_mask("1236")], np.int32),
                      rbe2_slave_ptr=np.array([0, 2], np.int64),
                      rbe2_slaves=np.array([idx(1, ny), idx(2, ny)], np.int32),
                      node_R=node_R, node_ids=np.arange(1, coords.shape[0] + 1), k6rot=250.0, name="skewed_plane")
    return m


def with_offset_bar(m):
    bp = m.bar_prop.copy()
    bp[0, 12:18] = [0.0, 0.0, 5.0, 0.0, 0.0, 5.0]
    return dataclasses.replace(m, bar_prop=bp)


def with_unused_nodes(m, extra=5):
    coords = np.vstack([m.coords, np.arange(extra * 3, dtype=float).reshape(extra, 3) + 1000.0])
    R = None if m.node_R is None else np.concatenate([m.node_R, np.repeat(np.eye(3)[None], extra, 0)])
    return dataclasses.replace(m, coords=coords, node_R=R, node_ids=np.arange(1, coords.shape[0] + 1))


def warped(m):
    """Lift one corner of the first quad out of plane (non-flat element)."""
    c = m.coords.copy()
    n = m.q4_nodes[0, 2]
    R = rotation(np.random.default_rng(0))
    c[n] = c[n] + 0.5 * np.cross(c[m.q4_nodes[0, 1]] - c[m.q4_nodes[0, 0]], c[m.q4_nodes[0, 3]] - c[m.q4_nodes[0, 0]]) / 100.0
    del R
    return dataclasses.replace(m, coords=c)


def plate_axis_rbe2(n=6, size=120.0, cm="123"):
    """Flat plate with an RBE2 whose slave lies on its master's grid row: the
    offset is along x, so the image of the slave's translations has no theta_x
    term and the master's theta_x row holds fewer columns than its other rows."""
    p = D.plate_c1(n=n, size=size)
    nn = n + 1
    idx = lambda i, j: j * nn + i
    j = n // 2
    return dataclasses.replace(p, rbe2_master=np.array([idx(2, j)], np.int32), rbe2_cm=np.array([D.cm_mask(cm)], np.int32),
                               rbe2_slave_ptr=np.array([0, 1], np.int64), rbe2_slaves=np.array([idx(n - 1, j)], np.int32),
                               name="plate_axis_rbe2")


def without_shells(m):
    """The deck's line elements and constraints only (shells removed)."""
    return dataclasses.replace(m, q4_nodes=np.zeros((0, 4), np.int32), q4_prop=np.zeros((0, D.N_SHELL_PROP)),
                               t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, D.N_SHELL_PROP)),
                               name=m.name + "_bars_only")


def bars_only_barrel():
    """The 72 x 24 barrel with its shells removed: CBEAM rings, CBAR longerons
    and the RBE2 end ring, whose centre node's rows sum terms up to ~3e4 times
    their row max."""
    return without_shells(D.barrel_small(seed=2, n_circ=72, n_axial=24))


def single_quad4():
    return D.plate_c1(n=1)


def single_cell_tria3():
    """One skewed, arbitrarily oriented quad cell split into two CTRIA3, nothing else."""
    rng = np.random.default_rng(8)
    P = np.array([[0.0, 0.0, 0.0], [23.0, 1.5, 0.0], [25.0, 19.0, 0.0], [-2.0, 17.0, 0.0]])
    coords = P @ rotation(rng).T + rng.uniform(-50, 50, 3)
    tris = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    prop = np.array([D.shell_prop_row(1.7, 70000.0, 0.33), D.shell_prop_row(2.3, 70000.0, 0.33)])
    p = D.plate_c1(n=1)
    return dataclasses.replace(p, coords=coords, q4_nodes=np.zeros((0, 4), np.int32), q4_prop=np.zeros((0, D.N_SHELL_PROP)),
                               t3_nodes=tris, t3_prop=prop, node_ids=np.arange(1, 5), spc_dofs=None,
                               force=np.zeros(24), name="single_cell_tria3")
