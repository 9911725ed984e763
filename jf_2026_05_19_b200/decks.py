"""Seeded synthetic decks for the element hot path, as flat structure-of-arrays.

The reference consumes Nastran bulk data that its parser and model builder turn
into a nested ``Dict`` model (OpenJFEM ``src/ModelBuilder.jl:421-826``).  The
element hot path only needs what that builder hands to ``assemble_stiffness``
(``src/solver/assembly.jl:1953-2536``): grid coordinates in node-index order
(sorted GRID IDs), per-node CD frames, shell connectivity with PSHELL/MAT1
data, bar connectivity with PBARL section data, RBE2 sets and PARAM K6ROT.
``ModelArrays`` holds exactly that, already resolved the way the reference's
parser resolves it:

* PSHELL ``BEND_RATIO`` is 0 when MID2 is blank, else 12I/T^3 (default 1.0);
  ``TS_T`` defaults to 5/6 (``src/parsing/extract_properties.jl:3-31``).
* MAT1 completes G from E and NU (``src/parsing/extract_materials.jl:3-28``).
* PBARL BAR/I section properties and Cowper shear factors follow
  ``src/parsing/extract_properties.jl:33-190,536-609`` (see ``pbarl_section``).

The five workloads are the ones the path is measured on: a 40x40 CQUAD4
plate, a 2000x1000 mm stiffened panel with CTRIA3 splits and CBAR stringers,
256 panel variants, a ~1M-shell barrel with CBEAM rings, CBAR longerons and an
RBE2 end ring, and a serving mix of model families.  All inputs are synthetic
and seeded; no external dataset is involved.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

# Column layout of the per-shell property table (one row per element).
SHELL_PROP_COLS = ("h", "E", "nu", "G", "br", "tst", "Gs")
# Column layout of the per-bar property table.
BAR_PROP_COLS = ("A", "I1", "I2", "I12", "J", "K1", "K2", "E", "G",
                 "vx", "vy", "vz", "wax", "way", "waz", "wbx", "wby", "wbz")
N_SHELL_PROP = len(SHELL_PROP_COLS)
N_BAR_PROP = len(BAR_PROP_COLS)


@dataclasses.dataclass
class ModelArrays:
    """Flat model handed to the assembly boundary (0-based node indices)."""

    coords: np.ndarray                      # (n, 3) f64, basic system
    q4_nodes: np.ndarray                    # (nq, 4) int32
    q4_prop: np.ndarray                     # (nq, 7) f64, SHELL_PROP_COLS
    t3_nodes: np.ndarray                    # (nt, 3) int32
    t3_prop: np.ndarray                     # (nt, 7) f64
    bar_nodes: np.ndarray                   # (nb, 2) int32
    bar_prop: np.ndarray                    # (nb, 18) f64, BAR_PROP_COLS
    bar_pin: np.ndarray                     # (nb, 2) int32, PA/PB
    rbe2_master: np.ndarray                 # (nr,) int32
    rbe2_cm: np.ndarray                     # (nr,) int32, component digits as a 6-bit mask
    rbe2_slave_ptr: np.ndarray              # (nr+1,) int64
    rbe2_slaves: np.ndarray                 # (ns,) int32
    node_R: Optional[np.ndarray] = None     # (n, 3, 3) f64 CD frames, None = all basic
    node_ids: Optional[np.ndarray] = None   # (n,) int64 sorted GRID IDs
    k6rot: float = 100.0
    param_snorm: float = 0.0
    name: str = "model"
    # Loads/BCs for a static preload (used by the SOL 105 consumer in tests)
    spc_dofs: Optional[np.ndarray] = None   # 0-based constrained dof indices
    force: Optional[np.ndarray] = None      # (ndof,) f64
    # Element IDs in handle order and PBARL stress-recovery points (C1 C2 D1 D2
    # E1 E2 F1 F2, then +1 for ROD/TUBE/TUBE2 sections, else -1), when the deck
    # came from a model dictionary
    q4_eid: Optional[np.ndarray] = None
    t3_eid: Optional[np.ndarray] = None
    bar_eid: Optional[np.ndarray] = None
    bar_points: Optional[np.ndarray] = None  # (nb, 9) f64
    shell_order: Optional[np.ndarray] = None  # shell record index (CQUAD4s, then CTRIA3s) in dictionary order

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def ndof(self) -> int:
        return 6 * self.n_nodes

    @property
    def n_elements(self) -> int:
        return int(self.q4_nodes.shape[0] + self.t3_nodes.shape[0] + self.bar_nodes.shape[0])

    def counts(self) -> dict:
        return {"quad4": int(self.q4_nodes.shape[0]), "tria3": int(self.t3_nodes.shape[0]),
                "bar": int(self.bar_nodes.shape[0]), "nodes": self.n_nodes,
                "rbe2_slaves": int(self.rbe2_slaves.shape[0])}

    def with_thickness(self, q4_h: np.ndarray, t3_h: np.ndarray) -> "ModelArrays":
        """Copy with new per-element shell thicknesses (PSHELL T update)."""
        q = self.q4_prop.copy(); q[:, 0] = q4_h
        t = self.t3_prop.copy(); t[:, 0] = t3_h
        return dataclasses.replace(self, q4_prop=q, t3_prop=t)


# ---------------------------------------------------------------------------
# material / section helpers (parser semantics)
# ---------------------------------------------------------------------------

def mat1_complete(E: float, G: Optional[float], nu: Optional[float]):
    """MAT1 E/G/NU completion as ``extract_mats`` does it."""
    E = 0.0 if E is None else float(E)
    G = 0.0 if G is None else float(G)
    nu = -1.0 if nu is None else float(nu)
    if E > 0 and G > 0 and nu < 0:
        nu = E / (2 * G) - 1.0
    elif E > 0 and nu >= 0 and G <= 0:
        G = E / (2 * (1 + nu))
    elif G > 0 and nu >= 0 and E <= 0:
        E = 2 * G * (1 + nu)
    if nu < 0:
        nu = 0.3
    return E, G, nu


def shell_prop_row(h: float, E: float, nu: float, G: Optional[float] = None,
                   br: float = 1.0, tst: float = 5.0 / 6.0) -> np.ndarray:
    """One PSHELL/MAT1 row (MID2 = MID3 = MID, so the shear material is MAT1 itself)."""
    E, G, nu = mat1_complete(E, G, nu)
    Gs = G if G > 0 else (E / (2 * (1 + nu)) if E > 0 else 0.0)
    return np.array([h, E, nu, G, br, tst, Gs], dtype=np.float64)


def pbarl_section(kind: str, dims):
    """(A, I1, I2, J, K1, K2) for PBARL BAR or I, Cowper factors with nu=0.3."""
    kind = kind.upper()
    nu = 0.3
    if kind == "BAR":
        w, h = dims
        A = w * h
        I1 = w * h ** 3 / 12
        I2 = h * w ** 3 / 12
        if w >= h and w > 0:
            J = w * h ** 3 / 3 * (1 - 0.63 * h / w)
        elif h > 0:
            J = h * w ** 3 / 3 * (1 - 0.63 * w / h)
        else:
            J = I1 + I2
        K = 10.0 * (1.0 + nu) / (12.0 + 11.0 * nu)
        return A, I1, I2, J, K, K
    if kind == "I":
        H, Bb, Bt, tw, tfb, tft = dims
        hw = H - tfb - tft
        A = Bb * tfb + hw * tw + Bt * tft
        yb = (Bb * tfb * tfb / 2 + hw * tw * (tfb + hw / 2) + Bt * tft * (H - tft / 2)) / A
        I1 = (Bb * tfb ** 3 / 12 + Bb * tfb * (yb - tfb / 2) ** 2 + tw * hw ** 3 / 12
              + tw * hw * (yb - tfb - hw / 2) ** 2 + Bt * tft ** 3 / 12 + Bt * tft * (yb - (H - tft / 2)) ** 2)
        I2 = tfb * Bb ** 3 / 12 + hw * tw ** 3 / 12 + tft * Bt ** 3 / 12
        J = (Bb * tfb ** 3 + hw * tw ** 3 + Bt * tft ** 3) / 3
        hw2 = max(H - tfb - tft, 0.0)
        K1 = min(hw2 * tw / A, 1.0)
        K2 = min((Bb * tfb + Bt * tft) / A, 1.0)
        return A, I1, I2, J, K1, K2
    raise ValueError(f"PBARL type {kind} not generated here")


def bar_prop_row(section, E: float, G: float, v, wa=(0.0, 0.0, 0.0), wb=(0.0, 0.0, 0.0), I12: float = 0.0):
    A, I1, I2, J, K1, K2 = section
    return np.array([A, I1, I2, I12, J, K1, K2, E, G, *v, *wa, *wb], dtype=np.float64)


def _empty_rbe2():
    return (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(1, np.int64), np.zeros(0, np.int32))


def cm_mask(digits: str) -> int:
    m = 0
    for ch in str(digits):
        if ch.isdigit() and 1 <= int(ch) <= 6:
            m |= 1 << (int(ch) - 1)
    return m


# ---------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------

def _grid_quads(nx: int, ny: int, node_index):
    """Quads of an (nx x ny)-cell structured grid, counter-clockwise, mesh order."""
    i = np.arange(nx)
    j = np.arange(ny)
    I, J = np.meshgrid(i, j, indexing="xy")  # row-major over j then i
    I = I.ravel(); J = J.ravel()
    n1 = node_index(I, J); n2 = node_index(I + 1, J)
    n3 = node_index(I + 1, J + 1); n4 = node_index(I, J + 1)
    return np.stack([n1, n2, n3, n4], axis=1).astype(np.int32)


def _split_quads(quads: np.ndarray, frac: float, rng: np.random.Generator):
    """Split a seeded random fraction of quads into CTRIA3 pairs (diagonal 1-3)."""
    n = quads.shape[0]
    k = int(round(frac * n))
    pick = np.zeros(n, bool)
    if k > 0:
        pick[rng.choice(n, size=k, replace=False)] = True
    keep = quads[~pick]
    sp = quads[pick]
    tris = np.empty((2 * sp.shape[0], 3), np.int32)
    tris[0::2] = sp[:, [0, 1, 2]]
    tris[1::2] = sp[:, [0, 2, 3]]
    return keep, tris, pick


def plate_c1(seed: int = 0, n: int = 40, size: float = 400.0, h: float = 2.0,
             E: float = 70000.0, nu: float = 0.33, edge_force: float = 1.0) -> ModelArrays:
    """40x40 CQUAD4 simply supported plate under uniform x-edge compression."""
    del seed
    nn = n + 1
    xs = np.linspace(0.0, size, nn)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    coords = np.stack([X.ravel(), Y.ravel(), np.zeros(nn * nn)], axis=1)
    idx = lambda i, j: j * nn + i
    quads = _grid_quads(n, n, idx)
    prop = np.tile(shell_prop_row(h, E, nu), (quads.shape[0], 1))
    m = ModelArrays(coords=coords, q4_nodes=quads, q4_prop=prop,
                    t3_nodes=np.zeros((0, 3), np.int32), t3_prop=np.zeros((0, N_SHELL_PROP)),
                    bar_nodes=np.zeros((0, 2), np.int32), bar_prop=np.zeros((0, N_BAR_PROP)),
                    bar_pin=np.zeros((0, 2), np.int32),
                    rbe2_master=_empty_rbe2()[0], rbe2_cm=_empty_rbe2()[1],
                    rbe2_slave_ptr=_empty_rbe2()[2], rbe2_slaves=_empty_rbe2()[3],
                    node_ids=np.arange(1, nn * nn + 1, dtype=np.int64), name=f"plate_{n}x{n}")
    # boundary: all edges w=0, corner (0,0) pinned in-plane, (size,0) y pinned
    ndof = m.ndof
    spc = []
    for j in range(nn):
        for i in range(nn):
            if i in (0, n) or j in (0, n):
                spc.append(6 * idx(i, j) + 2)
    spc += [6 * idx(0, 0) + 0, 6 * idx(0, 0) + 1, 6 * idx(n, 0) + 1]
    f = np.zeros(ndof)
    # consistent nodal loads of a uniform edge line force on x = 0 and x = size
    dy = size / n
    for j in range(nn):
        w = dy * (0.5 if j in (0, n) else 1.0) * edge_force
        f[6 * idx(0, j) + 0] += w
        f[6 * idx(n, j) + 0] -= w
    m.spc_dofs = np.array(sorted(set(spc)), np.int64)
    m.force = f
    return m


def stiffened_panel_c2(seed: int = 0, lx: float = 2000.0, ly: float = 1000.0, esize: float = 10.0,
                       tri_frac: float = 0.10, h_lo: float = 1.5, h_hi: float = 3.0,
                       E: float = 70000.0, nu: float = 0.33, stringer_every: int = 10,
                       stringer_dims=(20.0, 4.0), stringer_offset: float = 12.0,
                       h_override: Optional[np.ndarray] = None, end_force: float = 5.0,
                       name: str = "stiffened_panel") -> ModelArrays:
    """2000x1000 panel, 10 mm CQUAD4 skin, 10% CTRIA3 pairs, CBAR stringers in x.

    Stringers run along every ``stringer_every``-th grid line of constant y
    (interior lines, 10 of them for the default mesh: 2,000 CBARs), PBARL BAR
    20x4 with a ``stringer_offset`` mm WA=WB offset along +z.
    """
    rng = np.random.default_rng(seed)
    nx = int(round(lx / esize)); ny = int(round(ly / esize))
    nxn, nyn = nx + 1, ny + 1
    xs = np.linspace(0.0, lx, nxn); ys = np.linspace(0.0, ly, nyn)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    coords = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    idx = lambda i, j: j * nxn + i
    quads = _grid_quads(nx, ny, idx)
    keep, tris, pick = _split_quads(quads, tri_frac, rng)
    if h_override is None:
        h_all = rng.uniform(h_lo, h_hi, size=quads.shape[0])
    else:
        h_all = np.asarray(h_override, dtype=np.float64)
    base = shell_prop_row(1.0, E, nu)
    q4_prop = np.tile(base, (keep.shape[0], 1)); q4_prop[:, 0] = h_all[~pick]
    t3_prop = np.tile(base, (tris.shape[0], 1)); t3_prop[:, 0] = np.repeat(h_all[pick], 2)
    Ec, Gc, nuc = mat1_complete(E, None, nu)
    sec = pbarl_section("BAR", stringer_dims)
    bars = []
    rows = []
    off = (0.0, 0.0, stringer_offset)
    for j in range(stringer_every // 2, nyn, stringer_every):
        for i in range(nx):
            bars.append((idx(i, j), idx(i + 1, j)))
            rows.append(bar_prop_row(sec, Ec, Gc, (0.0, 0.0, 1.0), off, off))
    bar_nodes = np.array(bars, np.int32).reshape(-1, 2)
    bar_prop = np.array(rows, np.float64).reshape(-1, N_BAR_PROP)
    m = ModelArrays(coords=coords, q4_nodes=keep, q4_prop=q4_prop, t3_nodes=tris, t3_prop=t3_prop,
                    bar_nodes=bar_nodes, bar_prop=bar_prop, bar_pin=np.zeros((bar_nodes.shape[0], 2), np.int32),
                    rbe2_master=_empty_rbe2()[0], rbe2_cm=_empty_rbe2()[1],
                    rbe2_slave_ptr=_empty_rbe2()[2], rbe2_slaves=_empty_rbe2()[3],
                    node_ids=np.arange(1, coords.shape[0] + 1, dtype=np.int64), name=name)
    # far end (x=0) clamped, loaded end x=lx: axial compression, rotations free
    spc = []
    for j in range(nyn):
        spc += [6 * idx(0, j) + d for d in range(6)]
    for j in range(nyn):
        spc += [6 * idx(nx, j) + 1, 6 * idx(nx, j) + 2]
    f = np.zeros(m.ndof)
    dyy = ly / ny
    for j in range(nyn):
        f[6 * idx(nx, j)] -= end_force * dyy * (0.5 if j in (0, ny) else 1.0)
    m.spc_dofs = np.array(sorted(set(spc)), np.int64)
    m.force = f
    return m


def panel_variant_c3(variant: int, seed: int = 0, no_offset: bool = False) -> ModelArrays:
    """One of the 256 design variants: lognormal thickness, stringer height U[15,25]."""
    rng = np.random.default_rng(10_000 + 7919 * variant + seed)
    nq = 200 * 100
    h = 2.2 * np.exp(0.15 * rng.standard_normal(nq))
    sh = rng.uniform(15.0, 25.0)
    return stiffened_panel_c2(seed=seed, h_override=h, stringer_dims=(sh, 4.0),
                              stringer_offset=0.0 if no_offset else 12.0, name=f"panel_variant_{variant}")


def barrel_c4(seed: int = 0, radius: float = 2000.0, length: float = 6000.0, n_circ: int = 1440,
              n_axial: int = 696, tri_frac: float = 0.10, h0: float = 1.6, E: float = 70000.0,
              nu: float = 0.33, ring_every: int = 58, longeron_every: int = 20,
              axial_force: float = 20.0, with_rbe2: bool = True, name: str = "barrel") -> ModelArrays:
    """Cylindrical barrel: ~1M shells, CBEAM rings, CBAR longerons, RBE2 end.

    Defaults give 1440 x 696 cells (1,002,240 quad cells, 10% split into CTRIA3
    pairs), rings every 58 cells axially (500 mm) and longerons every 20 cells
    circumferentially (5 degrees).  The z = length end ring is tied by one RBE2
    (CM=123456) to a centre node; z = 0 is clamped.
    """
    rng = np.random.default_rng(seed)
    th = np.arange(n_circ) * (2.0 * math.pi / n_circ)
    zs = np.linspace(0.0, length, n_axial + 1)
    T, Z = np.meshgrid(th, zs, indexing="xy")
    ring_coords = np.stack([radius * np.cos(T).ravel(), radius * np.sin(T).ravel(), Z.ravel()], axis=1)
    n_ring_nodes = ring_coords.shape[0]
    coords = ring_coords
    if with_rbe2:
        coords = np.vstack([ring_coords, [[0.0, 0.0, length]]])
    idx = lambda i, j: j * n_circ + (i % n_circ)
    quads = _grid_quads(n_circ, n_axial, idx)
    keep, tris, pick = _split_quads(quads, tri_frac, rng)
    h_all = h0 * rng.uniform(0.9, 1.1, size=quads.shape[0])
    base = shell_prop_row(1.0, E, nu)
    q4_prop = np.tile(base, (keep.shape[0], 1)); q4_prop[:, 0] = h_all[~pick]
    t3_prop = np.tile(base, (tris.shape[0], 1)); t3_prop[:, 0] = np.repeat(h_all[pick], 2)
    Ec, Gc, _ = mat1_complete(E, None, nu)
    ring_sec = pbarl_section("I", (80.0, 40.0, 40.0, 3.0, 3.0, 3.0))
    long_sec = pbarl_section("BAR", (20.0, 4.0))
    bars = []
    rows = []
    for j in range(0, n_axial + 1, ring_every):
        for i in range(n_circ):
            a, b = idx(i, j), idx(i + 1, j)
            bars.append((a, b))
            mid = 0.5 * (ring_coords[a] + ring_coords[b])
            v = (mid[0], mid[1], 0.0)  # radial orientation vector
            rows.append(bar_prop_row(ring_sec, Ec, Gc, v))
    for i in range(0, n_circ, longeron_every):
        for j in range(n_axial):
            a, b = idx(i, j), idx(i, j + 1)
            bars.append((a, b))
            p = ring_coords[a]
            rows.append(bar_prop_row(long_sec, Ec, Gc, (p[0], p[1], 0.0)))
    bar_nodes = np.array(bars, np.int32)
    bar_prop = np.array(rows, np.float64)
    if with_rbe2:
        master = np.array([n_ring_nodes], np.int32)
        cm = np.array([cm_mask("123456")], np.int32)
        slaves = np.array([idx(i, n_axial) for i in range(n_circ)], np.int32)
        sptr = np.array([0, slaves.shape[0]], np.int64)
    else:
        master, cm, sptr, slaves = _empty_rbe2()
    m = ModelArrays(coords=coords, q4_nodes=keep, q4_prop=q4_prop, t3_nodes=tris, t3_prop=t3_prop,
                    bar_nodes=bar_nodes, bar_prop=bar_prop, bar_pin=np.zeros((bar_nodes.shape[0], 2), np.int32),
                    rbe2_master=master, rbe2_cm=cm, rbe2_slave_ptr=sptr, rbe2_slaves=slaves,
                    node_ids=np.arange(1, coords.shape[0] + 1, dtype=np.int64), name=name)
    spc = [6 * idx(i, 0) + d for i in range(n_circ) for d in range(6)]
    f = np.zeros(m.ndof)
    if with_rbe2:
        f[6 * n_ring_nodes + 2] = -axial_force * 2.0 * math.pi * radius
    m.spc_dofs = np.array(sorted(spc), np.int64)
    m.force = f
    return m


def barrel_small(seed: int = 0, n_circ: int = 72, n_axial: int = 24, **kw) -> ModelArrays:
    """Scaled-down barrel with the same element families (parity-test size)."""
    kw.setdefault("ring_every", max(1, n_axial // 4))
    kw.setdefault("longeron_every", max(1, n_circ // 12))
    return barrel_c4(seed=seed, n_circ=n_circ, n_axial=n_axial, name="barrel_small", **kw)


def serving_families(seed: int = 0, scale: float = 1.0):
    """Eight model families spanning 2k to 500k elements (plate, panel, barrel)."""
    fams = []
    specs = [("plate", 45), ("plate", 100), ("panel", 0.5), ("panel", 1.0),
             ("barrel", (240, 96)), ("barrel", (480, 160)), ("barrel", (720, 348)), ("barrel", (960, 432))]
    for k, (kind, arg) in enumerate(specs):
        if kind == "plate":
            n = max(2, int(round(arg * math.sqrt(scale))))
            fams.append(plate_c1(seed=seed + k, n=n))
        elif kind == "panel":
            fams.append(stiffened_panel_c2(seed=seed + k, lx=2000.0 * arg, esize=10.0 / math.sqrt(scale) if scale < 1 else 10.0,
                                           stringer_offset=0.0, name=f"panel_{k}"))
        else:
            nc, na = arg
            nc = max(24, int(nc * math.sqrt(scale)) // 24 * 24)
            na = max(12, int(na * math.sqrt(scale)) // 12 * 12)
            fams.append(barrel_c4(seed=seed + k, n_circ=nc, n_axial=na, ring_every=na // 12,
                                  longeron_every=nc // 72 if nc >= 72 else 1, name=f"barrel_{k}"))
    return fams


def smooth_displacement(m: ModelArrays, seed: int = 0, amp: float = 1e-2) -> np.ndarray:
    """Seeded smooth displacement field (all 6 dofs) for kernel-only KG timing."""
    rng = np.random.default_rng(seed)
    X = m.coords
    span = np.maximum(np.ptp(X, axis=0), 1.0)
    k = rng.uniform(0.5, 2.0, size=(6, 3)) * (2 * math.pi) / span
    ph = rng.uniform(0, 2 * math.pi, size=(6,))
    u = np.empty((m.n_nodes, 6))
    for d in range(6):
        scale = amp if d < 3 else amp * 1e-2
        u[:, d] = scale * np.sin(X @ k[d] + ph[d])
    return u.ravel()
