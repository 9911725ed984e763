"""Host-side mirror of the reference's assembly and output-recovery calls, backed by the CUDA library.

Same names, arguments and return values (or filled dictionaries) as OpenJFEM's

    Solver.assemble_stiffness(model; bending_incomp, shear_center_only,
        membrane_incomp, pcomp_membrane_incomp, snorm_angle_override,
        iso_no_incomp)                                   src/solver/assembly.jl:1953-1956
    Solver.assemble_geometric_stiffness(model, id_map, node_coords, node_R,
        ndof, u_global, snorm_normals, rbe3_map; snorm_angle_override,
        buckling_subcase, static_load_id, timings)       src/solver/assembly.jl:4382-4386

and the per-element loops of the SOL 101 output recovery that follows the
static solve,

    recover_shell_stresses!(model, id_map, X, node_R, u_global, snorm_normals,
        stresses, results_json)                          src/solver/stress_recovery.jl:163-430
    recover_bar_stresses!(model, id_map, X, node_R, u_global, stresses,
        results_json)                                    src/solver/stress_recovery.jl:432-593

``model`` is the nested dictionary the reference's model builder produces
(``GRIDs``, ``CORDs``, ``CSHELLs``, ``PSHELLs``, ``MATs``, ``CBARs``,
``CBEAMs``, ``PBARLs``, ``RBE2s``, ``PARAM_K6ROT``, ``PARAM_SNORM``).
Matrices come back as ``scipy.sparse.csc_matrix`` built from the library's
SparseMatrixCSC arrays (1-based colptr/rowval converted to 0-based).
Inputs that leave the reference's default branch raise ``NotImplementedError``
(the library's JFG_ERR_UNSUPPORTED); inputs on which the reference itself
raises raise ``RuntimeError`` with the reference location.
"""
from __future__ import annotations

import re

import numpy as np
import scipy.sparse as sp

from .abi import JFG_ERR_REFERENCE_RAISES, JFG_ERR_UNSUPPORTED
from .decks import N_BAR_PROP, N_SHELL_PROP, ModelArrays, cm_mask, mat1_complete
from .native import GpuModel, JfgError

_HANDLES: dict = {}


def _raise(err: JfgError):
    if err.status == JFG_ERR_UNSUPPORTED:
        raise NotImplementedError(err.msg) from err
    if err.status == JFG_ERR_REFERENCE_RAISES:
        raise RuntimeError(err.msg) from err
    raise err


def public_id(key, entry) -> int:
    """Element ID of a model-dictionary entry (_stress_entry_public_id,
    stress_recovery.jl:3-14): its "ID", else the key, else the key's leading integer."""
    if isinstance(entry, dict) and "ID" in entry:
        try:
            return int(str(entry["ID"]))
        except ValueError:
            pass
    try:
        return int(str(key))
    except ValueError:
        m = re.match(r"^-?\d+", str(key))
        return int(m.group(0)) if m else 0


def model_arrays_from_dict(model: dict) -> tuple:
    """Flatten a reference model dictionary into ModelArrays and the id map."""
    grids = model["GRIDs"]
    ids = sorted(int(k) for k in grids)
    id_map = {gid: i + 1 for i, gid in enumerate(ids)}        # 1-based like the reference
    n = len(ids)
    if n == 0:
        raise RuntimeError("No nodes found in model — is this a standalone BDF or an INCLUDE fragment?")
    coords = np.zeros((n, 3))
    node_R = np.repeat(np.eye(3)[None], n, axis=0)
    any_cd = False
    cords = model.get("CORDs", {})
    for g in grids.values():
        i = id_map[int(g["ID"])] - 1
        coords[i] = g["X"]
        cd = int(g.get("CD", 0))
        if cd != 0 and str(cd) in cords:
            c = cords[str(cd)]
            node_R[i] = np.column_stack([c["U"], c["V"], c["W"]])
            any_cd = True
    pshells, mats = model.get("PSHELLs", {}), model.get("MATs", {})

    def shell_row(el):
        prop = pshells[str(el["PID"])]
        if prop.get("TYPE", "") == "PCOMP_CLT":
            raise NotImplementedError("PCOMP laminates leave the isotropic default branch")
        mat = mats[str(prop["MID"])]
        if mat.get("TYPE", "MAT1") not in ("MAT1", ""):
            raise NotImplementedError(f"{mat.get('TYPE')} leaves the MAT1 default branch")
        E, G, nu = mat1_complete(mat.get("E"), mat.get("G"), mat.get("NU"))
        mid3 = prop.get("MID3", 0)
        smat = mats.get(str(mid3), mat) if mid3 else mat
        Es, Gs, nus = mat1_complete(smat.get("E"), smat.get("G"), smat.get("NU"))
        if Gs <= 0:
            Gs = Es / (2 * (1 + nus)) if Es > 0 else 0.0
        return [prop["T"], E, nu, G, prop.get("BEND_RATIO", 1.0), prop.get("TS_T", 5.0 / 6.0), Gs]

    q4n, q4p, t3n, t3p, q4e, t3e, order = [], [], [], [], [], [], []
    for key, el in model.get("CSHELLs", {}).items():
        if str(el["PID"]) not in pshells or str(pshells[str(el["PID"])]["MID"]) not in mats:
            continue
        nids = el["NODES"]
        if any(nid not in id_map for nid in nids):
            continue
        if len(nids) not in (3, 4):
            raise NotImplementedError("CQUAD8/CTRIA6 expansion is outside the supported element set")
        row = shell_row(el)
        idx = [id_map[nid] - 1 for nid in nids]
        (q4n if len(nids) == 4 else t3n).append(idx)
        (q4p if len(nids) == 4 else t3p).append(row)
        (q4e if len(nids) == 4 else t3e).append(public_id(key, el))
        order.append((len(nids) == 4, len(q4e if len(nids) == 4 else t3e) - 1))
    pbarls = model.get("PBARLs", {})
    bn, bp, bpin, be, bpts = [], [], [], [], []
    for group in ("CBARs", "CBEAMs"):
        for key, bar in model.get(group, {}).items():
            pid = str(bar["PID"])
            if pid not in pbarls:
                continue
            prop = pbarls[pid]
            if str(prop["MID"]) not in mats:
                continue
            if bar["GA"] not in id_map or bar["GB"] not in id_map:
                continue
            mat = mats[str(prop["MID"])]
            E, G, nu = mat1_complete(mat.get("E"), mat.get("G"), mat.get("NU"))
            ga = id_map[bar["GA"]] - 1
            g0 = int(bar.get("G0", 0) or 0)
            if g0 > 0 and g0 in id_map:
                v = coords[id_map[g0] - 1] - coords[ga]
            else:
                v = np.asarray(bar.get("V", [0.0, 0.0, 0.0]), float)
            I1 = prop.get("I1", prop.get("I", 0.0))
            I2 = prop.get("I2", prop.get("I", 0.0))
            bp.append([prop["A"], I1, I2, prop.get("I12", 0.0), prop["J"], prop.get("K1", 0.0), prop.get("K2", 0.0),
                       E, G, *v, *bar.get("WA", [0.0, 0.0, 0.0]), *bar.get("WB", [0.0, 0.0, 0.0])])
            bn.append([ga, id_map[bar["GB"]] - 1])
            bpin.append([int(bar.get("PA", 0) or 0), int(bar.get("PB", 0) or 0)])
            be.append(public_id(key, bar))
            sign = 1.0 if str(prop.get("TYPE", "")).upper() in ("ROD", "TUBE", "TUBE2") else -1.0
            bpts.append([float(prop.get(k, 0.0)) for k in ("C1", "C2", "D1", "D2", "E1", "E2", "F1", "F2")] + [sign])
    masters, cms, sptr, slaves = [], [], [0], []
    for rbe in model.get("RBE2s", {}).values():
        if rbe["GN"] not in id_map:
            continue
        masters.append(id_map[rbe["GN"]] - 1)
        cms.append(cm_mask(str(rbe["CM"])))
        slaves += [id_map[g] - 1 for g in rbe["GM"] if g in id_map]
        sptr.append(len(slaves))
    for other in ("RBE3s", "RBE1s", "RSPLINEs", "MPCs", "CRODs", "CONRODs", "CELAS1s", "CBUSHs", "DMIGs"):
        if model.get(other):
            raise NotImplementedError(f"{other} are outside the supported element set")
    m = ModelArrays(
        coords=coords,
        q4_nodes=np.array(q4n, np.int32).reshape(-1, 4), q4_prop=np.array(q4p, float).reshape(-1, N_SHELL_PROP),
        t3_nodes=np.array(t3n, np.int32).reshape(-1, 3), t3_prop=np.array(t3p, float).reshape(-1, N_SHELL_PROP),
        bar_nodes=np.array(bn, np.int32).reshape(-1, 2), bar_prop=np.array(bp, float).reshape(-1, N_BAR_PROP),
        bar_pin=np.array(bpin, np.int32).reshape(-1, 2), rbe2_master=np.array(masters, np.int32),
        rbe2_cm=np.array(cms, np.int32), rbe2_slave_ptr=np.array(sptr, np.int64), rbe2_slaves=np.array(slaves, np.int32),
        node_R=node_R if any_cd else None, node_ids=np.array(ids, np.int64),
        k6rot=float(model.get("PARAM_K6ROT", 100.0)), param_snorm=float(model.get("PARAM_SNORM", 0.0)),
        q4_eid=np.array(q4e, np.int64), t3_eid=np.array(t3e, np.int64), bar_eid=np.array(be, np.int64),
        bar_points=np.array(bpts, float).reshape(-1, 9),
        shell_order=np.array([i if quad else len(q4e) + i for quad, i in order], np.int64))
    return m, id_map, coords, [node_R[i] for i in range(n)]


def _same_structure(a: ModelArrays, b: ModelArrays) -> bool:
    same = lambda x, y: (x is None and y is None) or (x is not None and y is not None and x.shape == y.shape
                                                      and np.array_equal(x, y))
    props_ok = (same(a.q4_prop[:, 1:], b.q4_prop[:, 1:]) and same(a.t3_prop[:, 1:], b.t3_prop[:, 1:]))
    return (props_ok and same(a.coords, b.coords) and same(a.node_R, b.node_R) and same(a.q4_nodes, b.q4_nodes)
            and same(a.t3_nodes, b.t3_nodes) and same(a.bar_nodes, b.bar_nodes) and same(a.bar_prop, b.bar_prop)
            and same(a.bar_pin, b.bar_pin) and same(a.rbe2_master, b.rbe2_master) and same(a.rbe2_cm, b.rbe2_cm)
            and same(a.rbe2_slave_ptr, b.rbe2_slave_ptr) and same(a.rbe2_slaves, b.rbe2_slaves)
            and a.k6rot == b.k6rot and a.param_snorm == b.param_snorm)


def _handle(model, m):
    """Device handle for `model`: reused while the mesh is unchanged, thickness
    updates applied in place (the reference re-assembles from the dictionary on
    every call, so the dictionary is re-read each time)."""
    key = id(model)
    h = _HANDLES.get(key)
    if h is not None and h[0] is model and _same_structure(h[2], m):
        g, old = h[1], h[2]
        if not (np.array_equal(old.q4_prop[:, 0], m.q4_prop[:, 0]) and np.array_equal(old.t3_prop[:, 0], m.t3_prop[:, 0])):
            try:
                g.update_thickness(m.q4_prop[:, 0], m.t3_prop[:, 0])
            except JfgError as err:
                _raise(err)
            _HANDLES[key] = (model, g, m)
        return g
    if h is not None:
        h[1].close()
    try:
        g = GpuModel(m)
    except JfgError as err:
        _raise(err)
    _HANDLES[key] = (model, g, m)
    return g


def _csc(g: GpuModel, nz):
    colptr, rowval = g.pattern()
    return sp.csc_matrix((nz, rowval - 1, colptr - 1), shape=(g.ndof, g.ndof))


def assemble_stiffness(model, *, bending_incomp=True, shear_center_only=False, membrane_incomp=True,
                       pcomp_membrane_incomp=False, snorm_angle_override=None, iso_no_incomp=False):
    """K and the side outputs of assemble_stiffness (assembly.jl:4374)."""
    if not bending_incomp or shear_center_only or iso_no_incomp:
        raise NotImplementedError("only the static-K default branch (bending_incomp=true, "
                                  "shear_center_only=false, iso_no_incomp=false) is supported")
    if snorm_angle_override is not None and float(snorm_angle_override) > 0:
        raise NotImplementedError("PARAM,SNORM > 0 leaves the default branch")
    del membrane_incomp, pcomp_membrane_incomp   # flat isotropic shells use Wilson modes either way
    m, id_map, coords, node_R = model_arrays_from_dict(model)
    g = _handle(model, m)
    try:
        nz, mx, diag = g.assemble_k()
        dep, ptr, ind, coef = g.constraint_map()
    except JfgError as err:
        _raise(err)
    rbe3_map = {int(dep[i]): [(int(ind[t]), float(coef[t])) for t in range(ptr[i], ptr[i + 1])] for i in range(len(dep))}
    return _csc(g, nz), id_map, coords, g.ndof, node_R, mx, rbe3_map, {}, diag


def assemble_geometric_stiffness(model, id_map, node_coords, node_R, ndof, u_global, snorm_normals, rbe3_map, *,
                                 snorm_angle_override=None, buckling_subcase=None, static_load_id=None, timings=None):
    """Kg of assemble_geometric_stiffness (assembly.jl:6634)."""
    del id_map, node_coords, node_R, rbe3_map, buckling_subcase, static_load_id
    if snorm_normals:
        raise NotImplementedError("SNORM normals leave the default branch")
    if snorm_angle_override is not None and float(snorm_angle_override) > 0:
        raise NotImplementedError("PARAM,SNORM > 0 leaves the default branch")
    m, _, _, _ = model_arrays_from_dict(model)
    g = _handle(model, m)
    u = np.asarray(u_global, np.float64)
    if u.shape != (ndof,) or ndof != g.ndof:
        raise ValueError("u_global does not match the model's dof count")
    try:
        nz = g.assemble_kg(u)
    except JfgError as err:
        _raise(err)
    if timings is not None:
        el, red, tot = g.timing()
        timings.clear()
        timings.update({"shells": el / 1e3, "sparse_build": red / 1e3, "total": tot / 1e3})
    return _csc(g, nz)


def _recovery_inputs(model, u_global):
    m, _, _, _ = model_arrays_from_dict(model)
    g = _handle(model, m)
    u = np.asarray(u_global, np.float64)
    if u.shape != (g.ndof,):
        raise ValueError("u_global does not match the model's dof count")
    return m, g, u


def _pressure_deck(model) -> bool:
    """Model-level conditions of _quad4_pressure_resultant_moment_scale
    (stress_recovery.jl:131-161) that the library cannot see; it adds "no bars,
    no RBE2" itself.  MAT1 entries are taken as carrying E and NU (the parser
    completes them)."""
    if len(model.get("PLOAD4s", []) or []) < 4 or len(model.get("CSHELLs", {}) or {}) < 4:
        return False
    return not any(model.get(k) for k in ("RBE3s", "RSPLINEs", "MPCs", "CRODs", "CONRODs"))


def recover_shell_stresses(model, id_map, X, node_R, u_global, snorm_normals, stresses, results_json):
    """recover_shell_stresses! (stress_recovery.jl:163-430): per CQUAD4/CTRIA3 the
    max principal z1 stress into ``stresses[eid]`` and the "forces", "forces_bilin",
    "stresses" and "strains" rows into ``results_json``, in the dictionary's order."""
    del id_map, X, node_R
    if snorm_normals:
        raise NotImplementedError("SNORM normals leave the default branch")
    m, g, u = _recovery_inputs(model, u_global)
    try:
        shell, _ = g.recover_stresses(u, None, _pressure_deck(model))
    except JfgError as err:
        _raise(err)
    nq = m.q4_nodes.shape[0]
    forces = results_json.setdefault("forces", {})
    bilin = results_json.setdefault("forces_bilin", {})
    sres = results_json.setdefault("stresses", {})
    eres = results_json.setdefault("strains", {})
    ids = m.node_ids if m.node_ids is not None else np.arange(1, m.n_nodes + 1)
    f = lambda v: float(v)
    for i in m.shell_order:
        r = shell[i]
        if r[21] == 0.0:
            continue  # the reference's try block failed: no entries
        quad = i < nq
        j = i if quad else i - nq
        eid = int(m.q4_eid[j] if quad else m.t3_eid[j])
        T = float((m.q4_prop if quad else m.t3_prop)[j, 0])
        key = "quad4" if quad else "tria3"
        stresses[eid] = f(r[20])
        row = {"eid": eid, "fx": f(r[0]), "fy": f(r[1]), "fxy": f(r[2]), "mx": f(r[3]), "my": f(r[4]), "mxy": f(r[5]),
               "qx": f(r[6]), "qy": f(r[7])}
        forces.setdefault(key, []).append(row)
        if quad:
            rows = [dict(row, grid_id="CEN/4")]
            for k in range(4):
                rows.append({"eid": eid, "grid_id": int(ids[m.q4_nodes[j, k]]),
                             "fx": f(r[22 + 3 * k]), "fy": f(r[23 + 3 * k]), "fxy": f(r[24 + 3 * k]),
                             "mx": f(r[34 + 3 * k]), "my": f(r[35 + 3 * k]), "mxy": f(r[36 + 3 * k]),
                             "qx": f(r[6]), "qy": f(r[7])})
            bilin.setdefault("quad4", []).extend(rows)
        sz1, sz2, ez1, ez2 = r[8:11], r[11:14], r[14:17], r[17:20]

        def st(s, t, vm):
            return {"fiber_dist": t, "normal_x": f(s[0]), "normal_y": f(s[1]), "shear_xy": f(s[2]), "von_mises": f(vm),
                    "major": 0.0, "minor": 0.0}

        def sn(e, t):
            return {"fiber_dist": t, "normal_x": f(e[0]), "normal_y": f(e[1]), "shear_xy": f(e[2]), "major": 0.0, "minor": 0.0}

        sres.setdefault(key, []).append({"eid": eid, "z1": st(sz1, -T / 2, r[46]), "z2": st(sz2, T / 2, r[47])})
        eres.setdefault(key, []).append({"eid": eid, "z1": sn((ez1 + ez2) / 2.0, 0.0), "z2": sn((ez1 - ez2) / T, -1.0)})


def recover_bar_stresses(model, id_map, X, node_R, u_global, stresses, results_json):
    """recover_bar_stresses! (stress_recovery.jl:432-593): CBAR then CBEAM end
    forces into results_json["forces"]["cbar"], section-point stresses into
    results_json["stresses"]["cbar"] and |axial stress| into ``stresses[eid]``."""
    del id_map, X, node_R
    m, g, u = _recovery_inputs(model, u_global)
    try:
        _, bar = g.recover_stresses(u, m.bar_points)
    except JfgError as err:
        _raise(err)
    forces = results_json.setdefault("forces", {}).setdefault("cbar", [])
    sres = results_json.setdefault("stresses", {}).setdefault("cbar", [])
    names = ("axial", "shear_1", "shear_2", "torque", "moment_a1", "moment_a2", "moment_b1", "moment_b2")
    for i in range(bar.shape[0]):
        r = bar[i]
        if r[17] == 0.0:
            continue  # zero-length bar
        eid = int(m.bar_eid[i])
        stresses[eid] = abs(float(r[8]))
        forces.append({"eid": eid, **{n: float(r[k]) for k, n in enumerate(names)}})
        sres.append({"eid": eid, "end_a": {f"p{j + 1}": float(r[9 + j]) for j in range(4)},
                     "end_b": {f"p{j + 1}": float(r[13 + j]) for j in range(4)}, "axial": float(r[8])})


def release(model=None):
    """Drop cached device handles (all, or the one of `model`)."""
    keys = list(_HANDLES) if model is None else [id(model)]
    for k in keys:
        h = _HANDLES.pop(k, None)
        if h is not None:
            h[1].close()


def model_dict_from_arrays(m: ModelArrays) -> dict:
    """Reference-style model dictionary for a ModelArrays deck (test and example use)."""
    ids = m.node_ids if m.node_ids is not None else np.arange(1, m.n_nodes + 1)
    model = {"GRIDs": {}, "CORDs": {}, "CSHELLs": {}, "PSHELLs": {}, "MATs": {}, "CBARs": {}, "PBARLs": {},
             "RBE2s": {}, "PARAM_K6ROT": m.k6rot, "PARAM_SNORM": m.param_snorm}
    for i in range(m.n_nodes):
        cd = 0
        if m.node_R is not None and not np.allclose(m.node_R[i], np.eye(3)):
            cd = 1000 + i
            R = m.node_R[i]
            model["CORDs"][str(cd)] = {"U": R[:, 0].tolist(), "V": R[:, 1].tolist(), "W": R[:, 2].tolist()}
        model["GRIDs"][str(int(ids[i]))] = {"ID": int(ids[i]), "X": m.coords[i].tolist(), "CD": cd}
    eid = 1
    for nodes, props in ((m.q4_nodes, m.q4_prop), (m.t3_nodes, m.t3_prop)):
        for k in range(nodes.shape[0]):
            h, E, nu, G, br, tst, Gs = props[k]
            model["MATs"][str(eid)] = {"MID": eid, "E": E, "G": G, "NU": nu}
            prop = {"PID": eid, "MID": eid, "MID2": eid, "MID3": 0, "T": h, "BEND_RATIO": br, "TS_T": tst}
            if Gs != G:
                model["MATs"][str(eid + 10_000_000)] = {"MID": eid + 10_000_000, "E": 0.0, "G": Gs, "NU": 0.3}
                prop["MID3"] = eid + 10_000_000
            model["PSHELLs"][str(eid)] = prop
            model["CSHELLs"][str(eid)] = {"ID": eid, "PID": eid, "NODES": [int(ids[j]) for j in nodes[k]]}
            eid += 1
    for k in range(m.bar_nodes.shape[0]):
        r = m.bar_prop[k]
        model["MATs"][str(eid)] = {"MID": eid, "E": r[7], "G": r[8], "NU": -1.0}
        model["PBARLs"][str(eid)] = {"PID": eid, "MID": eid, "A": r[0], "I1": r[1], "I2": r[2], "I12": r[3],
                                     "J": r[4], "K1": r[5], "K2": r[6]}
        model["CBARs"][str(eid)] = {"ID": eid, "PID": eid, "GA": int(ids[m.bar_nodes[k, 0]]),
                                    "GB": int(ids[m.bar_nodes[k, 1]]), "V": r[9:12].tolist(),
                                    "WA": r[12:15].tolist(), "WB": r[15:18].tolist(),
                                    "PA": int(m.bar_pin[k, 0]), "PB": int(m.bar_pin[k, 1])}
        eid += 1
    for r in range(m.rbe2_master.shape[0]):
        digits = "".join(str(c + 1) for c in range(6) if m.rbe2_cm[r] & (1 << c))
        model["RBE2s"][str(eid)] = {"GN": int(ids[m.rbe2_master[r]]), "CM": int(digits),
                                    "GM": [int(ids[s]) for s in m.rbe2_slaves[m.rbe2_slave_ptr[r]:m.rbe2_slave_ptr[r + 1]]]}
        eid += 1
    return model
