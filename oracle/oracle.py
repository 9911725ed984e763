"""ctypes wrapper of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker / reference arm.  The
product library never imports it.  Parity unpinned (see jfem_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

from jf_2026_05_19_b200.abi import JfgModelDesc, make_desc
from jf_2026_05_19_b200.decks import ModelArrays

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "jfem_oracle.cpp")):
        subprocess.run(["make", "-C", HERE, "-B" if force else "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        pd = C.POINTER(C.c_double)
        pi64 = C.POINTER(C.c_int64)
        L.oracle_assemble_k.argtypes = [C.POINTER(JfgModelDesc), C.POINTER(C.c_void_p)]
        L.oracle_assemble_kg.argtypes = [C.POINTER(JfgModelDesc), pd, C.POINTER(C.c_void_p)]
        L.oracle_nnz.argtypes = [C.c_void_p]; L.oracle_nnz.restype = C.c_int64
        L.oracle_ndof.argtypes = [C.c_void_p]; L.oracle_ndof.restype = C.c_int64
        L.oracle_error.argtypes = [C.c_void_p]; L.oracle_error.restype = C.c_char_p
        L.oracle_max_elem_stiff.argtypes = [C.c_void_p]; L.oracle_max_elem_stiff.restype = C.c_double
        L.oracle_fetch.argtypes = [C.c_void_p, pi64, pi64, pd, pd]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_q4_stiffness_local.argtypes = [pd, pd, C.c_double, pd]
        L.oracle_t3_stiffness_local.argtypes = [pd, pd, C.c_double, pd]
        L.oracle_constraint_map.argtypes = [C.POINTER(JfgModelDesc), pi64, pi64, pi64, pd]
        L.oracle_constraint_map.restype = C.c_int64
        L.oracle_num_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_q4_generic_local.argtypes = [pd, C.c_double, C.c_double, C.c_double, pd, pd]
        L.oracle_t3_generic_local.argtypes = [pd, C.c_double, C.c_double, C.c_double, pd, pd]
        pu8 = C.POINTER(C.c_uint8)
        L.oracle_dkdh.argtypes = [C.POINTER(JfgModelDesc), pd, pd, pd, pd, pd, pu8, pu8, pd]
        L.oracle_recover.argtypes = [C.POINTER(JfgModelDesc), pd, pd, C.c_int32, pd, pd]
        L.oracle_kg_contract.argtypes = [C.POINTER(JfgModelDesc), pd, pd, pd, pd, pd]
        L.oracle_kg_contract.restype = C.c_int
        L.oracle_set_abs_sums.argtypes = [C.c_int]
        L.oracle_fetch_abs_sums.argtypes = [C.c_void_p, pd]
        L.oracle_fetch_abs_sums.restype = C.c_int
        L.oracle_phase_seconds.argtypes = [C.c_void_p, pd]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"oracle status {status}: {msg}")
        self.status = status


def _fetch(h, with_diag):
    L = lib()
    nnz = L.oracle_nnz(h); ndof = L.oracle_ndof(h)
    colptr = np.empty(ndof + 1, np.int64); rowval = np.empty(nnz, np.int64); nzval = np.empty(nnz)
    diag = np.empty(ndof) if with_diag else None
    pd = C.POINTER(C.c_double); pi64 = C.POINTER(C.c_int64)
    L.oracle_fetch(h, colptr.ctypes.data_as(pi64), rowval.ctypes.data_as(pi64), nzval.ctypes.data_as(pd),
                   diag.ctypes.data_as(pd) if diag is not None else C.cast(None, pd))
    return colptr, rowval, nzval, diag


def _detail(h, nnz, abs_sums):
    """Phase seconds and, when asked for, the per-entry sums of |term|."""
    L = lib()
    t = np.zeros(2)
    L.oracle_phase_seconds(h, t.ctypes.data_as(C.POINTER(C.c_double)))
    out = {"t_elements": float(t[0]), "t_sparse": float(t[1])}
    if abs_sums:
        a = np.empty(nnz)
        if L.oracle_fetch_abs_sums(h, a.ctypes.data_as(C.POINTER(C.c_double))):
            raise RuntimeError("oracle abs sums were not computed")
        out["abs_sums"] = a
    return out


def assemble_k(m: ModelArrays, detail: bool = False, abs_sums: bool = False):
    """Returns (colptr, rowval, nzval, max_elem_stiff, orig_diag), 1-based CSC.

    With detail=True a sixth item is a dict with the phase times (element
    loops, redistribution + sparse) and, with abs_sums=True, the per-entry
    sums of |term| (the scale of each entry's summation rounding)."""
    L = lib()
    d, keep = make_desc(m)
    h = C.c_void_p()
    L.oracle_set_abs_sums(int(abs_sums))
    try:
        st = L.oracle_assemble_k(C.byref(d), C.byref(h))
    finally:
        L.oracle_set_abs_sums(0)
    try:
        if st != 0:
            raise OracleError(st, L.oracle_error(h).decode())
        colptr, rowval, nzval, diag = _fetch(h, True)
        res = (colptr, rowval, nzval, L.oracle_max_elem_stiff(h), diag)
        return res + (_detail(h, len(nzval), abs_sums),) if detail else res
    finally:
        L.oracle_free(h)
        del keep


def assemble_kg(m: ModelArrays, u: np.ndarray, detail: bool = False, abs_sums: bool = False):
    """Returns (colptr, rowval, nzval); a fourth item as in assemble_k with detail=True."""
    L = lib()
    d, keep = make_desc(m)
    u = np.ascontiguousarray(u, np.float64)
    h = C.c_void_p()
    L.oracle_set_abs_sums(int(abs_sums))
    try:
        st = L.oracle_assemble_kg(C.byref(d), u.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    finally:
        L.oracle_set_abs_sums(0)
    try:
        if st != 0:
            raise OracleError(st, L.oracle_error(h).decode())
        colptr, rowval, nzval, _ = _fetch(h, False)
        res = (colptr, rowval, nzval)
        return res + (_detail(h, len(nzval), abs_sums),) if detail else res
    finally:
        L.oracle_free(h)
        del keep


def constraint_map(m: ModelArrays):
    L = lib()
    d, keep = make_desc(m)
    n = L.oracle_constraint_map(C.byref(d), None, None, None, None)
    dep = np.empty(n, np.int64); ptr = np.empty(n + 1, np.int64)
    L.oracle_constraint_map(C.byref(d), dep.ctypes.data_as(C.POINTER(C.c_int64)), ptr.ctypes.data_as(C.POINTER(C.c_int64)), None, None)
    ind = np.empty(ptr[-1], np.int64); coef = np.empty(ptr[-1])
    L.oracle_constraint_map(C.byref(d), dep.ctypes.data_as(C.POINTER(C.c_int64)), ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                            ind.ctypes.data_as(C.POINTER(C.c_int64)), coef.ctypes.data_as(C.POINTER(C.c_double)))
    del keep
    return dep, ptr, ind, coef


def q4_local(lc: np.ndarray, prop: np.ndarray, k6rot: float = 100.0) -> np.ndarray:
    L = lib()
    lc = np.ascontiguousarray(lc, np.float64).reshape(8)
    prop = np.ascontiguousarray(prop, np.float64).reshape(7)
    out = np.empty((24, 24))
    pd = C.POINTER(C.c_double)
    L.oracle_q4_stiffness_local(lc.ctypes.data_as(pd), prop.ctypes.data_as(pd), k6rot, out.ctypes.data_as(pd))
    return out


def t3_local(lc: np.ndarray, prop: np.ndarray, k6rot: float = 100.0) -> np.ndarray:
    L = lib()
    lc = np.ascontiguousarray(lc, np.float64).reshape(6)
    prop = np.ascontiguousarray(prop, np.float64).reshape(7)
    out = np.empty((18, 18))
    pd = C.POINTER(C.c_double)
    L.oracle_t3_stiffness_local(lc.ctypes.data_as(pd), prop.ctypes.data_as(pd), k6rot, out.ctypes.data_as(pd))
    return out


def q4_generic_local(lc: np.ndarray, E: float, nu: float, h: float):
    """(K, dK/dh) of stiffness_quad4_generic in the element frame (24 x 24 each)."""
    L = lib()
    lc = np.ascontiguousarray(lc, np.float64).reshape(8)
    K, dK = np.empty((24, 24)), np.empty((24, 24))
    pd = C.POINTER(C.c_double)
    L.oracle_q4_generic_local(lc.ctypes.data_as(pd), E, nu, h, K.ctypes.data_as(pd), dK.ctypes.data_as(pd))
    return K, dK


def t3_generic_local(lc: np.ndarray, E: float, nu: float, h: float):
    """(K, dK/dh) of stiffness_tria3_generic in the element frame (18 x 18 each)."""
    L = lib()
    lc = np.ascontiguousarray(lc, np.float64).reshape(6)
    K, dK = np.empty((18, 18)), np.empty((18, 18))
    pd = C.POINTER(C.c_double)
    L.oracle_t3_generic_local(lc.ctypes.data_as(pd), E, nu, h, K.ctypes.data_as(pd), dK.ctypes.data_as(pd))
    return K, dK


def dkdh(m: ModelArrays, a=None, b=None, u=None, mask_q4=None, mask_t3=None):
    """Shell-thickness sensitivities of the model (see oracle_dkdh): per-element
    contractions a_e' dK_e/dh b_e (CQUAD4, CTRIA3) when a and b are given, and
    the pseudo-load dK/dh u over the masked elements (all when no mask) when u
    is given."""
    L = lib()
    desc, keep = make_desc(m)
    pd, pu8 = C.POINTER(C.c_double), C.POINTER(C.c_uint8)
    nq, nt, ndof = m.q4_nodes.shape[0], m.t3_nodes.shape[0], 6 * m.coords.shape[0]
    arr = lambda x, dt: None if x is None else np.ascontiguousarray(x, dt)
    a, b, u = arr(a, np.float64), arr(b, np.float64), arr(u, np.float64)
    mq = arr(mask_q4 if mask_q4 is not None or u is None else np.ones(nq), np.uint8)
    mt = arr(mask_t3 if mask_t3 is not None or u is None else np.ones(nt), np.uint8)
    cq = np.zeros(nq) if a is not None else None
    ct = np.zeros(nt) if a is not None else None
    load = np.zeros(ndof) if u is not None else None
    ptr = lambda x, t: None if x is None else x.ctypes.data_as(t)
    L.oracle_dkdh(C.byref(desc), ptr(a, pd), ptr(b, pd), ptr(cq, pd), ptr(ct, pd), ptr(u, pd), ptr(mq, pu8), ptr(mt, pu8),
                  ptr(load, pd))
    del keep
    return cq, ct, load


SHELL_REC, BAR_REC, BAR_POINTS = 48, 18, 9
RECOVER_PRESSURE_DECK = 1


def recover(m: ModelArrays, u, bar_points=None, flags: int = 0):
    """SOL 101 output recovery of the model (see oracle_recover): the shell
    records (CQUAD4s then CTRIA3s, SHELL_REC values each) and the bar records
    (BAR_REC values each) for displacement u (ndof)."""
    L = lib()
    desc, keep = make_desc(m)
    pd = C.POINTER(C.c_double)
    ns, nb = m.q4_nodes.shape[0] + m.t3_nodes.shape[0], m.bar_nodes.shape[0]
    u = np.ascontiguousarray(u, np.float64)
    pts = None if bar_points is None else np.ascontiguousarray(bar_points, np.float64).reshape(nb, BAR_POINTS)
    shell = np.zeros((ns, SHELL_REC))
    bar = np.zeros((nb, BAR_REC))
    L.oracle_recover(C.byref(desc), u.ctypes.data_as(pd), None if pts is None else pts.ctypes.data_as(pd), int(flags),
                     shell.ctypes.data_as(pd), bar.ctypes.data_as(pd))
    del keep
    return shell, bar


def kg_contract(m: ModelArrays, u, a, b):
    """Per-element a_e' KG_e(u) b_e of every CQUAD4 and CTRIA3 (see oracle_kg_contract)."""
    L = lib()
    desc, keep = make_desc(m)
    pd = C.POINTER(C.c_double)
    u, a, b = (np.ascontiguousarray(x, np.float64) for x in (u, a, b))
    cq, ct = np.zeros(m.q4_nodes.shape[0]), np.zeros(m.t3_nodes.shape[0])
    st = L.oracle_kg_contract(C.byref(desc), u.ctypes.data_as(pd), a.ctypes.data_as(pd), b.ctypes.data_as(pd),
                              cq.ctypes.data_as(pd), ct.ctypes.data_as(pd))
    del keep
    if st:
        raise RuntimeError(f"oracle_kg_contract status {st}")
    return cq, ct


def to_scipy(colptr, rowval, nzval, ndof):
    return sp.csc_matrix((nzval, rowval - 1, colptr - 1), shape=(ndof, ndof))


def set_threads(n: int):
    lib().oracle_set_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())
