"""ctypes view of ``include/jfem_gpu.h``: the model descriptor and status codes.

``make_desc`` turns a :class:`~jf_2026_05_19_b200.decks.ModelArrays` into a
``jfg_model_desc`` whose pointers reference contiguous numpy buffers; the
returned keep-alive tuple must outlive every call that uses the descriptor.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .decks import ModelArrays, N_BAR_PROP, N_SHELL_PROP

JFG_OK = 0
JFG_ERR_INVALID = 1
JFG_ERR_UNSUPPORTED = 2
JFG_ERR_CUDA = 3
JFG_ERR_TIMEOUT = 4
JFG_ERR_STATE = 5
JFG_ERR_NOMEM = 6
JFG_ERR_REFERENCE_RAISES = 7

# output recovery records (jfg_recover_stresses)
SHELL_REC = 48
BAR_REC = 18
BAR_POINTS = 9
RECOVER_PRESSURE_DECK = 1

STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "UNSUPPORTED", 3: "CUDA", 4: "TIMEOUT",
                5: "STATE", 6: "NOMEM", 7: "REFERENCE_RAISES"}

_pd = C.POINTER(C.c_double)
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)


class JfgModelDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("coords", _pd),
        ("node_R", _pd),
        ("n_quad4", C.c_int64),
        ("quad4_nodes", _pi32),
        ("quad4_prop", _pd),
        ("n_tria3", C.c_int64),
        ("tria3_nodes", _pi32),
        ("tria3_prop", _pd),
        ("n_bar", C.c_int64),
        ("bar_nodes", _pi32),
        ("bar_prop", _pd),
        ("bar_pin", _pi32),
        ("n_rbe2", C.c_int64),
        ("rbe2_master", _pi32),
        ("rbe2_cm", _pi32),
        ("rbe2_slave_ptr", _pi64),
        ("rbe2_slaves", _pi32),
        ("k6rot", C.c_double),
        ("param_snorm", C.c_double),
    ]


def _c(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a


def _ptr(a, ctype):
    if a is None or a.size == 0:
        # a valid non-null pointer for empty arrays keeps the C side simple
        a = np.zeros(1, dtype=np.float64 if ctype is _pd else (np.int64 if ctype is _pi64 else np.int32))
        return a, a.ctypes.data_as(ctype)
    return a, a.ctypes.data_as(ctype)


def make_desc(m: ModelArrays):
    keep = []

    def P(a, dtype, ctype):
        if a is None:
            return C.cast(None, ctype)
        arr = _c(a, dtype)
        arr, p = _ptr(arr, ctype)
        keep.append(arr)
        return p

    d = JfgModelDesc()
    d.n_nodes = m.n_nodes
    d.coords = P(m.coords, np.float64, _pd)
    d.node_R = P(None if m.node_R is None else m.node_R.reshape(-1, 9), np.float64, _pd)
    d.n_quad4 = int(m.q4_nodes.shape[0])
    d.quad4_nodes = P(m.q4_nodes, np.int32, _pi32)
    d.quad4_prop = P(m.q4_prop.reshape(-1, N_SHELL_PROP), np.float64, _pd)
    d.n_tria3 = int(m.t3_nodes.shape[0])
    d.tria3_nodes = P(m.t3_nodes, np.int32, _pi32)
    d.tria3_prop = P(m.t3_prop.reshape(-1, N_SHELL_PROP), np.float64, _pd)
    d.n_bar = int(m.bar_nodes.shape[0])
    d.bar_nodes = P(m.bar_nodes, np.int32, _pi32)
    d.bar_prop = P(m.bar_prop.reshape(-1, N_BAR_PROP), np.float64, _pd)
    d.bar_pin = P(m.bar_pin, np.int32, _pi32)
    d.n_rbe2 = int(m.rbe2_master.shape[0])
    d.rbe2_master = P(m.rbe2_master, np.int32, _pi32)
    d.rbe2_cm = P(m.rbe2_cm, np.int32, _pi32)
    d.rbe2_slave_ptr = P(m.rbe2_slave_ptr, np.int64, _pi64)
    d.rbe2_slaves = P(m.rbe2_slaves, np.int32, _pi32)
    d.k6rot = float(m.k6rot)
    d.param_snorm = float(m.param_snorm)
    return d, tuple(keep)
