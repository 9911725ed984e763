"""ctypes binding of ``libjfemgpu.so`` and a handle class over it.

The product path is the CUDA library only: if the shared object is missing
or no CUDA device is visible, the calls raise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import abi
from .abi import BAR_POINTS, BAR_REC, RECOVER_PRESSURE_DECK, SHELL_REC, JfgModelDesc, make_desc
from .decks import ModelArrays

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libjfemgpu.so")

# every entry point declared in include/jfem_gpu.h
EXPORTS = ("jfg_model_create", "jfg_pattern", "jfg_pattern_fill", "jfg_assemble_k", "jfg_assemble_kg",
           "jfg_assemble_k_device", "jfg_assemble_kg_device", "jfg_update_properties", "jfg_constraint_map",
           "jfg_set_stream", "jfg_last_timing", "jfg_kernel_timing", "jfg_timing_accumulated", "jfg_model_stats", "jfg_model_counts", "jfg_batch_workspace_bytes",
           "jfg_batch_reserve", "jfg_assemble_batch_device", "jfg_ff_set_free", "jfg_ff_extract_device",
           "jfg_ff_fetch", "jfg_ff_device_arrays", "jfg_dkdh_contract", "jfg_dkdh_load",
           "jfg_dkdh_contract_device", "jfg_dkdh_load_device", "jfg_recover_stresses",
           "jfg_recover_stresses_device", "jfg_kg_contract", "jfg_kg_contract_device", "jfg_server_create", "jfg_server_submit", "jfg_server_wait",
           "jfg_server_result", "jfg_server_release", "jfg_server_stats", "jfg_server_family_batch",
           "jfg_server_hold", "jfg_server_last_error", "jfg_server_destroy", "jfg_group_create", "jfg_group_member", "jfg_autotune", "jfg_launch_config", "jfg_assemble_batch_device_ws",
           "jfg_shell_thickness", "jfg_server_create_units", "jfg_kg_transfer_entries",
           "jfg_assemble_k_quad4_noalloc", "jfg_model_destroy", "jfg_last_error",
           "jfg_version")

_lib = None

_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)


class JfgError(RuntimeError):
    """Nonzero jfg_status, with the handle's message (the reference's error(...))."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"jfg status {status} ({abi.STATUS_NAMES.get(status, '?')}): {msg}")
        self.status = status
        self.msg = msg


def load(path: str = LIB_PATH):
    """Load the library (building it first when the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    from . import build as _b
    if path == LIB_PATH and _b.needs_build():
        try:
            _b.build()
        except Exception as exc:  # pragma: no cover - reported loudly below
            raise RuntimeError(f"CUDA library {path} is missing or stale and could not be built: {exc}") from exc
    L = C.CDLL(path)
    L.jfg_version.restype = C.c_char_p
    ver = L.jfg_version().decode()
    if path == LIB_PATH and not ver.endswith("src " + _b.source_hash()):
        raise RuntimeError(f"{path} was built from other sources ({ver}); rebuild it (jf_2026_05_19_b200/build.py --force)")
    L.jfg_model_create.argtypes = [C.POINTER(JfgModelDesc), C.POINTER(C.c_void_p)]
    L.jfg_model_create.restype = C.c_int32
    L.jfg_group_create.argtypes = [C.c_int32, C.POINTER(C.POINTER(JfgModelDesc)), C.POINTER(C.c_void_p)]
    L.jfg_group_create.restype = C.c_int32
    L.jfg_group_member.argtypes = [C.c_void_p, C.c_int32, _pi64]
    L.jfg_group_member.restype = C.c_int32
    _pi32 = C.POINTER(C.c_int32)
    L.jfg_autotune.argtypes = [C.c_void_p, C.c_int32, _pi32]
    L.jfg_autotune.restype = C.c_int32
    L.jfg_launch_config.argtypes = [C.c_void_p, _pi32, _pi32]
    L.jfg_launch_config.restype = C.c_int32
    L.jfg_assemble_batch_device_ws.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64] + [C.c_void_p] * 3 + \
        [C.c_int64] + [C.c_void_p] * 4
    L.jfg_assemble_batch_device_ws.restype = C.c_int32
    L.jfg_kg_transfer_entries.argtypes = [C.c_void_p, _pi64]
    L.jfg_kg_transfer_entries.restype = C.c_int32
    L.jfg_shell_thickness.argtypes = [C.c_void_p, _pd]
    L.jfg_shell_thickness.restype = C.c_int32
    L.jfg_server_create_units.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32, _pi32, _pi32, C.c_int32,
                                          C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.jfg_server_create_units.restype = C.c_int32
    L.jfg_pattern.argtypes = [C.c_void_p, _pi64, _pi64]
    L.jfg_pattern_fill.argtypes = [C.c_void_p, _pi64, _pi64]
    L.jfg_assemble_k.argtypes = [C.c_void_p, _pd, _pd, _pd]
    L.jfg_assemble_kg.argtypes = [C.c_void_p, _pd, _pd]
    L.jfg_assemble_k_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jfg_assemble_kg_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.jfg_update_properties.argtypes = [C.c_void_p, _pd, _pd]
    L.jfg_constraint_map.argtypes = [C.c_void_p, _pi64, _pi64, _pi64, _pi64, _pi64, _pd]
    L.jfg_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.jfg_last_timing.argtypes = [C.c_void_p, _pd, _pd, _pd]
    L.jfg_kernel_timing.argtypes = [C.c_void_p, _pd]
    L.jfg_model_stats.argtypes = [C.c_void_p, _pi64]
    L.jfg_assemble_k_quad4_noalloc.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                               C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jfg_timing_accumulated.argtypes = [C.c_void_p, C.c_int, _pd, _pi64, C.c_int]
    L.jfg_batch_workspace_bytes.argtypes = [C.c_void_p, C.c_int32, _pi64]
    L.jfg_batch_reserve.argtypes = [C.c_void_p, C.c_int32]
    L.jfg_assemble_batch_device.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jfg_model_counts.argtypes = [C.c_void_p, _pi64]
    L.jfg_ff_set_free.argtypes = [C.c_void_p, _pi64, C.c_int64]
    _pu8 = C.POINTER(C.c_uint8)
    L.jfg_dkdh_contract.argtypes = [C.c_void_p, _pd, _pd, _pd, _pd]
    L.jfg_dkdh_load.argtypes = [C.c_void_p, _pd, _pu8, _pu8, _pd]
    L.jfg_dkdh_contract_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jfg_dkdh_load_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jfg_recover_stresses.argtypes = [C.c_void_p, _pd, _pd, C.c_int32, _pd, _pd]
    L.jfg_kg_contract.argtypes = [C.c_void_p, _pd, _pd, _pd, _pd, _pd]
    L.jfg_kg_contract_device.argtypes = [C.c_void_p] + [C.c_void_p] * 5
    L.jfg_recover_stresses_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    L.jfg_ff_extract_device.argtypes = [C.c_void_p, C.c_void_p, _pi64, _pd, _pd]
    L.jfg_ff_fetch.argtypes = [C.c_void_p, _pi64, _pi64, _pd]
    L.jfg_ff_device_arrays.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    _pp = C.POINTER(C.c_void_p)
    L.jfg_server_create.argtypes = [_pp, _pp, C.c_int32, C.c_int64, C.c_int32, C.c_int32, _pp]
    L.jfg_server_submit.argtypes = [C.c_void_p, C.c_int32, _pd, C.c_int32, _pi64]
    L.jfg_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_int32)]
    L.jfg_server_result.argtypes = [C.c_void_p, C.c_int64, _pp, _pp, _pp, _pd]
    L.jfg_server_release.argtypes = [C.c_void_p, C.c_int64]
    L.jfg_server_stats.argtypes = [C.c_void_p, _pi64]
    L.jfg_server_family_batch.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
    L.jfg_server_hold.argtypes = [C.c_void_p, C.c_int32]
    L.jfg_server_last_error.argtypes = [C.c_void_p]
    L.jfg_server_last_error.restype = C.c_char_p
    L.jfg_server_destroy.argtypes = [C.c_void_p]
    L.jfg_server_destroy.restype = None
    L.jfg_model_destroy.argtypes = [C.c_void_p]
    L.jfg_model_destroy.restype = None
    L.jfg_last_error.argtypes = [C.c_void_p]
    L.jfg_last_error.restype = C.c_char_p
    L.jfg_version.restype = C.c_char_p
    for name in ("jfg_pattern", "jfg_pattern_fill", "jfg_assemble_k", "jfg_assemble_kg", "jfg_assemble_k_device",
                 "jfg_assemble_kg_device", "jfg_update_properties", "jfg_constraint_map", "jfg_set_stream",
                 "jfg_last_timing", "jfg_kernel_timing", "jfg_timing_accumulated", "jfg_model_stats",
                 "jfg_assemble_k_quad4_noalloc", "jfg_model_counts", "jfg_batch_workspace_bytes", "jfg_batch_reserve",
                 "jfg_assemble_batch_device", "jfg_server_create", "jfg_server_submit", "jfg_server_wait",
                 "jfg_server_result", "jfg_server_release", "jfg_server_stats", "jfg_server_family_batch",
                 "jfg_server_hold", "jfg_ff_set_free", "jfg_ff_extract_device", "jfg_ff_fetch",
                 "jfg_ff_device_arrays"):
        getattr(L, name).restype = C.c_int32
    _lib = L
    return L


def _ptr(a: Optional[np.ndarray], ctype):
    return C.cast(None, ctype) if a is None else a.ctypes.data_as(ctype)


class GpuModel:
    """One jfg_model handle: mesh, pattern and scatter map resident on the GPU."""

    def __init__(self, m: ModelArrays):
        self.L = load()
        self.model = m
        self.h = C.c_void_p()
        d, keep = make_desc(m)
        st = self.L.jfg_model_create(C.byref(d), C.byref(self.h))
        del keep
        self._finish_create(st)

    def _finish_create(self, st: int):
        if st != 0:
            msg = self.L.jfg_last_error(self.h).decode()
            self.L.jfg_model_destroy(self.h)
            self.h = C.c_void_p()
            raise JfgError(st, msg)
        nd = C.c_int64(); nnz = C.c_int64()
        self._check(self.L.jfg_pattern(self.h, C.byref(nd), C.byref(nnz)))
        self.ndof = int(nd.value)
        self.nnz = int(nnz.value)
        self._pattern = None

    def _check(self, st: int):
        if st != 0:
            raise JfgError(st, self.L.jfg_last_error(self.h).decode())

    @property
    def counts(self) -> list:
        """[n_nodes, n_quad4, n_tria3, n_bar] of this handle."""
        o = np.zeros(4, np.int64)
        self._check(self.L.jfg_model_counts(self.h, _ptr(o, _pi64)))
        return o.tolist()

    def close(self):
        if self.h:
            self.L.jfg_model_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- launch shapes -----------------------------------------------------
    CONFIG_KEYS = ("quad4_warps", "tria3_k_warps", "tria3_kg_threads", "bar_k_threads", "bar_kg_threads")

    def autotune(self, read: bool = True, write: bool = True) -> dict:
        """Time the candidate CTA shapes on this model and keep the fastest (jfg_autotune)."""
        c = np.zeros(5, np.int32)
        flags = (1 if read else 0) | (2 if write else 0)
        self._check(self.L.jfg_autotune(self.h, flags, c.ctypes.data_as(C.POINTER(C.c_int32))))
        return dict(zip(self.CONFIG_KEYS, (int(x) for x in c)))

    def launch_config(self, cfg: Optional[dict] = None) -> dict:
        pi32 = C.POINTER(C.c_int32)
        cin = None if cfg is None else np.array([cfg[k] for k in self.CONFIG_KEYS], np.int32)
        c = np.zeros(5, np.int32)
        self._check(self.L.jfg_launch_config(self.h, None if cin is None else cin.ctypes.data_as(pi32),
                                             c.ctypes.data_as(pi32)))
        return dict(zip(self.CONFIG_KEYS, (int(x) for x in c)))

    # -- pattern -----------------------------------------------------------
    def pattern(self):
        """(colptr, rowval), 1-based int64, SparseMatrixCSC layout."""
        if self._pattern is None:
            colptr = np.empty(self.ndof + 1, np.int64)
            rowval = np.empty(self.nnz, np.int64)
            self._check(self.L.jfg_pattern_fill(self.h, _ptr(colptr, _pi64), _ptr(rowval, _pi64)))
            self._pattern = (colptr, rowval)
        return self._pattern

    # -- host-buffer assembly (the reference-facing calls) -----------------
    def assemble_k(self, nzval: Optional[np.ndarray] = None, want_diag: bool = True,
                   diag_out: Optional[np.ndarray] = None):
        """K values (and max_elem_stiff, orig_diag) into host arrays; pass pinned
        arrays as nzval / diag_out to avoid pageable copies."""
        nz = np.empty(self.nnz) if nzval is None else nzval
        mx = np.zeros(1)
        diag = (np.empty(self.ndof) if diag_out is None else diag_out) if want_diag else None
        self._check(self.L.jfg_assemble_k(self.h, _ptr(nz, _pd), _ptr(mx, _pd), _ptr(diag, _pd)))
        return nz, float(mx[0]), diag

    def assemble_kg(self, u: np.ndarray, nzval: Optional[np.ndarray] = None):
        u = np.ascontiguousarray(u, np.float64)
        if u.shape != (self.ndof,):
            raise ValueError(f"u_global must have {self.ndof} entries")
        nz = np.empty(self.nnz) if nzval is None else nzval
        self._check(self.L.jfg_assemble_kg(self.h, _ptr(u, _pd), _ptr(nz, _pd)))
        return nz

    # -- device-resident assembly (torch CUDA tensors or raw pointers) ------
    def assemble_k_device(self, nz_ptr: int, max_ptr: int = 0, diag_ptr: int = 0):
        self._check(self.L.jfg_assemble_k_device(self.h, C.c_void_p(nz_ptr), C.c_void_p(max_ptr or None),
                                                 C.c_void_p(diag_ptr or None)))

    def assemble_kg_device(self, u_ptr: int, nz_ptr: int):
        self._check(self.L.jfg_assemble_kg_device(self.h, C.c_void_p(u_ptr), C.c_void_p(nz_ptr)))

    # -- batched variants (device pointers) --------------------------------
    def batch_workspace_bytes(self, n_var: int) -> int:
        b = C.c_int64()
        self._check(self.L.jfg_batch_workspace_bytes(self.h, int(n_var), C.byref(b)))
        return b.value

    def batch_reserve(self, n_var: int):
        self._check(self.L.jfg_batch_reserve(self.h, int(n_var)))

    def assemble_batch_device(self, n_var: int, h_ptr: int = 0, bar_prop_ptr: int = 0, u_ptr: int = 0,
                              u_stride: Optional[int] = None, nzk_ptr: int = 0, max_ptr: int = 0, diag_ptr: int = 0,
                              nzkg_ptr: int = 0):
        """K and/or KG for n_var variants sharing this model's mesh and pattern."""
        us = self.ndof if u_stride is None else int(u_stride)
        v = lambda p: C.c_void_p(p or None)
        self._check(self.L.jfg_assemble_batch_device(self.h, int(n_var), v(h_ptr), v(bar_prop_ptr), v(u_ptr), us,
                                                     v(nzk_ptr), v(max_ptr), v(diag_ptr), v(nzkg_ptr)))

    # -- free-dof submatrices (K_ff / Kg_ff) ----------------------------------
    def ff_set_free(self, free0: np.ndarray):
        """Free dofs as 0-based indices (sorted); stored 1-based by the library."""
        f = np.ascontiguousarray(np.asarray(free0, np.int64) + 1)
        self._check(self.L.jfg_ff_set_free(self.h, _ptr(f, _pi64), int(f.shape[0])))
        self._n_free = int(f.shape[0])

    def ff_extract(self, nz_ptr: int):
        """0.5 (A_ff + A_ff') of device values; returns (colptr, rowval, nzval, max|A_ff|, max|A_ff - A_ff'|)."""
        nnz = C.c_int64(); a = C.c_double(); b = C.c_double()
        self._check(self.L.jfg_ff_extract_device(self.h, C.c_void_p(nz_ptr), C.byref(nnz), C.byref(a), C.byref(b)))
        colptr = np.empty(self._n_free + 1, np.int64)
        rowval = np.empty(nnz.value, np.int64)
        val = np.empty(nnz.value)
        self._check(self.L.jfg_ff_fetch(self.h, _ptr(colptr, _pi64), _ptr(rowval, _pi64), _ptr(val, _pd)))
        return colptr, rowval, val, a.value, b.value

    def dkdh_contract(self, a: np.ndarray, b: np.ndarray):
        """Per-element a_e' dK_e/dh b_e of the shell-thickness sensitivity element:
        (c_q4, c_t3) arrays (jfg_dkdh_contract)."""
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        nq, nt = self.counts[1], self.counts[2]
        cq, ct = np.zeros(nq), np.zeros(nt)
        self._check(self.L.jfg_dkdh_contract(self.h, _ptr(a, _pd), _ptr(b, _pd), _ptr(cq, _pd), _ptr(ct, _pd)))
        return cq, ct

    def dkdh_load(self, u: np.ndarray, mask_q4: Optional[np.ndarray] = None, mask_t3: Optional[np.ndarray] = None):
        """Pseudo-load sum_e T' dK_e/dh T u_e over the masked elements (None = all of that type)."""
        u = np.ascontiguousarray(u, np.float64)
        pu8 = C.POINTER(C.c_uint8)
        mq = None if mask_q4 is None else np.ascontiguousarray(mask_q4, np.uint8)
        mt = None if mask_t3 is None else np.ascontiguousarray(mask_t3, np.uint8)
        out = np.empty(self.ndof)
        self._check(self.L.jfg_dkdh_load(self.h, _ptr(u, _pd), None if mq is None else mq.ctypes.data_as(pu8),
                                         None if mt is None else mt.ctypes.data_as(pu8), _ptr(out, _pd)))
        return out

    def dkdh_contract_device(self, a_ptr: int, b_ptr: int, cq_ptr: Optional[int], ct_ptr: Optional[int]):
        self._check(self.L.jfg_dkdh_contract_device(self.h, C.c_void_p(a_ptr), C.c_void_p(b_ptr), C.c_void_p(cq_ptr or None),
                                                    C.c_void_p(ct_ptr or None)))

    def dkdh_load_device(self, u_ptr: int, mq_ptr: Optional[int], mt_ptr: Optional[int], out_ptr: int):
        self._check(self.L.jfg_dkdh_load_device(self.h, C.c_void_p(u_ptr), C.c_void_p(mq_ptr or None),
                                                C.c_void_p(mt_ptr or None), C.c_void_p(out_ptr)))

    def kg_contract(self, u: np.ndarray, a: np.ndarray, b: np.ndarray):
        """Per-element a_e' KG_e(u) b_e of every CQUAD4 and CTRIA3 (jfg_kg_contract);
        divided by the element thickness, with a = b = phi, the buckling thickness
        sensitivity phi' dKG_e/dh phi."""
        u, a, b = (np.ascontiguousarray(x, np.float64) for x in (u, a, b))
        nq, nt = self.counts[1], self.counts[2]
        cq, ct = np.zeros(nq), np.zeros(nt)
        self._check(self.L.jfg_kg_contract(self.h, _ptr(u, _pd), _ptr(a, _pd), _ptr(b, _pd), _ptr(cq, _pd), _ptr(ct, _pd)))
        return cq, ct

    def kg_contract_device(self, u_ptr: int, a_ptr: int, b_ptr: int, cq_ptr: Optional[int], ct_ptr: Optional[int]):
        self._check(self.L.jfg_kg_contract_device(self.h, C.c_void_p(u_ptr), C.c_void_p(a_ptr), C.c_void_p(b_ptr),
                                                  C.c_void_p(cq_ptr or None), C.c_void_p(ct_ptr or None)))

    def recover_stresses(self, u: np.ndarray, bar_points: Optional[np.ndarray] = None, pressure_deck: bool = False):
        """SOL 101 output recovery (jfg_recover_stresses): shell records
        (n_quad4 + n_tria3, SHELL_REC) and bar records (n_bar, BAR_REC)."""
        u = np.ascontiguousarray(u, np.float64)
        nq, nt, nb = self.counts[1], self.counts[2], self.counts[3]
        pts = None if bar_points is None else np.ascontiguousarray(bar_points, np.float64).reshape(nb, BAR_POINTS)
        shell = np.empty((nq + nt, SHELL_REC))
        bar = np.empty((nb, BAR_REC))
        self._check(self.L.jfg_recover_stresses(self.h, _ptr(u, _pd), _ptr(pts, _pd), RECOVER_PRESSURE_DECK if pressure_deck else 0,
                                                _ptr(shell, _pd), _ptr(bar, _pd)))
        return shell, bar

    def recover_stresses_device(self, u_ptr: int, points_ptr: Optional[int], flags: int, shell_ptr: Optional[int],
                                bar_ptr: Optional[int]):
        self._check(self.L.jfg_recover_stresses_device(self.h, C.c_void_p(u_ptr), C.c_void_p(points_ptr or None), int(flags),
                                                       C.c_void_p(shell_ptr or None), C.c_void_p(bar_ptr or None)))

    def set_stream(self, stream_ptr: int):
        self._check(self.L.jfg_set_stream(self.h, C.c_void_p(stream_ptr or None)))

    def update_thickness(self, q4_h: Optional[np.ndarray], t3_h: Optional[np.ndarray]):
        q = None if q4_h is None else np.ascontiguousarray(q4_h, np.float64)
        t = None if t3_h is None else np.ascontiguousarray(t3_h, np.float64)
        self._check(self.L.jfg_update_properties(self.h, _ptr(q, _pd), _ptr(t, _pd)))

    def timing(self):
        a = C.c_double(); b = C.c_double(); c = C.c_double()
        self._check(self.L.jfg_last_timing(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def kernel_timing(self) -> dict:
        ms = np.zeros(6)
        self._check(self.L.jfg_kernel_timing(self.h, _ptr(ms, _pd)))
        return dict(zip(("quad4", "tria3", "bar", "dof_reduce", "block_reduce", "diag"), ms.tolist()))

    def timing_accumulated(self, kind: str, reset: bool = True):
        """Summed per-kernel ms and call count of 'k' or 'kg' assemblies."""
        ms = np.zeros(6); n = C.c_int64()
        self._check(self.L.jfg_timing_accumulated(self.h, 0 if kind == "k" else 1, _ptr(ms, _pd), C.byref(n), int(reset)))
        return dict(zip(("quad4", "tria3", "bar", "dof_reduce", "block_reduce", "diag"), ms.tolist())), int(n.value)

    def kg_transfer_entries(self) -> int:
        """KG values a pageable host-buffer call moves over the bus (-1 before the first such call)."""
        n = C.c_int64()
        self._check(self.L.jfg_kg_transfer_entries(self.h, C.byref(n)))
        return int(n.value)

    def stats(self) -> dict:
        out = np.zeros(8, np.int64)
        self._check(self.L.jfg_model_stats(self.h, _ptr(out, _pi64)))
        keys = ("staging_values", "n_blocks", "nnz", "dof_contribs", "dof_raw_values", "element_pairs", "n_diag",
                "device_bytes_in_use")
        return dict(zip(keys, (int(x) for x in out)))

    def constraint_map(self):
        nd = C.c_int64(); nt = C.c_int64()
        self._check(self.L.jfg_constraint_map(self.h, C.byref(nd), C.byref(nt), None, None, None, None))
        dep = np.empty(nd.value, np.int64); ptr = np.empty(nd.value + 1, np.int64)
        ind = np.empty(nt.value, np.int64); coef = np.empty(nt.value)
        self._check(self.L.jfg_constraint_map(self.h, None, None, _ptr(dep, _pi64), _ptr(ptr, _pi64),
                                              _ptr(ind, _pi64), _ptr(coef, _pd)))
        return dep, ptr, ind, coef


def version() -> str:
    return load().jfg_version().decode()


SERVE_BATCHED, SERVE_SERIAL = 0, 1



class GpuGroup(GpuModel):
    """A group handle (jfg_group_create): several models side by side in one
    handle, so each launch takes bins from all of them.  Every GpuModel call
    works on the group; member(i) gives a member's offsets and member_values /
    member_pattern its slice of the group's arrays."""

    def __init__(self, models):
        self.L = load()
        self.models = list(models)
        self.model = None
        self.h = C.c_void_p()
        pairs = [make_desc(m) for m in self.models]
        arr = (C.POINTER(JfgModelDesc) * len(pairs))(*[C.pointer(d) for d, _ in pairs])
        st = self.L.jfg_group_create(len(pairs), arr, C.byref(self.h))
        del pairs, arr
        self._finish_create(st)

    def member(self, i: int) -> dict:
        o = np.zeros(8, np.int64)
        self._check(self.L.jfg_group_member(self.h, int(i), _ptr(o, _pi64)))
        keys = ("n_nodes", "node_off", "nnz", "nnz_off", "quad4_off", "tria3_off", "bar_off", "elements")
        return dict(zip(keys, (int(x) for x in o)))

    def member_values(self, nz: np.ndarray, i: int) -> np.ndarray:
        """Member i's nonzeros (CSC order) out of a group-wide value array."""
        d = self.member(i)
        return nz[d["nnz_off"]:d["nnz_off"] + d["nnz"]]

    def member_dofs(self, v: np.ndarray, i: int) -> np.ndarray:
        d = self.member(i)
        return v[6 * d["node_off"]:6 * (d["node_off"] + d["n_nodes"])]

    def member_pattern(self, i: int):
        """Member i's (colptr, rowval), 1-based, as its own handle would give them."""
        cp, rv = self.pattern()
        d = self.member(i)
        a, n = 6 * d["node_off"], 6 * d["n_nodes"]
        colptr = cp[a:a + n + 1] - d["nnz_off"]
        rowval = rv[d["nnz_off"]:d["nnz_off"] + d["nnz"]] - a
        return colptr, rowval

class Server:
    """Device-resident request loop over model families (jfg_server_* in the C ABI).

    Each request carries a new shell-thickness vector for one family and gets
    that family's K (and KG when the family has a displacement field); the
    results stay on the device until released.  The GpuModel handles must
    outlive the server, which uses them exclusively while it runs.
    """

    def __init__(self, models, u=None, hbm_budget_bytes: int = 150 * 10**9, max_batch: int = 32,
                 policy: int = SERVE_BATCHED, family_map=None):
        """models: the launch units (GpuModel or GpuGroup handles), u: one
        displacement field per unit (the group's concatenation for a group) or
        None.  family_map: per family (unit, member), member -1 for a plain
        handle; by default one plain unit per family (jfg_server_create_units)."""
        self.L = load()
        self.models = list(models)
        n = len(self.models)
        fmap = family_map if family_map is not None else [(i, -1) for i in range(n)]
        hs = (C.c_void_p * n)(*[m.h.value for m in self.models])
        self._u = [None if (u is None or u[i] is None) else np.ascontiguousarray(u[i], np.float64) for i in range(n)]
        us = (C.c_void_p * n)(*[None if a is None else a.ctypes.data for a in self._u])
        fu = np.array([f[0] for f in fmap], np.int32)
        fm = np.array([f[1] for f in fmap], np.int32)
        out = C.c_void_p()
        pi32 = C.POINTER(C.c_int32)
        st = self.L.jfg_server_create_units(hs, us, n, fu.ctypes.data_as(pi32), fm.ctypes.data_as(pi32), len(fmap),
                                            int(hbm_budget_bytes), int(max_batch), int(policy), C.byref(out))
        if st != 0:
            raise JfgError(st, "jfg_server_create_units failed (status %d)" % st)
        self.s = out.value
        self.n_shell = []
        for uidx, mem in fmap:
            g = self.models[uidx]
            if mem < 0:
                self.n_shell.append(int(g.counts[1] + g.counts[2]))
            else:
                mm = g.models[mem]
                self.n_shell.append(int(mm.q4_nodes.shape[0] + mm.t3_nodes.shape[0]))

    def _check(self, st: int):
        if st != 0:
            raise JfgError(st, self.L.jfg_server_last_error(self.s).decode())

    def submit(self, family: int, h: np.ndarray, keep: bool = True) -> int:
        h = np.ascontiguousarray(h, np.float64)
        if h.shape != (self.n_shell[family],):
            raise ValueError(f"family {family} takes {self.n_shell[family]} thicknesses")
        t = C.c_int64()
        self._check(self.L.jfg_server_submit(self.s, int(family), _ptr(h, _pd), int(keep), C.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> bool:
        d = C.c_int32()
        self._check(self.L.jfg_server_wait(self.s, int(ticket), float(timeout), C.byref(d)))
        return bool(d.value)

    def result(self, ticket: int):
        """(K ptr, KG ptr or None, max ptr, (t_submit, t_launch, t_done)) of a finished request."""
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        t = np.zeros(3)
        self._check(self.L.jfg_server_result(self.s, int(ticket), C.byref(a), C.byref(b), C.byref(c), _ptr(t, _pd)))
        return a.value, b.value, c.value, tuple(t.tolist())

    def release(self, ticket: int):
        self._check(self.L.jfg_server_release(self.s, int(ticket)))

    def stats(self) -> dict:
        o = np.zeros(6, np.int64)
        self._check(self.L.jfg_server_stats(self.s, _ptr(o, _pi64)))
        return dict(zip(("submitted", "completed", "batches", "max_batch", "pool_peak_bytes", "queued"), o.tolist()))

    def hold(self, on: bool = True):
        """Queue requests without launching them while on; off admits the queue."""
        self._check(self.L.jfg_server_hold(self.s, int(on)))

    def batch_limit(self, family: int) -> int:
        b = C.c_int32()
        self._check(self.L.jfg_server_family_batch(self.s, int(family), C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "s", None):
            self.L.jfg_server_destroy(self.s)
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
