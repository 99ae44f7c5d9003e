"""ctypes binding of libqbc_b200.so (include/qbc_b200.h).

Loading fails loudly when the library is missing: there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libqbc_b200.so")

QBC_OK, QBC_EINVAL, QBC_EIO, QBC_EGRAPH, QBC_ECUDA, QBC_ENOMEM, QBC_EDEVICE, QBC_ETIMEOUT, QBC_EBUSY = range(9)
QBC_INDEX_MHL, QBC_INDEX_H2H, QBC_INDEX_CSR = 0, 1, 2
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "EIO", 3: "EGRAPH", 4: "ECUDA", 5: "ENOMEM", 6: "EDEVICE",
                7: "ETIMEOUT", 8: "EBUSY"}

i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "qbc_last_error": (C.c_char_p, []),
    "qbc_version": (C.c_char_p, []),
    "qbc_graph_read": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "qbc_graph_from_lines": (C.c_int, [C.c_int, C.c_int, i32p, i32p, i32p, C.POINTER(vp)]),
    "qbc_graph_info": (C.c_int, [vp, i32p, i32p]),
    "qbc_graph_arcs": (C.c_int, [vp, i32p, i32p, i32p]),
    "qbc_graph_free": (None, [vp]),
    "qbc_read_order": (C.c_int, [C.c_char_p, C.c_int32, i32p]),
    "qbc_read_query": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, i32p, i32p]),
    "qbc_min_degree_order": (C.c_int, [vp, i32p]),
    "qbc_index_build": (C.c_int, [vp, C.c_int, i32p, C.c_int, C.POINTER(vp)]),
    "qbc_index_upload": (C.c_int, [vp, C.c_int]),
    "qbc_index_save": (C.c_int, [vp, C.c_char_p]),
    "qbc_index_load": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "qbc_index_build_device": (C.c_int, [vp, C.c_int, i32p, C.c_int, C.POINTER(vp)]),
    "qbc_index_release_device": (C.c_int, [vp]),
    "qbc_index_info": (C.c_int, [vp, i64p]),
    "qbc_index_scan_entries": (C.c_int, [vp, i32p, C.c_int32, i64p]),
    "qbc_index_group_entries": (C.c_int, [vp, i32p, C.c_int32, C.c_int32, i64p]),
    "qbc_index_label_group": (C.c_int, [vp, i32p]),
    "qbc_index_label_kernel": (C.c_int, [vp, C.c_char_p, C.c_int32]),
    "qbc_index_free": (None, [vp]),
    "qbc_index_export": (C.c_int, [vp, i32p, i32p, i32p, i64p, i32p, i32p, i32p]),
    "qbc_index_set_tuning": (C.c_int, [vp, i32p, C.c_int32]),
    "qbc_index_get_tuning": (C.c_int, [vp, i32p, C.c_int32]),
    "qbc_bc_all": (C.c_int, [vp, f64p]),
    "qbc_bc_sources": (C.c_int, [vp, i32p, C.c_int32, f64p]),
    "qbc_bc_plain": (C.c_int, [vp, i32p, C.c_int32, f64p]),
    "qbc_bc_sources_device": (C.c_int, [vp, vp, C.c_int32, vp, vp]),
    "qbc_bc_query": (C.c_int, [vp, i32p, C.c_int32, f64p]),
    "qbc_bc_query_batch": (C.c_int, [vp, i32p, i32p, C.c_int32, i32p, C.c_int32, f64p]),
    "qbc_index_profile": (C.c_int, [vp, C.c_int]),
    "qbc_index_stats": (C.c_int, [vp, f64p]),
    "qbc_bc_source_static": (C.c_int, [vp, C.c_int32, vp, vp]),
    "qbc_rows": (C.c_int, [vp, i32p, C.c_int32, i32p, u32p, i32p]),
    "qbc_autotune": (C.c_int, [vp, i32p, C.c_int32, i32p, C.c_int32, f64p]),
    "qbc_serve_open": (C.c_int, [vp, i32p, C.c_int32, i64p, C.c_int32, C.POINTER(vp)]),
    "qbc_serve_submit": (C.c_int, [vp, i32p, C.c_int32, i64p]),
    "qbc_serve_poll": (C.c_int, [vp, C.c_int64, f64p, f64p, i32p]),
    "qbc_serve_wait": (C.c_int, [vp, C.c_int64, C.c_double, f64p, f64p, i32p]),
    "qbc_serve_stats": (C.c_int, [vp, f64p, C.c_int32]),
    "qbc_serve_close": (C.c_int, [vp]),
}


class QbcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{STATUS_NAMES.get(code, code)}] {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m gpu_betweennesscentrality_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != QBC_OK:
        raise QbcError(rc, lib().qbc_last_error().decode())


def ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)
