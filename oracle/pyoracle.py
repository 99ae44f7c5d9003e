"""ctypes bindings of the oracle (liboracle.so) and of the compiled reference (_ref/libref_cpu.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by bench.py's CPU-baseline
and --impl reference legs.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_CPU_PATH = os.path.join(HERE, "_ref", "libref_cpu.so")

i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)


class _Arcs(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("off", i32p), ("head", i32p), ("w", i32p)]


class _TC(C.Structure):
    _fields_ = [("n", C.c_int), ("tree_width", C.c_int), ("tree_height", C.c_int),
                ("del_order", i32p), ("rank", i32p), ("vertex", i32p), ("parent", i32p), ("height", i32p),
                ("child_off", i32p), ("child", i32p),
                ("nb_off", i64p), ("nb", i32p), ("nb_len", i32p), ("nb_cnt", u32p), ("nb_hop", u32p),
                ("pos_off", i64p), ("pos", i32p),
                ("lab_off", i64p), ("dis", i32p), ("cnt", u32p), ("hop", u32p),
                ("euler_len", C.c_int), ("rmq_levels", C.c_int), ("euler_pos", i32p), ("rmq", i32p)]


class _H2H(C.Structure):
    _fields_ = [("n", C.c_int), ("rank", i32p), ("uvertex", i32p), ("parent", i32p), ("height", i32p),
                ("child_off", i32p), ("child", i32p),
                ("vert_off", i64p), ("vert", i32p), ("vert_w", i32p),
                ("pos_off", i64p), ("pos", i32p), ("dis_off", i64p), ("dis", i32p),
                ("popt_off", i64p), ("popt", i32p),
                ("euler_len", C.c_int), ("rmq_levels", C.c_int), ("to_rmq", i32p), ("rmq", i32p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        L.orc_arcs_build.argtypes = [C.c_int, C.c_int, i32p, i32p, i32p, C.POINTER(C.POINTER(_Arcs))]
        L.orc_arcs_free.argtypes = [C.POINTER(_Arcs)]
        L.orc_tc_build.argtypes = [C.c_int, C.c_int, i32p, i32p, i32p, C.POINTER(C.POINTER(_TC))]
        L.orc_tc_free.argtypes = [C.POINTER(_TC)]
        L.orc_h2h_build.argtypes = [C.POINTER(_Arcs), i32p, C.POINTER(C.POINTER(_H2H))]
        L.orc_h2h_free.argtypes = [C.POINTER(_H2H)]
        L.orc_mhl_rows.argtypes = [C.POINTER(_TC), C.c_int, i32p, u32p, i32p]
        L.orc_qbc_dist.argtypes = [C.POINTER(_H2H), C.c_int, i32p]
        L.orc_mhl_bc.argtypes = [C.POINTER(_TC), C.POINTER(_Arcs), i32p, C.c_int, f64p, C.c_int]
        L.orc_qbc_bc.argtypes = [C.POINTER(_H2H), C.POINTER(_Arcs), i32p, C.c_int, f64p, C.c_int]
        L.orc_rq_bc.argtypes = [C.POINTER(_TC), i32p, C.c_int, f64p, C.c_int]
        L.orc_brandes_bc.argtypes = [C.POINTER(_Arcs), i32p, C.c_int, f64p, C.c_int]
        L.orc_dijkstra_rows.argtypes = [C.POINTER(_Arcs), C.c_int, i32p, u32p, i32p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _arr(ptr, count, dtype):
    if count == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)


class Arcs:
    """Graph::ReadGraph arc list (src/Graph.cpp:4-37)."""

    def __init__(self, n, u1, v1, w):
        self._u, self._v, self._w = _i32(u1), _i32(v1), _i32(w)
        ptr = C.POINTER(_Arcs)()
        rc = lib().orc_arcs_build(int(n), self._u.shape[0], _p(self._u, i32p), _p(self._v, i32p),
                                  _p(self._w, i32p), C.byref(ptr))
        if rc:
            raise ValueError(f"orc_arcs_build failed ({rc})")
        self.ptr = ptr
        s = ptr.contents
        self.n, self.m = s.n, s.m
        self.off = _arr(s.off, self.n + 1, np.int32)
        self.head = _arr(s.head, self.m, np.int32)
        self.w = _arr(s.w, self.m, np.int32)

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.orc_arcs_free(self.ptr)
            self.ptr = None

    def bc(self, sources=None, nthreads=0):
        return _bc_call(lambda src, ns, out: lib().orc_brandes_bc(self.ptr, src, ns, out, nthreads), self.n, sources)

    def dijkstra_rows(self, source):
        d = np.empty(self.n, np.int32); c = np.empty(self.n, np.uint32); h = np.empty(self.n, np.int32)
        if lib().orc_dijkstra_rows(self.ptr, int(source), _p(d, i32p), _p(c, u32p), _p(h, i32p)):
            raise ValueError("bad source")
        return d, c, h


def _bc_call(fn, n, sources):
    out = np.zeros(n, np.float64)
    if sources is None:
        rc = fn(None, 0, _p(out, f64p))
    else:
        s = _i32(sources)
        rc = fn(_p(s, i32p), s.shape[0], _p(out, f64p))
    if rc:
        raise RuntimeError(f"oracle call failed ({rc})")
    return out


class TreeCount:
    """TreeDecomp restated (src/TreeCount/TreeDecomp.cpp)."""

    def __init__(self, n, u1, v1, w):
        u, v, ww = _i32(u1), _i32(v1), _i32(w)
        ptr = C.POINTER(_TC)()
        rc = lib().orc_tc_build(int(n), u.shape[0], _p(u, i32p), _p(v, i32p), _p(ww, i32p), C.byref(ptr))
        if rc:
            raise ValueError(f"orc_tc_build failed ({rc})")
        self.ptr = ptr
        s = ptr.contents
        self.n = n = s.n
        self.tree_width, self.tree_height = s.tree_width, s.tree_height
        self.del_order = _arr(s.del_order, n, np.int32)
        self.rank = _arr(s.rank, n + 1, np.int32)
        self.parent = _arr(s.parent, n, np.int32)
        self.height = _arr(s.height, n, np.int32)
        self.lab_off = _arr(s.lab_off, n + 1, np.int64)
        L = int(self.lab_off[-1])
        self.dis = _arr(s.dis, L, np.int32)
        self.cnt = _arr(s.cnt, L, np.uint32)
        self.hop = _arr(s.hop, L, np.uint32)
        self.pos_off = _arr(s.pos_off, n + 1, np.int64)
        self.pos = _arr(s.pos, int(self.pos_off[-1]), np.int32)
        self.euler_pos = _arr(s.euler_pos, n, np.int32)

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.orc_tc_free(self.ptr)
            self.ptr = None

    def rows(self, source):
        d = np.empty(self.n, np.int32); c = np.empty(self.n, np.uint32); h = np.empty(self.n, np.int32)
        if lib().orc_mhl_rows(self.ptr, int(source), _p(d, i32p), _p(c, u32p), _p(h, i32p)):
            raise ValueError("bad source")
        return d, c, h

    def bc(self, arcs: Arcs, sources=None, nthreads=0):
        return _bc_call(lambda src, ns, out: lib().orc_mhl_bc(self.ptr, arcs.ptr, src, ns, out, nthreads),
                        self.n, sources)

    def rq(self, points, nthreads=0):
        p = _i32(points)
        out = np.zeros(p.shape[0], np.float64)
        if lib().orc_rq_bc(self.ptr, _p(p, i32p), p.shape[0], _p(out, f64p), nthreads):
            raise ValueError("bad query point")
        return out


class H2H:
    """QBC's H2H index restated (src/buildIndex.cpp)."""

    def __init__(self, arcs: Arcs, node_order):
        self._arcs = arcs
        o = _i32(node_order)
        ptr = C.POINTER(_H2H)()
        rc = lib().orc_h2h_build(arcs.ptr, _p(o, i32p), C.byref(ptr))
        if rc:
            raise ValueError(f"orc_h2h_build failed ({rc})")
        self.ptr = ptr
        s = ptr.contents
        self.n = n = s.n
        self.rank = _arr(s.rank, n, np.int32)
        self.parent = _arr(s.parent, n, np.int32)
        self.height = _arr(s.height, n, np.int32)
        self.dis_off = _arr(s.dis_off, n + 1, np.int64)
        self.dis = _arr(s.dis, int(self.dis_off[-1]), np.int32)
        self.popt_off = _arr(s.popt_off, n + 1, np.int64)
        self.popt = _arr(s.popt, int(self.popt_off[-1]), np.int32)

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.orc_h2h_free(self.ptr)
            self.ptr = None

    def dist(self, source):
        d = np.empty(self.n, np.int32)
        if lib().orc_qbc_dist(self.ptr, int(source), _p(d, i32p)):
            raise ValueError("bad source")
        return d

    def bc(self, sources=None, nthreads=0):
        return _bc_call(lambda src, ns, out: lib().orc_qbc_bc(self.ptr, self._arcs.ptr, src, ns, out, nthreads),
                        self.n, sources)


# ---------------------------------------------------------------- compiled reference (CPU parts)
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_CPU_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_CPU_PATH)
        L.ref_tc_new.restype = C.c_void_p
        L.ref_tc_new.argtypes = [C.c_char_p, C.c_char_p]
        L.ref_tc_free.argtypes = [C.c_void_p]
        L.ref_tc_sizes.argtypes = [C.c_void_p, i64p]
        L.ref_tc_export.argtypes = [C.c_void_p, i32p, i32p, i32p, i32p, i64p, i32p, u32p, u32p, i64p, i32p, i32p]
        L.ref_tc_count_hop.argtypes = [C.c_void_p, C.c_int, C.c_int, u32p]
        L.ref_h2h_new.restype = C.c_void_p
        L.ref_h2h_new.argtypes = [C.c_char_p, C.c_char_p]
        L.ref_h2h_free.argtypes = [C.c_void_p]
        L.ref_h2h_sizes.argtypes = [C.c_void_p, i64p]
        L.ref_h2h_export.argtypes = [C.c_void_p, i32p, i32p, i32p, i32p, i64p, i32p, i64p, i32p]
        _ref = L
    return _ref


class RefTreeCount:
    """The reference's own TreeDecomp, run on a graph file (index dump goes to dump_path)."""

    def __init__(self, graph_path: str, dump_path: str):
        L = ref_lib()
        self.h = L.ref_tc_new(graph_path.encode(), dump_path.encode())
        sz = np.zeros(7, np.int64)
        L.ref_tc_sizes(self.h, _p(sz, i64p))
        n, nl, npos = int(sz[0]), int(sz[1]), int(sz[2])
        self.n, self.tree_width, self.tree_height = n, int(sz[3]), int(sz[4])
        self.del_order = np.zeros(n, np.int32); self.rank = np.zeros(n + 1, np.int32)
        self.parent = np.zeros(n, np.int32); self.height = np.zeros(n, np.int32)
        self.lab_off = np.zeros(n + 1, np.int64); self.dis = np.zeros(nl, np.int32)
        self.cnt = np.zeros(nl, np.uint32); self.hop = np.zeros(nl, np.uint32)
        self.pos_off = np.zeros(n + 1, np.int64); self.pos = np.zeros(npos, np.int32)
        self.euler_pos = np.zeros(n, np.int32)
        L.ref_tc_export(self.h, _p(self.del_order, i32p), _p(self.rank, i32p), _p(self.parent, i32p),
                        _p(self.height, i32p), _p(self.lab_off, i64p), _p(self.dis, i32p), _p(self.cnt, u32p),
                        _p(self.hop, u32p), _p(self.pos_off, i64p), _p(self.pos, i32p), _p(self.euler_pos, i32p))

    def count_hop(self, p1: int, q1: int):
        c = C.c_uint32(0)
        hop = ref_lib().ref_tc_count_hop(self.h, int(p1), int(q1), C.byref(c))
        return int(c.value), int(hop)

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_tc_free(self.h)
            self.h = None


class RefH2H:
    def __init__(self, graph_path: str, order_path: str):
        L = ref_lib()
        self.h = L.ref_h2h_new(graph_path.encode(), order_path.encode())
        sz = np.zeros(4, np.int64)
        L.ref_h2h_sizes(self.h, _p(sz, i64p))
        n, nd, npo = int(sz[0]), int(sz[1]), int(sz[2])
        self.n = n
        self.rank = np.zeros(n, np.int32); self.uvertex = np.zeros(n, np.int32)
        self.parent = np.zeros(n, np.int32); self.height = np.zeros(n, np.int32)
        self.dis_off = np.zeros(n + 1, np.int64); self.dis = np.zeros(nd, np.int32)
        self.popt_off = np.zeros(n + 1, np.int64); self.popt = np.zeros(npo, np.int32)
        L.ref_h2h_export(self.h, _p(self.rank, i32p), _p(self.uvertex, i32p), _p(self.parent, i32p),
                         _p(self.height, i32p), _p(self.dis_off, i64p), _p(self.dis, i32p),
                         _p(self.popt_off, i64p), _p(self.popt, i32p))

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_h2h_free(self.h)
            self.h = None
