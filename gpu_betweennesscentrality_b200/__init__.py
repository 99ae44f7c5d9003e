"""B200-native query-based betweenness centrality (QBC / MHL-QBC / RQ).

Host-side mirror of the reference's driver API (``class Graph``, include/Graph.h:64-200) over the
C ABI of ``libqbc_b200.so``:

    g = Graph(device=0)
    g.ReadGraph("graph.txt")                      # src/Graph.cpp:4
    g.brandesBCIndexGPU_5("graph.txt")            # MHL-QBC (MHLQBC.cu:495) -> g.BC
    g.brandesBCIndexGPU_5("graph.txt", "order")   # QBC with an order file (QBC.cu:419) -> g.BC
    g.brandesBCIndexGPU_PointBatch("graph.txt", points, q)   # RQ (RQ.cu:465) -> g.h_PointBC

``Index`` exposes the lower-level calls (rows, partial BC over a source list, plain path, device
pointers) used by tests and the benchmark.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Optional, Sequence

import numpy as np

from .capi import (QBC_INDEX_CSR, QBC_INDEX_H2H, QBC_INDEX_MHL, QbcError, check, f64p, i32, i32p, i64p, lib, ptr,
                   u32p)

__all__ = ["Graph", "Index", "QbcError", "QBC_INDEX_MHL", "QBC_INDEX_H2H", "QBC_INDEX_CSR", "read_order", "read_query"]


class _GraphHandle:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        if self.h and lib is not None:
            try:
                lib().qbc_graph_free(self.h)
            except Exception:
                pass
            self.h = None


def _graph_from_path(path: str) -> _GraphHandle:
    h = C.c_void_p()
    check(lib().qbc_graph_read(path.encode(), C.byref(h)))
    return _GraphHandle(h)


def _graph_from_lines(n: int, u1, v1, w) -> _GraphHandle:
    u1, v1, w = i32(u1), i32(v1), i32(w)
    h = C.c_void_p()
    check(lib().qbc_graph_from_lines(int(n), int(u1.shape[0]), ptr(u1, i32p), ptr(v1, i32p), ptr(w, i32p), C.byref(h)))
    return _GraphHandle(h)


def _graph_info(gh: _GraphHandle):
    n, m = C.c_int32(), C.c_int32()
    check(lib().qbc_graph_info(gh.h, C.byref(n), C.byref(m)))
    return n.value, m.value


def read_order(path: str, n: int) -> np.ndarray:
    o = np.empty(n, np.int32)
    check(lib().qbc_read_order(path.encode(), int(n), ptr(o, i32p)))
    return o


def read_query(path: str, n: int) -> np.ndarray:
    q = C.c_int32()
    check(lib().qbc_read_query(path.encode(), int(n), 0, C.byref(q), None))
    ids = np.empty(q.value, np.int32)
    check(lib().qbc_read_query(path.encode(), int(n), int(q.value), C.byref(q), ptr(ids, i32p)))
    return ids


class Index:
    """Tree-decomposition index of a graph, resident on one GPU.  ``on_device`` fills the label
    rows on the GPU (``qbc_index_build_device``); otherwise they are built on the host and uploaded
    to ``device`` (None: host only)."""

    def __init__(self, graph: _GraphHandle, kind: int = QBC_INDEX_MHL, node_order=None, nthreads: int = 0,
                 device: Optional[int] = 0, on_device: bool = False):
        self._graph = graph
        h = C.c_void_p()
        o = None if node_order is None else i32(node_order)
        optr = None if o is None else ptr(o, i32p)
        if on_device:
            if device is None:
                raise QbcError(1, "a device build needs a device")
            check(lib().qbc_index_build_device(graph.h, int(kind), optr, int(device), C.byref(h)))
        else:
            check(lib().qbc_index_build(graph.h, int(kind), optr, int(nthreads), C.byref(h)))
        self.h = h
        info = self.info()
        self.n = int(info[0])
        self.kind = kind
        if device is not None and not on_device:
            self.upload(device)

    @classmethod
    def load(cls, path: str, device: Optional[int] = 0) -> "Index":
        """Index saved by ``save`` (on-disk format of ``qbc_index_save``), uploaded to ``device``."""
        self = cls.__new__(cls)
        self._graph = None
        h = C.c_void_p()
        check(lib().qbc_index_load(str(path).encode(), C.byref(h)))
        self.h = h
        info = self.info()
        self.n = int(info[0])
        self.kind = int(info[6])
        if device is not None:
            self.upload(device)
        return self

    def save(self, path: str) -> None:
        check(lib().qbc_index_save(self.h, str(path).encode()))

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().qbc_index_free(self.h)
            except Exception:
                pass
            self.h = None

    def upload(self, device: int = 0):
        check(lib().qbc_index_upload(self.h, int(device)))

    def release_device(self):
        check(lib().qbc_index_release_device(self.h))

    def info(self) -> np.ndarray:
        info = np.zeros(8, np.int64)
        check(lib().qbc_index_info(self.h, ptr(info, i64p)))
        return info

    def export(self):
        info = self.info()
        n, L = int(info[0]), int(info[2])
        d = dict(vid_of=np.empty(n, np.int32), depth=np.empty(n, np.int32), send=np.empty(n, np.int32),
                 lab_off=np.empty(n + 1, np.int64), dis=np.empty(L, np.int32), anc=np.empty(L, np.int32))
        ch = np.empty(2 * L, np.int32) if self.kind == QBC_INDEX_MHL else None
        check(lib().qbc_index_export(self.h, ptr(d["vid_of"], i32p), ptr(d["depth"], i32p), ptr(d["send"], i32p),
                                     ptr(d["lab_off"], i64p), ptr(d["dis"], i32p),
                                     None if ch is None else ptr(ch, i32p), ptr(d["anc"], i32p)))
        d["ch"] = ch
        return d

    def scan_entries(self, sources: Sequence[int]) -> int:
        s = i32(sources)
        e = C.c_int64()
        check(lib().qbc_index_scan_entries(self.h, ptr(s, i32p), int(s.shape[0]), C.byref(e)))
        return int(e.value)

    def group_entries(self, sources: Sequence[int], group: int = 32) -> int:
        """Label entries the batched scan copies from target rows for CTAs of ``group`` sources."""
        s = i32(sources)
        e = C.c_int64()
        check(lib().qbc_index_group_entries(self.h, ptr(s, i32p), int(s.shape[0]), int(group), C.byref(e)))
        return int(e.value)

    def label_group(self) -> int:
        """Sources per CTA of the batched label scan under the current tuning (0: label-free index)."""
        g = np.zeros(1, np.int32)
        check(lib().qbc_index_label_group(self.h, ptr(g, i32p)))
        return int(g[0])

    def label_kernel(self) -> str:
        """Name of the kernel the batched per-source rows come from under the current tuning."""
        buf = C.create_string_buffer(64)
        check(lib().qbc_index_label_kernel(self.h, buf, 64))
        return buf.value.decode()

    TUNING_KEYS = ("lanes_per_source", "label_threads", "split", "chunk", "dep_threads", "dep_form", "queue_depth",
                   "label_warps", "label_tile", "label_passes", "sweep_delta", "sweep_threads", "label_sources",
                   "label_stream")

    def set_tuning(self, lanes_per_source=0, label_threads=256, split=0, chunk=0, dep_threads=256, dep_form=0,
                   queue_depth=0, label_warps=0, label_tile=0, label_passes=0, sweep_delta=0, sweep_threads=0,
                   label_sources=0, label_stream=0):
        p = i32([lanes_per_source, label_threads, split, chunk, dep_threads, dep_form, queue_depth, label_warps,
                 label_tile, label_passes, sweep_delta, sweep_threads, label_sources, label_stream])
        check(lib().qbc_index_set_tuning(self.h, ptr(p, i32p), len(self.TUNING_KEYS)))

    def get_tuning(self):
        p = np.zeros(len(self.TUNING_KEYS), np.int32)
        check(lib().qbc_index_get_tuning(self.h, ptr(p, i32p), len(self.TUNING_KEYS)))
        return dict(zip(self.TUNING_KEYS, p.tolist()))

    def autotune(self, sample, path: Optional[str] = None) -> dict:
        """Times candidate tunings on a sweep over ``sample`` (vids), keeps the fastest on the index
        and returns it; with ``path`` it is also written there as JSON (``load_tuning`` reads it)."""
        s = i32(sample)
        p = np.zeros(len(self.TUNING_KEYS), np.int32)
        ms = C.c_double()
        check(lib().qbc_autotune(self.h, ptr(s, i32p), int(s.shape[0]), ptr(p, i32p), len(self.TUNING_KEYS),
                                 C.byref(ms)))
        res = dict(tuning=dict(zip(self.TUNING_KEYS, p.tolist())), ms_per_source=float(ms.value),
                   sample_sources=int(s.shape[0]), n=self.n)
        if path:
            with open(path, "w") as f:
                json.dump(res, f, indent=1)
        return res

    def load_tuning(self, path: str) -> dict:
        with open(path) as f:
            t = json.load(f)["tuning"]
        self.set_tuning(**{k: int(t[k]) for k in self.TUNING_KEYS if k in t})
        return self.get_tuning()

    def serve(self, sources=None, max_active: int = 64, pool_bytes: int = 0, max_queue: int = 0, chunk: int = 0):
        """Opens the served RQ loop on this index (see ``serve.Server``)."""
        from .serve import Server

        return Server(self, sources, max_active, pool_bytes, max_queue, chunk)

    def profile(self, on: bool = True) -> None:
        check(lib().qbc_index_profile(self.h, 1 if on else 0))

    def stats(self) -> dict:
        out = np.zeros(5, np.float64)
        check(lib().qbc_index_stats(self.h, ptr(out, f64p)))
        return dict(label_ms=out[0], label_launches=int(out[1]), dep_ms=out[2], dep_launches=int(out[3]),
                    launches=int(out[4]))

    def bc_all(self) -> np.ndarray:
        out = np.zeros(self.n, np.float64)
        check(lib().qbc_bc_all(self.h, ptr(out, f64p)))
        return out

    def bc_sources(self, sources) -> np.ndarray:
        s = i32(sources)
        out = np.zeros(self.n, np.float64)
        check(lib().qbc_bc_sources(self.h, ptr(s, i32p), int(s.shape[0]), ptr(out, f64p)))
        return out

    def bc_plain(self, sources) -> np.ndarray:
        s = i32(sources)
        out = np.zeros(self.n, np.float64)
        check(lib().qbc_bc_plain(self.h, ptr(s, i32p), int(s.shape[0]), ptr(out, f64p)))
        return out

    def bc_sources_device(self, d_sources_ptr: int, ns: int, d_bc_ptr: int, stream_ptr: int = 0) -> None:
        check(lib().qbc_bc_sources_device(self.h, C.c_void_p(d_sources_ptr), int(ns), C.c_void_p(d_bc_ptr),
                                          C.c_void_p(stream_ptr) if stream_ptr else None))

    def bc_query(self, points) -> np.ndarray:
        p = i32(points)
        out = np.zeros(p.shape[0], np.float64)
        check(lib().qbc_bc_query(self.h, ptr(p, i32p), int(p.shape[0]), ptr(out, f64p)))
        return out

    def bc_query_batch(self, sets: Sequence[Sequence[int]], sources=None):
        flat = i32(np.concatenate([np.asarray(s, np.int32) for s in sets]) if sets else np.zeros(0, np.int32))
        off = i32(np.concatenate([[0], np.cumsum([len(s) for s in sets])]))
        out = np.zeros(flat.shape[0], np.float64)
        src = None if sources is None else i32(sources)
        check(lib().qbc_bc_query_batch(self.h, ptr(flat, i32p), ptr(off, i32p), len(sets),
                                       None if src is None else ptr(src, i32p),
                                       0 if src is None else int(src.shape[0]), ptr(out, f64p)))
        return [out[off[i]:off[i + 1]] for i in range(len(sets))]

    def rows(self, sources, counts: bool = True):
        s = i32(sources)
        ns = int(s.shape[0])
        d = np.empty((ns, self.n), np.int32)
        c = np.empty((ns, self.n), np.uint32) if counts else None
        h = np.empty((ns, self.n), np.int32) if counts else None
        check(lib().qbc_rows(self.h, ptr(s, i32p), ns, ptr(d, i32p), None if c is None else ptr(c, u32p),
                             None if h is None else ptr(h, i32p)))
        return d, c, h


class Graph:
    """Mirror of the reference's ``Graph`` driver class (include/Graph.h:64-200)."""

    def __init__(self, device: int = 0, nthreads: int = 0):
        self.device = device
        self.nthreads = nthreads
        self.nodenum = 0
        self.edgenum = 0
        self.BC: Optional[np.ndarray] = None
        self.h_PointBC: Optional[np.ndarray] = None
        self._g: Optional[_GraphHandle] = None
        self.index: Optional[Index] = None

    def ReadGraph(self, graphname: str) -> None:
        self._g = _graph_from_path(graphname)
        self.nodenum, self.edgenum = _graph_info(self._g)

    def ReadLines(self, n: int, u1, v1, w) -> None:
        """Same as ReadGraph from in-memory arc lines (1-based ids)."""
        self._g = _graph_from_lines(n, u1, v1, w)
        self.nodenum, self.edgenum = _graph_info(self._g)

    def arcs(self):
        off = np.empty(self.nodenum + 1, np.int32)
        head = np.empty(self.edgenum, np.int32)
        w = np.empty(self.edgenum, np.int32)
        check(lib().qbc_graph_arcs(self._g.h, ptr(off, i32p), ptr(head, i32p), ptr(w, i32p)))
        return off, head, w

    def min_degree_order(self) -> np.ndarray:
        o = np.empty(self.nodenum, np.int32)
        check(lib().qbc_min_degree_order(self._g.h, ptr(o, i32p)))
        return o

    def build_index(self, kind=QBC_INDEX_MHL, node_order=None, upload: bool = True, on_device: bool = False) -> Index:
        """Builds the index on the host and uploads it to ``self.device`` unless ``upload`` is False;
        with ``on_device`` the label rows are filled on ``self.device`` instead.  ``QBC_INDEX_CSR``
        keeps no labels (rows come from shortest-path sweeps over the arc list on the device)."""
        if self._g is None:
            raise QbcError(1, "ReadGraph first")
        self.index = Index(self._g, kind, node_order, self.nthreads, self.device if (upload or on_device) else None,
                           on_device=on_device)
        return self.index

    def brandesBCIndexGPU_5(self, roadName: str, orderFile: Optional[str] = None) -> None:
        if orderFile is None:
            idx = self.build_index(QBC_INDEX_MHL, on_device=True)
        else:
            idx = self.build_index(QBC_INDEX_H2H, read_order(orderFile, self.nodenum), on_device=True)
        self.BC = idx.bc_all()

    def brandesBCIndexGPU_PointBatch(self, roadName: str, points, querySize: int) -> None:
        pts = i32(points)[:querySize]
        idx = self.build_index(QBC_INDEX_MHL, on_device=True)
        self.h_PointBC = idx.bc_query(pts)
