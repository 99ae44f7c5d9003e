"""GPU: label rows filled on the device (qbc_index_build_device) equal the host builder's rows
bit-for-bit (dist, count bits, hop, ancestor ids), for MHL and H2H indexes, and give the same BC."""
import os

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
import pyoracle as O
from conftest import GOLDEN, rel_err
from gpu_betweennesscentrality_b200 import synth
from util import BC_RTOL, grid_lines

pytestmark = pytest.mark.gpu

FIELDS = ("vid_of", "depth", "send", "lab_off", "dis", "anc")


def _pair(n, u, v, w, kind=Q.QBC_INDEX_MHL, order=None):
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    host = g.build_index(kind, order, upload=False)
    dev = g.build_index(kind, order, on_device=True)
    return host, dev


def _same_rows(host, dev):
    a, b = host.export(), dev.export()
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    if a["ch"] is not None:
        assert np.array_equal(a["ch"], b["ch"])


def test_mhl_rows_2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    host, dev = _pair(n, u, v, w)
    bc = dev.bc_all()  # before export: rows only on the device
    _same_rows(host, dev)
    assert rel_err(bc, O.TreeCount(n, u, v, w).bc(O.Arcs(n, u, v, w))) <= BC_RTOL


def test_h2h_rows_2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    order = Q.read_order(os.path.join(GOLDEN, "g2k.order"), n)
    host, dev = _pair(n, u, v, w, Q.QBC_INDEX_H2H, order)
    bc = dev.bc_all()
    _same_rows(host, dev)
    assert rel_err(bc, O.H2H(O.Arcs(n, u, v, w), order).bc()) <= BC_RTOL


@pytest.mark.parametrize("n_target,seed,sc", [(3000, 6, 0.02), (20000, 3, 0.0)])
def test_mhl_rows_generated(n_target, seed, sc):
    n, u, v, w = grid_lines(n_target, seed=seed, shortcut_frac=sc)
    host, dev = _pair(n, u, v, w)
    srcs = np.arange(0, n, max(1, n // 40), dtype=np.int32)
    got = dev.bc_sources(srcs)
    _same_rows(host, dev)
    host.upload(0)
    assert rel_err(got, host.bc_sources(srcs)) <= BC_RTOL


def test_release_and_reupload_keeps_rows():
    n, u, v, w = grid_lines(800, seed=2)
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    dev = g.build_index(on_device=True)
    a = dev.bc_all()
    dev.release_device()  # rows come back to the host first
    dev.upload(0)
    assert rel_err(dev.bc_all(), a) <= BC_RTOL


def test_saved_device_index_cold_start(tmp_path):
    """a device-built index saved to disk and loaded back serves the same BC (no rebuild)"""
    n, u, v, w = grid_lines(2000, seed=5)
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    dev = g.build_index(on_device=True)
    a = dev.bc_all()
    p = str(tmp_path / "dev.qbcidx")
    dev.save(p)
    back = Q.Index.load(p, device=0)
    assert rel_err(back.bc_all(), a) <= BC_RTOL
    with back.serve() as srv:
        pts = np.array([0, n // 2, n - 1], np.int32)
        assert rel_err(srv.wait(srv.submit(pts), 60.0)[0], a[pts]) <= BC_RTOL


@pytest.mark.parametrize("name", ["single", "pair", "path3", "star5", "cycle4", "path40"])
def test_known_graphs_device_build(name):
    from util import KNOWN, lines_of

    n, edges, expect = KNOWN[name]
    nn, u, v, w = lines_of(edges, n)
    host, dev = _pair(nn, u, v, w)
    bc = dev.bc_all()
    _same_rows(host, dev)
    assert np.allclose(bc, expect, rtol=0, atol=1e-9)


@pytest.mark.parametrize("tail", [64, 700, 100000])
def test_mhl_rows_dense_tail_2k(monkeypatch, tail):
    """the last `tail` vertices of the min-degree elimination eliminated on the device as a dense
    matrix (all of them for 100000): same picks, separators, tree and rows as the host"""
    monkeypatch.setenv("QBC_DENSE_TAIL", str(tail))
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    host, dev = _pair(n, u, v, w)
    bc = dev.bc_all()
    _same_rows(host, dev)
    assert rel_err(bc, O.TreeCount(n, u, v, w).bc(O.Arcs(n, u, v, w))) <= BC_RTOL


@pytest.mark.parametrize("n_target,seed,sc,tail", [(3000, 6, 0.02, 3000), (20000, 3, 0.0, 2500)])
def test_mhl_rows_dense_tail_generated(monkeypatch, n_target, seed, sc, tail):
    """shortcut vertices (more than four arcs, long shortcuts) and a 20k grid with a 2,500-vertex
    dense tail: rows bit-identical to the host build"""
    monkeypatch.setenv("QBC_DENSE_TAIL", str(tail))
    n, u, v, w = grid_lines(n_target, seed=seed, shortcut_frac=sc)
    host, dev = _pair(n, u, v, w)
    _same_rows(host, dev)


def test_mhl_rows_dense_tail_200k(monkeypatch, graph_cache):
    """200k grid: the default device build (host elimination) and one with a 16,384-vertex dense
    tail on the device give identical trees and rows"""
    path = synth.cached_graph(graph_cache, 200000, seed=1)
    g = Q.Graph(device=0)
    g.ReadGraph(path)
    monkeypatch.setenv("QBC_DENSE_TAIL", "0")
    a = g.build_index(on_device=True).export()
    monkeypatch.setenv("QBC_DENSE_TAIL", "16384")
    b = g.build_index(on_device=True).export()
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["ch"], b["ch"])
