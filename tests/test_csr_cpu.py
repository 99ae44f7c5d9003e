"""CPU: the label-free index (QBC_INDEX_CSR) -- host build, connectivity rule, on-disk round trip,
tuning fields -- without a GPU.  Its per-source rows and BC are checked on the GPU in
test_gpu_csr.py."""
import os

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
from conftest import GOLDEN
from gpu_betweennesscentrality_b200 import capi, synth
from util import grid_lines, lines_of


def _graph(n, u, v, w):
    g = Q.Graph()
    g.ReadLines(n, u, v, w)
    return g


def test_csr_index_keeps_arcs_in_vid_order():
    n, u, v, w = grid_lines(3000, seed=4, shortcut_frac=0.02)
    g = _graph(n, u, v, w)
    idx = g.build_index(Q.QBC_INDEX_CSR, upload=False)
    info = idx.info()
    off, head, wt = g.arcs()
    assert info[0] == n and info[1] == head.shape[0]
    assert info[2] == 0 and info[3] == 0 and info[6] == Q.QBC_INDEX_CSR  # no label entries, no tree
    ex = idx.export()
    assert np.array_equal(ex["vid_of"], np.arange(n))
    assert np.array_equal(ex["send"], np.arange(1, n + 1))
    assert not ex["depth"].any() and not ex["lab_off"].any()
    assert idx.scan_entries(np.arange(0, n, 7)) == 0


def test_csr_index_rejects_disconnected_graph():
    n, u, v, w = lines_of([(0, 1, 3), (2, 3, 4)], 4)
    g = _graph(n, u, v, w)
    with pytest.raises(Q.QbcError) as e:
        g.build_index(Q.QBC_INDEX_CSR, upload=False)
    assert e.value.code == capi.QBC_EGRAPH


def test_csr_index_file_round_trip(tmp_path):
    n, u, v, w = grid_lines(2000, seed=3, shortcut_frac=0.02)
    g = _graph(n, u, v, w)
    idx = g.build_index(Q.QBC_INDEX_CSR, upload=False)
    p = str(tmp_path / "csr.qbcidx")
    idx.save(p)
    back = Q.Index.load(p, device=None)
    assert back.kind == Q.QBC_INDEX_CSR
    assert np.array_equal(back.info(), idx.info())
    a, b = idx.export(), back.export()
    for f in ("vid_of", "depth", "send", "lab_off"):
        assert np.array_equal(a[f], b[f]), f
    # a flipped payload byte is refused
    raw = bytearray(open(p, "rb").read())
    raw[len(raw) // 2] ^= 0x5A
    bad = str(tmp_path / "bad.qbcidx")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(Q.QbcError) as e:
        Q.Index.load(bad, device=None)
    assert e.value.code == capi.QBC_EIO


def test_tuning_fields_round_trip():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    idx = _graph(n, u, v, w).build_index(Q.QBC_INDEX_CSR, upload=False)
    idx.set_tuning(sweep_delta=500, sweep_threads=512, dep_threads=128)
    t = idx.get_tuning()
    assert t["sweep_delta"] == 500 and t["sweep_threads"] == 512 and t["dep_threads"] == 128
    idx.set_tuning(sweep_threads=1024)
    assert idx.get_tuning()["sweep_threads"] == 1024
    idx.set_tuning(sweep_threads=2048)  # four 512-thread CTAs per SM
    assert idx.get_tuning()["sweep_threads"] == 2048
    for bad in (dict(sweep_threads=384), dict(sweep_delta=-1)):
        with pytest.raises(Q.QbcError) as e:
            idx.set_tuning(**bad)
        assert e.value.code == capi.QBC_EINVAL
