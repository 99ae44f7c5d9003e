"""CPU: the on-disk index format (qbc_index_save / qbc_index_load) round-trips every array of MHL
and H2H indexes, and damaged, truncated or foreign files are refused with QBC_EIO."""
import os

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
from conftest import GOLDEN
from gpu_betweennesscentrality_b200 import capi, synth
from util import grid_lines

FIELDS = ("vid_of", "depth", "send", "lab_off", "dis", "anc", "ch")


def _same(a, b):
    ea, eb = a.export(), b.export()
    for f in FIELDS:
        if ea[f] is None:
            assert eb[f] is None
        else:
            assert np.array_equal(ea[f], eb[f]), f
    assert np.array_equal(a.info(), b.info())


@pytest.fixture(scope="module")
def g2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = Q.Graph()
    g.ReadLines(n, u, v, w)
    return n, g


def test_mhl_round_trip(g2k, tmp_path):
    n, g = g2k
    idx = g.build_index(upload=False)
    p = str(tmp_path / "g2k.qbcidx")
    idx.save(p)
    _same(idx, Q.Index.load(p, device=None))


def test_h2h_round_trip(g2k, tmp_path):
    n, g = g2k
    order = Q.read_order(os.path.join(GOLDEN, "g2k.order"), n)
    idx = g.build_index(Q.QBC_INDEX_H2H, order, upload=False)
    p = str(tmp_path / "g2k_h2h.qbcidx")
    idx.save(p)
    back = Q.Index.load(p, device=None)
    assert back.kind == Q.QBC_INDEX_H2H
    _same(idx, back)


def test_shortcut_graph_round_trip(tmp_path):
    n, u, v, w = grid_lines(1500, seed=4, shortcut_frac=0.02)
    g = Q.Graph()
    g.ReadLines(n, u, v, w)
    idx = g.build_index(upload=False)
    p = str(tmp_path / "sc.qbcidx")
    idx.save(p)
    _same(idx, Q.Index.load(p, device=None))


@pytest.mark.parametrize("damage", ["flip", "truncate", "magic", "grow"])
def test_damaged_files_refused(g2k, tmp_path, damage):
    n, g = g2k
    idx = g.build_index(upload=False)
    p = str(tmp_path / "x.qbcidx")
    idx.save(p)
    raw = bytearray(open(p, "rb").read())
    if damage == "flip":
        raw[len(raw) // 2] ^= 0x40
    elif damage == "truncate":
        raw = raw[: len(raw) - 100]
    elif damage == "magic":
        raw[0:8] = b"NOTANIDX"
    else:
        raw += b"\0" * 16
    open(p, "wb").write(bytes(raw))
    with pytest.raises(Q.QbcError) as e:
        Q.Index.load(p, device=None)
    assert e.value.code == capi.QBC_EIO


def test_missing_file_refused(tmp_path):
    with pytest.raises(Q.QbcError) as e:
        Q.Index.load(str(tmp_path / "none.qbcidx"), device=None)
    assert e.value.code == capi.QBC_EIO
