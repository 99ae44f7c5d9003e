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


FNV_BASIS, FNV_PRIME, M64 = 1469598103934665603, 1099511628211, (1 << 64) - 1


def _word_hash(body: bytes) -> int:
    """restatement of the version-2 checksum: FNV-1a's xor-multiply on 64-bit little-endian words
    in four interleaved lanes, the last block zero-padded, lanes and byte count folded"""
    pad = body + b"\0" * (-len(body) % 32)
    words = np.frombuffer(pad, dtype="<u8").tolist()
    lanes = [FNV_BASIS ^ q for q in range(4)]
    for i, w in enumerate(words):
        q = i & 3
        lanes[q] = ((lanes[q] ^ w) * FNV_PRIME) & M64
    h = FNV_BASIS
    for q in range(4):
        h = ((h ^ lanes[q]) * FNV_PRIME) & M64
    return ((h ^ len(body)) * FNV_PRIME) & M64


def _byte_fnv(body: bytes) -> int:
    h = FNV_BASIS
    for c in body:
        h = ((h ^ c) * FNV_PRIME) & M64
    return h


def _small_index():
    n, u, v, w = grid_lines(300, seed=6)
    g = Q.Graph()
    g.ReadLines(n, u, v, w)
    return g.build_index(upload=False)


def test_checksum_is_the_word_lane_fnv(tmp_path):
    idx = _small_index()
    p = str(tmp_path / "s.qbcidx")
    idx.save(p)
    raw = open(p, "rb").read()
    assert raw[:8] == b"QBCIDX02" and int.from_bytes(raw[8:12], "little") == 2
    assert int.from_bytes(raw[-8:], "little") == _word_hash(raw[:-8])


def test_version1_files_still_load(tmp_path):
    """the first format (same layout, magic QBCIDX01, version 1, byte-wise FNV-1a) is read as is"""
    idx = _small_index()
    p = str(tmp_path / "s.qbcidx")
    idx.save(p)
    body = bytearray(open(p, "rb").read()[:-8])
    body[0:8] = b"QBCIDX01"
    body[8:12] = (1).to_bytes(4, "little")
    v1 = str(tmp_path / "v1.qbcidx")
    open(v1, "wb").write(bytes(body) + _byte_fnv(bytes(body)).to_bytes(8, "little"))
    _same(idx, Q.Index.load(v1, device=None))
    body[len(body) // 3] ^= 0x01
    open(v1, "wb").write(bytes(body) + _byte_fnv(bytes(body[:len(body) // 3])).to_bytes(8, "little"))
    with pytest.raises(Q.QbcError) as e:
        Q.Index.load(v1, device=None)
    assert e.value.code == capi.QBC_EIO


@pytest.mark.parametrize("where", [9, 40, -9, -20, -40])
def test_any_changed_byte_is_refused(tmp_path, where):
    """header, first words, and bytes of the zero-padded last block"""
    idx = _small_index()
    p = str(tmp_path / "s.qbcidx")
    idx.save(p)
    raw = bytearray(open(p, "rb").read())
    raw[where] ^= 0x10
    open(p, "wb").write(bytes(raw))
    with pytest.raises(Q.QbcError) as e:
        Q.Index.load(p, device=None)
    assert e.value.code == capi.QBC_EIO
