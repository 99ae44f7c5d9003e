"""CPU: the oracle (oracle/oracle.c) pinned against the reference's own compiled CPU code, the
reference GPU outputs committed under tests/golden/, and an independent Dijkstra-Brandes."""
import os

import numpy as np
import pytest

import pyoracle as O
from conftest import GOLDEN, rel_err
from gpu_betweennesscentrality_b200 import synth
from util import BC_RTOL, KNOWN, grid_lines, lines_of

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")


@pytest.fixture(scope="module")
def g2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    return n, u, v, w, O.TreeCount(n, u, v, w), O.Arcs(n, u, v, w)


@needs_ref
def test_treecount_matches_reference_labels(g2k, tmp_path):
    n, u, v, w, tc, _ = g2k
    rt = O.RefTreeCount(os.path.join(GOLDEN, "g2k.txt"), str(tmp_path / "dump"))
    for name in ["del_order", "rank", "parent", "height", "lab_off", "dis", "cnt", "hop", "pos_off", "pos",
                 "euler_pos"]:
        assert np.array_equal(getattr(tc, name), getattr(rt, name)), name
    assert (tc.tree_width, tc.tree_height) == (rt.tree_width, rt.tree_height)


@needs_ref
def test_treecount_matches_reference_labels_shortcuts(tmp_path):
    g = synth.grid_graph(1500, seed=4, shortcut_frac=0.02)
    p = str(tmp_path / "g.txt")
    synth.write_graph(p, g)
    n, u, v, w = synth.read_graph_lines(p)
    tc = O.TreeCount(n, u, v, w)
    rt = O.RefTreeCount(p, str(tmp_path / "dump"))
    for name in ["del_order", "parent", "height", "dis", "cnt", "hop", "pos"]:
        assert np.array_equal(getattr(tc, name), getattr(rt, name)), name


@needs_ref
def test_reference_separator_count_query_agrees(g2k, tmp_path):
    """TreeDecomp::DistanceCountQuery (separator-only scan, TreeDecomp.cpp:568-628) gives the same
    path count as the full-ancestor scan of MHLQBC.cu:379-392 restated in the oracle.  Its hop value
    can exceed the true maximum hop count (the GPU scan's value, which Dijkstra confirms); no BC
    path uses that CPU query, so only the count is pinned here."""
    n, u, v, w, tc, _ = g2k
    rt = O.RefTreeCount(os.path.join(GOLDEN, "g2k.txt"), str(tmp_path / "dump"))
    rng = np.random.default_rng(3)
    for s in rng.choice(n, 5, replace=False):
        d, c, h = tc.rows(int(s))
        for t in rng.choice(n, 40, replace=False):
            if t == s:
                continue
            cc, hh = rt.count_hop(int(s) + 1, int(t) + 1)
            assert cc == int(c[t]) and hh >= int(h[t])


@needs_ref
def test_h2h_matches_reference(g2k):
    n, u, v, w, tc, arcs = g2k
    order = O.np.loadtxt(os.path.join(GOLDEN, "g2k.order"), skiprows=1, dtype=np.int64)
    node_order = np.empty(n, np.int32)
    node_order[order[:, 0]] = order[:, 1]
    h = O.H2H(arcs, node_order)
    rh = O.RefH2H(os.path.join(GOLDEN, "g2k.txt"), os.path.join(GOLDEN, "g2k.order"))
    for name in ["rank", "parent", "height", "dis_off", "dis"]:
        assert np.array_equal(getattr(h, name), getattr(rh, name)), name
    for p in range(n):
        a = set(h.popt[h.popt_off[p]:h.popt_off[p + 1]].tolist())
        b = set(rh.popt[rh.popt_off[p]:rh.popt_off[p + 1]].tolist())
        assert a == b


def test_rows_match_dijkstra(g2k):
    n, u, v, w, tc, arcs = g2k
    for s in [0, 1, 777, n - 1]:
        d1, c1, h1 = tc.rows(s)
        d2, c2, h2 = arcs.dijkstra_rows(s)
        assert np.array_equal(d1, d2) and np.array_equal(c1, c2) and np.array_equal(h1, h2)


def test_mhl_qbc_rq_bc_match_brandes(g2k):
    n, u, v, w, tc, arcs = g2k
    full = arcs.bc()
    assert rel_err(tc.bc(arcs), full) <= BC_RTOL
    order = np.loadtxt(os.path.join(GOLDEN, "g2k.order"), skiprows=1, dtype=np.int64)
    node_order = np.empty(n, np.int32)
    node_order[order[:, 0]] = order[:, 1]
    assert rel_err(O.H2H(arcs, node_order).bc(), full) <= BC_RTOL
    q = np.loadtxt(os.path.join(GOLDEN, "g2k.query"), skiprows=1, dtype=np.int64) - 1
    assert rel_err(tc.rq(q), full[q]) <= BC_RTOL


@pytest.mark.parametrize("name", sorted(KNOWN))
def test_known_answers(name):
    n, edges, expect = KNOWN[name]
    nn, u, v, w = lines_of(edges, n)
    arcs = O.Arcs(nn, u, v, w)
    full = arcs.bc()
    if expect is not None:
        assert np.allclose(full, expect, rtol=0, atol=1e-12)
    if n >= 2:
        tc = O.TreeCount(nn, u, v, w)
        assert rel_err(tc.bc(arcs), full) <= BC_RTOL


def test_shortcut_graph_counts():
    n, u, v, w = grid_lines(1200, seed=9, shortcut_frac=0.02)
    tc = O.TreeCount(n, u, v, w)
    arcs = O.Arcs(n, u, v, w)
    for s in [3, 500, 1100]:
        d1, c1, h1 = tc.rows(s)
        d2, c2, h2 = arcs.dijkstra_rows(s)
        assert np.array_equal(d1, d2) and np.array_equal(c1, c2) and np.array_equal(h1, h2)


def _golden(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated (tests/golden/make_golden.py on a B200)")
    return np.loadtxt(p)


def test_oracle_matches_reference_gpu_mhl(g2k):
    n, u, v, w, tc, arcs = g2k
    ref = _golden("ref_g2k_mhl.txt")
    assert ref.shape[0] == n and np.array_equal(ref[:, 0].astype(int), np.arange(1, n + 1))
    assert rel_err(tc.bc(arcs), ref[:, 1]) <= BC_RTOL


def test_oracle_matches_reference_gpu_qbc(g2k):
    n, u, v, w, tc, arcs = g2k
    ref = _golden("ref_g2k_qbc.txt")
    order = np.loadtxt(os.path.join(GOLDEN, "g2k.order"), skiprows=1, dtype=np.int64)
    node_order = np.empty(n, np.int32)
    node_order[order[:, 0]] = order[:, 1]
    assert rel_err(O.H2H(arcs, node_order).bc(), ref[:, 1]) <= BC_RTOL


def test_oracle_matches_reference_gpu_rq(g2k):
    n, u, v, w, tc, arcs = g2k
    ref = _golden("ref_g2k_rq.txt")
    q = ref[:, 0].astype(np.int64) - 1
    assert rel_err(tc.rq(q), ref[:, 1]) <= BC_RTOL


def test_oracle_matches_reference_gpu_la(la_path):
    """The reference's GPU BC of its own LosAngeles graph equals Dijkstra-Brandes over all sources."""
    p = os.path.join(GOLDEN, "ref_la_mhl.npz")
    if not os.path.exists(p):
        pytest.skip("ref_la_mhl.npz not generated")
    ref = np.load(p)["bc"]
    n, u, v, w = synth.read_graph_lines(la_path)
    assert ref.shape[0] == n
    assert rel_err(O.Arcs(n, u, v, w).bc(), ref) <= BC_RTOL


def test_rq_pair_product_wraps_where_half_delta_does_not():
    """The reference's RQ pair kernel multiplies the two path counts as int32, (int)(sigma_vs *
    sigma_vt) (RQ.cu:456), which wraps once the product passes 2^31; BC restricted to the query set
    (1/2 sum_s delta_s(v), MHLQBC.cu's quantity, with the same 32-bit counts) has no such product.
    Where counts stay small (the 2k grid) the two agree to 1e-9; on the 24 x 24 unit grid (counts up
    to C(46,23)) the pair formula departs from it.  This library's RQ follows 1/2 sum delta."""
    from util import unit_grid_lines

    n, u, v, w = unit_grid_lines()
    tc, arcs = O.TreeCount(n, u, v, w), O.Arcs(n, u, v, w)
    q = np.array([0, 11, 24 * 11 + 11, 24 * 12 + 12, 300, n - 1], np.int32)
    half_delta = arcs.bc()[q]
    pair = tc.rq(q)
    assert rel_err(tc.bc(arcs)[q], half_delta) <= BC_RTOL
    assert rel_err(pair, half_delta) > 1e-3  # the wrapped products differ by orders of magnitude
    n2, u2, v2, w2 = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    tc2, arcs2 = O.TreeCount(n2, u2, v2, w2), O.Arcs(n2, u2, v2, w2)
    q2 = np.arange(0, n2, 97, dtype=np.int32)
    assert rel_err(tc2.rq(q2), arcs2.bc()[q2]) <= BC_RTOL

