"""GPU: the label-free index (QBC_INDEX_CSR).  Per-source rows from the device shortest-path sweep
must equal, bit for bit, the oracle's Dijkstra rows (distance, 32-bit wrapping path count, largest
hop count over shortest paths) and the TreeCount label rows where those exist; BC must agree with the
oracle's Dijkstra-Brandes, the label path and the reference's own GPU outputs within BC_RTOL = 1e-9
relative.  Covers the workloads whose tree decomposition is too wide for labels: the seeded grids
with 2 % random shortcuts at 200k (RQ, q = 4,096) and 1M vertices (batched / served RQ), on seeded
source samples (partial BC over the sample)."""
import os

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
import pyoracle as O
from conftest import GOLDEN, rel_err
from gpu_betweennesscentrality_b200 import synth
from gpu_betweennesscentrality_b200.serve import request_sets
from util import BC_RTOL, KNOWN, grid_lines, lines_of, unit_grid_lines

pytestmark = pytest.mark.gpu


def _csr(n, u, v, w, **tuning):
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    idx = g.build_index(Q.QBC_INDEX_CSR)
    if tuning:
        idx.set_tuning(**tuning)
    return idx


def _rows_equal_dijkstra(idx, arcs, srcs):
    d, c, h = idx.rows(srcs)
    for k, s in enumerate(srcs):
        d0, c0, h0 = arcs.dijkstra_rows(int(s))
        assert np.array_equal(d[k], d0), f"dist of source {s}"
        assert np.array_equal(c[k], c0), f"count of source {s}"
        assert np.array_equal(h[k], h0), f"hop of source {s}"


@pytest.fixture(scope="module")
def g2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    return n, u, v, w, _csr(n, u, v, w), O.TreeCount(n, u, v, w), O.Arcs(n, u, v, w)


def test_rows_equal_treecount_labels_all_sources_2k(g2k):
    n, u, v, w, idx, tc, arcs = g2k
    d, c, h = idx.rows(np.arange(n, dtype=np.int32))
    for s in range(n):
        d0, c0, h0 = tc.rows(s)
        assert np.array_equal(d[s], d0) and np.array_equal(c[s], c0) and np.array_equal(h[s], h0), s


def test_full_bc_2k_matches_oracle_and_reference_gpu(g2k):
    n, u, v, w, idx, tc, arcs = g2k
    bc = idx.bc_all()
    assert rel_err(bc, arcs.bc()) <= BC_RTOL
    assert rel_err(bc, tc.bc(arcs)) <= BC_RTOL
    p = os.path.join(GOLDEN, "ref_g2k_mhl.txt")
    if os.path.exists(p):
        assert rel_err(bc, np.loadtxt(p)[:, 1]) <= BC_RTOL


@pytest.mark.parametrize("n_target,seed,sc", [(3000, 4, 0.02), (5000, 9, 0.05), (2500, 2, 0.0), (8000, 12, 0.02)])
def test_rows_and_full_bc_shortcut_graphs(n_target, seed, sc):
    n, u, v, w = grid_lines(n_target, seed=seed, shortcut_frac=sc)
    idx = _csr(n, u, v, w)
    arcs = O.Arcs(n, u, v, w)
    _rows_equal_dijkstra(idx, arcs, np.random.default_rng(seed).choice(n, 24, replace=False).astype(np.int32))
    assert rel_err(idx.bc_all(), arcs.bc()) <= BC_RTOL


@pytest.mark.parametrize("delta,threads", [(1, 256), (37, 512), (1000, 256), (1 << 20, 512), (0, 512), (0, 1024),
                                           (1, 1024), (0, 2048), (37, 2048)])
def test_bucket_widths_and_threads_give_identical_rows(delta, threads):
    """bucket width 1 (label-setting), the default, and one bucket holding every distance
    (Bellman-Ford on the whole graph) all reach the same fixed point"""
    n, u, v, w = grid_lines(3000, seed=4, shortcut_frac=0.02)
    base = _csr(n, u, v, w)
    alt = _csr(n, u, v, w, sweep_delta=delta, sweep_threads=threads)
    srcs = np.arange(0, n, 29, dtype=np.int32)
    for a, b in zip(base.rows(srcs), alt.rows(srcs)):
        assert np.array_equal(a, b)
    assert rel_err(alt.bc_sources(srcs), base.bc_sources(srcs)) <= BC_RTOL


@pytest.mark.parametrize("name", sorted(KNOWN))
def test_known_graphs(name):
    n, edges, expect = KNOWN[name]
    n, u, v, w = lines_of(edges, n)
    idx = _csr(n, u, v, w)
    bc = idx.bc_all()
    ref = O.Arcs(n, u, v, w).bc() if expect is None else np.asarray(expect, np.float64)
    assert rel_err(bc, ref) <= BC_RTOL


def test_wrapping_counts_unit_grid():
    """unit weights on a 24 x 24 grid: corner-to-corner path counts exceed 2^32 and wrap"""
    n, u, v, w = unit_grid_lines()
    idx = _csr(n, u, v, w)
    arcs = O.Arcs(n, u, v, w)
    _rows_equal_dijkstra(idx, arcs, np.array([0, 23, 24 * 12 + 5, n - 1], np.int32))
    assert rel_err(idx.bc_all(), arcs.bc()) <= BC_RTOL


def test_plain_path_equals_batched(g2k):
    n, u, v, w, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 37, dtype=np.int32)
    ref = idx.bc_sources(srcs)
    assert rel_err(idx.bc_plain(srcs), ref) <= BC_RTOL
    assert rel_err(ref, arcs.bc(srcs)) <= BC_RTOL


@pytest.mark.parametrize("delta", [0, 1, 1 << 20])
def test_plain_whole_gpu_sweep_matches_batched_shortcut_graph(delta):
    """the plain path sweeps one source with every CTA of a cooperative launch: same BC as the
    one-CTA-per-source batched sweep and the oracle, for label-setting, default and single-bucket
    widths"""
    n, u, v, w = grid_lines(5000, seed=9, shortcut_frac=0.05)
    idx = _csr(n, u, v, w, sweep_delta=delta)
    srcs = np.array([0, 17, 2500, n - 1], np.int32)
    ref = O.Arcs(n, u, v, w).bc(srcs)
    assert rel_err(idx.bc_plain(srcs), ref) <= BC_RTOL
    assert rel_err(idx.bc_sources(srcs), ref) <= BC_RTOL


def test_query_batch_and_served_requests(g2k):
    n, u, v, w, idx, tc, arcs = g2k
    full = arcs.bc()
    sets = request_sets(n, 16, 4, 1500, seed=5)
    for s, o in zip(sets, idx.bc_query_batch(sets)):
        assert rel_err(o, full[s]) <= BC_RTOL
    with idx.serve(max_active=8, chunk=256) as srv:
        tickets = [srv.submit(s) for s in sets[:6]]
        outs = [srv.wait(t, timeout_s=120.0) for t in tickets]
    for s, o in zip(sets[:6], outs):
        assert o is not None and rel_err(o[0], full[s]) <= BC_RTOL


def test_autotune_keeps_results(g2k):
    n, u, v, w, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 5, dtype=np.int32)
    before = idx.bc_sources(srcs)
    t = idx.autotune(srcs)
    assert t["tuning"]["sweep_threads"] in (0, 256, 512, 2048)
    assert rel_err(idx.bc_sources(srcs), before) <= BC_RTOL
    idx.set_tuning()


def test_la_graph_matches_reference_gpu(la_path):
    n, u, v, w = synth.read_graph_lines(la_path)
    g = Q.Graph(device=0)
    g.ReadGraph(la_path)
    idx = g.build_index(Q.QBC_INDEX_CSR)
    arcs = O.Arcs(n, u, v, w)
    _rows_equal_dijkstra(idx, arcs, np.arange(0, n, 4999, dtype=np.int32))
    p = os.path.join(GOLDEN, "ref_la_mhl.npz")
    if os.path.exists(p):
        assert rel_err(idx.bc_all(), np.load(p)["bc"]) <= BC_RTOL


def _sample(n, k, seed):
    return np.sort(np.random.default_rng(seed).choice(n, k, replace=False)).astype(np.int32)


def test_rq_200k_with_shortcuts_query_4096():
    """RQ on the 200,000-vertex grid + 2 % shortcuts with a uniform query set of 4,096 vertices:
    rows bit-exact, the sampled sweep's partial BC and the query set's values at 1e-9"""
    n, u, v, w = grid_lines(200000, seed=1, shortcut_frac=0.02)
    idx = _csr(n, u, v, w)
    arcs = O.Arcs(n, u, v, w)
    _rows_equal_dijkstra(idx, arcs, _sample(n, 3, 7))
    sample = _sample(n, 96, 8)
    part = idx.bc_sources(sample)
    assert rel_err(part, arcs.bc(sample)) <= BC_RTOL
    q = synth.query_set(n, 4096, seed=2)
    got = idx.bc_query_batch([q], sources=sample)[0]
    assert rel_err(got, part[q]) <= BC_RTOL


def test_1m_with_shortcuts_sample():
    """the 1,000,000-vertex grid + 2 % shortcuts: rows bit-exact, partial BC of a source sample,
    batched and plain paths agree"""
    n, u, v, w = grid_lines(1000000, seed=1, shortcut_frac=0.02)
    idx = _csr(n, u, v, w)
    arcs = O.Arcs(n, u, v, w)
    _rows_equal_dijkstra(idx, arcs, _sample(n, 2, 9))
    sample = _sample(n, 48, 10)
    part = idx.bc_sources(sample)
    assert rel_err(part, arcs.bc(sample)) <= BC_RTOL
    assert rel_err(idx.bc_plain(sample[:4]), arcs.bc(sample[:4])) <= BC_RTOL
