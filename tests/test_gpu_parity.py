"""GPU parity: the CUDA path (through the C ABI) against the oracle and the reference's own GPU
outputs.  Integers (dist / count bits / hop) bit-exact; BC within BC_RTOL = 1e-9 relative."""
import os
import subprocess

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
import pyoracle as O
from conftest import GOLDEN, ROOT, rel_err
from gpu_betweennesscentrality_b200 import capi, synth
from util import BC_RTOL, KNOWN, grid_lines, lines_of, unit_grid_lines

pytestmark = pytest.mark.gpu


def _graph(n, u, v, w):
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    return g


@pytest.fixture(scope="module")
def g2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = _graph(n, u, v, w)
    idx = g.build_index()
    return n, u, v, w, g, idx, O.TreeCount(n, u, v, w), O.Arcs(n, u, v, w)


def _order_g2k(n):
    return Q.read_order(os.path.join(GOLDEN, "g2k.order"), n)


def test_rows_bit_exact_all_sources_2k(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(n, dtype=np.int32)
    d, c, h = idx.rows(srcs)
    for s in range(0, n, 1):
        d0, c0, h0 = tc.rows(s)
        assert np.array_equal(d[s], d0), s
        assert np.array_equal(c[s], c0), s
        assert np.array_equal(h[s], h0), s


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
def test_rows_identical_across_tunings(g2k, lanes):
    """the packed-key kernel (auto) and every general-kernel lane split give identical rows"""
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 13, dtype=np.int32)
    base = idx.rows(srcs)
    idx.set_tuning(lanes_per_source=lanes, label_threads=128 if lanes > 4 else 256, split=3)
    try:
        alt = idx.rows(srcs)
    finally:
        idx.set_tuning()
    for a, b in zip(base, alt):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("warps,tile,passes", [(16, 0, 0), (8, 0, 0), (16, 32, 1), (8, 48, 1), (16, 8, 1),
                                               (16, 32, 2), (8, 48, 2), (16, 8, 2), (8, 20, 0),
                                               (12, 0, 0), (12, 32, 0), (12, 8, 0), (12, 44, 0),
                                               (20, 0, 0), (20, 40, 0), (20, 40, 2)])
def test_packed_kernel_tiles_and_warps(g2k, warps, tile, passes):
    """rows longer than the shared-memory tile: several tile passes (state kept in the output rows)
    or one pass with the entries beyond the tile from global memory: same rows, same BC"""
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 11, dtype=np.int32)
    base = idx.rows(srcs)
    idx.set_tuning(label_warps=warps, label_tile=tile, label_passes=passes)
    try:
        alt = idx.rows(srcs)
        bc = idx.bc_sources(srcs)
    finally:
        idx.set_tuning()
    for a, b in zip(base, alt):
        assert np.array_equal(a, b)
    assert rel_err(bc, tc.bc(arcs, srcs)) <= BC_RTOL


@pytest.mark.parametrize("warps,stream", [(0, 0), (8, 1), (12, 1), (16, 1), (8, 2), (12, 2), (16, 2)])
def test_tall_tree_kernel_forced_2k(g2k, warps, stream):
    """the 16-source forms of the packed scan (lane pairs: two targets per warp; target rows whole
    and double-buffered, or in 64-entry blocks through a cp.async ring) forced on the 2k graph: a
    ragged last group of sources, target chunks cut by n, ties -- rows bit-identical to the
    32-source kernel's, BC against the oracle"""
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(3, n, 11, dtype=np.int32)  # 182 sources: 11 groups of 16 and one of 6
    idx.set_tuning(label_sources=32)
    try:
        assert idx.label_group() == 32
        assert idx.label_kernel() == "k_label_scan_packed"
        base = idx.rows(srcs)
        idx.set_tuning(label_sources=16, label_warps=warps, label_stream=stream)
        assert idx.label_group() == 16
        assert idx.label_kernel() == ("k_label_scan_tall" if stream == 2 else "k_label_scan_rows16")
        alt = idx.rows(srcs)
        bc = idx.bc_sources(srcs)
    finally:
        idx.set_tuning()
    for a, b in zip(base, alt):
        assert np.array_equal(a, b)
    assert rel_err(bc, tc.bc(arcs, srcs)) <= BC_RTOL


@pytest.mark.parametrize("stream", [1, 2])
def test_tall_tree_kernel_unit_weight_ties(stream):
    """unit weights on a 40 x 40 lattice: most pairs have many shortest paths through several hubs
    (the scan's tie branch); the tall-tree kernel's rows equal the oracle's"""
    side = 40
    edges = [(r * side + c, r * side + c + 1, 1) for r in range(side) for c in range(side - 1)]
    edges += [(r * side + c, (r + 1) * side + c, 1) for r in range(side - 1) for c in range(side)]
    nn, u, v, w = lines_of(edges, side * side)
    g = _graph(nn, u, v, w)
    idx = g.build_index()
    tc = O.TreeCount(nn, u, v, w)
    srcs = np.arange(0, nn, 37, dtype=np.int32)
    idx.set_tuning(label_sources=16, label_stream=stream)
    try:
        d, c, h = idx.rows(srcs)
        bc = idx.bc_sources(srcs)
    finally:
        idx.set_tuning()
    for k, s in enumerate(srcs):
        d0, c0, h0 = tc.rows(int(s))
        assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0)
    assert rel_err(bc, tc.bc(O.Arcs(nn, u, v, w), srcs)) <= BC_RTOL


def test_bc_all_2k_matches_oracle_and_reference(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    bc = idx.bc_all()
    assert rel_err(bc, tc.bc(arcs)) <= BC_RTOL
    p = os.path.join(GOLDEN, "ref_g2k_mhl.txt")
    if os.path.exists(p):
        ref = np.loadtxt(p)
        assert rel_err(bc, ref[:, 1]) <= BC_RTOL


def test_plain_path_matches_batched(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 9, dtype=np.int32)
    assert rel_err(idx.bc_plain(srcs), idx.bc_sources(srcs)) <= BC_RTOL
    assert rel_err(idx.bc_sources(srcs), tc.bc(arcs, srcs)) <= BC_RTOL


@pytest.mark.parametrize("form", [1, 2, 3, 4])
def test_dependency_forms_agree(g2k, form):
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 5, dtype=np.int32)
    idx.set_tuning(dep_form=form)
    try:
        bc = idx.bc_sources(srcs)
    finally:
        idx.set_tuning()
    assert rel_err(bc, tc.bc(arcs, srcs)) <= BC_RTOL


@pytest.mark.parametrize("form", [1, 2, 3, 4])
def test_deep_dag_layer_counters_in_global_memory(form):
    """a 2,500-vertex path: hop layers up to 2,499 exceed the shared-memory layer counters of the
    CTA-per-source forms (2,046 layers for the pipelined one) and the warp forms' queues, so those
    count layers in their per-slot global arrays.  One shortest path per pair, so
    BC(v_i) = i * (n - 1 - i) exactly."""
    n = 2500
    nn, u, v, w = lines_of([(i, i + 1, 1 + i % 7) for i in range(n - 1)], n)
    g = Q.Graph(device=0)
    g.ReadLines(nn, u, v, w)
    idx = g.build_index()
    idx.set_tuning(dep_form=form)
    try:
        bc = idx.bc_all()
    finally:
        idx.set_tuning()
    i = np.arange(n, dtype=np.float64)
    assert np.allclose(bc, i * (n - 1 - i), rtol=1e-12, atol=0)


def test_device_source_list_any_order(g2k):
    """qbc_bc_sources_device takes the source list in any order, with repeats (it is sorted into
    tree order on the device): the same BC as the host entry point over the same multiset"""
    import torch

    n, u, v, w, g, idx, tc, arcs = g2k
    rng = np.random.default_rng(5)
    srcs = rng.choice(n, 700, replace=True).astype(np.int32)  # unsorted, with repeats
    d_src = torch.from_numpy(srcs).to("cuda:0")
    d_bc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    idx.set_tuning(chunk=256)  # several chunks out of the one sorted list
    try:
        idx.bc_sources_device(d_src.data_ptr(), int(srcs.shape[0]), d_bc.data_ptr())
        torch.cuda.synchronize()
        host = idx.bc_sources(srcs)
    finally:
        idx.set_tuning()
    assert rel_err(d_bc.cpu().numpy(), host) <= BC_RTOL
    assert rel_err(host, tc.bc(arcs, srcs)) <= BC_RTOL


def test_bc_repeatable_and_chunked(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    a = idx.bc_all()
    idx.set_tuning(chunk=96)
    try:
        b = idx.bc_all()
    finally:
        idx.set_tuning()
    assert rel_err(a, b) <= BC_RTOL


def test_qbc_h2h_2k(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    order = _order_g2k(n)
    gi = _graph(n, u, v, w)
    hidx = gi.build_index(Q.QBC_INDEX_H2H, order)
    h2 = O.H2H(arcs, order)
    srcs = np.arange(0, n, 7, dtype=np.int32)
    d, c, hop = hidx.rows(srcs)
    for k, s in enumerate(srcs):
        assert np.array_equal(d[k], h2.dist(int(s)))
        d0, c0, h0 = tc.rows(int(s))
        assert np.array_equal(c[k], c0)  # device Kahn sigma == TreeCount counts
        assert np.array_equal(hop[k], h0)  # Kahn wave == max-hop layer
    bc = hidx.bc_all()
    assert rel_err(bc, h2.bc()) <= BC_RTOL
    p = os.path.join(GOLDEN, "ref_g2k_qbc.txt")
    if os.path.exists(p):
        assert rel_err(bc, np.loadtxt(p)[:, 1]) <= BC_RTOL


def test_rq_2k(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    q = Q.read_query(os.path.join(GOLDEN, "g2k.query"), n)
    out = idx.bc_query(q)
    assert rel_err(out, tc.rq(q)) <= BC_RTOL
    p = os.path.join(GOLDEN, "ref_g2k_rq.txt")
    if os.path.exists(p):
        ref = np.loadtxt(p)
        assert np.array_equal(ref[:, 0].astype(int) - 1, q)
        assert rel_err(out, ref[:, 1]) <= BC_RTOL
    sets = [q[:3], q[3:], q[::-1]]
    outs = idx.bc_query_batch(sets)
    for s_, o_ in zip(sets, outs):
        assert rel_err(o_, idx.bc_query(s_)) <= BC_RTOL


def test_rq_follows_half_delta_where_the_pair_product_wraps():
    """RQ of a query set is BC restricted to it (1/2 sum_s delta_s); on the 24 x 24 unit grid the
    reference's int32 pair product (RQ.cu:456) wraps and its RQ departs from that value, which this
    library keeps (label and label-free indexes)"""
    n, u, v, w = unit_grid_lines()
    q = np.array([0, 11, 24 * 11 + 11, 24 * 12 + 12, 300, n - 1], np.int32)
    half_delta = O.Arcs(n, u, v, w).bc()[q]
    g = _graph(n, u, v, w)
    assert rel_err(g.build_index().bc_query(q), half_delta) <= BC_RTOL
    assert rel_err(g.build_index(Q.QBC_INDEX_CSR).bc_query(q), half_delta) <= BC_RTOL


def test_full_bc_50k_matches_reference_gpu_golden():
    """all-source BC of the benchmark's 50k grid against the reference's own GPU driver
    (MHLQBC.cu:495-537, run unmodified on a B200 by tests/golden/make_golden.py --g50k)"""
    p = os.path.join(GOLDEN, "ref_g50k_mhl.npz")
    if not os.path.exists(p):
        pytest.skip("50k reference golden not generated")
    ref = np.load(p)["bc"]
    n, u, v, w = grid_lines(50000, seed=1)
    g = _graph(n, u, v, w)
    assert rel_err(g.build_index(on_device=True).bc_all(), ref) <= BC_RTOL
    assert rel_err(g.build_index(Q.QBC_INDEX_CSR).bc_all(), ref) <= BC_RTOL


@pytest.mark.parametrize("name", sorted(KNOWN))
def test_known_graphs(name):
    n, edges, expect = KNOWN[name]
    nn, u, v, w = lines_of(edges, n)
    g = _graph(nn, u, v, w)
    idx = g.build_index()
    bc = idx.bc_all()
    full = O.Arcs(nn, u, v, w).bc()
    assert rel_err(bc, full) <= BC_RTOL
    if expect is not None:
        assert np.allclose(bc, expect, rtol=0, atol=1e-9)
    d, c, h = idx.rows(np.arange(n, dtype=np.int32))
    arcs = O.Arcs(nn, u, v, w)
    for s in range(n):
        d0, c0, h0 = arcs.dijkstra_rows(s)
        assert np.array_equal(d[s], d0) and np.array_equal(c[s], c0) and np.array_equal(h[s], h0)


def test_shortcut_graph_rows_and_bc():
    n, u, v, w = grid_lines(3000, seed=6, shortcut_frac=0.02)
    g = _graph(n, u, v, w)
    idx = g.build_index()
    tc = O.TreeCount(n, u, v, w)
    srcs = np.arange(0, n, 97, dtype=np.int32)
    d, c, h = idx.rows(srcs)
    for k, s in enumerate(srcs):
        d0, c0, h0 = tc.rows(int(s))
        assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0)
    want = tc.bc(O.Arcs(n, u, v, w), srcs)
    try:
        for form in (0, 1, 2, 3, 4):  # shortcut vertices have more than four arcs
            idx.set_tuning(dep_form=form, queue_depth=64 if form == 3 else 0)
            assert rel_err(idx.bc_sources(srcs), want) <= BC_RTOL, form
    finally:
        idx.set_tuning()


def test_50k_sampled_rows_and_partial_bc(graph_cache):
    path = synth.cached_graph(graph_cache, 50000, seed=1)
    n, u, v, w = synth.read_graph_lines(path)
    g = Q.Graph(device=0)
    g.ReadGraph(path)
    idx = g.build_index()
    tc = O.TreeCount(n, u, v, w)
    rng = np.random.default_rng(21)
    srcs = np.sort(rng.choice(n, 48, replace=False)).astype(np.int32)
    d, c, h = idx.rows(srcs[:12])
    for k, s in enumerate(srcs[:12]):
        d0, c0, h0 = tc.rows(int(s))
        assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0)
    assert rel_err(idx.bc_sources(srcs), tc.bc(O.Arcs(n, u, v, w), srcs)) <= BC_RTOL


def test_200k_tall_tree_rows_and_partial_bc(graph_cache):
    """the 200k grid's tree (height 1,088) is taller than the 32-source kernel's shared tile: the
    default is the tall-tree form (16 sources per CTA, whole rows in shared memory); the 32-source
    kernel reads entries beyond its tile from global memory, takes further tile passes, or with 16
    warps a longer global tail -- rows bit-exact and partial BC against the oracle in every case"""
    path = synth.cached_graph(graph_cache, 200000, seed=1)
    n, u, v, w = synth.read_graph_lines(path)
    g = Q.Graph(device=0)
    g.ReadGraph(path)
    idx = g.build_index(on_device=True)
    assert idx.info()[3] > 1024
    tc = O.TreeCount(n, u, v, w)
    rng = np.random.default_rng(22)
    srcs = np.sort(rng.choice(n, 16, replace=False)).astype(np.int32)
    want = [tc.rows(int(s)) for s in srcs[:4]]
    try:
        assert idx.label_group() == 16
        for tune in ({}, {"label_sources": 32}, {"label_warps": 16}, {"label_passes": 2}, {"label_warps": 12},
                     {"label_sources": 16, "label_warps": 8}, {"label_sources": 16, "label_stream": 1}):
            idx.set_tuning(**tune)
            d, c, h = idx.rows(srcs[:4])
            for k in range(4):
                d0, c0, h0 = want[k]
                assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0), tune
    finally:
        idx.set_tuning()
    assert rel_err(idx.bc_sources(srcs), tc.bc(O.Arcs(n, u, v, w), srcs)) <= BC_RTOL


def test_la_full_bc_matches_reference_gpu(la_path):
    p = os.path.join(GOLDEN, "ref_la_mhl.npz")
    g = Q.Graph(device=0)
    g.ReadGraph(la_path)
    idx = g.build_index()
    n, u, v, w = synth.read_graph_lines(la_path)
    tc = O.TreeCount(n, u, v, w)
    srcs = np.arange(0, n, 997, dtype=np.int32)
    d, c, h = idx.rows(srcs)
    for k, s in enumerate(srcs):
        d0, c0, h0 = tc.rows(int(s))
        assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0)
    bc = idx.bc_all()
    if os.path.exists(p):
        assert rel_err(bc, np.load(p)["bc"]) <= BC_RTOL
    assert rel_err(idx.bc_sources(srcs), tc.bc(O.Arcs(n, u, v, w), srcs)) <= BC_RTOL


def test_row_copy_wait_timeout_is_reported_and_the_index_recovers(g2k):
    """A label-row copy wait that runs out sets the error word; the warp waits out its copies in
    flight, the dependency pass skips the partial rows, the call returns QBC_EDEVICE, and the next
    call on the same index is correct.  QBC_TEST_ROW_WAIT_SPINS=0 makes every wait give up at once."""
    n, u, v, w, g, idx, tc, arcs = g2k
    srcs = np.arange(0, n, 7, dtype=np.int32)
    ref = idx.bc_sources(srcs)
    os.environ["QBC_TEST_ROW_WAIT_SPINS"] = "0"
    try:
        with pytest.raises(Q.QbcError) as e:
            idx.bc_sources(srcs)
        assert e.value.code == capi.QBC_EDEVICE and "copy wait" in str(e.value)
    finally:
        del os.environ["QBC_TEST_ROW_WAIT_SPINS"]
    assert rel_err(idx.bc_sources(srcs), ref) <= BC_RTOL
    d, c, h = idx.rows(srcs[:5])
    for k, s_ in enumerate(srcs[:5]):
        d0, c0, h0 = tc.rows(int(s_))
        assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0)


def test_errors_are_reported(g2k):
    n, u, v, w, g, idx, tc, arcs = g2k
    with pytest.raises(Q.QbcError):
        idx.bc_sources(np.array([0, n], np.int32))
    with pytest.raises(Q.QbcError):
        idx.bc_query(np.array([-1], np.int32))
    # the index is still usable afterwards
    assert rel_err(idx.bc_sources(np.arange(5, dtype=np.int32)), tc.bc(arcs, np.arange(5, dtype=np.int32))) <= BC_RTOL


def test_cli_drop_in(tmp_path):
    g = os.path.join(GOLDEN, "g2k.txt")
    binp = os.path.join(ROOT, "gpu_betweennesscentrality_b200", "bin")
    env = dict(os.environ, QBC_OUTPUT_DIGITS="17")
    r = subprocess.run([os.path.join(binp, "MHLQBC"), g, "0", str(tmp_path / "mhl.txt")], capture_output=True,
                       text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "seconds (---totalTime---)" in r.stdout and r.stdout.startswith("roadDataPath:")
    out = np.loadtxt(tmp_path / "mhl.txt", skiprows=1)
    n, u, vv, w = synth.read_graph_lines(g)
    ref = O.TreeCount(n, u, vv, w).bc(O.Arcs(n, u, vv, w))
    assert rel_err(out[:, 1], ref) <= BC_RTOL
    std = tmp_path / "std.txt"  # standard-BC file format of QBC.cu:632-638: "n m" then "vid bc"
    std.write_text(f"{n} {u.shape[0]}\n" + "".join(f"{i + 1} {x:.17g}\n" for i, x in enumerate(ref)))
    r = subprocess.run([os.path.join(binp, "QBC"), g, os.path.join(GOLDEN, "g2k.order"), "0", str(tmp_path / "q.txt"),
                        str(std)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "BC value is correct" in r.stdout
    # a tighter tolerance through QBC_STD_TOL, and a planted error it catches
    bad = tmp_path / "bad.txt"
    bad.write_text(f"{n} {u.shape[0]}\n" + "".join(f"{i + 1} {x + (1e-6 if i == 5 else 0):.17g}\n" for i, x in enumerate(ref)))
    env2 = dict(env, QBC_STD_TOL="1e-8")
    r = subprocess.run([os.path.join(binp, "QBC"), g, os.path.join(GOLDEN, "g2k.order"), "0", str(tmp_path / "q2.txt"),
                        str(bad)], capture_output=True, text=True, env=env2, timeout=300)
    assert r.returncode == 1 and "not correct for node 5" in r.stdout
    r = subprocess.run([os.path.join(binp, "RQ"), g, os.path.join(GOLDEN, "g2k.query"), "0"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "The number of vertices to query: 10" in r.stdout and "vertexID" in r.stdout


def test_wrapping_counts_on_device():
    """32-bit path counts that wrap (unit-weight 24 x 24 grid) are bit-exact on the device, and BC
    (computed from the wrapped counts, as the reference does) agrees with the oracle"""
    n, u, v, w = unit_grid_lines()
    g = _graph(n, u, v, w)
    for idx in (g.build_index(), g.build_index(on_device=True)):
        tc = O.TreeCount(n, u, v, w)
        srcs = np.array([0, 100, n - 1], np.int32)
        d, c, h = idx.rows(srcs)
        for k, s in enumerate(srcs):
            d0, c0, h0 = tc.rows(int(s))
            assert np.array_equal(d[k], d0) and np.array_equal(c[k], c0) and np.array_equal(h[k], h0)
        assert int(c[0][-1]) == 4273388464
        assert rel_err(idx.bc_all(), tc.bc(O.Arcs(n, u, v, w))) <= BC_RTOL
