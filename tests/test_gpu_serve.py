"""GPU: batched sweeps (graph-replayed), the autotuner and the served RQ loop.  Every answer must
equal BC restricted to the query set (the reference's RQ, RQ.cu:465-531) within BC_RTOL = 1e-9, and a
served request's answer must not depend on what else is in flight."""
import json
import os
import threading
import time

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
import pyoracle as O
from conftest import GOLDEN, rel_err
from gpu_betweennesscentrality_b200 import capi, synth
from gpu_betweennesscentrality_b200.serve import poisson_load, request_sets
from util import BC_RTOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g2k():
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    idx = g.build_index()
    full = O.TreeCount(n, u, v, w).bc(O.Arcs(n, u, v, w))
    return n, idx, full


def test_graph_replayed_sweep_matches_stream_path(g2k):
    n, idx, full = g2k
    a = idx.bc_all()
    b = idx.bc_all()  # second call replays the captured graph
    c = idx.bc_sources(np.arange(n, dtype=np.int32))
    assert rel_err(a, full) <= BC_RTOL and rel_err(b, full) <= BC_RTOL and rel_err(c, full) <= BC_RTOL


def test_query_batch_64_sets(g2k):
    n, idx, full = g2k
    sets = request_sets(n, 64, 16, 16384, seed=2)
    outs = idx.bc_query_batch(sets)
    for s, o in zip(sets, outs):
        assert o.shape == s.shape and rel_err(o, full[s]) <= BC_RTOL
    # partial sums over a source sample
    sample = np.arange(0, n, 3, dtype=np.int32)
    part = idx.bc_sources(sample)
    outs = idx.bc_query_batch(sets[:5], sources=sample)
    for s, o in zip(sets[:5], outs):
        assert rel_err(o, part[s]) <= BC_RTOL


def test_tuning_change_recaptures(g2k):
    n, idx, full = g2k
    idx.bc_all()
    idx.set_tuning(chunk=256, dep_form=2)
    try:
        assert rel_err(idx.bc_all(), full) <= BC_RTOL
        idx.set_tuning(chunk=256, dep_form=1, queue_depth=128)
        assert rel_err(idx.bc_all(), full) <= BC_RTOL
    finally:
        idx.set_tuning()
    assert rel_err(idx.bc_all(), full) <= BC_RTOL


def test_autotune_keeps_results(g2k, tmp_path):
    n, idx, full = g2k
    path = str(tmp_path / "tuning.json")
    try:
        res = idx.autotune(np.arange(0, n, 2, dtype=np.int32), path=path)
        assert res["ms_per_source"] > 0 and set(res["tuning"]) == set(Q.Index.TUNING_KEYS)
        assert rel_err(idx.bc_all(), full) <= BC_RTOL
        idx.set_tuning()
        got = idx.load_tuning(path)
        assert got == json.load(open(path))["tuning"]
        assert rel_err(idx.bc_all(), full) <= BC_RTOL
    finally:
        idx.set_tuning()


def test_serve_alone_and_in_the_mix(g2k):
    n, idx, full = g2k
    idx.set_tuning(chunk=256)  # 8 chunks per turn: requests overlap at many boundaries
    try:
        probe = request_sets(n, 1, 300, 300, seed=11)[0]
        with idx.serve(max_active=8) as srv:
            alone, _ = srv.wait(srv.submit(probe))
            assert rel_err(alone, full[probe]) <= BC_RTOL
            mix = request_sets(n, 30, 1, 2000, seed=12)
            tickets = []
            for i, s in enumerate(mix):
                tickets.append((s, srv.submit(s)))
                if i == 10:
                    tickets.append((probe, srv.submit(probe)))
                if i % 3 == 0:
                    time.sleep(0.002)
            for s, t in tickets:
                vals, (ts, ta, td) = srv.wait(t, 120.0)
                assert ts <= ta <= td
                assert rel_err(vals, full[s]) <= BC_RTOL
                if s is probe:
                    assert rel_err(vals, alone) <= BC_RTOL
            st = srv.stats()
            assert st["turns"] >= 1 and st["done"] == len(tickets) + 1 and st["active"] == 0
            assert st["chunks_per_turn"] == 8 and st["sources_per_turn"] == n
    finally:
        idx.set_tuning()


def test_serve_admission_by_pool_memory(g2k):
    n, idx, full = g2k
    idx.set_tuning(chunk=512)
    try:
        sets = request_sets(n, 4, 200, 200, seed=13)
        # room for one request of 200 vertices at a time (16 B per vertex)
        with idx.serve(max_active=64, pool_bytes=16 * 300) as srv:
            with pytest.raises(Q.QbcError) as e:
                srv.submit(np.arange(301, dtype=np.int32))
            assert e.value.code == capi.QBC_EINVAL
            ts = [srv.submit(s) for s in sets]
            res = [srv.wait(t, 120.0) for t in ts]
            for s, (vals, _) in zip(sets, res):
                assert rel_err(vals, full[s]) <= BC_RTOL
            times = sorted(r[1] for r in res)
            for a, b in zip(times, times[1:]):
                assert b[1] >= a[2] - 1e-3  # admitted only after the previous one released its pool range
    finally:
        idx.set_tuning()


def test_serve_holds_the_index(g2k):
    n, idx, full = g2k
    srv = idx.serve()
    try:
        with pytest.raises(Q.QbcError) as e:
            idx.bc_all()
        assert e.value.code == capi.QBC_EBUSY
        with pytest.raises(Q.QbcError):
            idx.set_tuning(chunk=128)
        with pytest.raises(Q.QbcError):
            idx.serve()
        empty = srv.submit(np.zeros(0, np.int32))
        assert srv.wait(empty)[0].shape == (0,)
        with pytest.raises(Q.QbcError):
            srv.submit(np.array([n], np.int32))
    finally:
        srv.close()
    assert rel_err(idx.bc_all(), full) <= BC_RTOL


def test_serve_source_sample_and_threads(g2k):
    n, idx, full = g2k
    sample = np.arange(0, n, 5, dtype=np.int32)
    part = idx.bc_sources(sample)
    sets = request_sets(n, 12, 1, 500, seed=14)
    got = {}
    with idx.serve(sources=sample) as srv:
        def client(k):
            got[k] = srv.wait(srv.submit(sets[k]), 120.0)[0]

        th = [threading.Thread(target=client, args=(k,)) for k in range(len(sets))]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for k, s in enumerate(sets):
        assert rel_err(got[k], part[s]) <= BC_RTOL


def test_serve_own_chunk_size(g2k):
    n, idx, full = g2k
    sets = request_sets(n, 6, 1, 900, seed=16)
    with idx.serve(chunk=90) as srv:  # rounded up to a multiple of 32: 96 sources per admission point
        res = [srv.wait(srv.submit(s), 120.0)[0] for s in sets]
        st = srv.stats()
    assert st["chunks_per_turn"] == (n + 95) // 96
    for s, vals in zip(sets, res):
        assert rel_err(vals, full[s]) <= BC_RTOL


def test_poisson_load_2k(g2k):
    n, idx, full = g2k
    idx.set_tuning(chunk=256)
    try:
        sets = request_sets(n, 40, 1, 8192, seed=15)
        with idx.serve(max_active=16) as srv:
            r = poisson_load(srv, sets, rate=400.0, seed=3, keep=True, timeout_s=120.0)
        assert r["p99_ms"] >= r["p50_ms"] > 0 and r["requests"] == 40
        for s, vals in zip(sets, r["results"]):
            assert rel_err(vals, full[s]) <= BC_RTOL
    finally:
        idx.set_tuning()


@pytest.mark.parametrize("name", ["single", "pair", "path3", "star5", "path40"])
def test_batch_and_serve_on_small_graphs(name):
    from util import KNOWN, lines_of

    n, edges, expect = KNOWN[name]
    nn, u, v, w = lines_of(edges, n)
    g = Q.Graph(device=0)
    g.ReadLines(nn, u, v, w)
    idx = g.build_index()
    want = np.asarray(expect, np.float64)
    sets = [np.arange(n, dtype=np.int32), np.array([n - 1], np.int32), np.zeros(0, np.int32)]
    outs = idx.bc_query_batch(sets)
    for s_, o in zip(sets, outs):
        assert np.allclose(o, want[s_], rtol=0, atol=1e-9)
    with idx.serve(max_active=2) as srv:
        ts = [srv.submit(s_) for s_ in sets]
        for s_, t in zip(sets, ts):
            assert np.allclose(srv.wait(t, 60.0)[0], want[s_], rtol=0, atol=1e-9)


def test_close_while_clients_wait(g2k):
    """closing the server fails the requests still queued; threads blocked in wait return with an
    error instead of hanging, and the index is usable again"""
    n, idx, full = g2k
    idx.set_tuning(chunk=64)
    try:
        srv = idx.serve(max_active=1)
        sets = request_sets(n, 30, 500, 500, seed=17)
        tickets = [srv.submit(s) for s in sets]
        errors, entered = [], []

        def client(t, ev):
            ev.set()
            try:
                srv.wait(t, 60.0)
            except Q.QbcError as e:
                errors.append(e.code)

        for t in tickets[-5:]:
            ev = threading.Event()
            th = threading.Thread(target=client, args=(t, ev))
            th.start()
            entered.append((th, ev))
        for th, ev in entered:
            ev.wait(10.0)
        time.sleep(0.02)  # the clients are inside the blocking wait call
        srv.close()
        for th, _ in entered:
            th.join(60.0)
        assert not any(th.is_alive() for th, _ in entered)
        assert all(code == capi.QBC_EBUSY for code in errors)  # cancelled by close
    finally:
        idx.set_tuning()
    assert rel_err(idx.bc_all(), full) <= BC_RTOL


def test_la_query_batch_and_served_match_reference_gpu(la_path, la_query_path):
    """the reference's own query batch on its LosAngeles graph: batched and served RQ equal the
    reference GPU's BC of those vertices (RQ = BC restricted to the set)"""
    p = os.path.join(GOLDEN, "ref_la_mhl.npz")
    if not os.path.exists(p):
        pytest.skip("ref_la_mhl.npz not generated")
    ref = np.load(p)["bc"]
    g = Q.Graph(device=0)
    g.ReadGraph(la_path)
    idx = g.build_index(on_device=True)
    q = Q.read_query(la_query_path, g.nodenum)
    sets = [q, q[::-1], q[:3]]
    for s_, o in zip(sets, idx.bc_query_batch(sets)):
        assert rel_err(o, ref[s_]) <= BC_RTOL
    with idx.serve() as srv:
        ts = [srv.submit(s_) for s_ in sets]
        for s_, t in zip(sets, ts):
            assert rel_err(srv.wait(t, 120.0)[0], ref[s_]) <= BC_RTOL
