"""Served RQ: Python handle of the library's request loop (qbc_serve_* in include/qbc_b200.h) and a
Poisson load driver that measures its latency.

The loop runs natively on its own host thread and CUDA stream.  It keeps sweeping the index's
sources chunk by chunk while requests are in flight, admits a request (a vertex set) at a chunk
boundary when a slot and pool memory are free, and completes it one full turn over the sources
later.  Every request's answer is therefore BC restricted to its vertex set (the reference's RQ,
RQ.cu:465-531), the same as ``Index.bc_query`` on that set alone.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Optional

import numpy as np

from .capi import check, f64p, i32, i32p, i64p, lib, ptr

STAT_KEYS = ("chunks", "turns", "done", "active", "queued", "pool_used", "pool_cap", "chunks_per_turn",
             "sources_per_turn")


class Server:
    def __init__(self, index, sources=None, max_active: int = 64, pool_bytes: int = 0, max_queue: int = 0,
                 chunk: int = 0):
        self.index = index
        self.h = C.c_void_p()
        src = None if sources is None else i32(sources)
        opts = np.array([max_active, pool_bytes, max_queue, chunk], np.int64)
        check(lib().qbc_serve_open(index.h, None if src is None else ptr(src, i32p),
                                   0 if src is None else int(src.shape[0]), ptr(opts, i64p), 4, C.byref(self.h)))
        self._sizes = {}

    def submit(self, points) -> int:
        p = i32(points)
        t = C.c_int64()
        check(lib().qbc_serve_submit(self.h, ptr(p, i32p) if p.shape[0] else None, int(p.shape[0]), C.byref(t)))
        self._sizes[t.value] = int(p.shape[0])
        return t.value

    def poll(self, ticket: int):
        """(values, (submit, admit, done) seconds) when complete, else None."""
        out = np.zeros(max(1, self._sizes[ticket]), np.float64)
        times = np.zeros(3, np.float64)
        done = C.c_int32()
        check(lib().qbc_serve_poll(self.h, int(ticket), ptr(out, f64p), ptr(times, f64p), C.byref(done)))
        if not done.value:
            return None
        q = self._sizes.pop(ticket)
        return out[:q], tuple(times)

    def wait(self, ticket: int, timeout_s: float = -1.0):
        out = np.zeros(max(1, self._sizes[ticket]), np.float64)
        times = np.zeros(3, np.float64)
        done = C.c_int32()
        check(lib().qbc_serve_wait(self.h, int(ticket), float(timeout_s), ptr(out, f64p), ptr(times, f64p),
                                   C.byref(done)))
        if not done.value:
            return None
        q = self._sizes.pop(ticket)
        return out[:q], tuple(times)

    def stats(self) -> dict:
        out = np.zeros(len(STAT_KEYS), np.float64)
        check(lib().qbc_serve_stats(self.h, ptr(out, f64p), len(STAT_KEYS)))
        return dict(zip(STAT_KEYS, out.tolist()))

    def close(self) -> None:
        if self.h:
            check(lib().qbc_serve_close(self.h))
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def log_uniform_sizes(rng: np.random.Generator, count: int, lo: int, hi: int) -> np.ndarray:
    """Integer sizes with log(size) uniform on [log lo, log hi]."""
    return np.minimum(hi, np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count)))).astype(np.int64)


def request_sets(n: int, count: int, lo: int, hi: int, seed: int):
    """`count` uniform random vertex sets (no repeats inside a set) of log-uniform sizes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = log_uniform_sizes(rng, count, lo, min(hi, n))
    return [np.sort(rng.choice(n, int(q), replace=False)).astype(np.int32) for q in sizes]


def poisson_load(server: Server, sets, rate: float, seed: int = 3, keep: bool = False,
                 timeout_s: Optional[float] = None) -> dict:
    """Submits `sets` at Poisson arrival times of `rate` requests/s and waits for all of them.
    Latency of a request = its completion minus its submission, as the server's clock records them."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(sets)))
    t0 = time.perf_counter()
    tickets = []
    for at, s in zip(arrivals, sets):
        dt = t0 + at - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        tickets.append(server.submit(s))
    lat, wait, results, first, last = [], [], [], None, None
    for t in tickets:
        r = server.wait(t, -1.0 if timeout_s is None else timeout_s)
        if r is None:
            raise TimeoutError(f"request {t} not done within {timeout_s} s")
        vals, (ts, ta, td) = r
        lat.append(td - ts)
        wait.append(ta - ts)
        first = ts if first is None else min(first, ts)
        last = td if last is None else max(last, td)
        if keep:
            results.append(vals)
    lat = np.array(lat)
    span = max(last - first, 1e-9)
    st = server.stats()
    out = dict(rate=rate, requests=len(sets), p50_ms=float(np.percentile(lat, 50) * 1e3),
               p99_ms=float(np.percentile(lat, 99) * 1e3), mean_ms=float(lat.mean() * 1e3),
               max_ms=float(lat.max() * 1e3), admit_wait_p99_ms=float(np.percentile(wait, 99) * 1e3),
               span_s=span, requests_per_s=len(sets) / span,
               query_vertices=int(sum(len(s) for s in sets)),
               effective_sources_per_s=len(sets) * st["sources_per_turn"] / span)
    if keep:
        out["results"] = results
    return out
