"""Benchmark: MHL-QBC all-vertex BC on a seeded 50k-vertex perturbed-grid road graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--n 50000]

One step = one full pass of the hot path over the workload: BC from all n sources (n source
sweeps: label scan for dist/count/hop rows, SP-DAG level bucketing, FP64 dependency backprop).
`value` is whole-job sources/s timed with CUDA events on the launching stream (index resident in
HBM); `e2e` is the same metric through the public C-ABI call with host buffers (source list H2D,
BC D2H inside the timed region).  With N>1 ranks (torchrun) each rank sweeps a contiguous share
of the sources and the partial BC vectors are summed with one NCCL all-reduce (strong scaling).

--impl reference times the reference algorithm's CPU restatement (oracle/, the reference itself
has no CPU BC path) on the host cores over a bounded source sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CACHE = os.environ.get("QBC_BENCH_CACHE", os.path.join(tempfile.gettempdir(), "qbc_bench_cache"))
METRIC = "sources/s (MHL-QBC all-vertex BC, exact counts)"


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _config(n_actual, m_und, ns, args, extra=None):
    what = "full BC" if ns >= n_actual else f"partial BC over a seeded sample of {ns} sources"
    sc = (f" + {args.shortcuts:.0%} random shortcut edges (weights 500..5000)" if args.shortcuts else "")
    c = {"workload": f"MHL-QBC {what}, seeded perturbed grid n={n_actual} (~{m_und} undirected edges, "
                     f"27% lattice edges deleted, weights round(euclid*U[0.8,1.2]) in 1..1000){sc}",
         "n": n_actual, "edges_undirected": m_und, "sources_per_step": ns, "graph_seed": args.seed,
         "parallelism": f"source-sharded x{args.gpus}" if args.gpus > 1 else "1 GPU",
         "l2": "working set (index + per-source scratch) > 126 MB L2; L2 additionally flushed between steps"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(args):
    """CPU restatement of the reference's per-source loop, all host threads, bounded sample."""
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from gpu_betweennesscentrality_b200 import synth

    path = synth.cached_graph(CACHE, args.n, seed=args.seed, shortcut_frac=args.shortcuts)
    n, u, v, w = synth.read_graph_lines(path)
    tc = pyoracle.TreeCount(n, u, v, w)
    arcs = pyoracle.Arcs(n, u, v, w)
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(11)
    # size the per-step sample for ~ (budget / steps) seconds of CPU work
    probe = rng.choice(n, size=min(n, 2 * cores), replace=False).astype(np.int32)
    t = time.perf_counter()
    tc.bc(arcs, probe, nthreads=cores)
    per_src = (time.perf_counter() - t) / probe.shape[0]
    budget = float(os.environ.get("QBC_REF_BUDGET_S", "120"))
    per_step = max(cores, int(budget / max(1, args.steps + args.warmup) / max(per_src, 1e-6)))
    per_step = min(per_step, n)
    for _ in range(args.warmup):
        tc.bc(arcs, rng.choice(n, size=min(per_step, n), replace=False).astype(np.int32), nthreads=cores)
    times = []
    for _ in range(args.steps):
        s = rng.choice(n, size=per_step, replace=False).astype(np.int32)
        t = time.perf_counter()
        tc.bc(arcs, s, nthreads=cores)
        times.append(time.perf_counter() - t)
    tot = sum(times)
    val = per_step * args.steps / tot
    sample = f"{per_step} random sources per step of the n={n} all-source workload, {args.steps} steps"
    out = {"metric": METRIC, "value": val, "unit": "sources/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "int32 dist/count, f64 dependency", "data": "synthetic",
           "impl": "reference",
           # the same workload as the B200 arm; each timed step here is a bounded sample of it
           "config": _config(n, int(u.shape[0]) // 2, args.sample if 0 < args.sample < n else n, args),
           "cpu_baseline": {"value": val, "unit": "sources/s", "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": val, "unit": "sources/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def cpu_baseline(path, seconds=12.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from gpu_betweennesscentrality_b200 import synth

    n, u, v, w = synth.read_graph_lines(path)
    tc = pyoracle.TreeCount(n, u, v, w)
    arcs = pyoracle.Arcs(n, u, v, w)
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(5)
    probe = rng.choice(n, size=min(n, 2 * cores), replace=False).astype(np.int32)
    t = time.perf_counter()
    tc.bc(arcs, probe, nthreads=cores)
    per = (time.perf_counter() - t) / probe.shape[0]
    k = int(min(n, max(cores, seconds / max(per, 1e-6))))
    s = rng.choice(n, size=k, replace=False).astype(np.int32)
    t = time.perf_counter()
    tc.bc(arcs, s, nthreads=cores)
    dt = time.perf_counter() - t
    return {"value": k / dt, "unit": "sources/s", "cores": cores, "kind": "port",
            "sample": f"{k} random sources of the same n={n} graph, oracle restatement of MHLQBC.cu:302-472 "
                      f"(OpenMP over sources), {dt:.1f} s"}


def rq_measurements(idx, n, sweep_value, args, sources=None):
    """Batched RQ (64 query sets, sizes log-uniform in 16..16384, one graph-replayed sweep) against
    the plain per-set calls, and the served loop under Poisson arrivals at three rates (request sizes
    log-uniform in 1..8192).  Host-timed through the public API with host buffers."""
    from gpu_betweennesscentrality_b200.serve import poisson_load, request_sets

    sets = request_sets(n, 64, 16, 16384, seed=2)
    ns = n if sources is None else int(len(sources))
    idx.bc_query_batch(sets, sources=sources)  # capture + warm
    reps = 3
    t = time.perf_counter()
    for _ in range(reps):
        outs = idx.bc_query_batch(sets, sources=sources)
    t_batch = (time.perf_counter() - t) / reps
    k_plain = 4  # 64 sequential per-set sweeps would take 64 sweeps; 4 of them are timed
    t = time.perf_counter()
    plain_outs = [idx.bc_query(s) if sources is None else idx.bc_query_batch([s], sources=sources)[0]
                  for s in sets[:k_plain]]
    t_plain_set = (time.perf_counter() - t) / k_plain
    diff = max(float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) for a, b in zip(outs, plain_outs))
    batched = {"max_rel_diff_vs_plain": diff, "sets": 64, "query_vertices": int(sum(len(s) for s in sets)), "ms": t_batch * 1e3,
               "sources_per_s": 64 * ns / t_batch,
               "plain_per_set_ms": t_plain_set * 1e3, "plain_sources_per_s": ns / t_plain_set,
               "speedup_vs_64_sequential": 64 * t_plain_set / t_batch,
               "note": f"plain = one qbc_bc_query call (one full sweep) per set, {k_plain} of 64 timed; "
                       "batched = one qbc_bc_query_batch call, one graph-replayed sweep for all 64 sets"}
    # served: slots = 64 concurrent requests; one turn over the sources takes n / sweep rate
    turn_s = ns / sweep_value
    slots = 64
    capacity = slots / turn_s
    chunk = max(256, (ns // 8 + 31) // 32 * 32)  # about 8 admission points per turn
    served = {"slots": slots, "turn_ms": turn_s * 1e3, "capacity_requests_per_s": capacity,
              "chunk_sources": min(chunk, idx.get_tuning()["chunk"] or chunk), "rates": []}
    for i, frac in enumerate((0.5, 0.8, 0.95)):
        rate = frac * capacity
        count = max(20, int(rate * args.served_seconds))
        reqs = request_sets(n, count, 1, 8192, seed=100 + i)
        with idx.serve(sources=sources, max_active=slots, chunk=chunk) as srv:
            r = poisson_load(srv, reqs, rate=rate, seed=3 + i)
        r["rate_fraction_of_capacity"] = frac
        served["rates"].append({k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()})
    return {"batched_rq": batched, "served_rq": served}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=50000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chunk", type=int, default=0, help="sources per scratch buffer (0: sized from free HBM)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tuning instead of autotuning")
    ap.add_argument("--sample", type=int, default=0,
                    help="sources per step: a seeded sample of this many vertices (0: all n, the full BC)")
    ap.add_argument("--shortcuts", type=float, default=0.0, help="fraction of n random shortcut edges (500..5000)")
    ap.add_argument("--host-build", action="store_true", help="fill the label rows on the host (default: on the GPU)")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="set a tuning field (Index.TUNING_KEYS) instead of autotuning it; repeatable")
    ap.add_argument("--no-rq", action="store_true", help="skip the batched and served RQ measurements")
    ap.add_argument("--served-seconds", type=float, default=8.0, help="arrival window per served rate")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    import gpu_betweennesscentrality_b200 as q
    from gpu_betweennesscentrality_b200 import synth

    rank, world, local = _env_rank()
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    if rank == 0:
        path = synth.cached_graph(CACHE, args.n, seed=args.seed, shortcut_frac=args.shortcuts)
    if world > 1:
        dist.barrier(device_ids=[local])
    path = synth.cached_graph(CACHE, args.n, seed=args.seed, shortcut_frac=args.shortcuts)

    G = q.Graph(device=local)
    t = time.perf_counter()
    G.ReadGraph(path)
    t_read = time.perf_counter() - t
    t = time.perf_counter()
    if args.host_build:
        idx = G.build_index(upload=False)
    else:  # elimination and tree on the host, label rows filled on the GPU
        idx = G.build_index(on_device=True)
        torch.cuda.synchronize()
    t_build = time.perf_counter() - t
    if args.chunk or args.tune:
        fixed = {"chunk": args.chunk}
        fixed.update({k: int(v) for k, v in (t.split("=", 1) for t in args.tune)})
        idx.set_tuning(**fixed)
    t = time.perf_counter()
    if args.host_build:
        idx.upload(local)
        torch.cuda.synchronize()
    t_upload = time.perf_counter() - t
    info = idx.info()
    n = G.nodenum
    ex_vid = idx.export()["vid_of"]  # tid order keeps each CTA's sources close in the tree
    if args.sample and args.sample < n:
        # a seeded sample of sources, kept in tid order
        tid_of = np.empty(n, np.int64)
        tid_of[ex_vid] = np.arange(n)
        pick = np.random.default_rng(args.seed + 1).choice(n, args.sample, replace=False)
        ex_vid = ex_vid[np.sort(tid_of[pick])]
    n_sources = int(ex_vid.shape[0])
    tune = None
    if not args.no_autotune and not args.chunk and not args.tune:
        t = time.perf_counter()
        k = int(min(8192, max(512, 8192 * 50000 / n)))  # about 50 ms of sweep per trial
        sample = ex_vid[:: max(1, n_sources // k)][:k]
        tune = idx.autotune(sample)
        tune["seconds"] = round(time.perf_counter() - t, 2)
    from gpu_betweennesscentrality_b200.shard import all_reduce_bc, max_over_ranks, shard_sources

    shard = shard_sources(ex_vid, world, rank)
    ns = int(shard.shape[0])

    stream = torch.cuda.Stream(device=dev)
    d_src = torch.from_numpy(shard).to(dev)
    d_bc = torch.zeros(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    def step():
        with torch.cuda.stream(stream):
            d_bc.zero_()
        idx.bc_sources_device(d_src.data_ptr(), ns, d_bc.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    if world > 1:
        dist.barrier(device_ids=[local])
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    idx.profile(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k)  # evicts L2 between timed steps (outside the events)
        torch.cuda.synchronize()
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    stats = idx.stats()
    idx.profile(False)
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    if world > 1:
        ms = max_over_ranks(ms, device=dev)
        all_reduce_bc(d_bc)  # the one exchange: sum of the ranks' partial BC vectors
        torch.cuda.synchronize()
    value = n_sources * args.steps / (ms / 1e3)

    # end to end through the C-ABI call with pinned host buffers: H2D of the source list and D2H of BC
    h_src = torch.from_numpy(shard).pin_memory()
    h_bc = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    idx.bc_sources(h_src.numpy())  # warm
    if world > 1:
        dist.barrier(device_ids=[local])
    t = time.perf_counter()
    for _ in range(e2e_steps):
        h_bc.numpy()[:] = idx.bc_sources(h_src.numpy())
    e2e_s = time.perf_counter() - t
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, device=dev)
    e2e_val = n_sources * e2e_steps / e2e_s

    # Roofline of the dominant kernel (the label scan).  Algorithmic bytes follow the per-source
    # label term of the workload's byte model: 12 B (dist, count, hop) per label entry a scan
    # consumes, sum over targets of depth(lca(s,t)) computed exactly from the index, plus 12 B of
    # dist/count/hop written per target.  The batched kernel fetches each target row once per
    # 32-source group and keeps source rows in shared memory, so achieved can exceed the HBM
    # peak; the DRAM bytes ncu measured for the same kernel (profiles/) are given as traffic, and
    # the inner loop's own roof (shared-memory wavefronts) as compute_roof.
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    entries = idx.scan_entries(shard)  # sum over (s,t) of label entries scanned
    label_bytes_step = 12.0 * entries + 12.0 * ns * n
    label_ms_step = stats["label_ms"] / args.steps
    launches_step = max(1.0, stats["label_launches"] / args.steps)
    per_launch_bytes = label_bytes_step / launches_step
    per_launch_ms = label_ms_step / launches_step
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "k_label_scan_packed_50k.md")
    if os.path.exists(prof) and args.n == 50000 and not args.shortcuts and n_sources == n:
        import re
        m = re.search(r"dram_bytes_per_source:\s*([0-9.e+]+)", open(prof).read())
        if m:
            traffic = float(m.group(1)) * ns / launches_step
    sm_mhz = (clk.get("sm_mhz") or 1965.0)
    ent_per_clk = entries / (label_ms_step / 1e3) / (sm_mhz * 1e6) / 148.0
    # plain path (one source per launch pair) on a sample, for the batched-vs-plain ratio
    plain = None
    if rank == 0 and world == 1:
        ps = shard[:: max(1, ns // 192)][:192]
        idx.bc_plain(ps[:8])
        torch.cuda.synchronize()
        t = time.perf_counter()
        idx.bc_plain(ps)
        plain = {"value": ps.shape[0] / (time.perf_counter() - t), "unit": "sources/s",
                 "sample": f"{ps.shape[0]} sources spread over the tid order, one label launch + one "
                           f"dependency launch each, host-timed with the final synchronisation"}
    rq = None
    if rank == 0 and world == 1 and not args.no_rq:
        rq = rq_measurements(idx, n, value, args, None if n_sources == n else ex_vid)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(path)
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "sources/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "strong", "vs_baseline": None,
               "dtype": "int32 dist / uint32 wrapping count / int32 hop; f64 dependency", "data": "synthetic",
               "config": _config(n, int(info[1]) // 2, n_sources, args,
                                 {"index": {"tree_height": int(info[3]), "tree_width": int(info[4]),
                                            "label_entries": int(info[7]), "device_bytes": int(info[5]),
                                            "build": "host" if args.host_build else "device rows",
                                            "build_s": round(t_build, 3), "read_s": round(t_read, 3),
                                            "upload_s": round(t_upload, 3)},
                                  "tuning": idx.get_tuning(), "autotune": tune}),
               "e2e": {"value": e2e_val, "unit": "sources/s", "h2d_bytes_per_step": int(4 * ns),
                       "d2h_bytes_per_step": int(8 * n), "steps": e2e_steps},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                            "kernel": "k_label_scan_packed",
                            "algorithmic_bytes_per_launch": per_launch_bytes,
                            "launch_ms": per_launch_ms,
                            "launches_per_step": launches_step,
                            "label_ms_per_step": label_ms_step,
                            "dependency_ms_per_step": stats["dep_ms"] / args.steps,
                            "compute_roof": {"unit": "label entries/clk/SM", "achieved": ent_per_clk,
                                             "peak": 25.6, "frac": ent_per_clk / 25.6,
                                             "issue_peak": 128.0 / 3.5,
                                             "note": "inner-loop model roofs: 5 shared-memory wavefronts per 128 "
                                                     "lane-entries (source-row LDS.128 + broadcast target row) "
                                                     "gives 25.6; 3.5 instructions per pair-entry at 128 lane-"
                                                     "instructions/clk/SM gives issue_peak; kernels moving 40-60 % "
                                                     "fewer wavefronts measured no faster, so issue and latency bind"},
                            "note": "algorithmic bytes = 12 B per label entry scanned + 12 B per target "
                                    "written; target rows are fetched once per 32-source group, so achieved "
                                    "exceeds HBM peak and DRAM traffic (profiles/) stays far below it"},
               "gpu_launches": int(stats["launches"]),
               "clocks": clk}
        if cpu is not None:
            out["cpu_baseline"] = cpu
        if plain is not None:
            out["plain"] = plain
            out["batched_vs_plain"] = value / plain["value"]
        if rq is not None:
            out.update(rq)
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
