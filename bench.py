"""Benchmark: MHL-QBC all-vertex BC on a seeded 50k-vertex perturbed-grid road graph, plus the
other configurations of the workload as extra keys.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--n 50000]

One step = one full pass of the hot path over the workload: BC from all n sources (n source
sweeps: label scan for dist/count/hop rows, SP-DAG level bucketing, FP64 dependency backprop).
`value` is whole-job sources/s timed with CUDA events on the launching stream (index resident in
HBM); `e2e` is the same metric through the public C-ABI call with host buffers (source list H2D,
BC D2H inside the timed region).  With N>1 ranks (torchrun) each rank sweeps a contiguous share
of the sources and the partial BC vectors are summed with one NCCL all-reduce (strong scaling).

Extra keys (1 GPU, rank 0):
  qbc_2k        QBC on the committed 2,024-vertex grid with its min-degree order file (H2H index):
                all-source BC on the GPU, next to the oracle's CPU restatement of QBC.cu's loop
                (index-distance rows + host Kahn sigma pass + backprop) on the host cores;
  rq_200k       RQ on the seeded 200,000-vertex grid + 2 % random shortcuts (label-free index):
                a seeded source sample sweeps once and answers a uniform 4,096-vertex query set;
  shortcuts_1m  the 1,000,000-vertex grid + 2 % shortcuts: sampled sweep rate, the plain
                one-source-per-launch path, batched RQ (64 query sets in one sweep) and served RQ
                (Poisson arrivals at three rates) with p50/p99 latency, and the sweep kernel's
                roofline.

--impl reference times the reference algorithm's CPU restatement (oracle/, the reference itself
has no CPU BC path) on the host cores over a bounded source sample.
"""
from __future__ import annotations

import argparse
import gc
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
GRID = "27% lattice edges deleted, weights round(euclid*U[0.8,1.2]) in 1..1000"


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _config(n_actual, m_und, ns, args, extra=None):
    what = "full BC" if ns >= n_actual else f"partial BC over a seeded sample of {ns} sources"
    sc = (f" + {args.shortcuts:.0%} random shortcut edges (weights 500..5000)" if args.shortcuts else "")
    c = {"workload": f"MHL-QBC {what}, seeded perturbed grid n={n_actual} (~{m_und} undirected edges, {GRID}){sc}",
         "n": n_actual, "edges_undirected": m_und, "sources_per_step": ns, "graph_seed": args.seed,
         "parallelism": f"source-sharded x{args.gpus}" if args.gpus > 1 else "1 GPU",
         "l2": "working set (index + per-source scratch) > 126 MB L2; L2 additionally flushed between steps"}
    if extra:
        c.update(extra)
    return c


def load_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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
        return self

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


# ------------------------------------------------------------------------------- CPU baselines
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


def _timed_cpu(fn, n, seconds, seed):
    """fn(sources) run on a source sample sized for about `seconds` of work; sources/s."""
    rng = np.random.default_rng(seed)
    cores = os.cpu_count() or 1
    probe = rng.choice(n, size=min(n, 2 * cores), replace=False).astype(np.int32)
    t = time.perf_counter()
    fn(probe)
    per = (time.perf_counter() - t) / probe.shape[0]
    k = int(min(n, max(cores, seconds / max(per, 1e-6))))
    s = rng.choice(n, size=k, replace=False).astype(np.int32)
    t = time.perf_counter()
    fn(s)
    dt = time.perf_counter() - t
    return k, dt, cores


def cpu_baseline(path, seconds=12.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from gpu_betweennesscentrality_b200 import synth

    n, u, v, w = synth.read_graph_lines(path)
    tc = pyoracle.TreeCount(n, u, v, w)
    arcs = pyoracle.Arcs(n, u, v, w)
    cores = os.cpu_count() or 1
    k, dt, _ = _timed_cpu(lambda s: tc.bc(arcs, s, nthreads=cores), n, seconds, 5)
    return {"value": k / dt, "unit": "sources/s", "cores": cores, "kind": "port",
            "sample": f"{k} random sources of the same n={n} graph, oracle restatement of MHLQBC.cu:302-472 "
                      f"(OpenMP over sources), {dt:.1f} s"}


def cpu_brandes_baseline(n, u, v, w, seconds=10.0):
    """The oracle's Dijkstra-Brandes (the reference cannot build its index on the shortcut graphs)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    arcs = pyoracle.Arcs(n, u, v, w)
    cores = os.cpu_count() or 1
    k, dt, _ = _timed_cpu(lambda s: arcs.bc(s, nthreads=cores), n, seconds, 6)
    return {"value": k / dt, "unit": "sources/s", "cores": cores, "kind": "port",
            "sample": f"{k} random sources of the same n={n} graph, the oracle's Dijkstra-Brandes (OpenMP over "
                      f"sources; the reference's TreeDecomp index build does not finish on this graph), {dt:.1f} s"}


# ------------------------------------------------------------------------------- device timing
def device_sweep(idx, src_vids, steps, warmup, dev, flush, barrier=None):
    """CUDA-event timing of `steps` partial-BC sweeps over src_vids (device-resident inputs) on one
    stream, L2 flushed between steps outside the events; `barrier` (multi-rank) runs between the
    warm-up and the timed steps.  Returns (ms per step list, kernel stats, the BC accumulator)."""
    import torch

    stream = torch.cuda.Stream(device=dev)
    d_src = torch.from_numpy(np.ascontiguousarray(src_vids, np.int32)).to(dev)
    d_bc = torch.zeros(idx.n, dtype=torch.float64, device=dev)

    def step():
        with torch.cuda.stream(stream):
            d_bc.zero_()
        idx.bc_sources_device(d_src.data_ptr(), int(d_src.shape[0]), d_bc.data_ptr(), stream.cuda_stream)

    for _ in range(warmup):
        step()
    stream.synchronize()
    if barrier:
        barrier()
    torch.cuda.synchronize()
    idx.profile(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(k)
        torch.cuda.synchronize()
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    stats = idx.stats()
    idx.profile(False)
    return [a.elapsed_time(b) for a, b in ev], stats, d_bc


def e2e_rate(idx, src_vids, steps):
    """sources/s through the C-ABI call with host buffers (source list H2D and BC D2H timed)."""
    import torch

    h_src = torch.from_numpy(np.ascontiguousarray(src_vids, np.int32)).pin_memory()
    h_bc = torch.zeros(idx.n, dtype=torch.float64).pin_memory()
    idx.bc_sources(h_src.numpy())  # warm
    t = time.perf_counter()
    for _ in range(steps):
        h_bc.numpy()[:] = idx.bc_sources(h_src.numpy())
    dt = time.perf_counter() - t
    return len(src_vids) * steps / dt, dt


def plain_rate(idx, sources, k):
    ps = np.ascontiguousarray(sources[:: max(1, len(sources) // k)][:k], np.int32)
    idx.bc_plain(ps[:1])
    t = time.perf_counter()
    idx.bc_plain(ps)
    return ps.shape[0] / (time.perf_counter() - t), int(ps.shape[0])


# ------------------------------------------------------------------------------- rooflines
L2_BYTES = 126e6


def label_roofline(idx, shard, n, stats, steps, peak, peak_src, sm_mhz):
    """Dominant kernel of the label path: the packed label scan.  DRAM model per launch: the target
    rows' label distances -- read once per launch when the distance array fits in three quarters
    of the L2 (50k: 69 MB; every CTA group then finds them in L2), else once per CTA group of sources (32;
    16 for the lane-pair forms), each row up to the group's deepest LCA depth (4 B per entry, exact
    from the index) -- plus the count/hop gather at each pair's minimising entry (8 B per pair) and
    the (dist, count, rho) records and hop layers written (20 B per pair).  Cross-checked against
    ncu in profiles/k_label_scan_packed_50k.md and profiles/k_label_scan_tall_200k.md.  The
    algorithmic figure of the workload's byte model (12 B per label entry scanned + 12 B per pair)
    is given as effective_bw: rows are reused by every source of a group, so it exceeds the HBM
    peak."""
    ns = len(shard)
    per_cta = idx.label_group() or 32
    tall = per_cta == 16
    dis_bytes = 4.0 * idx.info()[2]
    scan = idx.scan_entries(shard)
    label_ms_step = stats["label_ms"] / steps
    launches_step = max(1.0, stats["label_launches"] / steps)
    launch_ms = label_ms_step / launches_step
    if dis_bytes <= 0.75 * L2_BYTES:
        rows_step = dis_bytes * launches_step
    else:
        rows_step = 4.0 * idx.group_entries(shard, per_cta)
    dram_step = rows_step + 28.0 * ns * n
    algo_step = 12.0 * scan + 12.0 * ns * n
    achieved = dram_step / launches_step / (launch_ms / 1e3) / 1e9
    effective = algo_step / launches_step / (launch_ms / 1e3) / 1e9
    ent_per_clk = scan / (label_ms_step / 1e3) / (sm_mhz * 1e6) / 148.0
    smem_roof = 32.0 if tall else 256.0 / 12.0
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_source": peak_src,
            "kernel": idx.label_kernel(), "sources_per_cta": per_cta,
            "dram_model_bytes_per_launch": dram_step / launches_step, "launch_ms": launch_ms,
            "launches_per_step": launches_step, "label_ms_per_step": label_ms_step,
            "dependency_ms_per_step": stats["dep_ms"] / steps,
            "effective_bw": {"achieved": effective, "unit": "GB/s", "frac_of_hbm_peak": effective / peak,
                             "algorithmic_bytes_per_launch": algo_step / launches_step},
            "compute_roof": {"unit": "label entries/clk/SM", "achieved": ent_per_clk, "peak": smem_roof,
                             "frac": ent_per_clk / smem_roof, "issue_peak": 128.0 / 3.5,
                             "note": "shared-memory roof: a 16-byte shared load takes at least one wavefront "
                                     "per half-warp (2 for a full-warp broadcast, measured); " +
                                     ("16-source forms (rows16, tall): lane pairs share a source row, so 8 wavefronts per 8 "
                                      "entries of 32 pairs (32.0)" if tall else
                                      "32 distinct source rows + broadcast target: 12 wavefronts per 8 entries "
                                      "of 32 pairs (21.3)") +
                                     "; issue_peak: 3.5 instructions per pair-entry at 128 lane-instructions/clk/SM"},
            "note": "frac = modelled DRAM bytes per launch / launch time / measured HBM copy bandwidth; traffic "
                    "is not measured in this run (ncu figures for the same kernel are in profiles/)"}


def sweep_roofline(n, ns_step, stats, steps, peak, peak_src):
    """The label-free sweep kernel (k_sweep_rows).  DRAM model per source: each 16-byte record is
    initialised (16 B), then read and rewritten by the in-degree pass (32 B) -- 48 B per vertex (the
    batched sweep writes no hop layers: the dependency pass reads its wave queue); the frontier
    phases' scattered record visits come on top (DRAM sectors per visit), which ncu's traffic in
    profiles/ shows (~415 B per (source, vertex) at 200k + 2 %)."""
    ms_step = stats["label_ms"] / steps
    launches_step = max(1.0, stats["label_launches"] / steps)
    launch_ms = ms_step / launches_step
    dram_step = 48.0 * n * ns_step
    achieved = dram_step / launches_step / (launch_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_source": peak_src, "kernel": "k_sweep_rows",
            "dram_model_bytes_per_launch": dram_step / launches_step, "launch_ms": launch_ms,
            "launches_per_step": launches_step, "sweep_ms_per_step": ms_step,
            "dependency_ms_per_step": stats["dep_ms"] / steps,
            "note": "model = 48 B per (source, vertex): record init, in-degree pass read + write; the scattered "
                    "frontier visits are gathers of DRAM sectors (ncu: ~415 B per (source, vertex) moved)"}


# ------------------------------------------------------------------------------- RQ (batched / served)
def rq_measurements(idx, n, sweep_value, args, sources=None, plain_value=None):
    """Batched RQ (64 query sets, sizes log-uniform in 16..16384, one graph-replayed sweep) and the
    served loop under Poisson arrivals at three rates (request sizes log-uniform in 1..8192).
    Host-timed through the public API with host buffers."""
    from gpu_betweennesscentrality_b200.serve import poisson_load, request_sets

    sets = request_sets(n, 64, 16, 16384, seed=2)
    ns = n if sources is None else int(len(sources))
    idx.bc_query_batch(sets, sources=sources)  # capture + warm
    reps = 3
    t = time.perf_counter()
    for _ in range(reps):
        outs = idx.bc_query_batch(sets, sources=sources)
    t_batch = (time.perf_counter() - t) / reps
    one = [idx.bc_query(s) if sources is None else idx.bc_query_batch([s], sources=sources)[0] for s in sets[:2]]
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-12 * max(1.0, float(np.max(np.abs(b)))))))
    batched = {"sets": 64, "query_vertices": int(sum(len(s) for s in sets)), "ms": t_batch * 1e3,
               "sweep_sources_per_s": ns / t_batch, "max_rel_diff_vs_one_set": max(rel(a, b) for a, b in zip(outs, one)),
               "note": "one qbc_bc_query_batch call: one graph-replayed sweep over the sources answers all 64 sets "
                       "(RQ of a set is BC restricted to it, so the per-source work is shared); the device "
                       "throughput against the plain path is batched_vs_plain"}
    if plain_value:
        batched["plain_sources_per_s"] = plain_value
        batched["batched_vs_plain"] = (ns / t_batch) / plain_value
        batched["plain_64_sets_s"] = 64 * ns / plain_value
    # served: slots = 64 concurrent requests; one turn over the sources takes ns / sweep rate
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


# ------------------------------------------------------------------------------- extra configs
def _csr_index(q, n_target, sc, seed):
    from gpu_betweennesscentrality_b200 import synth

    t = time.perf_counter()
    g = synth.grid_graph(n_target, seed=seed, shortcut_frac=sc)
    u, v, w = g.arcs()
    t_gen = time.perf_counter() - t
    G = q.Graph(device=0)
    G.ReadLines(g.n, u, v, w)
    t = time.perf_counter()
    idx = G.build_index(q.QBC_INDEX_CSR)
    return g, (u, v, w), idx, {"generate_s": round(t_gen, 2), "build_upload_s": round(time.perf_counter() - t, 3)}


def config_shortcuts_1m(q, args, dev, flush, peak, peak_src):
    """Batched and served RQ on the 1,000,000-vertex grid + 2 % random shortcuts (label-free index)."""
    g, (u, v, w), idx, build = _csr_index(q, args.shortcut_n, 0.02, args.seed)
    n = g.n
    sample = np.sort(np.random.default_rng(args.seed + 1).choice(n, min(n, args.shortcut_sample), replace=False)).astype(np.int32)
    tune = None
    if not args.no_autotune:
        t = time.perf_counter()
        tune = idx.autotune(sample)  # the step's own sample: chunk and occupancy as timed
        tune["seconds"] = round(time.perf_counter() - t, 2)
    steps = min(args.steps, 5)
    clocks = ClockSampler(dev.index or 0).start()
    ms, stats, _ = device_sweep(idx, sample, steps, 3, dev, flush)
    clk = clocks.stop()
    value = len(sample) * steps / (sum(ms) / 1e3)
    e2e, _ = e2e_rate(idx, sample, 2)
    plain, k_plain = plain_rate(idx, sample, 8)
    out = {"workload": f"batched / served RQ on the seeded {n}-vertex perturbed grid + 2% random shortcut edges "
                       f"(weights 500..5000), label-free index (per-source shortest-path sweeps); a seeded sample of "
                       f"{len(sample)} sources per step (partial BC)",
           "n": n, "arcs": int(idx.info()[1]), "sources_per_step": int(len(sample)), "steps": steps, "warmup": 3,
           "value": value, "unit": "sources/s", "ms_per_step": sum(ms) / steps,
           "e2e": {"value": e2e, "unit": "sources/s", "h2d_bytes_per_step": int(4 * len(sample)),
                   "d2h_bytes_per_step": int(8 * n)},
           "plain": {"value": plain, "unit": "sources/s", "sample": f"{k_plain} sources, one sweep launch + one "
                                                                     "dependency launch each"},
           "batched_vs_plain": value / plain, "index": build, "tuning": idx.get_tuning(), "autotune": tune,
           "roofline": sweep_roofline(n, len(sample), stats, steps, peak, peak_src), "clocks": clk,
           "gpu_launches": int(stats["launches"])}
    if not args.no_rq:
        out.update(rq_measurements(idx, n, value, args, sample, plain))
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_brandes_baseline(n, u, v, w, seconds=8.0)
    del idx
    gc.collect()
    return out


def config_mhl_1m(q, args, dev, flush, peak, peak_src):
    """The label path on a tree too tall for the 32-source label kernel: MHL-QBC partial BC on the
    1,000,000-vertex grid without shortcuts (tree height 2,725), rows filled on the device (its
    last 16,384 eliminations too), default tuning: the 16-source tall-tree label kernel."""
    import torch
    from gpu_betweennesscentrality_b200 import synth

    t = time.perf_counter()
    g = synth.grid_graph(args.shortcut_n, seed=args.seed)
    u, v, w = g.arcs()
    t_gen = time.perf_counter() - t
    G = q.Graph(device=0)
    G.ReadLines(g.n, u, v, w)
    t = time.perf_counter()
    idx = G.build_index(on_device=True)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t
    info = idx.info()
    n = g.n
    sample = np.sort(np.random.default_rng(args.seed + 1).choice(n, min(n, 4096), replace=False)).astype(np.int32)
    steps = min(args.steps, 3)
    clocks = ClockSampler(dev.index or 0).start()
    ms, stats, _ = device_sweep(idx, sample, steps, 3, dev, flush)
    clk = clocks.stop()
    value = len(sample) * steps / (sum(ms) / 1e3)
    e2e, _ = e2e_rate(idx, sample, 1)
    roof = label_roofline(idx, sample, n, stats, steps, peak, peak_src, clk.get("sm_mhz") or 1965.0)
    out = {"workload": f"MHL-QBC partial BC over a seeded sample of {len(sample)} sources, seeded perturbed grid "
                       f"n={n} without shortcuts (tree height {int(info[3])}: the tall-tree label kernel)",
           "n": n, "sources_per_step": int(len(sample)), "steps": steps, "warmup": 3,
           "value": value, "unit": "sources/s", "ms_per_step": sum(ms) / steps,
           "e2e": {"value": e2e, "unit": "sources/s", "h2d_bytes_per_step": int(4 * len(sample)),
                   "d2h_bytes_per_step": int(8 * n)},
           "index": {"tree_height": int(info[3]), "tree_width": int(info[4]), "label_entries": int(info[2]),
                     "device_bytes": int(info[5]), "generate_s": round(t_gen, 2),
                     "build_s": round(t_build, 3), "build": "device rows and dense elimination tail"},
           "tuning": idx.get_tuning(), "roofline": roof, "clocks": clk, "gpu_launches": int(stats["launches"])}
    del idx, G
    gc.collect()
    return out


def config_rq_200k(q, args, dev, flush):
    """RQ on the 200,000-vertex grid + 2 % shortcuts with a uniform query set of 4,096 vertices."""
    from gpu_betweennesscentrality_b200 import synth

    g, _, idx, build = _csr_index(q, 200000, 0.02, args.seed)
    n = g.n
    sample = np.sort(np.random.default_rng(args.seed + 1).choice(n, min(n, 4096), replace=False)).astype(np.int32)
    query = synth.query_set(n, 4096, seed=2)
    steps = min(args.steps, 5)
    ms, stats, _ = device_sweep(idx, sample, steps, 3, dev, flush)
    value = len(sample) * steps / (sum(ms) / 1e3)
    idx.bc_query_batch([query], sources=sample)
    t = time.perf_counter()
    idx.bc_query_batch([query], sources=sample)
    t_q = time.perf_counter() - t
    plain, k_plain = plain_rate(idx, sample, 16)
    out = {"workload": f"RQ on the seeded {n}-vertex perturbed grid + 2% random shortcut edges, query set of 4096 "
                       f"uniform vertices; a seeded sample of {len(sample)} sources per step (partial sums)",
           "n": n, "value": value, "unit": "sources/s", "ms_per_step": sum(ms) / steps, "steps": steps,
           "query_call": {"ms": t_q * 1e3, "sources_per_s": len(sample) / t_q,
                          "note": "one qbc_bc_query_batch call with host buffers (sweep + pick of the 4096 values)"},
           "plain": {"value": plain, "unit": "sources/s", "sample": f"{k_plain} sources"},
           "batched_vs_plain": value / plain, "index": build, "gpu_launches": int(stats["launches"]),
           "sweep_ms_per_step": stats["label_ms"] / steps, "dependency_ms_per_step": stats["dep_ms"] / steps}
    del idx
    gc.collect()
    return out


def config_qbc_2k(q, args):
    """QBC (H2H index from the committed min-degree order file) on the committed 2,024-vertex grid."""
    from gpu_betweennesscentrality_b200 import synth

    gpath = os.path.join(ROOT, "tests", "golden", "g2k.txt")
    opath = os.path.join(ROOT, "tests", "golden", "g2k.order")
    G = q.Graph(device=0)
    G.ReadGraph(gpath)
    n = G.nodenum
    order = q.read_order(opath, n)
    idx = G.build_index(q.QBC_INDEX_H2H, order, on_device=True)
    idx.bc_all()
    reps = 10
    t = time.perf_counter()
    for _ in range(reps):
        idx.bc_all()
    dt = (time.perf_counter() - t) / reps
    plain, k_plain = plain_rate(idx, np.arange(n, dtype=np.int32), 64)
    out = {"workload": f"QBC all-vertex BC, H2H index from the min-degree order file, seeded grid n={n}",
           "n": n, "value": n / dt, "unit": "sources/s", "ms_per_all_source_bc": dt * 1e3,
           "note": "qbc_bc_all with host output (graph-replayed sweep + D2H), host-timed over 10 calls",
           "plain": {"value": plain, "unit": "sources/s", "sample": f"{k_plain} sources"}}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle

        nn, u, v, w = synth.read_graph_lines(gpath)
        arcs = pyoracle.Arcs(nn, u, v, w)
        h2h = pyoracle.H2H(arcs, order)
        cores = os.cpu_count() or 1
        h2h.bc(nthreads=cores)
        t = time.perf_counter()
        h2h.bc(nthreads=cores)
        dc = time.perf_counter() - t
        out["cpu_baseline"] = {"value": n / dc, "unit": "sources/s", "cores": cores, "kind": "port",
                               "sample": f"all {n} sources: the oracle's restatement of QBC.cu:243-397 + the host "
                                         f"Kahn sigma pass of QBC.cu:485-555, OpenMP over sources, {dc:.2f} s"}
    del idx
    gc.collect()
    return out


# ------------------------------------------------------------------------------- main
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
    ap.add_argument("--no-extra", action="store_true", help="skip the extra configurations (2k QBC, 200k/1M shortcuts)")
    ap.add_argument("--shortcut-n", type=int, default=1000000, help="vertices of the shortcut-graph configuration")
    ap.add_argument("--shortcut-sample", type=int, default=2048, help="sources per step on the shortcut graph")
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
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    clocks = ClockSampler(local).start()
    ms_list, stats, d_bc = device_sweep(idx, shard, args.steps, args.warmup, dev, flush,
                                        barrier=(lambda: dist.barrier(device_ids=[local])) if world > 1 else None)
    clk = clocks.stop()
    ms = sum(ms_list)
    if world > 1:
        ms = max_over_ranks(ms, device=dev)
        all_reduce_bc(d_bc)  # the one exchange: sum of the ranks' partial BC vectors
        torch.cuda.synchronize()
    value = n_sources * args.steps / (ms / 1e3)

    # end to end through the C-ABI call with pinned host buffers: H2D of the source list and D2H of BC
    e2e_steps = max(1, min(args.steps, 3))
    if world > 1:
        dist.barrier(device_ids=[local])
    e2e_val, e2e_s = e2e_rate(idx, shard, e2e_steps)
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, device=dev)
        e2e_val = n_sources * e2e_steps / e2e_s

    peak, peak_src = load_peak()
    roof = label_roofline(idx, shard, n, stats, args.steps, peak, peak_src, clk.get("sm_mhz") or 1965.0)
    tuning_now = idx.get_tuning()
    plain = None
    rq = None
    cpu = None
    extra = {}
    if rank == 0 and world == 1:
        p_val, p_k = plain_rate(idx, shard, 192)
        plain = {"value": p_val, "unit": "sources/s",
                 "sample": f"{p_k} sources spread over the tid order, one label launch + one dependency launch "
                           f"each, host-timed with the final synchronisation"}
        if not args.no_rq:
            rq = rq_measurements(idx, n, value, args, None if n_sources == n else ex_vid, p_val)
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(path)
        if not args.no_extra:
            del idx
            G.index = None  # the last reference: frees the 50k index and its scratch
            gc.collect()
            torch.cuda.empty_cache()
            extra["qbc_2k"] = config_qbc_2k(q, args)
            extra["rq_200k"] = config_rq_200k(q, args, dev, flush)
            extra["shortcuts_1m"] = config_shortcuts_1m(q, args, dev, flush, peak, peak_src)
            extra["mhl_1m"] = config_mhl_1m(q, args, dev, flush, peak, peak_src)
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
                                  "tuning": tuning_now, "autotune": tune}),
               "e2e": {"value": e2e_val, "unit": "sources/s", "h2d_bytes_per_step": int(4 * ns),
                       "d2h_bytes_per_step": int(8 * n), "steps": e2e_steps},
               "roofline": roof,
               "gpu_launches": int(stats["launches"]),
               "clocks": clk}
        if cpu is not None:
            out["cpu_baseline"] = cpu
        if plain is not None:
            out["plain"] = plain
            out["batched_vs_plain"] = value / plain["value"]
        if rq is not None:
            out.update(rq)
        out.update(extra)
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
