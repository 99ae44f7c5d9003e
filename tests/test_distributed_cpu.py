"""CPU: the multi-rank path's host logic with two gloo ranks.  Each rank computes the partial BC of
its contiguous source share (with the oracle, standing in for the device sweep), one all-reduce sums
them, and the result must equal the single-rank BC; timings reduce to the slowest rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import GOLDEN, ROOT, rel_err


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import sys

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import torch
    import torch.distributed as dist

    import pyoracle as O
    from gpu_betweennesscentrality_b200 import synth
    from gpu_betweennesscentrality_b200.shard import all_reduce_bc, max_over_ranks, shard_sources

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    tc, arcs = O.TreeCount(n, u, v, w), O.Arcs(n, u, v, w)
    order = np.arange(n, dtype=np.int32)[::-1].copy()
    mine = shard_sources(order, world, rank)
    part = torch.from_numpy(tc.bc(arcs, mine, nthreads=2))
    all_reduce_bc(part)
    slowest = max_over_ranks(10.0 + rank)
    np.save(os.path.join(out_dir, f"bc{rank}.npy"), part.numpy())
    np.save(os.path.join(out_dir, f"t{rank}.npy"), np.array([slowest, mine.shape[0]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_sum_to_the_full_bc(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    import sys

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    from gpu_betweennesscentrality_b200 import synth

    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    full = O.TreeCount(n, u, v, w).bc(O.Arcs(n, u, v, w))
    for r in range(world):
        bc = np.load(tmp_path / f"bc{r}.npy")
        assert rel_err(bc, full) <= 1e-9
        t = np.load(tmp_path / f"t{r}.npy")
        assert t[0] == 11.0
    sizes = [int(np.load(tmp_path / f"t{r}.npy")[1]) for r in range(world)]
    assert sum(sizes) == n and abs(sizes[0] - sizes[1]) <= 1


def test_shard_sources_partition():
    from gpu_betweennesscentrality_b200.shard import shard_sources

    order = np.arange(1001, dtype=np.int32)
    parts = [shard_sources(order, 4, r) for r in range(4)]
    assert np.array_equal(np.concatenate(parts), order)
    with pytest.raises(ValueError):
        shard_sources(order, 2, 2)


def _rank_leaves(rank, world, port, out_dir):
    """rank 1 joins the group, then leaves without taking part in the reduction; rank 0's
    all-reduce of its partial BC must end with an error within the group's timeout, not hang"""
    import sys
    import time

    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from gpu_betweennesscentrality_b200.shard import all_reduce_bc

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=15))
    if rank == 1:
        os._exit(0)
    t0 = time.time()
    try:
        all_reduce_bc(torch.ones(64, dtype=torch.float64))
        outcome = "completed"
    except Exception as e:  # the peer is gone: gloo reports a closed connection or a timeout
        outcome = "error: " + type(e).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write(f"{outcome}\n{time.time() - t0:.2f}\n")
    os._exit(0)


def test_a_rank_that_leaves_ends_the_reduction_with_an_error(tmp_path):
    world = 2
    mp.start_processes(_rank_leaves, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    outcome, seconds = open(tmp_path / "rank0.txt").read().split("\n")[:2]
    assert outcome.startswith("error"), outcome
    assert float(seconds) < 30.0
