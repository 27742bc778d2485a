"""The multi-GPU paths of bench.py on CPU, as two gloo ranks on 127.0.0.1.

Default (weak scaling, no data-path collective): each rank has its own
system (seeded by rank), timed separately; the job's time is the slowest
rank's and the whole-job throughput counts both ranks' targets.

--shard (strong scaling): the ranks share one system, each keeps its target
shard and zeros elsewhere, and one all-reduce combines the potentials."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    import time
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = dict(bench.CONFIGS[1], n_override=2000 + 500 * rank)
        x, y, z, q, off = bench.make_inputs(cfg, seed=rank)
        from oracle import oracle as O
        dist.barrier()
        t0 = time.perf_counter()
        O.treecode(x, y, z, None, x, y, z, q, None, 1, [0.0], 1, 1, 1, 0.7, 4, 200, 200, 1.0, -1.0, 0)
        ms = (time.perf_counter() - t0) * 1e3
        (job_ms,) = bench.max_over_ranks([ms], world, torch.device("cpu"))
        gathered = [None] * world
        dist.all_gather_object(gathered, (ms, float(x[0]), len(x)))
        if rank == 0:
            out.put((job_ms, gathered, bench.job_throughput(len(x), world, job_ms)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_ranks_weak_scaling_max_over_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
    assert all(p.exitcode == 0 for p in procs)
    job_ms, gathered, value = out.get(timeout=10)
    assert job_ms == max(g[0] for g in gathered)          # the slowest rank's time
    assert gathered[0][1] != gathered[1][1]               # each rank has its own system
    assert gathered[0][2] == 2000 and gathered[1][2] == 2500
    assert np.isclose(value, 2 * 2000 / (job_ms * 1e-3))


def _shard_rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = dict(bench.CONFIGS[1], n_override=3000)
        x, y, z, q, off = bench.make_inputs(cfg, seed=0)      # one system shared by the ranks
        from oracle import oracle as O
        full = O.treecode(x, y, z, None, x, y, z, q, None, 1, [0.0], 1, 1, 1, 0.7, 4, 200, 200, 1.0, -1.0, 0)
        # this rank's shard: a contiguous run of targets, the rest 0 (as the
        # library leaves the targets of other shards)
        lo, hi = rank * len(x) // world, (rank + 1) * len(x) // world
        part = np.zeros_like(full)
        part[lo:hi] = full[lo:hi]
        nonzero = int(np.count_nonzero(part))
        t = bench.combine_shards(torch.from_numpy(part.copy()), world)
        if rank == 0:
            out.put((np.array_equal(t.numpy(), full), nonzero))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_ranks_target_shards_combine_to_the_whole_system():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
    assert all(p.exitcode == 0 for p in procs)
    equal, nonzero = out.get(timeout=10)
    assert equal and nonzero == 1500
