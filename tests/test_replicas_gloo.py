"""Replicas over several ranks (world_size 2, gloo on CPU) and several
engines in one process: sharding by records, per-rank compute, and the gather
back into the reference's output order, through replicas.run_distributed and
replicas.run.  The per-shard compute here is the oracle (a host-logic test);
on GPUs the same code runs an engine per device (tests/test_gpu_replicas.py)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from gpupairhmm_b200 import replicas, synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import torch
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = synth.config1(seed=21, regions=30)
    seen = []

    def compute(device, part):
        seen.append((device, part.num_records))
        return oracle.batch_log10(part, nthreads=1)

    full = replicas.run_distributed(b, device=rank, compute=compute)
    lo, hi = replicas.shard(b, rank, world)[1:]
    assert seen == [(rank, replicas.shard(b, rank, world)[0].num_records)] and hi > lo
    if rank == 0:
        q.put(full)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_and_gather_reproduce_single_rank_order():
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    b = synth.config1(seed=21, regions=30)
    want = oracle.batch_log10(b).astype(np.float32)
    np.testing.assert_array_equal(full, want)


def test_shard_bounds_cover_and_balance():
    b = synth.config1(seed=4, regions=50)
    for world in (1, 2, 3, 8):
        bounds = replicas.shard_bounds(b, world)
        assert bounds[0][0] == 0 and bounds[-1][1] == b.num_records
        for (a0, a1), (b0, b1) in zip(bounds, bounds[1:]):
            assert a1 == b0 and a0 <= a1
        cells = replicas.record_cells(b)
        per = [cells[s:e].sum() for s, e in bounds]
        assert sum(per) == cells.sum()
        if world <= 3:
            assert max(per) <= cells.sum() / world + cells.max()


def test_in_process_replicas_gather_in_order():
    """replicas.run with three replicas (the oracle as compute): every shard is
    computed once, on its own device slot, and the gather gives the one-pass
    order; a failing replica is reported."""
    import oracle
    b = synth.config1(seed=22, regions=25)
    calls = []

    def compute(device, part):
        calls.append(device)
        return oracle.batch_log10(part, nthreads=1)

    full = replicas.run(b, devices=[3, 1, 2], compute=compute)
    assert sorted(calls) == [1, 2, 3]
    np.testing.assert_array_equal(full, oracle.batch_log10(b).astype(np.float32))

    def broken(device, part):
        if device == 1:
            raise ValueError("device lost")
        return oracle.batch_log10(part, nthreads=1)

    import pytest
    with pytest.raises(RuntimeError, match="replica 1"):
        replicas.run(b, devices=[0, 1], compute=broken)
