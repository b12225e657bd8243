"""Multi-GPU replicas: records are independent, so N GPUs run N independent
engines over contiguous record ranges and no data-path collective is needed
(the reference runs on one GPU only, main.cu:32).  The ranges are balanced by
DP cell count; results are gathered in record order on the host.

Two drivers over the same shard/gather logic:

* ``run(batch, devices)``: one process, one engine per listed device, the
  shards computed concurrently on host threads (the C calls release the GIL);
* ``run_distributed(batch, device)``: one process per GPU under
  torch.distributed; each rank computes its shard and the scores are
  all-gathered as host objects (the only exchange: the results).

Both take a ``compute(device, batch) -> scores`` callable; the default runs
an engine on the device.
"""
from __future__ import annotations

import threading

import numpy as np

from . import Batch


def record_cells(batch: Batch) -> np.ndarray:
    """Cells per record: (sum of its read lengths) x (sum of its haplotype lengths)."""
    rpr = np.asarray(batch.reads_per_record, dtype=np.int64)
    hpr = np.asarray(batch.haps_per_record, dtype=np.int64)
    cr = np.r_[0, np.cumsum(np.asarray(batch.read_lengths, dtype=np.int64))]
    ch = np.r_[0, np.cumsum(np.asarray(batch.hap_lengths, dtype=np.int64))]
    er, eh = np.cumsum(rpr), np.cumsum(hpr)
    return (cr[er] - cr[er - rpr]) * (ch[eh] - ch[eh - hpr])


def shard_bounds(batch: Batch, world: int) -> list[tuple[int, int]]:
    """Contiguous record ranges [first, last) per rank with near-equal cells."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.cumsum(record_cells(batch))
    total = int(c[-1]) if len(c) else 0
    bounds, start = [], 0
    for r in range(world):
        if r == world - 1:
            end = batch.num_records
        else:
            target = total * (r + 1) / world
            end = int(np.searchsorted(c, target, side="left")) + 1 if total else 0
            end = min(max(end, start), batch.num_records)
        bounds.append((start, end))
        start = end
    return bounds


def pair_offsets(batch: Batch) -> np.ndarray:
    """Output slot of each record's first pair (exclusive prefix of R*H)."""
    p = np.asarray(batch.reads_per_record, dtype=np.int64) * np.asarray(batch.haps_per_record, dtype=np.int64)
    return np.r_[0, np.cumsum(p)]


def shard(batch: Batch, rank: int, world: int) -> tuple[Batch, int, int]:
    """This rank's records and the slice [lo, hi) of the global score array they fill."""
    first, last = shard_bounds(batch, world)[rank]
    po = pair_offsets(batch)
    return batch.select_records(first, last), int(po[first]), int(po[last])


def gather(parts: list[tuple[int, int, np.ndarray]], total: int) -> np.ndarray:
    """Place per-rank scores back at their global slots."""
    out = np.empty(total, dtype=np.float32)
    filled = 0
    for lo, hi, s in parts:
        out[lo:hi] = s
        filled += hi - lo
    if filled != total:
        raise ValueError("shards do not cover the batch")
    return out


def engine_compute(device: int, part: Batch, engines: dict | None = None) -> np.ndarray:
    """Scores of `part` on `device`, through a cached engine when `engines`
    (a dict keyed by device) is given, else a fresh one."""
    from . import Engine
    if engines is not None:
        if device not in engines:
            engines[device] = Engine(device=device)
        return engines[device].compute(part)
    with Engine(device=device) as e:
        return e.compute(part)


def run(batch: Batch, devices=(0,), compute=None) -> np.ndarray:
    """Scores of the whole batch in the reference's output order, the records
    split into len(devices) cell-balanced ranges computed side by side (one
    engine per entry of `devices`; a device may be listed more than once)."""
    devices = list(devices)
    if not devices:
        raise ValueError("no devices")
    world = len(devices)
    if compute is None:
        engines: list[dict] = [{} for _ in devices]
        compute_at = lambda r, part: engine_compute(devices[r], part, engines[r])
    else:
        engines = []
        compute_at = lambda r, part: compute(devices[r], part)
    shards = [shard(batch, r, world) for r in range(world)]
    results: list = [None] * world
    errors: list = [None] * world

    def work(r):
        try:
            results[r] = np.asarray(compute_at(r, shards[r][0]), dtype=np.float32)
        except BaseException as e:  # reported on the calling thread
            errors[r] = e

    threads = [threading.Thread(target=work, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for d in engines:
        for e in d.values():
            e.close()
    for r, e in enumerate(errors):
        if e is not None:
            raise RuntimeError(f"replica {r} (device {devices[r]}) failed: {e}") from e
    for r, (_, lo, hi) in enumerate(shards):
        if len(results[r]) != hi - lo:
            raise ValueError(f"replica {r} returned {len(results[r])} scores for {hi - lo} pairs")
    return gather([(lo, hi, results[r]) for r, (_, lo, hi) in enumerate(shards)], batch.num_pairs)


def run_distributed(batch: Batch, device: int, compute=None, group=None) -> np.ndarray:
    """Process-per-GPU form under an initialised torch.distributed process
    group: this rank computes its shard of `batch` (every rank passes the same
    batch) on `device`; the shards' scores are all-gathered as host objects and
    every rank returns the whole array in output order."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    part, lo, hi = shard(batch, rank, world)
    s = np.asarray((compute or engine_compute)(device, part), dtype=np.float32)
    if len(s) != hi - lo:
        raise ValueError(f"rank {rank} computed {len(s)} scores for {hi - lo} pairs")
    parts: list = [None] * world
    dist.all_gather_object(parts, (lo, hi, s), group=group)
    return gather(parts, batch.num_pairs)
