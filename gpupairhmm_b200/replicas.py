"""Multi-GPU replicas: records are independent, so N GPUs run N independent
engines over contiguous record ranges and no data-path collective is needed
(the reference runs on one GPU only, main.cu:32).  The ranges are balanced by
DP cell count; results are gathered in record order on the host.
"""
from __future__ import annotations

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
