#!/usr/bin/env python
"""GCUPS of the PairHMM forward path on the uneven-length workload.

One step = one batch of synthetic records with the shapes of the uneven-length
configuration (20,000 regions, see gpupairhmm_b200/synth.py) through the
engine's C ABI (pairhmm_compute_host): upload from pinned host memory,
packing and work-list construction, the FP32 wavefront launches, the FP64
pass, and the download of the scores.

  value   cells / device time of the batch (CUDA events on the engine's stream
          around everything after the upload: inputs resident in HBM)
  e2e     cells / wall time of the blocking C-ABI call (host index, H2D, device
          work, D2H), pinned host buffers
  roofline  11 FP32 FLOP per DP cell / time of the FP32 wavefront launches,
          against an FFMA peak measured on the same GPU in the same run

Beside the headline line (single GPU only): the precision-stress and
long-read configurations at their stated sizes (`stress`, `long`: device
GCUPS, stage split, FP64 fractions, error against the FP64 oracle on a
sample), the plain per-launch FP32 form on the same batch (`plain`,
`vs_plain`), the reference's own gpuPairHMM binary built for sm_100a on the
same batch as record text (`reference_gpu`, `vs_reference_gpu`, both by the
binary's batch clock: upload, kernels, download), and the streaming service
(`serving`: 60 s at 2,000 regions/s, then a sweep of higher rates).

Multi-GPU (torchrun): each rank runs its own replica on its own batch (weak
scaling, no data-path collective); times are the max over ranks.

--impl reference: the reference's own CPU forward (align_host, built from its
sources into oracle/_ref/ with OpenMP over pairs) on all host cores, over a
bounded sample of the same workload per step; falls back to the FP64 oracle
port when the reference build is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GCUPS (PairHMM cells/s) at ≤1e-5 rel log10 err; p50/p99 region latency"
FLOPS_PER_CELL = 11  # M: 5, I: 3, D: 3 (FMA = 2 FLOP)
WORKLOAD = ("uneven lengths: 20,000 regions, R ~ lognormal(median 40, sigma 1.0) clipped 1-400, "
            "H ~ U{1..16}, read length {100,150,250} (.3/.5/.2) minus U{0..30}, "
            "haplotype = read + U{50..400}, base quality U{10..40}, ins/del 40, gcp 10")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu", "cli"], default="ours",
                    help="reference-gpu / cli: the reference's gpuPairHMM binary (oracle/_ref, built from its "
                         "sources) or our CLI on the same record file, GCUPS as the binary prints it")
    ap.add_argument("--mode", choices=["engine", "plain"], default="engine")
    ap.add_argument("--regions", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample size (seconds of work)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--accuracy-pairs", type=int, default=3000)
    ap.add_argument("--serving-seconds", type=float, default=60.0,
                    help="length of the streaming-service run at --serving-rate (0 = skip)")
    ap.add_argument("--serving-rate", type=float, default=2000.0, help="region arrivals per second")
    ap.add_argument("--sweep-rates", default="8000,20000,40000,60000",
                    help="further arrival rates of the serving sweep (comma separated, '' = none); "
                         "stops at the first rate whose p99 exceeds 1 s")
    ap.add_argument("--sweep-seconds", type=float, default=10.0)
    ap.add_argument("--no-extra-configs", action="store_true",
                    help="skip the precision-stress / long-read blocks, the plain form and the reference binary")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for ln in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) >= 10:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        pw = [float(r[4]) for r in rows if r[4].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_median": statistics.median(pw) if pw else None, "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------- helpers
def traffic_per_cell():
    """DRAM bytes per DP cell of the FP32 wavefront from the committed ncu
    summary (profiles/fp32_wavefront_traffic.json), or None."""
    p = ROOT / "profiles" / "fp32_wavefront_traffic.json"
    if not p.exists():
        return None
    try:
        return float(json.loads(p.read_text())["dram_bytes_per_cell"])
    except Exception:
        return None


def sample_records(batch, target_cells: int, rng: np.random.Generator):
    """Contiguous records from a random start with about target_cells cells."""
    from gpupairhmm_b200 import replicas
    c = replicas.record_cells(batch)
    start = int(rng.integers(0, max(1, batch.num_records - 1)))
    cs = np.cumsum(c[start:])
    end = start + int(np.searchsorted(cs, target_cells)) + 1
    end = min(end, batch.num_records)
    return batch.select_records(start, end), end - start


def cpu_rate(fn, batch, target_seconds: float, rng):
    """Time fn over a sample sized for about target_seconds; returns (GCUPS, sample text)."""
    probe, _ = sample_records(batch, int(2e8), rng)
    t = time.perf_counter()
    fn(probe)
    rate = probe.cells() / max(time.perf_counter() - t, 1e-6)
    sub, nrec = sample_records(batch, int(rate * target_seconds), rng)
    t = time.perf_counter()
    fn(sub)
    dt = time.perf_counter() - t
    return sub.cells() / dt / 1e9, f"{nrec} consecutive records, {sub.num_pairs} pairs, {sub.cells()} cells, {dt:.1f} s"


def accuracy(batch, scores, n, rng):
    import oracle
    pick = np.sort(rng.choice(batch.num_records, size=min(batch.num_records, max(1, n // 40)), replace=False))
    from gpupairhmm_b200 import replicas, synth
    po = replicas.pair_offsets(batch)
    parts = [batch.select_records(int(g), int(g) + 1) for g in pick]
    sub = synth.concat(parts)
    want = oracle.batch_log10(sub)
    got = np.concatenate([scores[po[g]:po[g + 1]] for g in pick]).astype(np.float64)
    err = np.abs(got - want)
    rel = err / np.maximum(np.abs(want), 1e-30)
    return {"sample_pairs": int(len(want)), "max_abs_log10": float(err.max()), "mean_abs_log10": float(err.mean()),
            "max_rel_log10": float(rel.max()), "within_1e-5_rel": bool(np.all(err <= 1e-5 * np.abs(want) + 1e-6))}


# ----------------------------------------------------------------- arms
def run_reference(args, cfg):
    """The reference's own CPU implementation, all host threads."""
    import oracle
    from gpupairhmm_b200 import synth
    batch = synth.config1(seed=args.seed, regions=args.regions)
    rng = np.random.default_rng(1234)
    ref_ok = oracle.ref_cpu() is not None
    fn = (lambda b: oracle.ref_batch_log10(b)) if ref_ok else (lambda b: oracle.batch_log10(b))
    kind = "reference" if ref_ok else "port"
    cores = os.cpu_count() or 1
    per_step = max(2.0, min(12.0, 120.0 / max(1, args.steps + args.warmup)))
    # size one step's sample from a probe, then run warmup + steps
    probe, _ = sample_records(batch, int(2e8), rng)
    t = time.perf_counter()
    fn(probe)
    rate = probe.cells() / max(time.perf_counter() - t, 1e-6)
    sub, nrec = sample_records(batch, int(rate * per_step), rng)
    for _ in range(args.warmup):
        fn(sub)
    t = time.perf_counter()
    for _ in range(args.steps):
        fn(sub)
    dt = time.perf_counter() - t
    value = sub.cells() * args.steps / dt / 1e9
    sample = (f"{nrec} consecutive records of the workload per step ({sub.num_pairs} pairs, {sub.cells()} cells); "
              f"{'reference align_host (gpuworker.cuh:1022-1098), FP32 cells, OpenMP over pairs' if ref_ok else 'FP64 oracle port'}")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_binary(args, cfg):
    """A gpuPairHMM-style binary on a record file of the workload (file parse,
    upload, compute, download; output to /dev/null as the reference skips
    formatting for it).  GCUPS as printed by the binary.  Three more runs write
    the scores to a regular file and are timed whole (`file_to_file`, median)."""
    import re
    from gpupairhmm_b200 import synth, CLI_PATH
    binary = ROOT / "oracle" / "_ref" / "gpuPairHMM" if args.impl == "reference-gpu" else CLI_PATH
    if not binary.exists():
        print(json.dumps({"impl": args.impl, "unavailable": f"{binary} not built"}))
        return
    batch = synth.config1(seed=args.seed, regions=args.regions)
    fd, path = tempfile.mkstemp(prefix="records_", suffix=".txt")
    os.close(fd)
    try:
        Path(path).write_text(synth.to_text(batch))
        in_bytes = os.path.getsize(path)
        vals = []
        for i in range(args.warmup + args.steps):
            out = subprocess.run([str(binary), "--inputfile", path, "--outputfile", "/dev/null",
                                  "--fileBatchsize", "0", "--transferBatchsize", "0"],
                                 capture_output=True, text=True, check=True).stdout
            m = re.search(r"Batch processing time: ([0-9.e+-]+)s \(([0-9.e+-]+) GCUPS\)", out)
            if i >= args.warmup:
                vals.append((float(m.group(1)), float(m.group(2))))
        # the whole command three times more with a regular output file: process
        # start, parse, compute and the "%.5f" text, by the wall clock around it
        # (median; our CLI also reports its host stage times with --verbose)
        fd2, opath = tempfile.mkstemp(prefix="scores_", suffix=".txt")
        os.close(fd2)
        f2f_runs, stages = [], None
        try:
            for _ in range(3):
                cmd = [str(binary), "--inputfile", path, "--outputfile", opath]
                if args.impl == "cli":
                    cmd.append("--verbose")
                t0 = time.perf_counter()
                out2 = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
                f2f_runs.append(time.perf_counter() - t0)
                m2 = re.search(r"Host stages: engine start-up ([0-9.e+-]+)s, parse ([0-9.e+-]+)s, "
                               r"format\+write ([0-9.e+-]+)s", out2)
                if m2:
                    stages = {"engine_start_s": float(m2.group(1)), "parse_s": float(m2.group(2)),
                              "format_write_s": float(m2.group(3))}
            f2f = statistics.median(f2f_runs)
            out_bytes = os.path.getsize(opath)
        finally:
            os.unlink(opath)
    finally:
        os.unlink(path)
    # median step: a single batch per process is exposed to one-off host stalls
    secs = statistics.median(v[0] for v in vals) * len(vals)
    value = batch.cells() * len(vals) / secs / 1e9
    print(json.dumps({"impl": args.impl, "metric": METRIC, "value": round(value, 3), "unit": "GCUPS",
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": round(secs / len(vals) * 1e3, 3), "higher_is_better": True,
                      "data": "synthetic", "config": dict(cfg, pairs=batch.num_pairs, cells=batch.cells()),
                      "timing": "the binary's own batch wall clock (upload, kernels, download; file "
                                "parsing excluded), whole batch at once; median over the steps",
                      "step_seconds": [round(v[0], 4) for v in vals],
                      "file_to_file": {"wall_s": round(f2f, 3), "gcups": round(batch.cells() / f2f / 1e9, 3),
                                       "runs_s": [round(x, 3) for x in f2f_runs], "last_run_stages": stages,
                                       "input_bytes": in_bytes,
                                       "output_bytes": out_bytes,
                                       "command": "--inputfile records --outputfile scores (default batch sizes); "
                                                  "median of 3"}}),
          flush=True)


def host_io(batch, regions=4000, reps=3):
    """Record-format throughput of the library on this host: parse (text ->
    SoA batch) and format (scores -> "%.5f" text) through the C ABI, on all host
    threads, best of `reps`, on the first `regions` records of the workload."""
    import ctypes
    import gpupairhmm_b200 as g
    from gpupairhmm_b200 import synth
    sub = batch.select_records(0, min(regions, batch.num_records))
    text = synth.to_text(sub).encode()
    L = g.lib()
    best_p = best_f = float("inf")
    h = ctypes.c_void_p()
    for _ in range(reps):
        if h.value:
            L.pairhmm_records_free(h)
        t0 = time.perf_counter()
        g._check_records(L.pairhmm_records_parse(text, len(text), ctypes.byref(h)))
        best_p = min(best_p, time.perf_counter() - t0)
    npairs = ctypes.c_int64()
    view = g._Batch()
    L.pairhmm_records_view(h, ctypes.byref(view), ctypes.byref(npairs))
    scores = (-np.random.default_rng(5).random(npairs.value) * 300).astype(np.float32)
    need = ctypes.c_int64()
    L.pairhmm_records_format(h, g._ptr(scores), None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(need.value + 1)
    for _ in range(reps):
        t0 = time.perf_counter()
        L.pairhmm_records_format(h, g._ptr(scores), buf, need.value + 1, ctypes.byref(need))
        best_f = min(best_f, time.perf_counter() - t0)
    L.pairhmm_records_free(h)
    return {"parse_gb_per_s": round(len(text) / best_p / 1e9, 3),
            "format_mscores_per_s": round(npairs.value / best_f / 1e6, 2),
            "threads": os.cpu_count() or 1,
            "sample": f"first {sub.num_records} records of the workload as record text: {len(text) / 1e6:.0f} MB, "
                      f"{npairs.value} pairs, {need.value / 1e6:.0f} MB of output; best of {reps}"}


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def _serve_stream(eng, pool, times, picks, cells_of, heavy=None):
    """Submit pool regions at the given arrival times, then collect.  Every
    pass of the loop submits all regions that have arrived by then in one
    ``submit_many`` call (busy wait while none is due).  Latency of a region =
    (call start - arrival) + the engine's submit-to-done time (which counts
    from the start of the call), so a submit loop that falls behind shows up
    in it.  Python's cyclic garbage collector is paused meanwhile (a
    collection would stall the submissions, not the service)."""
    import gc
    gc.collect()
    gc.disable()
    try:
        return _serve_stream_timed(eng, pool, times, picks, cells_of, heavy)
    finally:
        gc.enable()


def _serve_stream_timed(eng, pool, times, picks, cells_of, heavy):
    times = np.asarray(times, dtype=np.float64)
    n = len(times)
    t0 = time.perf_counter()
    tickets, sub, late = [], np.zeros(n), np.zeros(n)
    k = 0
    calls = 0
    while k < n:
        now = time.perf_counter() - t0
        if now < times[k]:
            continue
        j = int(np.searchsorted(times, now, side="right"))
        tickets += eng.submit_many(pool, picks[k:j])
        sub[k:j] = now
        late[k:j] = now - times[k:j]
        calls += 1
        k = j
    lat, done = [], []
    for i, tk in enumerate(tickets):
        while not eng.poll(tk):
            time.sleep(0.0002)
        ms = eng.latency_ms(tk)
        eng.drain(tk, pool.num_pairs[picks[i]])
        lat.append(late[i] * 1e3 + ms)
        done.append(sub[i] + ms / 1e3)
    span = max(done) if done else 1e-9
    cells = sum(cells_of[i] for i in picks)
    out = {"regions": n, "submit_calls": calls, "p50_ms": round(percentile(lat, 50), 3),
           "p99_ms": round(percentile(lat, 99), 3), "max_ms": round(max(lat), 3) if lat else 0.0,
           "gcups": round(cells / span / 1e9, 3), "span_s": round(span, 3),
           "offered_gcups": round(cells / max(float(times[-1]), 1e-9) / 1e9, 3) if n else 0.0}
    if heavy is not None and n:
        kind = np.asarray([heavy[i] for i in picks])
        lat = np.asarray(lat)
        for name, sel in (("single_tile", ~kind), ("multi_tile", kind)):
            if sel.any():
                out[name] = {"regions": int(sel.sum()), "p50_ms": round(percentile(lat[sel], 50), 3),
                             "p99_ms": round(percentile(lat[sel], 99), 3)}
    return out


def run_serving(args, local_rank):
    """Streaming service: regions arrive as a Poisson stream (the uneven-length
    region shapes, 5% long-read shapes) and are submitted to the engine's
    continuous-batching queue as they arrive.  Region shapes are drawn from a
    pool of 24,000 regions generated ahead of time (the generator is far slower
    than the arrival rates).  First the configured rate for the configured
    length, then a sweep of higher rates until p99 exceeds 1 s.  Beside it, the
    first 10 s of the configured stream through one blocking plain-FP32 call
    per region in arrival order (latency from arrival)."""
    import gpupairhmm_b200 as g
    from gpupairhmm_b200 import synth
    pool = g.RegionSet(synth.region_pool(seed=4, regions=24000, long_frac=0.05))
    cells_of = [r.cells() for r in pool.regions]
    times, picks = synth.poisson_arrivals(5, args.serving_rate, args.serving_seconds, len(pool))
    out = {"rate_per_s": args.serving_rate, "seconds": args.serving_seconds, "long_region_fraction": 0.05,
           "pool": "24,000 regions drawn ahead of time (seed 4), picked uniformly per arrival",
           "latency": "arrival to scores on the host (submission delay + submit-to-done)"}

    eng = g.Engine(device=local_rank)
    # regions with a read beyond the longest single tile run on the multi-tile slots
    single_max = max(m for m, _, _, kind in eng.tile_table() if kind != 1)
    heavy = [int(np.max(r.read_lengths)) > single_max for r in pool.regions]
    warm = eng.submit_many(pool, range(300))  # warm the queue's engines (a burst of both kinds)
    for i, tk in enumerate(warm):
        eng.drain(tk, pool.num_pairs[i])
    out["continuous_batching"] = _serve_stream(eng, pool, times, picks, cells_of, heavy)
    sweep = []
    for k, rate in enumerate(float(x) for x in args.sweep_rates.split(",") if x.strip()):
        tt, pp = synth.poisson_arrivals(6 + k, rate, args.sweep_seconds, len(pool))
        point = dict(rate_per_s=rate, seconds=args.sweep_seconds,
                     **_serve_stream(eng, pool, tt, pp, cells_of, heavy))
        sweep.append(point)
        if point["p99_ms"] > 1000.0:
            break
    out["sweep"] = sweep
    out["admission"] = eng.serving_stats()
    eng.close()

    # one region per blocking call, plain FP32 form, first 10 s of the stream
    pe = g.Engine(device=local_rank, mode=g.MODE_PLAIN)
    for r in pool.regions[:200]:
        pe.compute(r)
    n10 = int(np.searchsorted(times, min(10.0, args.serving_seconds), side="right"))
    lat = []
    t0 = time.perf_counter()
    for t_arr, i in zip(times[:n10], picks[:n10]):
        while time.perf_counter() - t0 < t_arr:
            pass
        pe.compute(pool[i])
        lat.append((time.perf_counter() - t0 - t_arr) * 1e3)
    span = time.perf_counter() - t0
    pe.close()
    cells10 = sum(cells_of[i] for i in picks[:n10])
    out["plain_per_region"] = {"regions": n10, "seconds_of_stream": min(10.0, args.serving_seconds),
                               "p50_ms": round(percentile(lat, 50), 3), "p99_ms": round(percentile(lat, 99), 3),
                               "max_ms": round(max(lat), 3), "gcups": round(cells10 / span / 1e9, 3),
                               "span_s": round(span, 3)}
    return out


def region_accuracy(batch, scores, regions, seed):
    """|log10 difference| against the FP64 oracle on every pair of `regions`
    randomly chosen records."""
    import oracle
    from gpupairhmm_b200 import replicas, synth
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(batch.num_records, size=min(batch.num_records, regions), replace=False))
    po = replicas.pair_offsets(batch)
    sub = synth.concat([batch.select_records(int(r), int(r) + 1) for r in pick])
    want = oracle.batch_log10(sub)
    got = np.concatenate([scores[po[r]:po[r + 1]] for r in pick]).astype(np.float64)
    err = np.abs(got - want)
    rel = err / np.maximum(np.abs(want), 1e-30)
    return {"sample_regions": int(len(pick)), "sample_pairs": int(len(want)), "sample_cells": int(sub.cells()),
            "max_abs_log10": float(err.max()), "mean_abs_log10": float(err.mean()),
            "max_rel_log10": float(rel.max()), "min_log10": float(want.min()),
            "within_1e-5_rel": bool(np.all(err <= 1e-5 * np.abs(want) + 1e-6))}


def run_config(name, batch, desc, steps, warmup, local_rank, acc_regions):
    """One configuration at its stated size through a one-pass engine (inputs
    page-locked; device time after the upload), its FP32-only result from the
    plain form (how many pairs the FP32 recurrence alone loses), and the error
    against the FP64 oracle on a sample of regions."""
    import torch
    import gpupairhmm_b200 as g
    pinned = batch.pin()
    scores = torch.empty(batch.num_pairs, dtype=torch.float32).pin_memory().numpy()
    eng = g.Engine(device=local_rank, pipeline_chunks=1)
    for _ in range(warmup):
        eng.compute(pinned, out=scores)
    dev = fp32 = fp64 = prep = 0.0
    for _ in range(steps):
        eng.compute(pinned, out=scores)
        st = eng.stats()
        dev += st.device_ms
        fp32 += st.fp32_ms
        fp64 += st.fp64_ms
        prep += st.prep_ms
    eng.close()
    cells = batch.cells()
    out = {"workload": desc, "pairs": batch.num_pairs, "cells": cells, "steps": steps,
           "gcups": round(cells * steps / (dev / 1e3) / 1e9, 3), "ms_per_step": round(dev / steps, 3),
           "stage_ms_per_step": {"prep": round(prep / steps, 3), "fp32": round(fp32 / steps, 3),
                                 "fp64": round(fp64 / steps, 3)},
           "fp64_fraction": round(st.rescued / batch.num_pairs, 5),
           "fp64_extended_fraction": round(st.rescued_ext / batch.num_pairs, 6),
           "fp64_pairs": int(st.rescued), "fp64_extended_pairs": int(st.rescued_ext)}
    pe = g.Engine(device=local_rank, mode=g.MODE_PLAIN, pipeline_chunks=1)
    fp32_only = pe.compute(pinned)
    pe.close()
    out["fp32_only_nonfinite_fraction"] = round(float(np.mean(~np.isfinite(fp32_only))), 5)
    out["accuracy"] = region_accuracy(batch, scores, acc_regions, seed=17)
    return out


def run_plain(batch_pinned, cells, steps, warmup, local_rank):
    """The plain per-launch FP32 form on the same batch: the reference's tile
    table and launch shape (one launch per length partition), FP32 only, device
    time with inputs resident."""
    import gpupairhmm_b200 as g
    pe = g.Engine(device=local_rank, mode=g.MODE_PLAIN, pipeline_chunks=1)
    for _ in range(warmup):
        pe.compute(batch_pinned)
    dev = 0.0
    for _ in range(steps):
        pe.compute(batch_pinned)
        dev += pe.stats().device_ms
    pe.close()
    return {"gcups": round(cells * steps / (dev / 1e3) / 1e9, 3), "ms_per_step": round(dev / steps, 3),
            "steps": steps, "form": "reference tile table (tuningconfigs.hpp:33-57), one non-persistent launch "
                                    "per partition, this engine's FP32 cell, no FP64 pass"}


def run_reference_binary(batch, steps):
    """The reference's gpuPairHMM, built from its sources for sm_100a into
    oracle/_ref, on the same batch as a record file; GCUPS by its own batch
    clock (upload, kernels, download), median over the runs."""
    import re
    from gpupairhmm_b200 import synth
    binary = ROOT / "oracle" / "_ref" / "gpuPairHMM"
    if not binary.exists():
        return {"unavailable": "oracle/_ref/gpuPairHMM not built"}
    fd, path = tempfile.mkstemp(prefix="records_", suffix=".txt")
    os.close(fd)
    try:
        Path(path).write_text(synth.to_text(batch))
        runs = []
        for _ in range(steps + 1):
            out = subprocess.run([str(binary), "--inputfile", path, "--outputfile", "/dev/null",
                                  "--fileBatchsize", "0", "--transferBatchsize", "0"],
                                 capture_output=True, text=True, timeout=600).stdout
            m = re.search(r"Batch processing time: ([0-9.e+-]+)s \(([0-9.e+-]+) GCUPS\)", out)
            if not m:
                return {"unavailable": "no batch time in the binary's output"}
            runs.append(float(m.group(1)))
    finally:
        os.unlink(path)
    sec = statistics.median(runs[1:])
    return {"gcups": round(batch.cells() / sec / 1e9, 3), "batch_seconds": [round(x, 4) for x in runs[1:]],
            "timing": "the binary's printed batch time (upload, kernels, download; file parse excluded), "
                      "median of the runs after one warm-up, no profiler attached",
            "build": "oracle/Makefile from the reference's sources, sm_100a, generic tuning table"}


def run_ours(args, cfg, rank, world, local_rank):
    import torch
    import gpupairhmm_b200 as g
    from gpupairhmm_b200 import synth

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))

    batch = synth.config1(seed=args.seed + rank, regions=args.regions)
    cells = batch.cells()
    pinned = batch.pin()
    mode = g.MODE_PLAIN if args.mode == "plain" else g.MODE_ENGINE
    # value: device time of one pass over the batch with its inputs in HBM (events
    # after the upload); e2e: the default host API call, which runs a batch this
    # large as chunks whose uploads overlap the previous chunk's kernels
    engine_dev = g.Engine(device=local_rank, mode=mode, pipeline_chunks=1)
    engine = g.Engine(device=local_rank, mode=mode)
    peak = g.probe_fp32_peak(local_rank, 100)
    scores = torch.empty(batch.num_pairs, dtype=torch.float32).pin_memory().numpy()  # page-locked output
    for _ in range(args.warmup):
        engine_dev.compute(pinned, out=scores)
        engine.compute(pinned, out=scores)

    props = torch.cuda.get_device_properties(local_rank)
    uuid = str(getattr(props, "uuid", "") or "")
    uuid = ("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or None)
    sampler = ClockSampler(uuid)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.25)
    dev_ms = fp32_ms = prep_ms = fp64_ms = 0.0
    launches = fp32_launches = h2d = d2h = rescued = rescued_ext = 0
    for _ in range(args.steps):
        engine_dev.compute(pinned, out=scores)
        st = engine_dev.stats()
        dev_ms += st.device_ms
        fp32_ms += st.fp32_ms
        prep_ms += st.prep_ms
        fp64_ms += st.fp64_ms
        launches += st.launches
        fp32_launches += st.fp32_launches
        rescued = st.rescued
        rescued_ext = st.rescued_ext
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        engine.compute(pinned, out=scores)
        st = engine.stats()
        h2d += st.h2d_bytes
        d2h += st.d2h_bytes
        launches += st.launches  # the end-to-end calls' kernels are in the timed region too
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    wall = t1 - t0
    times = np.array([wall, dev_ms / 1e3, fp32_ms / 1e3], dtype=np.float64)
    if dist:
        tt = torch.tensor(times, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        times = tt.cpu().numpy()
    wall, dev_s, fp32_s = (float(x) for x in times)
    total_cells = cells * args.steps * world

    if rank == 0:
        value = total_cells / dev_s / 1e9
        e2e = total_cells / wall / 1e9
        achieved = FLOPS_PER_CELL * cells * args.steps / fp32_s / 1e12
        tpc = traffic_per_cell()
        n_fp32_launches = max(1, fp32_launches // max(1, args.steps))
        rng = np.random.default_rng(99)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dev_s / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": dict(cfg, pairs=batch.num_pairs, cells=cells, rescued_fp64=rescued,
                           rescued_fp64_extended=rescued_ext, parallelism=f"replicas{world}"),
            "e2e": {"value": round(e2e, 3), "unit": "GCUPS", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps, "ms_per_step": round(wall / args.steps * 1e3, 3)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak, 3),
                         "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                         "traffic": (round(tpc * cells / n_fp32_launches) if tpc else None),
                         "peak_source": "FFMA throughput measured in this run on this GPU (MEASURED_PEAKS.json "
                                        "has no FP32 entry)",
                         "flop_per_cell": FLOPS_PER_CELL,
                         # 11 algorithmic FLOP per cell in 5 FMA-pipe instructions (4 FFMA + 1 FMUL)
                         "instruction_mix_ceiling": round(FLOPS_PER_CELL / 10, 4),
                         "kernel": "fp32_bucket_kernel (all length buckets)",
                         "stage_ms_per_step": {"prep": round(prep_ms / args.steps, 3),
                                               "fp32": round(fp32_ms / args.steps, 3),
                                               "fp64": round(fp64_ms / args.steps, 3)}},
            "clocks": clocks,
        }
        engine.close()
        engine_dev.close()
        extras = world == 1 and not args.no_extra_configs
        if extras:
            # the 1.5x target's denominator and the reference's own kernels, same batch
            line["plain"] = run_plain(pinned, cells, 3, 2, local_rank)
            line["vs_plain"] = round(value / line["plain"]["gcups"], 4)
            ref = run_reference_binary(batch, 3)
            line["reference_gpu"] = ref
            line["vs_reference_gpu"] = round(e2e / ref["gcups"], 4) if "gcups" in ref else None
        # the streaming-service run goes before anything that runs the OpenMP oracle
        # in this process (accuracy samples, CPU baseline): after it, the serving
        # threads saw periodic host stalls of several hundred ms
        if world == 1 and args.serving_seconds > 0:
            line["serving"] = run_serving(args, local_rank)
        if extras:
            line["stress"] = run_config(
                "stress", synth.config2(seed=2, regions=5000),
                "precision stress: 5,000 regions x R=64 x H=8, reads 250 bp, haplotypes 600 bp, half of the "
                "reads unrelated, base quality U{35..41}, ins/del 40, gcp 10", 3, 2, local_rank, 40)
            line["long"] = run_config(
                "long", synth.config3(seed=3, regions=2000),
                "long reads: 2,000 regions x R=16 x H=4, reads U{1000..2000}, haplotypes U{2000..5000} with "
                "1-50 bp indels, base quality U{5..40}, ins/del U{30..45} per position, gcp 10", 3, 2,
                local_rank, 16)
        if world == 1:
            line["host_io"] = host_io(batch)
        line["accuracy"] = accuracy(batch, scores, args.accuracy_pairs, rng)
        if world == 1 and not args.no_cpu_baseline:
            import oracle
            gc, desc = cpu_rate(lambda b: oracle.batch_log10(b), batch, args.cpu_seconds, rng)
            line["cpu_baseline"] = {"value": round(gc, 4), "unit": "GCUPS", "cores": os.cpu_count() or 1,
                                    "kind": "port", "sample": desc + "; FP64 oracle, OpenMP over pairs"}
        print(json.dumps(line), flush=True)
    else:
        engine.close()
        engine_dev.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = {"workload": WORKLOAD, "regions": args.regions, "seed": args.seed, "sigma": 1.0, "mode": args.mode,
           "l2": "inputs larger than L2 (packed batch ~1 GB vs 126 MB)"}
    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args, cfg)
        return
    if args.impl in ("reference-gpu", "cli"):
        if rank == 0:
            run_binary(args, cfg)
        return
    run_ours(args, cfg, rank, world, local_rank)


if __name__ == "__main__":
    main()
