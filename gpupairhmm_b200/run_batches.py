"""Throughput harness: run batches of one synthetic workload through the
engine and print, per batch, its pairs, cells, FP64 pairs and device stage
times (packing, FP32 wavefront, FP64 pass) and the call's wall time.  It is
this package's counterpart of the reference's kernel benchmark
(benchmark_peakperformance.cu:229-277), on the benchmark configurations'
shapes instead of uniform lengths, and the command the ncu summaries in
profiles/ name.

  python -m gpupairhmm_b200.run_batches --config uneven --regions 4000 --batches 2

Configurations (gpupairhmm_b200/synth.py): small (64 records, 32 reads x 4
haplotypes, 100/150 bp), uneven (uneven lengths), stress (FP32 + FP64 rescue,
half unrelated reads), long (long reads, multi-tile).
"""
from __future__ import annotations

import argparse

from . import MODE_ENGINE, MODE_PLAIN, Engine
from . import synth

CONFIGS = {
    "small": lambda n, seed: synth.config0(seed=seed, records=n or 64),
    "uneven": lambda n, seed, sigma=1.0: synth.config1(seed=seed, regions=n or 20000, sigma=sigma),
    "stress": lambda n, seed: synth.config2(seed=seed, regions=n or 5000),
    "long": lambda n, seed: synth.config3(seed=seed, regions=n or 2000),
}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=sorted(CONFIGS), default="uneven")
    ap.add_argument("--regions", type=int, default=0, help="records/regions (0 = the configuration's size)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--batches", type=int, default=2)
    ap.add_argument("--mode", choices=["engine", "plain"], default="engine")
    ap.add_argument("--pageable", action="store_true", help="pass pageable numpy arrays (default: page-locked)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--sigma", type=float, default=1.0,
                    help="uneven configuration: sigma of the lognormal reads-per-region count")
    ap.add_argument("--chunks", type=int, default=1,
                    help="pipeline_chunks of the engine (1 = one pass, whose stage times add up; 0 = auto)")
    a = ap.parse_args()
    batch = CONFIGS[a.config](a.regions, a.seed, a.sigma) if a.config == "uneven" else CONFIGS[a.config](a.regions, a.seed)
    inputs = batch if a.pageable else batch.pin()
    with Engine(device=a.device, mode=MODE_PLAIN if a.mode == "plain" else MODE_ENGINE,
                pipeline_chunks=a.chunks) as e:
        for i in range(a.batches):
            e.compute(inputs)
            s = e.stats()
            print(f"batch {i}: pairs {s.pairs} cells {s.cells} rescued {s.rescued} (extended {s.rescued_ext}) "
                  f"device {s.device_ms:.2f} ms "
                  f"(prep {s.prep_ms:.2f}, fp32 {s.fp32_ms:.2f}, fp64 {s.fp64_ms:.2f}) call {s.total_ms:.2f} ms",
                  flush=True)


if __name__ == "__main__":
    main()
