"""Autotuner for the engine's tile table on the local GPU.

For each read-length class (16 positions wide up to 1024, wider beyond) it
times every compiled single-tile configuration (G lanes x R positions, with
G*R >= the class's longest read) on synthetic pairs of that class -- read
length uniform in the class, haplotype length = read length + U{50..400},
base quality U{10..40}, ins/del 40 -- and keeps the fastest.  Classes beyond
the largest single tile are timed with the multi-tile configurations.
Adjacent classes with the same winner merge into one rule.

Outputs:
  gpupairhmm_b200/tuning_sm100a.json   every measurement and the table
  gpupairhmm_b200/csrc/tuned_table.inc the table compiled into the engine

  python -m gpupairhmm_b200.autotune [--pairs-per-class N] [--repeats K] [--only LO-HI]

--only re-times the classes inside [LO, HI] and keeps the earlier measurements
of the others (from tuning_sm100a.json) when it rebuilds the table.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import Batch, Engine
from .synth import ACGT, _Builder

HERE = Path(__file__).resolve().parent

SINGLE = [(G, R) for G in (4, 8, 16, 32) for R in (4, 8, 12, 16, 20, 24, 28, 32)
          if not (G >= 8 and R == 4)]
# tiles with R % 4 == 2 where G*R falls on a class bound that no other tile has
SINGLE += [(8, 14), (8, 18), (8, 22), (16, 10), (16, 14), (16, 18)]
MULTI = [(32, 16), (32, 20), (32, 24), (32, 28), (32, 32), (16, 32)]
PACKED = [(G, R) for G in (4, 8, 16, 32) for R in (8, 12, 16)] + [(16, 10)]  # two reads per group, packed FP32


def classes():
    out, lo = [], 0
    for hi in list(range(16, 1025, 16)) + [1152, 1280, 1536, 1792, 2048, 3072, 4096]:
        out.append((lo + 1, hi))
        lo = hi
    return out


def class_batch(lo: int, hi: int, pairs: int, seed: int) -> Batch:
    rng = np.random.default_rng(seed)
    b = _Builder()
    haps_per = 8
    n_rec = max(1, pairs // (4 * haps_per))
    for _ in range(n_rec):
        H = hi + rng.integers(50, 401, size=haps_per)  # every read fits in every haplotype
        haps = [ACGT[rng.integers(0, 4, size=int(n))] for n in H]
        L = rng.integers(lo, hi + 1, size=4)
        reads = []
        for l in L:
            h = haps[int(rng.integers(0, haps_per))]
            s = int(rng.integers(0, len(h) - l + 1))
            r = h[s:s + l].copy()
            m = rng.random(l) < 0.01
            r[m] = ACGT[rng.integers(0, 4, size=int(m.sum()))]
            reads.append(r)
        n = int(L.sum())
        b.add_concat(L, np.concatenate(reads), rng.integers(10, 41, size=n).astype(np.uint8),
                     np.full(n, 40, np.uint8), np.full(n, 40, np.uint8), H, np.concatenate(haps))
    return b.build()


def time_config(engine: Engine, batch: Batch, G: int, R: int, kind: int, repeats: int) -> float:
    """GCUPS of the FP32 launches for this configuration (kind 0 one tile,
    1 multi-tile, 2 packed) on this batch."""
    engine.set_tile_table([(1 << 30, G, R, 1)] if kind == 1 else [(G * R, G, R, kind), (1 << 30, 32, 32, 1)])
    engine.compute(batch)
    best = 0.0
    for _ in range(repeats):
        engine.compute(batch)
        st = engine.stats()
        best = max(best, st.cells / (st.fp32_ms * 1e-3) / 1e9)
    return best


def tune(pairs_per_class: int = 60000, repeats: int = 3, device: int = 0, only=None):
    eng = Engine(device=device, fp64_rescue=False)
    eng.set_tile_table([(1 << 30, 32, 32, 1)])
    results = []
    for ci, (lo, hi) in enumerate(classes()):
        if only and not (only[0] <= lo and hi <= only[1]):
            continue
        batch = class_batch(lo, hi, pairs_per_class if hi <= 1024 else max(512, pairs_per_class // 8), 1000 + ci)
        cands = [(G, R, 0) for G, R in SINGLE if G * R >= hi] if hi <= 1024 else []
        cands += [(G, R, 2) for G, R in PACKED if G * R >= hi]
        cands += [(G, R, 1) for G, R in MULTI if hi > 1024 or G * R < hi]
        timings = {}
        for G, R, kind in cands:
            timings[f"{G}x{R}{['', 'mt', 'p'][kind]}"] = time_config(eng, batch, G, R, kind, repeats)
        best = max(timings, key=timings.get)
        results.append({"lo": lo, "hi": hi, "best": best, "gcups": timings})
        print(f"[{lo:5d},{hi:5d}] best {best:10s} {timings[best]:8.1f} GCUPS "
              f"({len(timings)} candidates)", flush=True)
    eng.close()
    return results


def to_rules(results):
    rules = []
    for r in results:
        key = r["best"]
        kind = 1 if key.endswith("mt") else (2 if key.endswith("p") else 0)
        G, R = (int(x) for x in key.replace("mt", "").replace("p", "").split("x"))
        if rules and (rules[-1][1], rules[-1][2], rules[-1][3]) == (G, R, kind):
            rules[-1] = (r["hi"], G, R, kind)
        else:
            rules.append((r["hi"], G, R, kind))
    last = rules[-1]
    if last[3] == 1:
        rules[-1] = (1 << 30, last[1], last[2], 1)
    else:
        rules.append((1 << 30, 32, 32, 1))
    return rules


def write_outputs(results, rules):
    meta = {"device": "NVIDIA B200", "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            "rules": [{"max_len": a, "G": b, "R": c, "kind": ["single", "multi_tile", "packed"][d]}
                      for a, b, c, d in rules],
            "classes": results}
    (HERE / "tuning_sm100a.json").write_text(json.dumps(meta, indent=1))
    lines = ["// Generated by gpupairhmm_b200/autotune.py on a B200; see tuning_sm100a.json.",
             "// {max read length, G, R, multi-tile, packed}"]
    for a, b, c, d in rules:
        lines.append(f"{{{a if a < (1 << 30) else '1 << 30'}, {b}, {c}, {'true' if d == 1 else 'false'}, "
                     f"{'true' if d == 2 else 'false'}}},")
    (HERE / "csrc" / "tuned_table.inc").write_text("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs-per-class", type=int, default=60000,
                    help="pairs per length class: enough that a launch is not dominated by its tail")
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--outdir", default=None, help="also copy the outputs here")
    ap.add_argument("--only", default=None, help="LO-HI: re-time only the classes inside, keep the others")
    a = ap.parse_args()
    only = tuple(int(x) for x in a.only.split("-")) if a.only else None
    res = tune(a.pairs_per_class, a.repeats, a.device, only)
    if only:  # merge with the earlier measurements of the other classes
        new = {(r["lo"], r["hi"]): r for r in res}
        old = json.loads((HERE / "tuning_sm100a.json").read_text())["classes"]
        res = [new.get((r["lo"], r["hi"]), r) for r in old]
    rules = to_rules(res)
    write_outputs(res, rules)
    print("rules:", rules)
    if a.outdir:
        out = Path(a.outdir)
        out.mkdir(parents=True, exist_ok=True)
        (out / "tuning_sm100a.json").write_text((HERE / "tuning_sm100a.json").read_text())
        (out / "tuned_table.inc").write_text((HERE / "csrc" / "tuned_table.inc").read_text())


if __name__ == "__main__":
    main()
