"""Regenerate the golden fixtures in this directory.

readme_example.in / readme_example.expected
    The only known-answer vector the reference ships: the example record and
    its printed scores in the reference's README (README.md:45-61).  Read from
    the reference checkout, not typed in.

ref_gpu_<name>.in / ref_gpu_<name>.out
    Inputs generated here (seeded, gpupairhmm_b200.synth + edge cases) and the
    output of the reference's own GPU binary (oracle/_ref/gpuPairHMM, built
    from the reference sources by oracle/Makefile) on a B200.  Generating the
    outputs needs a GPU:  python tests/golden/make_golden.py --ref-gpu
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def readme_example(reference_dir: Path) -> None:
    text = (reference_dir / "README.md").read_text()
    blocks = re.findall(r"```\n(.*?)```", text, re.S)
    inp = [b for b in blocks if re.match(r"\d+ \d+\n[ACGTN]", b)]
    out = [b for b in blocks if re.match(r"\d+ \d+\n-?\d", b)]
    if len(inp) != 1 or len(out) != 1:
        raise SystemExit("README example blocks not found")
    (HERE / "readme_example.in").write_text(inp[0])
    (HERE / "readme_example.expected").write_text(out[0])


def edge_case_text(seed: int = 11) -> str:
    """Small records at the lengths where the reference's tiles change, plus
    N bases, lowercase bases and a single-position read."""
    import numpy as np
    rng = np.random.default_rng(seed)
    lines = []
    lens = [1, 2, 3, 4, 5, 15, 16, 17, 31, 32, 33, 47, 48, 49, 63, 64, 65, 100, 112, 113, 127, 128, 129,
            159, 160, 161, 255, 256, 257, 511, 512, 513, 1023, 1024, 1025, 1200]
    for L in lens:
        H = int(rng.integers(1, 4))
        lines.append(f"2 {H}")
        for _ in range(2):
            bases = "".join(rng.choice(list("ACGT"), size=L))
            if L > 8:
                pos = rng.integers(0, L, size=2)
                b = list(bases)
                b[pos[0]] = "N"
                b[pos[1]] = "a"
                bases = "".join(b)
            bq = "".join(chr(33 + int(q)) for q in rng.integers(10, 41, size=L))
            iq = "".join(chr(33 + int(q)) for q in rng.integers(30, 46, size=L))
            dq = "".join(chr(33 + int(q)) for q in rng.integers(30, 46, size=L))
            gq = "+" * L
            lines.append(" ".join([bases, bq, iq, dq, gq]))
        for _ in range(H):
            n = int(rng.integers(max(1, L // 2), 2 * L + 40))
            lines.append("".join(rng.choice(list("ACGTN"), size=n, p=[0.24, 0.24, 0.24, 0.24, 0.04])))
    return "\n".join(lines) + "\n"


def ref_gpu_inputs() -> dict[str, str]:
    from gpupairhmm_b200 import synth
    cases = {
        "cfg0": synth.to_text(synth.config0(seed=0)),
        "cfg1_small": synth.to_text(synth.config1(seed=5, regions=60)),
        "cfg2_small": synth.to_text(synth.config2(seed=6, regions=12)),
        "cfg3_small": synth.to_text(synth.config3(seed=7, regions=3)),
        "edges": edge_case_text(),
    }
    return cases


def ref_gpu(binary: Path, outdir: Path) -> None:
    outdir.mkdir(parents=True, exist_ok=True)
    for name, text in ref_gpu_inputs().items():
        inp = outdir / f"ref_gpu_{name}.in"
        out = outdir / f"ref_gpu_{name}.out"
        inp.write_text(text)
        subprocess.run([str(binary), "--inputfile", str(inp), "--outputfile", str(out)], check=True,
                       stdout=subprocess.DEVNULL)
        print("wrote", out)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-dir", default=os.environ.get("PAIRHMM_REFERENCE_DIR", ""),
                    help="reference checkout (default: PAIRHMM_REFERENCE_DIR)")
    ap.add_argument("--ref-gpu", action="store_true", help="run the reference GPU binary (needs a GPU)")
    ap.add_argument("--binary", default=str(ROOT / "oracle" / "_ref" / "gpuPairHMM"))
    ap.add_argument("--outdir", default=str(HERE))
    a = ap.parse_args()
    if a.reference_dir and Path(a.reference_dir).is_dir():
        readme_example(Path(a.reference_dir))
    if a.ref_gpu:
        ref_gpu(Path(a.binary), Path(a.outdir))


if __name__ == "__main__":
    main()
