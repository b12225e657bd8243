"""Writes ph2pr_table.inc: the probability table p(q) = float(10^(-q/10)) for
q = 0..127 as hexadecimal float literals, computed as the reference computes
it (double pow, rounded to float; gpuworker.cuh:473-486).  The allocation-free
entry point (noalloc.cu) compiles it into its constant memory, so the table is
part of the module image and needs no upload.

    python gpupairhmm_b200/csrc/ph2pr_table.py
"""
from pathlib import Path

import numpy as np


def table() -> list[float]:
    return [float(np.float32(10.0 ** (-q / 10.0))) for q in range(128)]


def main() -> None:
    vals = table()
    rows = [", ".join(f"{v.hex()}f" for v in vals[i:i + 4]) for i in range(0, 128, 4)]
    text = ("// p(q) = float(10^(-q/10)), q = 0..127 (gpuworker.cuh:473-486); written by ph2pr_table.py\n"
            + ",\n".join(rows) + "\n")
    Path(__file__).with_name("ph2pr_table.inc").write_text(text)


if __name__ == "__main__":
    main()
