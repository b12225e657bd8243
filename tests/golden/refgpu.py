"""Loader for the reference-GPU golden fixtures: regenerates each input from
its seed, checks it against the recorded SHA-256 (so the committed outputs
belong to exactly these inputs), and parses the reference's output file."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CASES = ["cfg0", "cfg1_small", "cfg2_small", "cfg3_small", "edges"]
_inputs = None


def inputs() -> dict[str, str]:
    global _inputs
    if _inputs is None:
        import make_golden  # noqa: E402  (same directory)
        _inputs = make_golden.ref_gpu_inputs()
    return _inputs


def load(name: str):
    """(input text, reference scores as float64 with -inf kept)."""
    text = inputs()[name]
    want_hash = json.loads((HERE / "ref_gpu_inputs.sha256.json").read_text())[name]
    if hashlib.sha256(text.encode()).hexdigest() != want_hash:
        raise AssertionError(f"regenerated input {name} differs from the one the reference ran on")
    lines = (HERE / f"ref_gpu_{name}.out").read_text().split("\n")
    vals, i = [], 0
    while i < len(lines) and lines[i]:
        R, H = (int(x) for x in lines[i].split())
        i += 1
        for _ in range(R):
            if H:
                vals += [float(v) for v in lines[i].split(" ")]
            i += 1
    return text, np.array(vals, dtype=np.float64)
