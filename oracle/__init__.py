"""PairHMM oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only to check or time against it.  The
product library never links, loads or calls anything here.

Contents
--------
* ``liboracle.so`` (built from ``pairhmm_oracle.c``): FP64 forward recurrence with
  exact power-of-two row rescaling, restating the reference's algorithm
  (citations in the C file).
* ``formats``: a plain-Python restatement of the reference's record file
  format (parser ``file_parser_worker.cu:50-218``, writer
  ``output_writer_worker.cu:84-135``).
* ``_ref/libref_cpu.so`` (optional, built by ``make ref`` where the reference
  sources exist): the reference's own CPU recurrence ``align_host``
  (``gpuworker.cuh:1022-1098``) behind a C ABI, used to pin the oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None
_REF = None


def build(reference_dir: str | None = None) -> None:
    """Compile the oracle, and the reference shim when a reference checkout is
    given (argument or PAIRHMM_REFERENCE_DIR)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    ref = reference_dir or os.environ.get("PAIRHMM_REFERENCE_DIR", "")
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REFERENCE_DIR={ref}"], check=True)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = ctypes.CDLL(str(path))
        L.oracle_pair_log10.restype = ctypes.c_double
        L.oracle_pair_log10.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.oracle_batch_log10.restype = ctypes.c_int64
        L.oracle_batch_log10.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 11 + [ctypes.c_void_p, ctypes.c_int]
        L.oracle_batch_log10_gcp.restype = ctypes.c_int64
        L.oracle_batch_log10_gcp.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 12 + [ctypes.c_void_p, ctypes.c_int]
        L.oracle_pair_log10_gcp.restype = ctypes.c_double
        L.oracle_pair_log10_gcp.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                                    ctypes.c_int]
        L.oracle_ph2pr.restype = ctypes.c_float
        L.oracle_ph2pr.argtypes = [ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def ref_cpu() -> ctypes.CDLL | None:
    """The reference's align_host behind a C ABI, or None when it was not built."""
    global _REF
    if _REF is None:
        path = HERE / "_ref" / "libref_cpu.so"
        if not path.exists():
            return None
        L = ctypes.CDLL(str(path))
        L.ref_align_host.restype = ctypes.c_double
        L.ref_align_host.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ubyte]
        L.ref_ph2pr.restype = ctypes.c_float
        L.ref_ph2pr.argtypes = [ctypes.c_int]
        L.ref_batch_align_host.restype = ctypes.c_longlong
        L.ref_batch_align_host.argtypes = [ctypes.c_longlong] + [ctypes.c_void_p] * 13 + [ctypes.c_int]
        _REF = L
    return _REF


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def pair_log10(read: bytes, bq, iq, dq, hap: bytes) -> float:
    """One pair; bases as ASCII bytes, qualities as Phred integers."""
    r = np.frombuffer(bytes(read), dtype=np.uint8).copy()
    h = np.frombuffer(bytes(hap), dtype=np.uint8).copy()
    b = np.asarray(bq, dtype=np.uint8).copy()
    i = np.asarray(iq, dtype=np.uint8).copy()
    d = np.asarray(dq, dtype=np.uint8).copy()
    return lib().oracle_pair_log10(_ptr(r), _ptr(b), _ptr(i), _ptr(d), len(r), _ptr(h), len(h))


def batch_log10(batch, nthreads: int = 0, gcp: bool = False) -> np.ndarray:
    """FP64 log10 likelihood per pair for a batch object exposing the SoA arrays
    (``reads_per_record``, ``haps_per_record``, ``read_bases``, ``base_quals``,
    ``ins_quals``, ``del_quals``, ``read_offsets``, ``read_lengths``,
    ``hap_bases``, ``hap_offsets``, ``hap_lengths``).  gcp=True takes eps and
    beta per read from ``gcp_quals`` at its first position (the product's gcp
    mode); otherwise the GPU path's constants."""
    rpr = np.ascontiguousarray(batch.reads_per_record, dtype=np.int32)
    hpr = np.ascontiguousarray(batch.haps_per_record, dtype=np.int32)
    arrs = [np.ascontiguousarray(getattr(batch, n), dtype=np.uint8)
            for n in ("read_bases", "base_quals", "ins_quals", "del_quals")]
    ro = np.ascontiguousarray(batch.read_offsets, dtype=np.int64)
    rl = np.ascontiguousarray(batch.read_lengths, dtype=np.int32)
    hb = np.ascontiguousarray(batch.hap_bases, dtype=np.uint8)
    ho = np.ascontiguousarray(batch.hap_offsets, dtype=np.int64)
    hl = np.ascontiguousarray(batch.hap_lengths, dtype=np.int32)
    npairs = int((rpr.astype(np.int64) * hpr).sum())
    out = np.empty(npairs, dtype=np.float64)
    if npairs == 0:
        return out
    if gcp:
        gq = np.ascontiguousarray(batch.gcp_quals, dtype=np.uint8)
        lib().oracle_batch_log10_gcp(len(rpr), _ptr(rpr), _ptr(hpr), *[_ptr(a) for a in arrs], _ptr(gq),
                                     _ptr(ro), _ptr(rl), _ptr(hb), _ptr(ho), _ptr(hl), _ptr(out), int(nthreads))
        return out
    lib().oracle_batch_log10(len(rpr), _ptr(rpr), _ptr(hpr), *[_ptr(a) for a in arrs],
                             _ptr(ro), _ptr(rl), _ptr(hb), _ptr(ho), _ptr(hl), _ptr(out), int(nthreads))
    return out


def ref_batch_log10(batch, nthreads: int = 0) -> np.ndarray:
    """The reference's own CPU recurrence (align_host, FP32 cells, double final
    sum) over a whole batch with OpenMP; requires oracle/_ref/libref_cpu.so."""
    L = ref_cpu()
    if L is None:
        raise RuntimeError("oracle/_ref/libref_cpu.so is not built")
    rpr = np.ascontiguousarray(batch.reads_per_record, dtype=np.int32)
    hpr = np.ascontiguousarray(batch.haps_per_record, dtype=np.int32)
    arrs = [np.ascontiguousarray(getattr(batch, n), dtype=np.uint8)
            for n in ("read_bases", "base_quals", "ins_quals", "del_quals")]
    gq = getattr(batch, "gcp_quals", None)
    gq = None if gq is None else np.ascontiguousarray(gq, dtype=np.uint8)
    ro = np.ascontiguousarray(batch.read_offsets, dtype=np.int64)
    rl = np.ascontiguousarray(batch.read_lengths, dtype=np.int32)
    hb = np.ascontiguousarray(batch.hap_bases, dtype=np.uint8)
    ho = np.ascontiguousarray(batch.hap_offsets, dtype=np.int64)
    hl = np.ascontiguousarray(batch.hap_lengths, dtype=np.int32)
    n = int((rpr.astype(np.int64) * hpr).sum())
    out = np.empty(n, dtype=np.float32)
    if n:
        L.ref_batch_align_host(len(rpr), _ptr(rpr), _ptr(hpr), *[_ptr(a) for a in arrs],
                               None if gq is None else _ptr(gq), _ptr(ro), _ptr(rl), _ptr(hb), _ptr(ho),
                               _ptr(hl), _ptr(out), int(nthreads))
    return out
