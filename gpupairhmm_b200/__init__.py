"""pairhmm_b200: PairHMM forward engine for NVIDIA B200 (sm_100a).

Python mirror of the C ABI in ``include/pairhmm_b200.h`` (ctypes).  The
operator surface follows the reference (asbschmidt/gpuPairHMM):

* ``Batch`` -- the structure-of-arrays batch of records
  (``BatchOfSequenceGroups``, common.cuh:109-201);
* ``Engine.compute(batch)`` -- per-pair float log10 likelihoods in the
  reference's output order (``processBatch_overlapped_float_coalesced_smem``,
  gpuworker.cuh:559-973);
* ``parse_records`` / ``format_scores`` -- the record file format
  (file_parser_worker.cu:50-218, output_writer_worker.cu:84-135), implemented
  in the C++ library;
* ``Engine.submit / poll / drain`` -- the continuous-batching request loop.

There is no CPU fallback: if ``libpairhmm_b200.so`` is missing, importing
this package raises.  Build it with ``make -C gpupairhmm_b200 -j``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpairhmm_b200.so"
CLI_PATH = HERE / "pairhmm_b200"

MODE_ENGINE = 0
MODE_PLAIN = 1

STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "region exceeds the device budget",
    5: "unknown ticket", 6: "timed out", 7: "unsupported", 8: "busy",
    9: "haplotype length above the no-alloc limit of 16384",
}


class PairHMMError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}" if message else STATUS.get(status, str(status)))


class _Batch(ctypes.Structure):
    _fields_ = [
        ("num_records", ctypes.c_int64),
        ("reads_per_record", ctypes.c_void_p),
        ("haps_per_record", ctypes.c_void_p),
        ("read_bases", ctypes.c_void_p),
        ("base_quals", ctypes.c_void_p),
        ("ins_quals", ctypes.c_void_p),
        ("del_quals", ctypes.c_void_p),
        ("gcp_quals", ctypes.c_void_p),
        ("read_offsets", ctypes.c_void_p),
        ("read_lengths", ctypes.c_void_p),
        ("hap_bases", ctypes.c_void_p),
        ("hap_offsets", ctypes.c_void_p),
        ("hap_lengths", ctypes.c_void_p),
    ]


class _Options(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("fp64_rescue", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("device_budget_bytes", ctypes.c_int64),
        ("pipeline_chunks", ctypes.c_int32),
        ("gcp", ctypes.c_int32),
    ]


class _Stats(ctypes.Structure):
    _fields_ = [
        ("pairs", ctypes.c_int64),
        ("cells", ctypes.c_int64),
        ("rescued", ctypes.c_int64),
        ("multi_tile_pairs", ctypes.c_int64),
        ("device_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("prep_ms", ctypes.c_double),
        ("fp32_ms", ctypes.c_double),
        ("fp64_ms", ctypes.c_double),
        ("launches", ctypes.c_int64),
        ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
        ("rescued_ext", ctypes.c_int64),
        ("fp32_launches", ctypes.c_int64),
    ]


class _ServingStats(ctypes.Structure):
    _fields_ = [
        ("regions", ctypes.c_int64),
        ("batches", ctypes.c_int64),
        ("max_batch_regions", ctypes.c_int64),
        ("max_batch_bytes", ctypes.c_int64),
        ("budget_per_slot", ctypes.c_int64),
        ("slots", ctypes.c_int32),
        ("max_in_flight", ctypes.c_int32),
    ]


# every symbol the header declares, with its ctypes signature
_P = ctypes.c_void_p
_SIGNATURES = {
    "pairhmm_default_options": (None, [_P]),
    "pairhmm_engine_create": (ctypes.c_int, [_P, _P]),
    "pairhmm_engine_destroy": (ctypes.c_int, [_P]),
    "pairhmm_compute_host": (ctypes.c_int, [_P, _P, _P]),
    "pairhmm_compute_device": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P]),
    "pairhmm_get_stats": (ctypes.c_int, [_P, _P]),
    "pairhmm_submit": (ctypes.c_int, [_P, _P, _P]),
    "pairhmm_submit_many": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P]),
    "pairhmm_poll": (ctypes.c_int, [_P, ctypes.c_uint64, _P]),
    "pairhmm_drain": (ctypes.c_int, [_P, ctypes.c_uint64, _P, ctypes.c_int64, ctypes.c_int32]),
    "pairhmm_region_latency_ms": (ctypes.c_int, [_P, ctypes.c_uint64, _P]),
    "pairhmm_serving_stats": (ctypes.c_int, [_P, _P]),
    "pairhmm_set_tile_table": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int32]),
    "pairhmm_get_tile_table": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int32, _P]),
    "pairhmm_probe_fp32_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _P]),
    "pairhmm_probe_fp64_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _P]),
    "pairhmm_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "pairhmm_last_error": (ctypes.c_char_p, [_P]),
    "pairhmm_batch_counts": (ctypes.c_int, [_P, _P, _P]),
    "pairhmm_version": (ctypes.c_char_p, []),
    "pairhmm_records_parse": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64, _P]),
    "pairhmm_records_view": (ctypes.c_int, [_P, _P, _P]),
    "pairhmm_records_format": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
    "pairhmm_records_free": (None, [_P]),
    "pairhmm_reader_open": (ctypes.c_int, [ctypes.c_char_p, _P]),
    "pairhmm_reader_next": (ctypes.c_int, [_P, ctypes.c_int64, _P]),
    "pairhmm_reader_close": (None, [_P]),
    "pairhmm_records_last_error": (ctypes.c_char_p, []),
    "pairhmm_set_host_threads": (None, [ctypes.c_int32]),
    "pairhmm_host_register": (ctypes.c_int, [_P, ctypes.c_size_t]),
    "pairhmm_host_unregister": (ctypes.c_int, [_P]),
    "pairhmm_forward_pairs_noalloc": (ctypes.c_int, [ctypes.c_int32] + [_P] * 6 + [ctypes.c_int64, ctypes.c_int32,
                                                                                  _P, _P]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the library once; raises when it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE} -j`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int, engine=None) -> None:
    if status != 0:
        msg = ""
        if engine is not None:
            msg = (lib().pairhmm_last_error(engine) or b"").decode(errors="replace")
        raise PairHMMError(status, msg)


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    # torch tensors (host or device)
    return a.data_ptr()


class RegionSet:
    """Regions prepared once for repeated serving submissions: arrays made
    contiguous and their C descriptors built ahead (``Engine.submit_many``
    then only copies descriptors)."""

    def __init__(self, regions):
        self.regions = [r.contiguous() for r in regions]
        self.structs = [r.as_struct() for r in self.regions]
        self.num_pairs = [r.num_pairs for r in self.regions]

    def __len__(self) -> int:
        return len(self.regions)

    def __getitem__(self, i: int) -> "Batch":
        return self.regions[i]


@dataclass
class Batch:
    """Records in the reference's SoA layout (host numpy arrays, or torch tensors
    on the device for ``Engine.compute_device``)."""
    reads_per_record: np.ndarray
    haps_per_record: np.ndarray
    read_bases: np.ndarray
    base_quals: np.ndarray
    ins_quals: np.ndarray
    del_quals: np.ndarray
    read_offsets: np.ndarray
    read_lengths: np.ndarray
    hap_bases: np.ndarray
    hap_offsets: np.ndarray
    hap_lengths: np.ndarray
    gcp_quals: np.ndarray | None = None

    @property
    def num_records(self) -> int:
        return int(len(self.reads_per_record))

    @property
    def num_pairs(self) -> int:
        return int((np.asarray(self.reads_per_record, dtype=np.int64) * np.asarray(self.haps_per_record)).sum())

    def cells(self) -> int:
        """Sum over records of (sum of read lengths) x (sum of haplotype lengths),
        the reference's DP cell count (gpuworker.cuh:495-520)."""
        rpr = np.asarray(self.reads_per_record, dtype=np.int64)
        hpr = np.asarray(self.haps_per_record, dtype=np.int64)
        cr = np.r_[0, np.cumsum(np.asarray(self.read_lengths, dtype=np.int64))]
        ch = np.r_[0, np.cumsum(np.asarray(self.hap_lengths, dtype=np.int64))]
        er, eh = np.cumsum(rpr), np.cumsum(hpr)
        rs = cr[er] - cr[er - rpr]
        hs = ch[eh] - ch[eh - hpr]
        return int((rs * hs).sum())

    def contiguous(self) -> "Batch":
        def c(a, dt):
            return None if a is None else np.ascontiguousarray(a, dtype=dt)
        return Batch(c(self.reads_per_record, np.int32), c(self.haps_per_record, np.int32),
                     c(self.read_bases, np.uint8), c(self.base_quals, np.uint8), c(self.ins_quals, np.uint8),
                     c(self.del_quals, np.uint8), c(self.read_offsets, np.int64), c(self.read_lengths, np.int32),
                     c(self.hap_bases, np.uint8), c(self.hap_offsets, np.int64), c(self.hap_lengths, np.int32),
                     c(self.gcp_quals, np.uint8))

    def as_struct(self) -> _Batch:
        s = _Batch()
        s.num_records = self.num_records
        for name, _ in _Batch._fields_[1:]:
            setattr(s, name, _ptr(getattr(self, name)))
        return s

    def select_records(self, first: int, last: int) -> "Batch":
        """Records [first, last) as a batch sharing the byte arrays (absolute offsets)."""
        rpr = np.asarray(self.reads_per_record)
        hpr = np.asarray(self.haps_per_record)
        r0, r1 = int(rpr[:first].sum()), int(rpr[:last].sum())
        h0, h1 = int(hpr[:first].sum()), int(hpr[:last].sum())
        return Batch(rpr[first:last], hpr[first:last], self.read_bases, self.base_quals, self.ins_quals,
                     self.del_quals, self.read_offsets[r0:r1], self.read_lengths[r0:r1], self.hap_bases,
                     self.hap_offsets[h0:h1], self.hap_lengths[h0:h1], self.gcp_quals).contiguous()

    def to_device(self, device="cuda"):
        import torch
        return Batch(*[None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(device)
                       for a in (self.reads_per_record, self.haps_per_record, self.read_bases, self.base_quals,
                                 self.ins_quals, self.del_quals, self.read_offsets, self.read_lengths,
                                 self.hap_bases, self.hap_offsets, self.hap_lengths, self.gcp_quals)])

    def pin(self):
        """Copies of the arrays in page-locked host memory (torch tensors)."""
        import torch
        return Batch(*[None if a is None else torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                       for a in (self.reads_per_record, self.haps_per_record, self.read_bases, self.base_quals,
                                 self.ins_quals, self.del_quals, self.read_offsets, self.read_lengths,
                                 self.hap_bases, self.hap_offsets, self.hap_lengths, self.gcp_quals)])


@dataclass
class Stats:
    pairs: int
    cells: int
    rescued: int
    multi_tile_pairs: int
    device_ms: float
    total_ms: float
    prep_ms: float
    fp32_ms: float
    fp64_ms: float
    launches: int
    h2d_bytes: int
    d2h_bytes: int
    rescued_ext: int = 0
    fp32_launches: int = 0


class Engine:
    """A device engine (resident tables, streams, device buffers)."""

    def __init__(self, device: int = 0, mode: int = MODE_ENGINE, fp64_rescue: bool = True,
                 use_graphs: bool = True, device_budget_bytes: int = 0, pipeline_chunks: int = 0,
                 gcp: bool = False):
        """gcp=True: eps and beta per read from its first gcp quality (the
        reference's CPU recurrence) instead of the GPU path's 0.1 / 0.9."""
        L = lib()
        o = _Options()
        L.pairhmm_default_options(ctypes.byref(o))
        o.device, o.mode, o.fp64_rescue, o.use_graphs = device, mode, int(fp64_rescue), int(use_graphs)
        o.device_budget_bytes = device_budget_bytes
        o.pipeline_chunks = pipeline_chunks
        o.gcp = int(gcp)
        h = ctypes.c_void_p()
        _check(L.pairhmm_engine_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._keep = []

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pairhmm_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def compute(self, batch: Batch, out: np.ndarray | None = None) -> np.ndarray:
        """Host arrays in, float32 log10 likelihood per pair out (blocking)."""
        # numpy arrays are made contiguous; pinned torch tensors are passed as they are
        b = batch.contiguous() if isinstance(batch.read_bases, np.ndarray) else batch
        n = b.num_pairs
        if out is None:
            out = np.empty(max(n, 0), dtype=np.float32)
        s = b.as_struct()
        _check(lib().pairhmm_compute_host(self._h, ctypes.byref(s), _ptr(out) if n else None), self._h)
        return out

    def compute_device(self, batch: Batch, scores, stream=None, max_read_length: int = 0,
                       max_hap_length: int = 0) -> None:
        """Device tensors in, device scores out, ordered on `stream` (torch stream or None)."""
        s = batch.as_struct()
        st = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        _check(lib().pairhmm_compute_device(self._h, ctypes.byref(s), max_read_length, max_hap_length,
                                            _ptr(scores), st), self._h)

    def stats(self) -> Stats:
        st = _Stats()
        _check(lib().pairhmm_get_stats(self._h, ctypes.byref(st)), self._h)
        return Stats(st.pairs, st.cells, st.rescued, st.multi_tile_pairs, st.device_ms, st.total_ms, st.prep_ms,
                     st.fp32_ms, st.fp64_ms, st.launches, st.h2d_bytes, st.d2h_bytes, st.rescued_ext,
                     st.fp32_launches)

    # ------------------------------------------------------------ serving
    def submit(self, region: Batch) -> int:
        r = region.contiguous()
        t = ctypes.c_uint64()
        s = r.as_struct()
        _check(lib().pairhmm_submit(self._h, ctypes.byref(s), ctypes.byref(t)), self._h)
        return int(t.value)

    def submit_many(self, regions, picks=None) -> list[int]:
        """Submit several regions in one call (one lock, one wake-up of the
        serving slots); returns their tickets in order.  ``regions`` is a list
        of batches, or a ``RegionSet`` with ``picks`` the indices to submit
        (a region may be picked more than once).  On an error none is queued."""
        if isinstance(regions, RegionSet):
            idx = range(len(regions)) if picks is None else picks
            structs = regions.structs
            arr = (_Batch * len(idx))(*[structs[i] for i in idx])
        else:
            keep = [r.contiguous() for r in regions]
            arr = (_Batch * len(keep))(*[r.as_struct() for r in keep])
        n = len(arr)
        if n == 0:
            return []
        t = (ctypes.c_uint64 * n)()
        _check(lib().pairhmm_submit_many(self._h, arr, n, t), self._h)
        return list(t)

    def poll(self, ticket: int) -> bool:
        d = ctypes.c_int32()
        _check(lib().pairhmm_poll(self._h, ticket, ctypes.byref(d)), self._h)
        return bool(d.value)

    def latency_ms(self, ticket: int) -> float:
        v = ctypes.c_double()
        _check(lib().pairhmm_region_latency_ms(self._h, ticket, ctypes.byref(v)), self._h)
        return float(v.value)

    def drain(self, ticket: int, num_scores: int, timeout_ms: int = -1) -> np.ndarray:
        out = np.empty(max(num_scores, 1), dtype=np.float32)
        _check(lib().pairhmm_drain(self._h, ticket, _ptr(out), num_scores, timeout_ms), self._h)
        return out[:num_scores]

    def serving_stats(self) -> dict:
        """Admission record of the serving queue (batches, most regions and
        bytes in one batch, slot budget, most batches in flight)."""
        st = _ServingStats()
        _check(lib().pairhmm_serving_stats(self._h, ctypes.byref(st)), self._h)
        return {name: int(getattr(st, name)) for name, _ in _ServingStats._fields_}

    # ------------------------------------------------------------ tuning
    def tile_table(self) -> list[tuple[int, int, int, int]]:
        """(max read length, G, R, kind) with kind 0 = one tile, 1 = multi-tile,
        2 = one tile, two reads per group in packed FP32."""
        n = ctypes.c_int32()
        _check(lib().pairhmm_get_tile_table(self._h, None, None, None, None, 0, ctypes.byref(n)), self._h)
        arrs = [np.zeros(n.value, dtype=np.int32) for _ in range(4)]
        _check(lib().pairhmm_get_tile_table(self._h, *[_ptr(a) for a in arrs], n.value, ctypes.byref(n)), self._h)
        return [(int(a), int(b), int(c), int(d)) for a, b, c, d in zip(*arrs)]

    def set_tile_table(self, rules) -> None:
        arrs = [np.array([int(r[i]) for r in rules], dtype=np.int32) for i in range(4)]
        _check(lib().pairhmm_set_tile_table(self._h, *[_ptr(a) for a in arrs], len(rules)), self._h)


def batch_counts(batch: Batch) -> tuple[int, int]:
    b = batch.contiguous()
    s = b.as_struct()
    p, c = ctypes.c_int64(), ctypes.c_int64()
    _check(lib().pairhmm_batch_counts(ctypes.byref(s), ctypes.byref(p), ctypes.byref(c)))
    return int(p.value), int(c.value)


def probe_fp32_peak(device: int = 0, milliseconds: int = 50) -> float:
    """Measured FP32 FMA throughput in TFLOP/s (2 FLOP per FMA)."""
    v = ctypes.c_double()
    _check(lib().pairhmm_probe_fp32_peak(device, milliseconds, ctypes.byref(v)))
    return float(v.value)


def probe_fp64_peak(device: int = 0, milliseconds: int = 50) -> float:
    """Measured FP64 FMA throughput in TFLOP/s (2 FLOP per FMA)."""
    v = ctypes.c_double()
    _check(lib().pairhmm_probe_fp64_peak(device, milliseconds, ctypes.byref(v)))
    return float(v.value)


PAIR_DTYPE = np.dtype([("read_offset", "<i8"), ("hap_offset", "<i8"), ("read_length", "<i4"),
                       ("hap_length", "<i4")])


def forward_pairs_noalloc(device: int, read_bases, base_quals, ins_quals, del_quals, hap_bases, pairs,
                          num_pairs: int, max_hap_length: int, scores, stream=None) -> None:
    """Allocation-free forward over a flat pair list (all arguments device
    tensors, `pairs` laid out as PAIR_DTYPE).  See pairhmm_forward_pairs_noalloc."""
    st = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    _check(lib().pairhmm_forward_pairs_noalloc(device, _ptr(read_bases), _ptr(base_quals), _ptr(ins_quals),
                                               _ptr(del_quals), _ptr(hap_bases), _ptr(pairs), num_pairs,
                                               max_hap_length, _ptr(scores), st))


def version() -> str:
    return lib().pairhmm_version().decode()


def _check_records(status: int) -> None:
    if status != 0:
        raise PairHMMError(status, (lib().pairhmm_records_last_error() or b"").decode(errors="replace"))


def set_host_threads(threads: int = 0) -> None:
    """Host threads for record parsing and formatting (0: the default, all
    hardware threads or PAIRHMM_HOST_THREADS)."""
    lib().pairhmm_set_host_threads(int(threads))


class Records:
    """Records parsed by the library's parser (file_parser_worker.cu rules)."""

    def __init__(self, text: str | bytes | None = None, *, handle: ctypes.c_void_p | None = None):
        if handle is None:
            data = text.encode() if isinstance(text, str) else bytes(text)
            handle = ctypes.c_void_p()
            _check_records(lib().pairhmm_records_parse(data, len(data), ctypes.byref(handle)))
        self._h = handle
        s = _Batch()
        n = ctypes.c_int64()
        _check(lib().pairhmm_records_view(self._h, ctypes.byref(s), ctypes.byref(n)))
        self.num_pairs = int(n.value)
        self.batch = self._batch_from_struct(s)

    def _batch_from_struct(self, s: _Batch) -> Batch:
        g = s.num_records
        def arr(ptr, n, dt):
            if n == 0 or not ptr:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                         shape=(n,)).copy()
        rpr = arr(s.reads_per_record, g, np.int32)
        hpr = arr(s.haps_per_record, g, np.int32)
        nr, nh = int(rpr.sum()), int(hpr.sum())
        rl = arr(s.read_lengths, nr, np.int32)
        ro = arr(s.read_offsets, nr, np.int64)
        hl = arr(s.hap_lengths, nh, np.int32)
        ho = arr(s.hap_offsets, nh, np.int64)
        rbytes = int(max((ro + rl + (4 - rl % 4)).max(), 0)) if nr else 0
        hbytes = int(max((ho + hl + (4 - hl % 4)).max(), 0)) if nh else 0
        return Batch(rpr, hpr, arr(s.read_bases, rbytes, np.uint8), arr(s.base_quals, rbytes, np.uint8),
                     arr(s.ins_quals, rbytes, np.uint8), arr(s.del_quals, rbytes, np.uint8), ro, rl,
                     arr(s.hap_bases, hbytes, np.uint8), ho, hl, arr(s.gcp_quals, rbytes, np.uint8))

    def format(self, scores: np.ndarray) -> str:
        sc = np.ascontiguousarray(scores, dtype=np.float32)
        need = ctypes.c_int64()
        _check(lib().pairhmm_records_format(self._h, _ptr(sc), None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value + 1)
        _check(lib().pairhmm_records_format(self._h, _ptr(sc), buf, need.value + 1, ctypes.byref(need)))
        return buf.raw[:need.value].decode()

    def close(self):
        if getattr(self, "_h", None):
            lib().pairhmm_records_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parse_records(text: str | bytes) -> Records:
    return Records(text)


class RecordFileReader:
    """A record file read batch by batch (FileParserWorker::run,
    file_parser_worker.cu:226-262): each batch holds whole records with at
    least ``min_pairs`` pairs (<= 0: the rest of the file)."""

    def __init__(self, path: str | os.PathLike):
        h = ctypes.c_void_p()
        _check_records(lib().pairhmm_reader_open(os.fsencode(path), ctypes.byref(h)))
        self._h = h

    def next(self, min_pairs: int = 0) -> Records | None:
        r = ctypes.c_void_p()
        _check_records(lib().pairhmm_reader_next(self._h, int(min_pairs), ctypes.byref(r)))
        return Records(handle=r) if r.value else None

    def batches(self, min_pairs: int = 0):
        while (r := self.next(min_pairs)) is not None:
            yield r

    def close(self):
        if getattr(self, "_h", None):
            lib().pairhmm_reader_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_records_file(path: str | os.PathLike) -> Records:
    return Records(Path(path).read_bytes())
