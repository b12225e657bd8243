"""Host-side logic that needs no GPU: the C ABI loads and exports every
declared symbol, the record parser/writer (C++) agrees with the plain-Python
restatement of the reference's format, batch accounting, and argument checks."""
import re

import numpy as np
import pytest

import gpupairhmm_b200 as g
from gpupairhmm_b200 import synth
from oracle import formats
from conftest import ROOT

HEADER = ROOT / "include" / "pairhmm_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pairhmm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = g.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python mirror binds each of them
    assert set(names) <= set(g._SIGNATURES), set(names) - set(g._SIGNATURES)


def test_version_and_status_strings():
    assert "sm_100a" in g.version()
    for s in range(9):
        assert g.lib().pairhmm_status_string(s)


def _texts():
    yield (ROOT / "tests" / "golden" / "readme_example.in").read_text()
    yield synth.to_text(synth.config0(seed=5, records=3))
    # lengths that are multiples of 4 get 4 bytes of padding
    yield "1 1\nACGT IIII IIII IIII ++++\nACGTACGT\n"
    # empty read set and empty haplotype set
    yield "0 2\nACGT\nAC\n2 0\nAC II II II ++\nACG III III III +++\n"
    # lowercase / other letters, lines with CR kept as haplotype bytes
    yield "1 2\nacgtN 5555I IIIII IIIII +++++\nACGTN\nAAAA\r\n"


@pytest.mark.parametrize("text", list(_texts()))
def test_parser_matches_python_restatement(text):
    recs = g.parse_records(text)
    want = formats.to_soa(formats.parse_text(text))
    b = recs.batch
    for name in ("reads_per_record", "haps_per_record", "read_offsets", "read_lengths", "hap_offsets",
                 "hap_lengths"):
        np.testing.assert_array_equal(np.asarray(getattr(b, name)), getattr(want, name), err_msg=name)
    n = len(want.read_bases)
    for name in ("read_bases", "base_quals", "ins_quals", "del_quals", "gcp_quals"):
        np.testing.assert_array_equal(np.asarray(getattr(b, name))[:n], getattr(want, name), err_msg=name)
    np.testing.assert_array_equal(np.asarray(b.hap_bases)[:len(want.hap_bases)], want.hap_bases)
    assert recs.num_pairs == int((want.reads_per_record.astype(np.int64) * want.haps_per_record).sum())


@pytest.mark.parametrize("text", list(_texts()))
def test_writer_matches_python_restatement(text):
    recs = g.parse_records(text)
    rng = np.random.default_rng(0)
    scores = (-rng.random(recs.num_pairs) * 50).astype(np.float32)
    assert recs.format(scores) == formats.format_scores(formats.parse_text(text), scores)


def test_parser_rejects_malformed_records():
    for bad in ("2 1\nACGT IIII IIII IIII ++++\n", "x y\n", "1 1\nACGT III\nAC\n"):
        with pytest.raises(g.PairHMMError):
            g.parse_records(bad)


def test_batch_counts_match_reference_formula():
    b = synth.config1(seed=3, regions=40)
    pairs, cells = g.batch_counts(b)
    assert pairs == b.num_pairs
    assert cells == b.cells()
    # reference formula (gpuworker.cuh:495-520), spelled out
    want, ri, hi = 0, 0, 0
    for R, H in zip(b.reads_per_record, b.haps_per_record):
        want += int(b.read_lengths[ri:ri + R].sum()) * int(b.hap_lengths[hi:hi + H].sum())
        ri += R
        hi += H
    assert cells == want


def test_batch_counts_reject_bad_lengths():
    b = synth.config0(seed=1, records=2)
    b.read_lengths[3] = 0
    with pytest.raises(g.PairHMMError):
        g.batch_counts(b)


def test_synthetic_generators_are_deterministic():
    a = synth.config1(seed=9, regions=5)
    b = synth.config1(seed=9, regions=5)
    for name in ("reads_per_record", "read_bases", "base_quals", "hap_bases", "read_lengths", "hap_lengths"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name))


def test_synthetic_shapes():
    b = synth.config2(seed=2, regions=3)
    assert set(np.asarray(b.read_lengths).tolist()) == {250}
    assert set(np.asarray(b.hap_lengths).tolist()) == {600}
    assert b.num_pairs == 3 * 64 * 8
    c = synth.config3(seed=2, regions=2)
    assert np.all((c.read_lengths >= 1000) & (c.read_lengths <= 2000))
    assert np.all((c.hap_lengths >= 2000) & (c.hap_lengths <= 5000))


def test_engine_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(g.PairHMMError) as e:
        g.Engine()
    assert e.value.status in (2, 7)


# --- multi-threaded record parsing and formatting -------------------------

def _c_printf5(values):
    """The C library's printf("%.5f") of each float (what the reference's
    writer calls, output_writer_worker.cu:118)."""
    import ctypes
    libc = ctypes.CDLL(None)
    buf = ctypes.create_string_buffer(64)
    out = []
    for v in values:
        libc.snprintf(buf, 64, b"%.5f", ctypes.c_double(float(v)))
        out.append(buf.value.decode())
    return out


def _fixed5_values():
    rng = np.random.default_rng(7)
    bits = rng.integers(0, 2**32, size=60000, dtype=np.uint64).astype(np.uint32)
    parts = [
        bits.view(np.float32),                                            # every exponent, NaN payloads
        (-rng.random(60000) * 400).astype(np.float32),                    # log10 scores
        (-rng.random(20000) * 1e-3).astype(np.float32),                   # near the last digit
        (np.arange(-4001, 4001, 2) / 64).astype(np.float32),              # exact ties k/64, k odd
        (np.arange(-200, 200) * 1e-5).astype(np.float32),                 # around each 5th digit
        np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 2.0**24, -(2.0**24), 2.0**24 - 1,
                  np.finfo(np.float32).max, -np.finfo(np.float32).max, np.finfo(np.float32).tiny,
                  -np.finfo(np.float32).smallest_subnormal, 5e-6, -5e-6, 1.5e-5, 0.5, -0.5],
                 dtype=np.float32),
    ]
    v = np.concatenate(parts)
    return v


def test_formatter_matches_c_printf():
    values = _fixed5_values()
    n = len(values)
    text = f"1 {n}\nACGT IIII IIII IIII ++++\n" + "A\n" * n
    recs = g.parse_records(text)
    out = recs.format(values)
    header, line = out.split("\n")[:2]
    assert header == f"1 {n}"
    got = line.split(" ")
    want = _c_printf5(values)
    bad = [(float(values[i]), got[i], want[i]) for i in range(n) if got[i] != want[i]]
    assert not bad, bad[:10]


def _batch_arrays(b):
    names = ("reads_per_record", "haps_per_record", "read_offsets", "read_lengths", "hap_offsets",
             "hap_lengths", "read_bases", "base_quals", "ins_quals", "del_quals", "gcp_quals", "hap_bases")
    return {k: np.asarray(getattr(b, k)) for k in names}


def test_parser_result_does_not_depend_on_threads():
    text = synth.to_text(synth.config1(seed=9, regions=300))  # a few MB: several threads
    try:
        g.set_host_threads(1)
        one = _batch_arrays(g.parse_records(text).batch)
        g.set_host_threads(7)
        many = g.parse_records(text)
        assert len(text) > 2 << 20
        got = _batch_arrays(many.batch)
        scores = (-np.random.default_rng(1).random(many.num_pairs) * 90).astype(np.float32)
        g.set_host_threads(7)
        f7 = many.format(scores)
        g.set_host_threads(1)
        f1 = many.format(scores)
    finally:
        g.set_host_threads(0)
    for k in one:
        np.testing.assert_array_equal(got[k], one[k], err_msg=k)
    assert f1 == f7


def test_parser_matches_restatement_on_uneven_records():
    text = synth.to_text(synth.config1(seed=4, regions=25))
    want = formats.to_soa(formats.parse_text(text))
    got = g.parse_records(text).batch
    for k in ("reads_per_record", "haps_per_record", "read_offsets", "read_lengths", "hap_offsets", "hap_lengths"):
        np.testing.assert_array_equal(np.asarray(getattr(got, k)), getattr(want, k), err_msg=k)
    for k in ("read_bases", "base_quals", "ins_quals", "del_quals", "gcp_quals"):
        np.testing.assert_array_equal(np.asarray(getattr(got, k))[:len(want.read_bases)], getattr(want, k), err_msg=k)


def _records_text(seed, n):
    """Records with blank separator lines, empty read and haplotype sets and no
    newline after the last line."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        R, H = int(rng.integers(0, 6)), int(rng.integers(0, 5))
        lines = [f"{R} {H}"]
        for _ in range(R):
            L = int(rng.integers(1, 40))
            bases = "".join(rng.choice(list("ACGTN"), L))
            quals = ["".join(chr(33 + int(q)) for q in rng.integers(0, 60, L)) for _ in range(4)]
            lines.append(" ".join([bases] + quals))
        lines += ["".join(rng.choice(list("ACGT"), int(rng.integers(1, 60)))) for _ in range(H)]
        out.append("\n".join(lines) + "\n" + ("\n" if i % 3 == 0 else ""))
    return "".join(out).rstrip("\n")


@pytest.mark.parametrize("min_pairs", [1, 5, 23, 0])
def test_reader_batches_concatenate_to_the_whole_file(tmp_path, min_pairs):
    text = _records_text(3, 200)
    path = tmp_path / "records.txt"
    path.write_text(text)
    whole = g.parse_records(text)
    w = whole.batch
    got_rpr, got_hpr, got_reads, got_haps, pairs = [], [], [], [], []
    with g.RecordFileReader(path) as rd:
        for recs in rd.batches(min_pairs):
            b = recs.batch
            got_rpr.append(np.asarray(b.reads_per_record))
            got_hpr.append(np.asarray(b.haps_per_record))
            for i in range(len(b.read_lengths)):
                o, L = int(b.read_offsets[i]), int(b.read_lengths[i])
                got_reads.append(bytes(b.read_bases[o:o + L]) + bytes(b.base_quals[o:o + L]))
            for j in range(len(b.hap_lengths)):
                o, n = int(b.hap_offsets[j]), int(b.hap_lengths[j])
                got_haps.append(bytes(b.hap_bases[o:o + n]))
            pairs.append(recs.num_pairs)
            rph = np.asarray(b.reads_per_record, np.int64) * np.asarray(b.haps_per_record)
            if min_pairs > 0:  # whole records, the fewest that reach min_pairs (the last batch may hold less)
                assert rph.sum() - rph[-1] < min_pairs
        assert rd.next(min_pairs) is None
    if min_pairs > 0:
        assert all(p >= min_pairs for p in pairs[:-1])
    else:
        assert len(pairs) == 1
    np.testing.assert_array_equal(np.concatenate(got_rpr), np.asarray(w.reads_per_record))
    np.testing.assert_array_equal(np.concatenate(got_hpr), np.asarray(w.haps_per_record))
    want_reads = [bytes(w.read_bases[o:o + L]) + bytes(w.base_quals[o:o + L])
                  for o, L in zip(np.asarray(w.read_offsets).tolist(), np.asarray(w.read_lengths).tolist())]
    want_haps = [bytes(w.hap_bases[o:o + n])
                 for o, n in zip(np.asarray(w.hap_offsets).tolist(), np.asarray(w.hap_lengths).tolist())]
    assert got_reads == want_reads and got_haps == want_haps
    assert sum(pairs) == whole.num_pairs


@pytest.mark.parametrize("text,message", [
    ("2 1\nACGT IIII IIII IIII ++++\n", "file ends inside a record's reads (line 2)"),
    ("1 2\nACGT IIII IIII IIII ++++\nAC\n", "file ends inside a record's haplotypes (line 3)"),
    ("x y\n", "malformed record header (line 1)"),
    ("1 1\nACGT III\nAC\n", "read line shorter than 5 fields of the read length (line 2)"),
    ("1 1\nACGTIIII\nAC\n", "read line without 5 space-separated fields (line 2)"),
    ("1 1\n ACGT IIII IIII IIII ++++\nAC\n", "read line without 5 space-separated fields (line 2)"),
    ("1 1\nACGT IIII IIII IIII ++++\n\nAC\n", "empty haplotype line (line 3)"),
    # two malformed records: the first in the file is named
    ("1 1\nAC II II II ++\nA\n\n2 1\nAC I\nAC II II II ++\nA\nzz\n",
     "read line shorter than 5 fields of the read length (line 6)"),
])
def test_parser_errors_name_the_first_bad_line(text, message):
    with pytest.raises(g.PairHMMError) as e:
        g.parse_records(text)
    assert message in str(e.value)


def test_reader_reports_a_missing_file(tmp_path):
    with pytest.raises(g.PairHMMError) as e:
        g.RecordFileReader(tmp_path / "none.txt")
    assert "could not open" in str(e.value)


def _random_record_text(seed: int, target_bytes: int) -> str:
    """Well-formed records of random shape: R and H from 0, read lengths 1..300,
    any printable quality characters, bases with N, lowercase and other letters."""
    rng = np.random.default_rng(seed)
    letters = np.frombuffer(b"ACGTACGTACGTNacgtRYX", dtype=np.uint8)
    out, size = [], 0
    while size < target_bytes:
        R, H = int(rng.integers(0, 9)), int(rng.integers(0, 6))
        lines = [f"{R} {H}"]
        for _ in range(R):
            L = int(rng.integers(1, 301))
            bases = letters[rng.integers(0, len(letters), L)].tobytes().decode()
            quals = [rng.integers(33, 127, L).astype(np.uint8).tobytes().decode() for _ in range(4)]
            lines.append(" ".join([bases] + quals))
        for _ in range(H):
            lines.append(letters[rng.integers(0, len(letters), int(rng.integers(1, 500)))].tobytes().decode())
        block = "\n".join(lines) + "\n"
        out.append(block)
        size += len(block)
    return "".join(out)


@pytest.mark.parametrize("seed,size", [(1, 20_000), (2, 200_000), (3, 2_600_000)])
def test_parser_random_records_match_restatement(seed, size):
    """The multi-threaded parser against the plain-Python restatement of the
    reference's parser rules, on one thread and on several."""
    text = _random_record_text(seed, size)
    want = formats.to_soa(formats.parse_text(text))
    try:
        for threads in (1, 6):
            g.set_host_threads(threads)
            b = g.parse_records(text).batch
            for k in ("reads_per_record", "haps_per_record", "read_offsets", "read_lengths", "hap_offsets",
                      "hap_lengths"):
                np.testing.assert_array_equal(np.asarray(getattr(b, k)), getattr(want, k), err_msg=f"{k} x{threads}")
            n = len(want.read_bases)
            for k in ("read_bases", "base_quals", "ins_quals", "del_quals", "gcp_quals"):
                np.testing.assert_array_equal(np.asarray(getattr(b, k))[:n], getattr(want, k), err_msg=f"{k} x{threads}")
            np.testing.assert_array_equal(np.asarray(b.hap_bases)[:len(want.hap_bases)], want.hap_bases)
    finally:
        g.set_host_threads(0)
