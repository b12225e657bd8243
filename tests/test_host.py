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
