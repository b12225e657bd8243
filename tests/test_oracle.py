"""The oracle, pinned: the reference README's known answers and the reference's
own CPU recurrence (align_host, gpuworker.cuh:1022-1098) built from its sources."""
import numpy as np
import pytest

import oracle
from oracle import formats
from conftest import ROOT, assert_log10_close

GOLDEN = ROOT / "tests" / "golden"


def test_readme_known_answers():
    recs = formats.parse_text((GOLDEN / "readme_example.in").read_text())
    got = oracle.batch_log10(formats.to_soa(recs))
    lines = (GOLDEN / "readme_example.expected").read_text().split("\n")
    want = np.array([float(x) for ln in lines[1:] if ln for x in ln.split()])
    # the README prints 6 significant digits of the reference's FP32 result
    assert np.max(np.abs(got - want)) <= 1e-5


def test_probability_table_matches_reference():
    ref = oracle.ref_cpu()
    if ref is None:
        pytest.skip("reference shim not built (no reference sources here)")
    for q in range(128):
        assert oracle.lib().oracle_ph2pr(q) == ref.ref_ph2pr(q)


def _rand_pair(rng, L, H, letters="ACGT"):
    read = bytes(rng.choice(list(letters.encode()), size=L).astype(np.uint8))
    hap = bytes(rng.choice(list(letters.encode()), size=H).astype(np.uint8))
    bq = rng.integers(5, 42, size=L).astype(np.uint8)
    iq = rng.integers(25, 46, size=L).astype(np.uint8)
    dq = rng.integers(25, 46, size=L).astype(np.uint8)
    return read, bq, iq, dq, hap


def test_oracle_matches_reference_align_host():
    """align_host runs in FP32 with a double final sum; compare where it has
    not lost range (it has no rescaling)."""
    ref = oracle.ref_cpu()
    if ref is None:
        pytest.skip("reference shim not built (no reference sources here)")
    rng = np.random.default_rng(1234)
    got, want = [], []
    for i in range(300):
        L = int(rng.integers(1, 200))
        H = int(rng.integers(1, 300))
        letters = "ACGTN" if i % 5 == 0 else "ACGT"
        read, bq, iq, dq, hap = _rand_pair(rng, L, H, letters)
        # related pairs three times in four: the read is a substring of the hap
        if i % 4 and H > L:
            s = int(rng.integers(0, H - L + 1))
            read = hap[s:s + L]
        o = oracle.pair_log10(read, bq, iq, dq, hap)
        r = ref.ref_align_host(np.frombuffer(hap, np.uint8).ctypes.data, H,
                               np.frombuffer(read, np.uint8).ctypes.data, L,
                               bq.ctypes.data, iq.ctypes.data, dq.ctypes.data, 10)
        if r > -60.0:
            got.append(o)
            want.append(r)
    assert len(got) > 150
    assert_log10_close(got, want, what="oracle vs align_host")


def test_oracle_rescaling_is_exact_for_far_underflow():
    """A 250 bp read against an unrelated 600 bp haplotype lies about 244
    decades below 1 (the cheapest explanation runs most of the read through the
    insertion state at 0.1 per base), far beyond FP32 and beyond the range of
    an unscaled double; row rescaling must keep it finite and ordered."""
    rng = np.random.default_rng(7)
    read, bq, iq, dq, hap = _rand_pair(rng, 250, 600)
    bq[:] = 40
    v = oracle.pair_log10(read, bq, iq, dq, hap)
    assert np.isfinite(v) and v < -200
    # a prefix of the same read must be more likely per the model's structure
    v2 = oracle.pair_log10(read[:200], bq[:200], iq[:200], dq[:200], hap)
    assert np.isfinite(v2) and v2 > v


def test_oracle_batch_order_matches_pairwise():
    from gpupairhmm_b200 import synth
    b = synth.config0(seed=3, records=3)
    full = oracle.batch_log10(b)
    k = 0
    ri, hi = 0, 0
    for g in range(b.num_records):
        R, H = int(b.reads_per_record[g]), int(b.haps_per_record[g])
        for r in range(R):
            o, L = int(b.read_offsets[ri + r]), int(b.read_lengths[ri + r])
            for h in range(H):
                ho, hn = int(b.hap_offsets[hi + h]), int(b.hap_lengths[hi + h])
                v = oracle.pair_log10(bytes(b.read_bases[o:o + L]), b.base_quals[o:o + L],
                                      b.ins_quals[o:o + L], b.del_quals[o:o + L],
                                      bytes(b.hap_bases[ho:ho + hn]))
                assert v == full[k]
                k += 1
        ri += R
        hi += H
    assert k == len(full)


def _pair_gcp(read, bq, iq, dq, hap, gcp):
    r = np.frombuffer(bytes(read), np.uint8).copy()
    h = np.frombuffer(bytes(hap), np.uint8).copy()
    return oracle.lib().oracle_pair_log10_gcp(r.ctypes.data, bq.ctypes.data, iq.ctypes.data, dq.ctypes.data,
                                              len(r), h.ctypes.data, len(h), int(gcp))


def test_oracle_gcp_mode_matches_reference_align_host():
    """gcp mode takes eps = p(gcp) and beta = 1 - eps from the read's first gcp
    quality: the reference's CPU recurrence (gpuworker.cuh:1009, 1048-1049)."""
    ref = oracle.ref_cpu()
    if ref is None:
        pytest.skip("reference shim not built (no reference sources here)")
    rng = np.random.default_rng(99)
    got, want = [], []
    for i in range(300):
        L = int(rng.integers(1, 160))
        H = int(rng.integers(1, 260))
        read, bq, iq, dq, hap = _rand_pair(rng, L, H)
        if i % 4 and H > L:
            s = int(rng.integers(0, H - L + 1))
            read = hap[s:s + L]
        gcp = int(rng.integers(1, 45))
        o = _pair_gcp(read, bq, iq, dq, hap, gcp)
        r = ref.ref_align_host(np.frombuffer(hap, np.uint8).ctypes.data, H,
                               np.frombuffer(read, np.uint8).ctypes.data, L,
                               bq.ctypes.data, iq.ctypes.data, dq.ctypes.data, gcp)
        if r > -60.0:
            got.append(o)
            want.append(r)
    assert len(got) > 150
    assert_log10_close(got, want, what="oracle gcp mode vs align_host")


def test_oracle_gcp_mode_batch():
    """Per read, the first position's gcp quality decides; gcp 10 everywhere is
    the GPU path's eps 0.1 and beta 0.9 exactly."""
    from gpupairhmm_b200 import synth
    b = synth.config0(seed=4, records=3)
    default = oracle.batch_log10(b)
    assert np.array_equal(oracle.batch_log10(b, gcp=True), default)  # synthetic gcp is 10
    rng = np.random.default_rng(5)
    gq = rng.integers(1, 41, size=len(b.gcp_quals)).astype(np.uint8)
    b2 = type(b)(**{**b.__dict__, "gcp_quals": gq})
    full = oracle.batch_log10(b2, gcp=True)
    k = 0
    ri, hi = 0, 0
    for g in range(b.num_records):
        R, H = int(b.reads_per_record[g]), int(b.haps_per_record[g])
        for r in range(R):
            o, L = int(b.read_offsets[ri + r]), int(b.read_lengths[ri + r])
            for h in range(H):
                ho, hn = int(b.hap_offsets[hi + h]), int(b.hap_lengths[hi + h])
                v = _pair_gcp(bytes(b.read_bases[o:o + L]), b.base_quals[o:o + L], b.ins_quals[o:o + L],
                              b.del_quals[o:o + L], bytes(b.hap_bases[ho:ho + hn]), int(gq[o]))
                assert v == full[k]
                k += 1
        ri += R
        hi += H
    assert not np.array_equal(full, default)
    ref = oracle.ref_cpu()
    if ref is not None:  # the reference's own batch loop over the same gcp array
        assert_log10_close(full, oracle.ref_batch_log10(b2), what="oracle gcp batch vs reference CPU batch")
