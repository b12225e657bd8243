"""The precision-stress and long-read configurations at a sizeable fraction of
their stated sizes, through the C ABI, against the FP64 oracle.

Tolerance: |gpu - oracle| <= 1e-5 * |oracle| + 1e-6 on log10 (conftest.RTOL/ATOL).

The FP64 pass has two tiers: scaled doubles (a fixed power-of-two scale, good
down to about 10^-599 * L*H) take every pair the FP32 pass flags; the pairs
below that go on to the per-lane-exponent tier.  The stats report both counts."""
import numpy as np
import pytest

import gpupairhmm_b200 as g
import oracle
from gpupairhmm_b200 import synth
from conftest import assert_log10_close

pytestmark = pytest.mark.gpu


def test_precision_stress_200_regions(engine):
    """200 regions x 64 reads x 8 haplotypes (102,400 pairs of 250 x 600):
    half of the reads unrelated, so about half of the pairs underflow FP32 and
    are recomputed in FP64; none is beyond the scaled tier's range."""
    b = synth.config2(seed=202, regions=200)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    st = engine.stats()
    assert st.pairs == b.num_pairs == 102400
    under = int((want < -67.0).sum())
    assert under > 0.4 * len(want)
    assert st.rescued >= under
    assert st.rescued_ext == 0
    assert np.isfinite(got).all()
    assert_log10_close(got, want, what="precision stress, 200 regions")


def test_long_reads_20_regions(engine):
    """20 regions x 16 reads x 4 haplotypes, reads 1,000-2,000 and haplotypes
    2,000-5,000 with 1-50 bp indels (multi-tile FP32 and FP64 kernels): most
    pairs underflow FP32, a few lie beyond 10^-600 and take the extended tier."""
    b = synth.config3(seed=303, regions=20)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    st = engine.stats()
    # reads above the largest single tile (1,024 positions) run multi-tile
    L = np.repeat(np.asarray(b.read_lengths), np.repeat(np.asarray(b.haps_per_record), b.reads_per_record))
    assert st.multi_tile_pairs == int((L > 1024).sum()) > 0
    deep = int((want < -640.0).sum())
    assert deep > 0
    assert st.rescued_ext >= deep
    assert st.rescued_ext <= int((want < -540.0).sum())
    assert np.isfinite(got).all()
    assert_log10_close(got, want, what="long reads, 20 regions")


def test_fp64_tiers_split_by_range(engine):
    """Unrelated reads on short haplotypes cost about a decade per base: pairs
    above about 10^-560 finish in the scaled tier, pairs below 10^-640 in the
    extended tier, and both agree with the oracle."""
    from test_gpu_parity import _record, _soa
    rng = np.random.default_rng(41)
    recs = [_record(rng, L, H, n_reads=2, n_haps=2, related=False)
            for L, H in [(150, 3), (400, 2), (520, 9), (560, 4), (700, 5), (900, 2), (1500, 30), (2100, 7)]]
    b = _soa(recs)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    st = engine.stats()
    assert (want > -560).sum() > 0 and (want < -640).sum() > 0
    assert int((want < -640).sum()) <= st.rescued_ext <= int((want < -540).sum())
    assert_log10_close(got, want, what="tiers")


def test_fused_and_separate_fp64_tiers_agree_bitwise(engine):
    """Up to 2,048 multi-tile pairs in a batch, the FP64 scaled tier runs a
    pair's extended form right after it in the same warp; above that the
    extended tier is a launch of its own.  A batch of 40 long-read regions
    (2,560 multi-tile pairs: separate launches) gives every region's scores
    bitwise as that region computed alone (64 pairs: fused)."""
    from gpupairhmm_b200 import replicas
    b = synth.config3(seed=505, regions=40)
    got = engine.compute(b)
    separate_ext = engine.stats().rescued_ext
    assert separate_ext > 0
    po = replicas.pair_offsets(b)
    fused_ext = 0
    for r in range(b.num_records):
        alone = engine.compute(b.select_records(r, r + 1))
        fused_ext += engine.stats().rescued_ext
        np.testing.assert_array_equal(alone, got[po[r]:po[r + 1]])
    assert fused_ext == separate_ext  # the same pairs take the extended form either way


def test_serving_matches_batch_on_long_and_stress_regions(engine):
    """Regions of both heavy configurations through the serving queue give the
    batch call's scores bitwise."""
    regions = [synth.config3(seed=404, regions=1), synth.config2(seed=405, regions=1),
               synth.config3(seed=406, regions=1)]
    want = [engine.compute(r) for r in regions]
    e = g.Engine()
    tickets = [e.submit(r) for r in regions]
    for tk, r, w in zip(tickets, regions, want):
        np.testing.assert_array_equal(e.drain(tk, r.num_pairs, timeout_ms=120000), w)
    e.close()


def test_uneven_workload_full_size_properties():
    """The uneven-length workload at its full size (20,000 regions, 10.9 M pairs):
    every score finite and at most 0 (a probability), the chunked host pipeline
    bitwise equal to one pass and to a repeated pass, and a random sample of
    2,000 pairs within the tolerance of the oracle."""
    from gpupairhmm_b200 import replicas
    b = synth.config1(seed=1, regions=20000)
    pinned = b.pin()
    one = g.Engine(pipeline_chunks=1)
    a = one.compute(pinned)
    st = one.stats()
    a2 = one.compute(pinned)
    one.close()
    chunked = g.Engine()  # 4 chunks at this size
    c = chunked.compute(pinned)
    chunked.close()
    assert st.pairs == b.num_pairs == len(a) and st.rescued_ext == 0
    assert np.isfinite(a).all() and (a <= 0.0).all()
    np.testing.assert_array_equal(a, a2)
    np.testing.assert_array_equal(a, c)
    # a random sample of whole records through the oracle
    rng = np.random.default_rng(5)
    po = replicas.pair_offsets(b)
    picks, n = [], 0
    while n < 2000:
        r = int(rng.integers(0, b.num_records))
        picks.append(r)
        n += int(po[r + 1] - po[r])
    sub = synth.concat([b.select_records(r, r + 1) for r in picks])
    got = np.concatenate([a[po[r]:po[r + 1]] for r in picks])
    assert_log10_close(got, oracle.batch_log10(sub), what="uneven workload sample")
