"""CUDA path vs the oracle, through the C ABI, on seeded inputs.

Tolerance: |gpu - oracle| <= 1e-5 * |oracle| + 1e-6 on log10 (conftest.RTOL/ATOL)."""
import numpy as np
import pytest

import gpupairhmm_b200 as g
import oracle
from gpupairhmm_b200 import synth
from conftest import ROOT, assert_log10_close

pytestmark = pytest.mark.gpu
GOLDEN = ROOT / "tests" / "golden"


def test_readme_known_answers(engine):
    recs = g.read_records_file(GOLDEN / "readme_example.in")
    got = engine.compute(recs.batch)
    lines = (GOLDEN / "readme_example.expected").read_text().split("\n")
    want = np.array([float(x) for ln in lines[1:] if ln for x in ln.split()])
    assert np.max(np.abs(got - want)) <= 1e-5
    assert_log10_close(got, oracle.batch_log10(recs.batch), what="readme")


@pytest.mark.parametrize("mode", ["engine", "plain"])
def test_config0_matches_oracle(mode, engine, plain_engine):
    e = engine if mode == "engine" else plain_engine
    b = synth.config0(seed=0)
    got = e.compute(b)
    st = e.stats()
    assert st.pairs == b.num_pairs and st.cells == b.cells()
    assert_log10_close(got, oracle.batch_log10(b), what=f"cfg0 {mode}")


def _record(rng, L, H, n_reads=2, n_haps=2, letters="ACGT", bq=(10, 41), idq=(30, 46), related=True):
    reads, haps = [], []
    for _ in range(n_haps):
        haps.append(bytes(rng.choice(list(letters.encode()), size=H).astype(np.uint8)))
    for i in range(n_reads):
        if related and H >= L and i % 2 == 0:
            s = int(rng.integers(0, H - L + 1))
            r = bytearray(haps[0][s:s + L])
        else:
            r = bytearray(rng.choice(list(letters.encode()), size=L).astype(np.uint8))
        q = [rng.integers(*bq, size=L), rng.integers(*idq, size=L), rng.integers(*idq, size=L)]
        reads.append((bytes(r), *[bytes(x.astype(np.uint8)) for x in q], bytes([10] * L)))
    from oracle.formats import Record
    return Record(reads=reads, haps=haps)


def _soa(records):
    from oracle.formats import to_soa
    s = to_soa(records)
    return g.Batch(s.reads_per_record, s.haps_per_record, s.read_bases, s.base_quals, s.ins_quals, s.del_quals,
                   s.read_offsets, s.read_lengths, s.hap_bases, s.hap_offsets, s.hap_lengths, s.gcp_quals)


def test_length_sweep_across_tile_boundaries(engine, plain_engine):
    rng = np.random.default_rng(5)
    lens = list(range(1, 41)) + [47, 48, 49, 63, 64, 65, 79, 80, 81, 95, 96, 97, 111, 112, 113, 127, 128, 129,
                                 159, 160, 161, 191, 192, 193, 223, 224, 225, 255, 256, 257, 319, 320, 321,
                                 383, 384, 385, 447, 448, 449, 511, 512, 513, 639, 640, 641, 767, 768, 769,
                                 895, 896, 897, 1023, 1024, 1025]
    recs = []
    for i, L in enumerate(lens):
        H = int(rng.choice([1, 2, 3, 5, 16, 17, L, L + 7, 2 * L + 3]))
        recs.append(_record(rng, L, max(H, 1), n_reads=2, n_haps=1 + i % 3))
    b = _soa(recs)
    want = oracle.batch_log10(b)
    assert_log10_close(engine.compute(b), want, what="sweep engine")
    # the plain form is FP32 only, like the reference: compare it in FP32 range
    ok = want > -60.0
    assert_log10_close(plain_engine.compute(b)[ok], want[ok], what="sweep plain")


@pytest.mark.parametrize("G,R", [(8, 14), (8, 18), (8, 22), (16, 10), (16, 14), (16, 18)])
def test_even_r_tiles_match_oracle(G, R):
    """Tiles with R % 4 == 2 (lanes start 8-byte aligned, a float2 tail table):
    read lengths at every lane and tile edge of the tile."""
    rng = np.random.default_rng(60 + G + R)
    T = G * R
    lens = sorted({1, 2, 3, R - 2, R - 1, R, R + 1, R + 2, 2 * R - 1, 2 * R, 2 * R + 1, T // 2 - 1, T // 2,
                   T - 3, T - 2, T - 1, T})
    recs = [_record(rng, L, int(rng.integers(max(L, 8), L + 300)), n_reads=2, n_haps=2) for L in lens]
    b = _soa(recs)
    e = g.Engine()
    e.set_tile_table([(T, G, R, 0), (1 << 30, 32, 32, 1)])
    got = e.compute(b)
    e.close()
    assert_log10_close(got, oracle.batch_log10(b), what=f"{G}x{R} tile")


def test_packed_even_r_tile_matches_oracle():
    """The packed kernel with R % 4 == 2 (16 x 10, lanes 8-byte aligned, the last
    two positions of a lane in their own table entry): read lengths at every lane
    and tile edge, records with odd read counts (one-read units)."""
    rng = np.random.default_rng(61)
    lens = sorted({1, 2, 3, 8, 9, 10, 11, 12, 19, 20, 21, 79, 80, 81, 129, 144, 150, 158, 159, 160})
    recs = [_record(rng, L, int(rng.integers(max(L, 8), L + 300)), n_reads=1 + i % 3, n_haps=2)
            for i, L in enumerate(lens)]
    b = _soa(recs)
    e = g.Engine()
    e.set_tile_table([(160, 16, 10, 2), (1 << 30, 32, 32, 1)])
    got = e.compute(b)
    e.close()
    assert_log10_close(got, oracle.batch_log10(b), what="packed 16x10 tile")


def test_haplotype_length_sweep(engine):
    rng = np.random.default_rng(6)
    recs = [_record(rng, 100, H, n_reads=3, n_haps=2) for H in
            list(range(1, 34)) + [63, 64, 65, 127, 128, 129, 1000, 4097, 5000]]
    b = _soa(recs)
    assert_log10_close(engine.compute(b), oracle.batch_log10(b), what="hap sweep")


def test_result_sum_over_long_haplotypes(engine, plain_engine):
    """Short reads on haplotypes of 5,000 and 16,384 positions: the result is a
    sum of thousands of rows of similar size and lies near zero, where the
    tolerance is tightest (1e-5 relative of a log10 near -1); every kernel form
    (scalar, packed, plain) must sum it without drift."""
    rng = np.random.default_rng(71)
    recs = [_record(rng, L, H, n_reads=3, n_haps=2) for L in (1, 2, 5, 16, 33, 100) for H in (5000, 16384)]
    b = _soa(recs)
    want = oracle.batch_log10(b)
    assert_log10_close(engine.compute(b), want, what="long haplotype sums, engine")
    ok = want > -60.0  # the plain form is FP32 only
    assert_log10_close(plain_engine.compute(b)[ok], want[ok], what="long haplotype sums, plain")
    e = g.Engine()
    e.set_tile_table(PACKED_TABLE)
    assert_log10_close(e.compute(b), want, what="long haplotype sums, packed")
    e.close()


def test_n_lowercase_and_odd_letters(engine):
    rng = np.random.default_rng(8)
    recs = [_record(rng, L, H, letters="ACGTNacgtX") for L, H in [(7, 9), (64, 80), (150, 300), (250, 260)]]
    b = _soa(recs)
    assert_log10_close(engine.compute(b), oracle.batch_log10(b), what="letters")


def test_quality_extremes_and_degenerate_alpha(engine):
    """Qualities 0..93 and ins/del qualities low enough that 1-(delta+sigma) is
    near or below zero (the FP32 kernel hands those pairs to the FP64 pass)."""
    rng = np.random.default_rng(9)
    recs = []
    for bq, idq in [((0, 94), (30, 46)), ((10, 41), (0, 4)), ((10, 41), (3, 4)), ((0, 3), (0, 94))]:
        for L, H in [(20, 40), (100, 150), (300, 400)]:
            recs.append(_record(rng, L, H, bq=bq, idq=idq))
    b = _soa(recs)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got))
    assert_log10_close(got[fin], want[fin], what="quality extremes")


def test_fp64_rescue_of_underflowing_pairs(engine):
    b = synth.config2(seed=12, regions=4)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    st = engine.stats()
    under = want < -67.0
    assert under.sum() > 0.3 * len(want)
    assert st.rescued >= under.sum()
    assert_log10_close(got, want, what="cfg2 with rescue")


def test_fp64_length_class_boundaries(engine):
    """Unrelated high-quality reads at every FP64 length-class edge (64, 96,
    128, 160, 192, 256 single tile, then multi-tile): all of them underflow FP32
    and are recomputed by the class's FP64 kernel."""
    rng = np.random.default_rng(22)
    recs = [_record(rng, L, 400, n_reads=2, n_haps=2, bq=(35, 42), related=False)
            for L in [1, 63, 64, 65, 95, 96, 97, 127, 128, 129, 159, 160, 161, 191, 192, 193, 255, 256, 257,
                      300, 511, 513]]
    b = _soa(recs)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    assert engine.stats().rescued >= int((want < -67.0).sum())
    assert_log10_close(got, want, what="FP64 class boundaries")


def test_rescue_disabled_keeps_fp32_results():
    e = g.Engine(fp64_rescue=False)
    b = synth.config2(seed=12, regions=2)
    want = oracle.batch_log10(b)
    got = e.compute(b)
    ok = want > -60.0
    assert_log10_close(got[ok], want[ok], what="cfg2 fp32 part")
    e.close()


def test_multi_tile_long_reads(engine, plain_engine):
    b = synth.config3(seed=13, regions=2)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    assert engine.stats().multi_tile_pairs > 0
    fin = want > -67
    assert_log10_close(got, want, what="cfg3 engine")
    assert_log10_close(plain_engine.compute(b)[fin], want[fin], what="cfg3 plain")


def test_very_long_read_many_tiles(engine):
    rng = np.random.default_rng(14)
    recs = [_record(rng, 4500, 5200, n_reads=2, n_haps=1), _record(rng, 2049, 300, n_reads=1, n_haps=2)]
    b = _soa(recs)
    assert_log10_close(engine.compute(b), oracle.batch_log10(b), what="long read")


def test_fp64_long_reads_short_haplotypes(engine):
    """Insertion-dominated pairs: every read position costs about a factor 10,
    so the FP64 pass carries values across hundreds of decades per tile."""
    rng = np.random.default_rng(21)
    recs = [_record(rng, L, H, n_reads=2, n_haps=2, related=False)
            for L, H in [(257, 1), (300, 2), (383, 3), (500, 4), (641, 5), (900, 1), (1300, 3), (2100, 7)]]
    b = _soa(recs)
    want = oracle.batch_log10(b)
    assert want.min() < -600
    assert_log10_close(engine.compute(b), want, what="long reads, short haplotypes")


def test_fp64_multi_tile_lengths(engine):
    """FP64 multi-tile pairs (512-position tiles, border rows through global
    memory): lengths at the single-tile bound and at 1 to 9 tiles, against
    haplotypes from 1 to 1,500 positions."""
    rng = np.random.default_rng(23)
    recs = [_record(rng, L, H, n_reads=2, n_haps=2, bq=(35, 42), related=False)
            for L, H in [(512, 300), (513, 300), (768, 60), (769, 2), (2048, 400), (2049, 9), (2300, 1500),
                         (4097, 120), (4500, 33)]]
    b = _soa(recs)
    want = oracle.batch_log10(b)
    got = engine.compute(b)
    assert engine.stats().rescued >= len(want) - 4  # unrelated high-quality reads: FP64 throughout
    assert np.isfinite(got).all()
    assert_log10_close(got, want, what="FP64 multi-tile lengths")


def test_empty_and_ragged_records(engine):
    rng = np.random.default_rng(15)
    from oracle.formats import Record
    recs = [_record(rng, 30, 40, n_reads=3, n_haps=2), Record(reads=[], haps=[b"ACGT"]),
            _record(rng, 5, 7, n_reads=1, n_haps=1), Record(reads=_record(rng, 9, 9).reads, haps=[]),
            _record(rng, 200, 90, n_reads=7, n_haps=5)]
    b = _soa(recs)
    got = engine.compute(b)
    assert len(got) == b.num_pairs
    assert_log10_close(got, oracle.batch_log10(b), what="ragged")
    # a batch without pairs
    e = _soa([Record(reads=[], haps=[b"AC"])])
    assert len(engine.compute(e)) == 0


def test_results_do_not_depend_on_batch_composition(engine):
    """Each pair's result is computed independently: alone, in a bigger batch
    and after shuffling the records it is bitwise the same."""
    b = synth.config1(seed=16, regions=40)
    full = engine.compute(b)
    po = np.r_[0, np.cumsum(b.reads_per_record.astype(np.int64) * b.haps_per_record)]
    for first, last in [(0, 1), (5, 9), (39, 40)]:
        part = engine.compute(b.select_records(first, last))
        np.testing.assert_array_equal(part, full[po[first]:po[last]])


def test_graphs_and_direct_launches_agree():
    b = synth.config1(seed=17, regions=20)
    a = g.Engine(use_graphs=True).compute(b)
    c = g.Engine(use_graphs=False).compute(b)
    np.testing.assert_array_equal(a, c)


def test_chunked_host_call_matches_one_pass():
    """A batch run as chunks on two alternating engines (uploads overlapping
    the previous chunk's kernels) gives bitwise the same scores and counts."""
    b = synth.concat([synth.config1(seed=31, regions=150), synth.config3(seed=32, regions=3),
                      synth.config2(seed=33, regions=2)])
    one = g.Engine(pipeline_chunks=1)
    want = one.compute(b)
    s1 = one.stats()
    one.close()
    for chunks in (2, 3, 5):
        e = g.Engine(pipeline_chunks=chunks)
        got = e.compute(b)
        got2 = e.compute(b.pin())
        s = e.stats()
        e.close()
        assert np.array_equal(got, want) and np.array_equal(got2, want), chunks
        assert (s.pairs, s.cells, s.rescued, s.multi_tile_pairs) == (s1.pairs, s1.cells, s1.rescued,
                                                                     s1.multi_tile_pairs)
        assert s.device_ms > 0


def test_repeat_calls_are_deterministic(engine):
    b = synth.config1(seed=18, regions=25)
    x = engine.compute(b)
    y = engine.compute(synth.config0(seed=3))
    z = engine.compute(b)
    np.testing.assert_array_equal(x, z)
    assert len(y) == 8192


def test_device_api_matches_host_api(engine):
    import torch
    b = synth.config1(seed=19, regions=15)
    host = engine.compute(b)
    d = b.to_device()
    scores = torch.empty(b.num_pairs, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    engine.compute_device(d, scores, stream=s)
    s.synchronize()
    np.testing.assert_array_equal(scores.cpu().numpy(), host)


def test_pinned_host_inputs(engine):
    b = synth.config0(seed=4, records=8)
    np.testing.assert_array_equal(engine.compute(b.pin()), engine.compute(b))


PACKED_TABLE = [(32, 4, 8, 2), (48, 4, 12, 2), (64, 4, 16, 2), (96, 8, 12, 2), (128, 8, 16, 2),
                (192, 16, 12, 2), (256, 16, 16, 2), (384, 32, 12, 2), (512, 32, 16, 2), (1024, 32, 32, 0),
                (1 << 30, 32, 32, 1)]


def test_packed_kernel_matches_oracle():
    """Two reads per group in packed FP32: odd read counts (one-read units),
    reads of different lengths in one unit, every packed tile size."""
    e = g.Engine()
    e.set_tile_table(PACKED_TABLE)
    rng = np.random.default_rng(31)
    recs = []
    for L in [1, 5, 17, 31, 33, 47, 64, 65, 95, 97, 128, 129, 191, 193, 256, 257, 383, 385, 511, 512]:
        H = int(rng.integers(1, 3 * L + 50))
        recs.append(_record(rng, L, H, n_reads=1 + L % 3, n_haps=1 + L % 4))
    b = synth.concat([_soa(recs), synth.config0(seed=2, records=3), synth.config2(seed=3, regions=1, reads=7, haps=3)])
    got = e.compute(b)
    assert_log10_close(got, oracle.batch_log10(b), what="packed")
    # scalar and packed single-tile kernels agree within the tolerance
    e2 = g.Engine()
    e2.set_tile_table([(r[0], r[1], r[2], 0 if r[3] == 2 else r[3]) for r in PACKED_TABLE])
    assert_log10_close(got, e2.compute(b), what="packed vs scalar")
    e.close()
    e2.close()


def test_tile_table_round_trip_and_validation():
    e = g.Engine()
    t = e.tile_table()
    assert t[-1][3]
    b = synth.config1(seed=20, regions=10)
    base = e.compute(b)
    # a coarser table (different tiles) gives the same results within tolerance
    e.set_tile_table([(128, 8, 16, 0), (256, 16, 16, 2), (512, 32, 16, 0), (1 << 30, 32, 32, 1)])
    assert e.tile_table()[1] == (256, 16, 16, 2)
    assert_log10_close(e.compute(b), base, what="alt table")
    with pytest.raises(g.PairHMMError):
        e.set_tile_table([(128, 4, 8, False), (1 << 30, 32, 32, True)])  # 128 > 4*8
    with pytest.raises(g.PairHMMError):
        e.set_tile_table([(128, 4, 32, False)])  # last rule must be multi-tile
    with pytest.raises(g.PairHMMError):
        e.set_tile_table([(128, 4, 32, 2), (1 << 30, 32, 32, 1)])  # no packed 4x32 kernel
    e.close()
