"""gcp mode (engine option gcp=1) vs the oracle's gcp mode, through the C ABI.

In gcp mode each read takes eps = p(gcp) and beta = 1 - eps from the gcp
quality of its first position, as the reference's CPU recurrence does
(gpuworker.cuh:1009, 1048-1049); the default keeps the GPU path's 0.1 / 0.9.
Tolerance: conftest.RTOL/ATOL on log10, as for every parity test."""
import numpy as np
import pytest

import gpupairhmm_b200 as g
import oracle
from gpupairhmm_b200 import synth
from conftest import assert_log10_close

pytestmark = pytest.mark.gpu

GCP_TABLE = [(64, 4, 16, 0), (128, 8, 16, 0), (160, 8, 20, 0), (256, 16, 16, 0), (512, 32, 16, 0),
             (1024, 32, 32, 0), (1 << 30, 32, 32, 1)]


@pytest.fixture(scope="module")
def gcp_engine():
    e = g.Engine(gcp=True)
    yield e
    e.close()


def with_gcp(b, seed, lo=1, hi=41):
    rng = np.random.default_rng(seed)
    gq = rng.integers(lo, hi, size=len(b.read_bases)).astype(np.uint8)
    return g.Batch(b.reads_per_record, b.haps_per_record, b.read_bases, b.base_quals, b.ins_quals, b.del_quals,
                   b.read_offsets, b.read_lengths, b.hap_bases, b.hap_offsets, b.hap_lengths, gq)


@pytest.mark.parametrize("name,make", [
    ("small", lambda: synth.config0(seed=30, records=24)),
    ("uneven", lambda: synth.config1(seed=31, regions=40)),
    ("rescue", lambda: synth.config2(seed=32, regions=3, reads=16, haps=4)),
    ("long", lambda: synth.config3(seed=33, regions=1)),
])
def test_gcp_mode_matches_oracle(gcp_engine, name, make):
    b = with_gcp(make(), seed=len(name))
    want = oracle.batch_log10(b, gcp=True)
    got = gcp_engine.compute(b)
    assert_log10_close(got, want, what=f"gcp mode, {name}")
    if name in ("rescue", "long"):  # FP32 underflows: the FP64 pass ran with the reads' own eps/beta
        assert gcp_engine.stats().rescued > 0
    if name == "long":
        assert gcp_engine.stats().multi_tile_pairs > 0
    # and the gcp qualities did change the model
    assert not np.allclose(want, oracle.batch_log10(b), rtol=1e-4)


def test_gcp_10_is_the_default_model(gcp_engine):
    """gcp quality 10 gives eps = p(10) = 0.1f and beta = 0.9f: the gcp kernels
    then compute what the default kernels with the same tiles compute, up to the
    final subtraction log10(S) - log10(beta*FLT_MAX/16): the default kernels take
    that constant (about 37.4) folded at compile time, the gcp kernels evaluate
    log10(beta) on the device, so results may differ by one float ulp of 37.4
    (3.8e-6), or by one ulp of the result where that is larger, and by nothing
    else."""
    b = synth.config1(seed=34, regions=30)  # synthetic gcp qualities are 10
    assert np.all(b.gcp_quals[b.read_bases != ord("N")] == 10)
    e = g.Engine()
    e.set_tile_table(GCP_TABLE)
    want = e.compute(b)
    e.close()
    got = gcp_engine.compute(b)
    d = np.abs(got.astype(np.float64) - want)
    bound = np.maximum(2.0 ** -18, np.spacing(np.abs(want)).astype(np.float64))  # 2^-18: ulp in [32, 64)
    assert np.all(d <= bound), (d.max(), int((d > bound).sum()))


def test_gcp_mode_serving_matches_batch_call(gcp_engine):
    regions = [with_gcp(synth.config1(seed=40 + i, regions=2), seed=i) for i in range(6)]
    want = [gcp_engine.compute(r) for r in regions]
    tickets = [gcp_engine.submit(r) for r in regions]
    for t, w in zip(tickets, want):
        got = gcp_engine.drain(t, len(w))
        assert_log10_close(got, w, what="gcp serving")


def test_gcp_mode_rejections():
    b = with_gcp(synth.config0(seed=35, records=2), seed=3)
    e = g.Engine(gcp=True)
    bad = b.gcp_quals.copy()
    bad[int(b.read_offsets[1])] = 0  # eps = 1, beta = 0
    with pytest.raises(g.PairHMMError) as err:
        e.compute(g.Batch(*[getattr(b, k) for k in ("reads_per_record", "haps_per_record", "read_bases",
                                                    "base_quals", "ins_quals", "del_quals", "read_offsets",
                                                    "read_lengths", "hap_bases", "hap_offsets",
                                                    "hap_lengths")], bad))
    assert "gcp quality 0" in str(err.value)
    no_gcp = g.Batch(*[getattr(b, k) for k in ("reads_per_record", "haps_per_record", "read_bases", "base_quals",
                                               "ins_quals", "del_quals", "read_offsets", "read_lengths",
                                               "hap_bases", "hap_offsets", "hap_lengths")], None)
    with pytest.raises(g.PairHMMError):
        e.compute(no_gcp)
    with pytest.raises(g.PairHMMError):  # packed kernels have no gcp form
        e.set_tile_table([(96, 8, 12, 2), (1 << 30, 32, 32, 1)])
    # the engine still works after the rejected calls
    assert_log10_close(e.compute(b), oracle.batch_log10(b, gcp=True), what="gcp after rejections")
    e.close()
    with pytest.raises(g.PairHMMError):
        g.Engine(mode=g.MODE_PLAIN, gcp=True)


def test_gcp_serving_matches_batch_call(gcp_engine):
    """gcp mode through the serving queue (the regions' gcp qualities travel with
    their other arrays into the merged batch): scores equal the batch call's
    bitwise, for short and multi-tile regions submitted together."""
    regions = [with_gcp(synth.config1(seed=600 + i, regions=1), 700 + i) for i in range(6)] + \
              [with_gcp(synth.config3(seed=610, regions=1), 710)]
    want = [gcp_engine.compute(r) for r in regions]
    e = g.Engine(gcp=True)
    tickets = e.submit_many(regions)
    for t, r, w in zip(tickets, regions, want):
        np.testing.assert_array_equal(e.drain(t, r.num_pairs, timeout_ms=120000), w)
    e.close()


def test_gcp_fused_and_separate_fp64_tiers_agree_bitwise(gcp_engine):
    """gcp mode, multi-tile FP64 pairs: a 40-region long-read batch (2,560
    multi-tile pairs, separate tier launches) gives each region's scores
    bitwise as the region alone (64 pairs, tiers fused in one launch)."""
    from gpupairhmm_b200 import replicas
    b = with_gcp(synth.config3(seed=620, regions=40), 720, lo=5, hi=41)
    got = gcp_engine.compute(b)
    assert gcp_engine.stats().rescued > 0
    po = replicas.pair_offsets(b)
    for r in range(b.num_records):
        np.testing.assert_array_equal(gcp_engine.compute(b.select_records(r, r + 1)), got[po[r]:po[r + 1]])
