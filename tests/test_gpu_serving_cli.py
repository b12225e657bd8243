"""Serving loop and command-line front end on the GPU."""
import subprocess
import threading
import time

import numpy as np
import pytest

import gpupairhmm_b200 as g
import oracle
from gpupairhmm_b200 import synth
from conftest import assert_log10_close

pytestmark = pytest.mark.gpu


def test_serving_results_equal_alone_and_in_the_mix():
    """Regions submitted while others are on the GPU are merged into shared
    batches; every region's scores equal its scores computed alone."""
    regions = [synth.config1(seed=100 + i, regions=1) for i in range(24)] + \
              [synth.config3(seed=200, regions=1)]
    alone_engine = g.Engine()
    alone = [alone_engine.compute(r) for r in regions]
    alone_engine.close()

    e = g.Engine()
    tickets = [None] * len(regions)

    def producer():
        for i, r in enumerate(regions):
            tickets[i] = e.submit(r)
            if i % 5 == 0:
                time.sleep(0.002)

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    for i, r in enumerate(regions):
        got = e.drain(tickets[i], r.num_pairs, timeout_ms=120000)
        np.testing.assert_array_equal(got, alone[i])
    e.close()


def test_serving_poll_latency_and_errors():
    e = g.Engine()
    r = synth.config0(seed=1, records=2)
    t = e.submit(r)
    deadline = time.time() + 60
    while not e.poll(t):
        assert time.time() < deadline
        time.sleep(0.001)
    assert e.latency_ms(t) > 0
    got = e.drain(t, r.num_pairs)
    assert_log10_close(got, oracle.batch_log10(r), what="served")
    with pytest.raises(g.PairHMMError) as err:
        e.poll(t)  # drained tickets are released
    assert err.value.status == 5
    e.close()


def test_serving_budget_rejects_oversized_region():
    e = g.Engine(device_budget_bytes=1 << 20)
    with pytest.raises(g.PairHMMError) as err:
        e.submit(synth.config0(seed=2, records=64))
    assert err.value.status == 4
    e.close()


def test_serving_admission_under_a_small_budget():
    """A device budget that holds only a few regions per slot batch: a burst of
    regions is admitted in many budget-limited batches, more than one slot
    batch is on the device at a time, no batch exceeds its slot's budget, and
    every region's scores equal the batch call's bitwise."""
    rng = np.random.default_rng(7)
    regions = []
    seed = 500
    while len(regions) < 48:
        r = synth.config1(seed=seed, regions=1)
        seed += 1
        if int(r.reads_per_record[0]) <= 60:
            regions.append(r)
    ref = g.Engine()
    want = [ref.compute(r) for r in regions]
    ref.close()
    e = g.Engine(device_budget_bytes=4 * 400_000)  # four slots
    order = rng.permutation(len(regions))
    tickets = {int(i): e.submit(regions[i]) for i in order}
    for i, r in enumerate(regions):
        np.testing.assert_array_equal(e.drain(tickets[i], r.num_pairs, timeout_ms=120000), want[i])
    st = e.serving_stats()
    e.close()
    assert st["regions"] == len(regions)
    assert st["budget_per_slot"] == 400_000
    assert 0 < st["max_batch_bytes"] <= st["budget_per_slot"]
    assert st["batches"] >= 8
    assert st["max_in_flight"] >= 2


def test_serving_concurrent_drains_of_one_ticket():
    """Two threads drain the same ticket: one gets the scores, the other an
    unknown-ticket error; nothing else breaks."""
    e = g.Engine()
    r = synth.config1(seed=77, regions=1)
    t = e.submit(r)
    results = []

    def drain():
        try:
            results.append(("ok", e.drain(t, r.num_pairs, timeout_ms=60000)))
        except g.PairHMMError as err:
            results.append(("err", err.status))

    ths = [threading.Thread(target=drain) for _ in range(2)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    kinds = sorted(k for k, _ in results)
    assert kinds == ["err", "ok"]
    assert [v for k, v in results if k == "err"] == [5]
    e.close()


def test_submit_many_matches_the_batch_call():
    """Regions submitted many per call -- a list, and a prepared region set with
    a region picked more than once -- give the batch call's scores bitwise."""
    regions = [synth.config1(seed=900 + i, regions=1) for i in range(20)] + [synth.config3(seed=901, regions=1)]
    ref = g.Engine()
    alone = [ref.compute(r) for r in regions]
    ref.close()
    e = g.Engine()
    tickets = e.submit_many(regions)
    assert len(set(tickets)) == len(regions)
    for t, r, want in zip(tickets, regions, alone):
        np.testing.assert_array_equal(e.drain(t, r.num_pairs, timeout_ms=120000), want)
    rs = g.RegionSet(regions)
    picks = np.array([3, 3, 20, 0, 7, 3])
    tickets = e.submit_many(rs, picks)
    for t, i in zip(tickets, picks):
        np.testing.assert_array_equal(e.drain(t, rs.num_pairs[i], timeout_ms=120000), alone[i])
    assert e.submit_many([]) == []
    e.close()


def test_submit_many_queues_nothing_when_a_region_is_bad():
    """One malformed region fails the whole call, names the region, and leaves
    the queue as it was."""
    good = [synth.config0(seed=10 + i, records=1) for i in range(4)]
    bad = synth.config0(seed=20, records=1)
    bad.read_lengths = np.array(bad.read_lengths, dtype=np.int32)
    bad.read_lengths[1] = 0
    e = g.Engine()
    with pytest.raises(g.PairHMMError) as err:
        e.submit_many(good[:2] + [bad] + good[2:])
    assert err.value.status == 1
    assert "region 2" in str(err.value)
    tickets = e.submit_many(good)
    for t, r in zip(tickets, good):
        assert_log10_close(e.drain(t, r.num_pairs, timeout_ms=60000), oracle.batch_log10(r), what="served")
    assert e.serving_stats()["regions"] == len(good)
    e.close()


def test_cli_end_to_end(tmp_path):
    b = synth.config0(seed=7, records=6)
    text = synth.to_text(b) + synth.to_text(synth.config3(seed=8, regions=1))
    inp = tmp_path / "in.txt"
    out = tmp_path / "out.txt"
    inp.write_text(text)
    res = subprocess.run([str(g.CLI_PATH), "--inputfile", str(inp), "--outputfile", str(out),
                          "--fileBatchsize", "500", "--transferBatchsize", "300"],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    assert "GCUPS" in res.stdout
    recs = g.parse_records(text)
    want = oracle.batch_log10(recs.batch)
    lines = out.read_text().split("\n")
    scores, i = [], 0
    for R, H in zip(recs.batch.reads_per_record, recs.batch.haps_per_record):
        assert lines[i] == f"{R} {H}"
        i += 1
        for _ in range(R):
            vals = lines[i].split(" ")
            assert len(vals) == H and all(len(v.split(".")[1]) == 5 for v in vals)
            scores += [float(v) for v in vals]
            i += 1
    fin = want > -67
    # printed with 5 decimals
    assert np.max(np.abs(np.array(scores)[fin] - want[fin])) <= 1e-5 * np.abs(want[fin]).max() + 6e-6


def test_cli_dev_null_and_plain_mode(tmp_path):
    inp = tmp_path / "in.txt"
    inp.write_text(synth.to_text(synth.config0(seed=9, records=2)))
    for args in (["--outputfile", "/dev/null"], ["--outputfile", str(tmp_path / "o.txt"), "--mode", "plain"]):
        res = subprocess.run([str(g.CLI_PATH), "--inputfile", str(inp), *args], capture_output=True, text=True,
                             timeout=300)
        assert res.returncode == 0, res.stderr


def test_cli_rejects_malformed_input(tmp_path):
    inp = tmp_path / "bad.txt"
    inp.write_text("2 1\nACGT IIII IIII IIII ++++\n")
    res = subprocess.run([str(g.CLI_PATH), "--inputfile", str(inp), "--outputfile", "/dev/null"],
                         capture_output=True, text=True, timeout=120)
    assert res.returncode != 0
