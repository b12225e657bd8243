"""GPU test of the allocation-free forward (pairhmm_forward_pairs_noalloc).

It runs on caller-owned device buffers and keeps its border scratch in a
statically allocated device array, so it is compared here with the regular
engine entry point (pairhmm_compute_host) on the same pairs: two calls in a
row, each within the parity tolerance, the second bit-identical to the first.
The file name sorts last so that the test also runs after every other GPU test
in a full session; it passes alone in a fresh process too.
"""
import numpy as np
import pytest

from conftest import RTOL, ATOL, assert_log10_close

pytestmark = pytest.mark.gpu

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def related_batch(seed: int = 11):
    """Records whose haplotypes are prefixes of one sequence with 0.2%
    substitutions and whose reads are substrings of it with 0.3% substitutions,
    so every read-haplotype score sits well inside FP32 range.  Read lengths reach 1800 (up to
    four 512-position tiles); one record has haplotypes close to 16384."""
    from gpupairhmm_b200.synth import _Builder

    rng = np.random.default_rng(seed)
    b = _Builder()
    shapes = [(6, 4, 40, 300, 60, 400)] * 40 + [(4, 3, 400, 1100, 200, 600)] * 12 + \
             [(3, 2, 1000, 1800, 100, 300)] * 4 + [(2, 2, 300, 1500, 14000, 14800)]
    for n_reads, n_haps, rlo, rhi, extra_lo, extra_hi in shapes:
        L = rng.integers(rlo, rhi + 1, size=n_reads)
        H = int(L.max()) + rng.integers(extra_lo, extra_hi + 1, size=n_haps)
        base = ACGT[rng.integers(0, 4, size=int(H.max()))]
        haps = []
        for h in H:
            hs = base[:h].copy()
            m = rng.random(h) < 0.002
            hs[m] = ACGT[rng.integers(0, 4, size=int(m.sum()))]
            haps.append(hs)
        reads = []
        for l in L:
            s = int(rng.integers(0, int(H.min()) - l + 1))
            r = base[s:s + l].copy()
            m = rng.random(l) < 0.003
            r[m] = ACGT[rng.integers(0, 4, size=int(m.sum()))]
            reads.append(r)
        n = int(L.sum())
        b.add_concat(L, np.concatenate(reads), rng.integers(20, 41, size=n).astype(np.uint8),
                     rng.integers(30, 46, size=n).astype(np.uint8), rng.integers(30, 46, size=n).astype(np.uint8),
                     H, np.concatenate(haps))
    return b.build()


def pair_list(batch):
    """Flat pair list in the order the engine writes scores: per record, read
    by read, each read against every haplotype of its record."""
    import gpupairhmm_b200 as g

    out = []
    r0 = h0 = 0
    for nr, nh in zip(batch.reads_per_record, batch.haps_per_record):
        for i in range(r0, r0 + int(nr)):
            for j in range(h0, h0 + int(nh)):
                out.append((batch.read_offsets[i], batch.hap_offsets[j], batch.read_lengths[i],
                            batch.hap_lengths[j]))
        r0 += int(nr)
        h0 += int(nh)
    return np.array(out, dtype=g.PAIR_DTYPE)


def test_noalloc_matches_engine_two_calls():
    import torch
    import gpupairhmm_b200 as g

    batch = related_batch()
    eng = g.Engine()
    want = eng.compute(batch)
    eng.close()
    pairs = pair_list(batch)
    assert len(pairs) == len(want)
    max_h = int(batch.hap_lengths.max())
    assert max_h <= 16384

    dev = torch.device("cuda:0")
    d = {k: torch.from_numpy(np.ascontiguousarray(getattr(batch, k))).to(dev)
         for k in ("read_bases", "base_quals", "ins_quals", "del_quals", "hap_bases")}
    dpairs = torch.from_numpy(pairs.view(np.uint8)).to(dev)
    scores = torch.full((len(pairs),), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    got = []
    for call in range(2):
        scores.fill_(-12345.0)  # the second call must write every score again
        g.forward_pairs_noalloc(0, d["read_bases"], d["base_quals"], d["ins_quals"], d["del_quals"],
                                d["hap_bases"], dpairs, len(pairs), max_h, scores, stream)
        torch.cuda.synchronize(dev)
        out = scores.cpu().numpy().copy()
        assert np.isfinite(out).all(), f"call {call}: non-finite scores"
        assert_log10_close(out, want, RTOL, ATOL, what=f"no-alloc call {call} vs engine")
        got.append(out)
    assert np.array_equal(got[0], got[1])


def test_noalloc_tile_edges_against_oracle():
    """The allocation-free kernel's own tile and lane residues, checked against
    the FP64 oracle directly: read lengths at the lane and 512-position tile
    edges (L - 1 = 15 mod 16 ends a read on a lane's last position), one-base
    reads and haplotypes, haplotypes of exactly the 16384 limit, on a side
    stream.  FP32 only: a pair below the FP32 range would be left out of the
    comparison (this set has none or almost none)."""
    import torch
    import gpupairhmm_b200 as g
    import oracle
    from gpupairhmm_b200.synth import _Builder

    rng = np.random.default_rng(13)
    b = _Builder()
    for L in (1, 16, 17, 511, 512, 513, 1024, 1025):
        H = np.array([1, 2, L + 40, 16384] if L <= 17 else [L + 40, 2000, 16384])
        base = ACGT[rng.integers(0, 4, size=16384)]
        haps = [base[:h].copy() for h in H]
        reads = []
        for _ in range(3):  # substrings of the common prefix, 0.3% substitutions
            s = int(rng.integers(0, 41))
            r = base[s:s + L].copy()
            m = rng.random(L) < 0.003
            r[m] = ACGT[rng.integers(0, 4, size=int(m.sum()))]
            reads.append(r)
        n = 3 * L
        b.add_concat(np.full(3, L), np.concatenate(reads), rng.integers(20, 41, size=n).astype(np.uint8),
                     rng.integers(30, 46, size=n).astype(np.uint8), rng.integers(30, 46, size=n).astype(np.uint8),
                     H, np.concatenate(haps))
    batch = b.build()
    want = oracle.batch_log10(batch)
    pairs = pair_list(batch)
    dev = torch.device("cuda:0")
    d = [torch.from_numpy(np.ascontiguousarray(getattr(batch, k))).to(dev)
         for k in ("read_bases", "base_quals", "ins_quals", "del_quals", "hap_bases")]
    dpairs = torch.from_numpy(pairs.view(np.uint8)).to(dev)
    scores = torch.full((len(pairs),), float("nan"), dtype=torch.float32, device=dev)
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        g.forward_pairs_noalloc(0, *d, dpairs, len(pairs), 16384, scores, side)
    side.synchronize()
    got = scores.cpu().numpy()
    ok = want > -60.0
    assert ok.sum() >= 0.9 * len(want)
    assert_log10_close(got[ok], want[ok], RTOL, ATOL, what="no-alloc tile edges vs oracle")


def test_noalloc_limits():
    import torch
    import gpupairhmm_b200 as g

    batch = related_batch(seed=12)
    pairs = pair_list(batch)[:64]
    dev = torch.device("cuda:0")
    d = [torch.from_numpy(np.ascontiguousarray(getattr(batch, k))).to(dev)
         for k in ("read_bases", "base_quals", "ins_quals", "del_quals", "hap_bases")]
    dpairs = torch.from_numpy(pairs.view(np.uint8)).to(dev)
    scores = torch.zeros(len(pairs), dtype=torch.float32, device=dev)
    with pytest.raises(g.PairHMMError) as e:
        g.forward_pairs_noalloc(0, *d, dpairs, len(pairs), 16385, scores)
    assert e.value.status == 9
    # a pair longer than the declared bound is not computed: NaN
    bound = int(pairs["hap_length"].min())
    g.forward_pairs_noalloc(0, *d, dpairs, len(pairs), bound, scores)
    torch.cuda.synchronize(dev)
    out = scores.cpu().numpy()
    over = pairs["hap_length"] > bound
    assert over.any() and np.isnan(out[over]).all() and np.isfinite(out[~over]).all()
