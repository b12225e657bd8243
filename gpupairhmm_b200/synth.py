"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No real sequencing data is available offline, so every benchmark and parity
case uses generated records with the described shapes, lengths and quality
distributions.  All generators are deterministic for a given seed.

  cfg0  plain FP32, small: 64 records x R=32 x H=4; 150 bp haplotypes from a
        region sequence with 0-3 SNPs and 1-5 bp indels each; 100 bp reads
        sampled from a haplotype with 1% substitutions; base quality U{10..40},
        ins/del quality 40, gcp 10.
  cfg1  uneven lengths: 20,000 regions; R ~ lognormal(median 40, sigma 1.0)
        clipped to 1..400; H ~ U{1..16}; read length from {100,150,250}
        (weights .3/.5/.2) minus U{0..30}; haplotype length = read length +
        U{50..400}; qualities as cfg0.  sigma is not given by the description;
        1.0 is used and the generated cell count is reported (about 5.7e11).
  cfg2  precision stress: 5,000 regions x R=64 x H=8, reads 250 bp, haplotypes
        600 bp, half of the reads unrelated random sequence, base quality
        U{35..41}.
  cfg3  long reads: 2,000 regions x R=16 x H=4, reads U{1000..2000}, haplotypes
        U{2000..5000} with 1-50 bp indels, base quality U{5..40}, ins/del
        quality U{30..45} per position.
  cfg4  streaming: Poisson arrivals at 2,000 regions/s; shapes from cfg1 with
        5% drawn from cfg3.
"""
from __future__ import annotations

import numpy as np

from . import Batch

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def _rand_seq(rng: np.random.Generator, n: int) -> np.ndarray:
    return ACGT[rng.integers(0, 4, size=n)]


def _mutate(rng: np.random.Generator, seq: np.ndarray, n_snps: int, n_indels: int, indel_max: int) -> np.ndarray:
    s = seq.copy()
    if n_snps and len(s):
        pos = rng.integers(0, len(s), size=n_snps)
        s[pos] = ACGT[(np.searchsorted(ACGT, s[pos]) + rng.integers(1, 4, size=n_snps)) % 4]
    for _ in range(n_indels):
        if len(s) < 2:
            break
        p = int(rng.integers(0, len(s)))
        k = int(rng.integers(1, indel_max + 1))
        if rng.random() < 0.5:
            s = np.concatenate([s[:p], _rand_seq(rng, k), s[p:]])
        else:
            s = np.concatenate([s[:p], s[p + k:]])
    return s


def _fit(seq: np.ndarray, n: int, rng: np.random.Generator) -> np.ndarray:
    if len(seq) >= n:
        return seq[:n]
    return np.concatenate([seq, _rand_seq(rng, n - len(seq))])


class _Builder:
    """Accumulates records into the SoA layout with the parser's 4-byte padding
    (4 - len % 4 bytes of 'N', quality 'N' - 33)."""

    def __init__(self):
        self.rpr, self.hpr = [], []
        self.rlen, self.hlen = [], []
        self.reads, self.bq, self.iq, self.dq, self.haps = [], [], [], [], []

    def add(self, reads, bq, iq, dq, haps):
        """Lists of per-sequence arrays."""
        self.add_concat(np.array([len(r) for r in reads], np.int64),
                        *(np.concatenate(x) if len(x) else np.zeros(0, np.uint8) for x in (reads, bq, iq, dq)),
                        np.array([len(h) for h in haps], np.int64),
                        np.concatenate(haps) if len(haps) else np.zeros(0, np.uint8))

    def add_concat(self, read_lens, reads, bq, iq, dq, hap_lens, haps):
        """One record from concatenated sequences and their lengths."""
        self.rpr.append(len(read_lens))
        self.hpr.append(len(hap_lens))
        self.rlen.append(np.asarray(read_lens, np.int64))
        self.hlen.append(np.asarray(hap_lens, np.int64))
        self.reads.append(reads)
        self.bq.append(bq)
        self.iq.append(iq)
        self.dq.append(dq)
        self.haps.append(haps)

    @staticmethod
    def _layout(lens):
        """Padded offsets and the destination index of every data byte."""
        pads = 4 - lens % 4
        offs = np.zeros(len(lens), dtype=np.int64)
        if len(lens):
            offs[1:] = np.cumsum(lens + pads)[:-1]
        total = int((lens + pads).sum())
        dest = np.arange(int(lens.sum()), dtype=np.int64) + np.repeat(offs - (np.cumsum(lens) - lens), lens)
        return offs, dest, total

    @staticmethod
    def _fill(dest, total, data, pad_byte):
        buf = np.full(total, pad_byte, dtype=np.uint8)
        buf[dest] = data
        return buf

    def build(self) -> Batch:
        rl = np.concatenate(self.rlen) if self.rlen else np.zeros(0, np.int64)
        hl = np.concatenate(self.hlen) if self.hlen else np.zeros(0, np.int64)
        cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0, np.uint8)
        ro, rdest, rtot = self._layout(rl)
        ho, hdest, htot = self._layout(hl)
        rb = self._fill(rdest, rtot, cat(self.reads), ord("N"))
        bq = self._fill(rdest, rtot, cat(self.bq), ord("N") - 33)
        iq = self._fill(rdest, rtot, cat(self.iq), ord("N") - 33)
        dq = self._fill(rdest, rtot, cat(self.dq), ord("N") - 33)
        hb = self._fill(hdest, htot, cat(self.haps), ord("N"))
        gq = np.where(rb == ord("N"), ord("N") - 33, 10).astype(np.uint8)
        return Batch(np.array(self.rpr, dtype=np.int32), np.array(self.hpr, dtype=np.int32), rb, bq, iq, dq,
                     ro, rl.astype(np.int32), hb, ho, hl.astype(np.int32), gq)


def _reads_from_haps(rng, haps, n_reads, lengths, err_rate):
    """Substrings of randomly chosen haplotypes with substitution errors;
    returns (concatenated reads, lengths)."""
    lengths = np.asarray(lengths, dtype=np.int64)
    hl = np.array([len(h) for h in haps], dtype=np.int64)
    hcat = np.concatenate(haps)
    hoff = np.r_[0, np.cumsum(hl)[:-1]]
    pick = rng.integers(0, len(haps), size=n_reads)
    span = np.maximum(hl[pick] - lengths + 1, 1)
    start = (rng.random(n_reads) * span).astype(np.int64)
    within = np.arange(int(lengths.sum())) - np.repeat(np.cumsum(lengths) - lengths, lengths)
    src = np.repeat(hoff[pick] + start, lengths) + within
    lim = np.repeat(hoff[pick] + hl[pick], lengths)
    out = np.where(src < lim, hcat[np.minimum(src, len(hcat) - 1)], ACGT[rng.integers(0, 4, size=len(src))])
    m = rng.random(len(out)) < err_rate
    if m.any():
        out[m] = ACGT[(np.searchsorted(ACGT, out[m]) + rng.integers(1, 4, size=int(m.sum()))) % 4]
    return out.astype(np.uint8), lengths


def config0(seed: int = 0, records: int = 64) -> Batch:
    rng = np.random.default_rng(seed)
    b = _Builder()
    for _ in range(records):
        base = _rand_seq(rng, 150)
        haps = [_fit(_mutate(rng, base, int(rng.integers(0, 4)), int(rng.integers(0, 2)), 5), 150, rng)
                for _ in range(4)]
        reads, rl = _reads_from_haps(rng, haps, 32, np.full(32, 100), 0.01)
        n = len(reads)
        b.add_concat(rl, reads, rng.integers(10, 41, size=n).astype(np.uint8), np.full(n, 40, np.uint8),
                     np.full(n, 40, np.uint8), np.array([len(h) for h in haps]), np.concatenate(haps))
    return b.build()


def _cfg1_region(rng, b: _Builder, sigma: float):
    R = int(np.clip(np.round(40.0 * np.exp(sigma * rng.standard_normal())), 1, 400))
    H = int(rng.integers(1, 17))
    Lb = int(rng.choice([100, 150, 250], p=[0.3, 0.5, 0.2]))
    hap_lens = Lb + rng.integers(50, 401, size=H)
    base = _rand_seq(rng, int(hap_lens.max()) + 60)
    haps = [_fit(_mutate(rng, base, int(rng.integers(0, 4)), int(rng.integers(0, 2)), 5), int(n), rng)
            for n in hap_lens]
    rl = Lb - rng.integers(0, 31, size=R)
    reads, rl = _reads_from_haps(rng, haps, R, rl, 0.01)
    n = len(reads)
    b.add_concat(rl, reads, rng.integers(10, 41, size=n).astype(np.uint8), np.full(n, 40, np.uint8),
                 np.full(n, 40, np.uint8), hap_lens, np.concatenate(haps))


def config1(seed: int = 1, regions: int = 20000, sigma: float = 1.0) -> Batch:
    rng = np.random.default_rng(seed)
    b = _Builder()
    for _ in range(regions):
        _cfg1_region(rng, b, sigma)
    return b.build()


def config2(seed: int = 2, regions: int = 5000, reads: int = 64, haps: int = 8) -> Batch:
    rng = np.random.default_rng(seed)
    b = _Builder()
    for _ in range(regions):
        base = _rand_seq(rng, 660)
        hs = [_fit(_mutate(rng, base, int(rng.integers(0, 4)), int(rng.integers(0, 2)), 5), 600, rng)
              for _ in range(haps)]
        half = reads // 2
        rel, _ = _reads_from_haps(rng, hs, reads - half, np.full(reads - half, 250), 0.01)
        unrel = _rand_seq(rng, 250 * half)  # unrelated reads
        allr = np.concatenate([rel, unrel]).reshape(reads, 250)[rng.permutation(reads)].reshape(-1)
        n = len(allr)
        b.add_concat(np.full(reads, 250), allr, rng.integers(35, 42, size=n).astype(np.uint8),
                     np.full(n, 40, np.uint8), np.full(n, 40, np.uint8), np.full(haps, 600), np.concatenate(hs))
    return b.build()


def _cfg3_region(rng, b: _Builder, R: int = 16, H: int = 4):
    hap_lens = rng.integers(2000, 5001, size=H)
    base = _rand_seq(rng, int(hap_lens.max()) + 200)
    hs = [_fit(_mutate(rng, base, int(rng.integers(0, 4)), int(rng.integers(1, 4)), 50), int(n), rng)
          for n in hap_lens]
    rl = rng.integers(1000, 2001, size=R)
    rs, rl = _reads_from_haps(rng, hs, R, rl, 0.01)
    n = len(rs)
    b.add_concat(rl, rs, rng.integers(5, 41, size=n).astype(np.uint8), rng.integers(30, 46, size=n).astype(np.uint8),
                 rng.integers(30, 46, size=n).astype(np.uint8), np.array([len(h) for h in hs]), np.concatenate(hs))


def config3(seed: int = 3, regions: int = 2000) -> Batch:
    rng = np.random.default_rng(seed)
    b = _Builder()
    for _ in range(regions):
        _cfg3_region(rng, b)
    return b.build()


def stream_regions(seed: int = 4, rate: float = 2000.0, seconds: float = 60.0, long_frac: float = 0.05,
                   sigma: float = 1.0):
    """cfg4: yields (arrival_time_s, Batch of one region) in arrival order."""
    rng = np.random.default_rng(seed)
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > seconds:
            return
        b = _Builder()
        if rng.random() < long_frac:
            _cfg3_region(rng, b)
        else:
            _cfg1_region(rng, b, sigma)
        yield t, b.build()


def region_pool(seed: int = 4, regions: int = 24000, long_frac: float = 0.05, sigma: float = 1.0) -> list:
    """cfg4 region shapes drawn ahead of time: `regions` independent regions
    (config-1 shapes, `long_frac` of them long-read shapes), each a contiguous
    Batch of one record.  Streams at any rate replay draws from this pool."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(regions):
        b = _Builder()
        if rng.random() < long_frac:
            _cfg3_region(rng, b)
        else:
            _cfg1_region(rng, b, sigma)
        out.append(b.build().contiguous())
    return out


def poisson_arrivals(seed: int, rate: float, seconds: float, pool_size: int):
    """Poisson arrival times at `rate` per second over `seconds`, each with a
    region drawn uniformly from a pool of `pool_size`: (times, pool indices)."""
    rng = np.random.default_rng(seed)
    n = int(rate * seconds * 1.2 + 100)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    while t[-1] < seconds:
        t = np.concatenate([t, t[-1] + np.cumsum(rng.exponential(1.0 / rate, size=n))])
    t = t[t <= seconds]
    return t, rng.integers(0, pool_size, size=len(t))


def concat(batches) -> Batch:
    """Records of several batches, in order, as one batch."""
    parts = list(batches)
    roff, hoff = 0, 0
    ro, ho = [], []
    for p in parts:
        ro.append(np.asarray(p.read_offsets, np.int64) + roff)
        ho.append(np.asarray(p.hap_offsets, np.int64) + hoff)
        roff += len(p.read_bases)
        hoff += len(p.hap_bases)
    cat = lambda name, dt: np.concatenate([np.asarray(getattr(p, name), dt) for p in parts])
    return Batch(cat("reads_per_record", np.int32), cat("haps_per_record", np.int32), cat("read_bases", np.uint8),
                 cat("base_quals", np.uint8), cat("ins_quals", np.uint8), cat("del_quals", np.uint8),
                 np.concatenate(ro), cat("read_lengths", np.int32), cat("hap_bases", np.uint8), np.concatenate(ho),
                 cat("hap_lengths", np.int32),
                 cat("gcp_quals", np.uint8) if all(p.gcp_quals is not None for p in parts) else None)


def to_text(b: Batch) -> str:
    """Render a batch in the record file format (qualities + 33)."""
    out = []
    rpr, hpr = np.asarray(b.reads_per_record), np.asarray(b.haps_per_record)
    ri = hi = 0
    gq = b.gcp_quals
    for g in range(len(rpr)):
        out.append(f"{int(rpr[g])} {int(hpr[g])}\n")
        for _ in range(int(rpr[g])):
            o, L = int(b.read_offsets[ri]), int(b.read_lengths[ri])
            fields = [bytes(b.read_bases[o:o + L])]
            for q in (b.base_quals, b.ins_quals, b.del_quals):
                fields.append(bytes((np.asarray(q[o:o + L], np.int64) + 33).astype(np.uint8)))
            g4 = np.full(L, 10, np.int64) if gq is None else np.asarray(gq[o:o + L], np.int64)
            fields.append(bytes((g4 + 33).astype(np.uint8)))
            out.append(b" ".join(fields).decode() + "\n")
            ri += 1
        for _ in range(int(hpr[g])):
            o, n = int(b.hap_offsets[hi]), int(b.hap_lengths[hi])
            out.append(bytes(b.hap_bases[o:o + n]).decode() + "\n")
            hi += 1
    return "".join(out)
