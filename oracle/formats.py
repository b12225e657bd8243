"""Plain-Python restatement of the reference's record file format -- TEST INFRASTRUCTURE ONLY.

Parser rules (file_parser_worker.cu):
  * a record header line ``R H`` (``:52-54``), then R read lines, then H haplotype lines;
  * a read line holds 5 equal-length strings separated by single spaces; field k
    starts at k*(L+1) where L is the position of the first space (``:101-133``):
    bases, base quality, insertion quality, deletion quality, gap-continuation quality;
  * qualities are stored as ASCII - 33 (``:95, 115-133``);
  * the haplotype length is the whole line length (``:139``);
  * every read/haplotype is padded by 4 - (len % 4) bytes of 'N' (so 1..4 bytes;
    a multiple of 4 still gets 4) and padded quality bytes are 'N'-33 = 45 (``:81-86``).

Writer rules (output_writer_worker.cu):
  * per record ``"%d %d\\n"`` (``:114``), then R lines of H ``"%.5f"`` values separated by
    single spaces (``:116-127``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def padding_length(n: int) -> int:
    """file_parser_worker.cu:81-83"""
    return 4 - (n % 4)


@dataclass
class Record:
    reads: list = field(default_factory=list)   # (bases, bq, iq, dq, gq) as bytes; quals already -33
    haps: list = field(default_factory=list)    # bases as bytes


def parse_text(text: str) -> list[Record]:
    lines = text.split("\n")
    out: list[Record] = []
    i = 0
    while i < len(lines):
        if lines[i] == "" and i == len(lines) - 1:
            break
        head = lines[i]
        sp = head.find(" ")
        R = int(head[:sp])
        H = int(head[sp:])
        i += 1
        rec = Record()
        for _ in range(R):
            ln = lines[i].encode()
            i += 1
            L = ln.find(b" ")
            fields = [ln[k * (L + 1): k * (L + 1) + L] for k in range(5)]
            quals = [bytes((c - 33) & 0xFF for c in f) for f in fields[1:]]
            rec.reads.append((fields[0], *quals))
        for _ in range(H):
            rec.haps.append(lines[i].encode())
            i += 1
        out.append(rec)
    return out


def format_scores(records: list[Record], scores) -> str:
    parts = []
    k = 0
    for rec in records:
        R, H = len(rec.reads), len(rec.haps)
        parts.append("%d %d\n" % (R, H))
        for _ in range(R):
            parts.append(" ".join("%.5f" % float(np.float32(scores[k + h])) for h in range(H)) + "\n")
            k += H
    return "".join(parts)


@dataclass
class SoABatch:
    """The reference's BatchOfSequenceGroups layout (common.cuh:109-201), with
    the parser's padding applied."""
    reads_per_record: np.ndarray
    haps_per_record: np.ndarray
    read_bases: np.ndarray
    base_quals: np.ndarray
    ins_quals: np.ndarray
    del_quals: np.ndarray
    gcp_quals: np.ndarray
    read_offsets: np.ndarray
    read_lengths: np.ndarray
    hap_bases: np.ndarray
    hap_offsets: np.ndarray
    hap_lengths: np.ndarray


def to_soa(records: list[Record]) -> SoABatch:
    rb, bq, iq, dq, gq, hb = bytearray(), bytearray(), bytearray(), bytearray(), bytearray(), bytearray()
    ro, rl, ho, hl = [], [], [], []
    for rec in records:
        for (b, q1, q2, q3, q4) in rec.reads:
            L = len(b)
            pad = padding_length(L)
            ro.append(len(rb))
            rl.append(L)
            rb += b + b"N" * pad
            for dst, q in ((bq, q1), (iq, q2), (dq, q3), (gq, q4)):
                dst += q + bytes([ord("N") - 33]) * pad
        for h in rec.haps:
            ho.append(len(hb))
            hl.append(len(h))
            hb += h + b"N" * padding_length(len(h))
    u8 = lambda x: np.frombuffer(bytes(x), dtype=np.uint8).copy()
    return SoABatch(
        reads_per_record=np.array([len(r.reads) for r in records], dtype=np.int32),
        haps_per_record=np.array([len(r.haps) for r in records], dtype=np.int32),
        read_bases=u8(rb), base_quals=u8(bq), ins_quals=u8(iq), del_quals=u8(dq), gcp_quals=u8(gq),
        read_offsets=np.array(ro, dtype=np.int64), read_lengths=np.array(rl, dtype=np.int32),
        hap_bases=u8(hb), hap_offsets=np.array(ho, dtype=np.int64), hap_lengths=np.array(hl, dtype=np.int32),
    )
