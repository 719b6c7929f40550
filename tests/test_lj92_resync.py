"""The statistical property the GPU lossless-JPEG decoder's chunking relies on,
checked on the CPU: a decode path started kOverlapBits (1536) bits before a
chunk boundary, at an arbitrary bit and in component phase 0, reaches the true
sample boundary at or after the chunk start for almost every chunk (the GPU
also tries the other component phase from that position, and fixes the rest
from the neighbouring chunk's exit).  Streams: 256x256 tiles with one fixed
table and with an optimal table per component, on noise (the slow case) and
on smooth data."""
import numpy as np
import pytest

from cpipe_b200.dng_synth import lj92_segment

LEAD, CHUNK = 1536, 1024


def _stream(seg):
    """(tables as {(length, code): category}, per-component table index,
    unstuffed bits) of a one-scan lossless-JPEG stream."""
    i = seg.index(b"\xff\xc4")
    n = int.from_bytes(seg[i + 2:i + 4], "big")
    body = seg[i + 4:i + 2 + n]
    tables, q = {}, 0
    while q < len(body):
        th, counts = body[q] & 15, list(body[q + 1:q + 17])
        vals = list(body[q + 17:q + 17 + sum(counts)])
        codes, code, k = {}, 0, 0
        for length in range(1, 17):
            for _ in range(counts[length - 1]):
                codes[(length, code)] = vals[k]
                code, k = code + 1, k + 1
            code <<= 1
        tables[th] = codes
        q += 17 + sum(counts)
    sos = seg.index(b"\xff\xda")
    ns = seg[sos + 4]
    sel = [seg[sos + 6 + 2 * c] >> 4 for c in range(ns)]
    p = sos + 2 + int.from_bytes(seg[sos + 2:sos + 4], "big")
    data = bytearray()
    while p < len(seg):
        if seg[p] == 0xFF:
            if seg[p + 1] != 0:
                break
            data.append(0xFF)  # a data 0xFF; its stuffed 0x00 is dropped
            p += 2
            continue
        data.append(seg[p])
        p += 1
    return [tables[t] for t in sel], np.unpackbits(np.frombuffer(bytes(data), np.uint8))


def _misses(seg, lead=LEAD):
    tabs, bits = _stream(seg)
    nf, nb = len(tabs), len(bits)

    def step(pos, ph):
        code = 0
        for length in range(1, 17):
            code = (code << 1) | (int(bits[pos + length - 1]) if pos + length - 1 < nb else 0)
            cat = tabs[ph].get((length, code))
            if cat is not None:
                return pos + length + (cat if 0 < cat < 16 else 0), (ph + 1) % nf
        return pos + 1, ph  # no code: one bit on, as the GPU paths do

    truth, pos, ph = set(), 0, 0
    for _ in range(256 * 256):
        truth.add(pos)
        pos, ph = step(pos, ph)
    chunks = range(2, nb // CHUNK)  # chunk 1 starts within the lead of the exact stream start
    miss = 0
    for c in chunks:
        pos, ph = c * CHUNK - lead, 0
        while pos < c * CHUNK:
            pos, ph = step(pos, ph)
        miss += pos not in truth
    return miss, len(chunks)


@pytest.mark.parametrize("tables", ["fixed", "per_component"])
@pytest.mark.parametrize("kind", ["noise", "smooth"])
def test_lead_paths_resynchronise(tables, kind):
    rng = np.random.default_rng(256)
    if kind == "noise":
        tile = rng.integers(0, 1024, (256, 256))
    else:
        tile = np.cumsum(rng.integers(-40, 41, (256, 256)), 1) % 1024
    seg = lj92_segment(tile.astype(np.uint16), 10, 2, tables)
    miss, n = _misses(seg)
    assert n > 100
    assert miss <= 0.01 * n, (miss, n)
    if tables == "per_component":
        # why the lead is this long: a quarter of it leaves far more chunks
        # unsynchronised under per-component tables
        short, _ = _misses(seg, LEAD // 4)
        assert short >= max(10, 5 * miss), (short, miss, n)
