"""Lossless JPEG (DNG Compression 7) on the CPU: the oracle codec's round
trips over predictors, component counts, bit depths and restart intervals;
the vectorised encoder equals the reference encoder byte for byte; the DNG
parse finds the segments of strip and tile files, and rejects a tile-only
file as the reference's parse does (it requires the strip tags,
OpcodeListParser.cpp:509-515)."""
import numpy as np
import oracle_dng as od
import oracle_lj92 as L
import pytest
from cpipe_b200 import _abi as A
from cpipe_b200 import dng
from cpipe_b200.dng_synth import build_dng


def smooth(h, w, bits, seed):
    rng = np.random.default_rng(seed)
    return (np.cumsum(rng.integers(-40, 41, (h, w)), 1) % (1 << bits)).astype(np.uint16)


@pytest.mark.parametrize("ps", range(1, 8))
@pytest.mark.parametrize("nf,bits,restart", [(2, 12, 0), (1, 16, 0), (4, 10, 0), (2, 14, 3), (2, 8, 5)])
def test_round_trip(ps, nf, bits, restart):
    for img in (smooth(12, 24, bits, ps), np.random.default_rng(ps).integers(0, 1 << bits, (12, 24)).astype(np.uint16)):
        assert np.array_equal(L.decode(L.encode(img, bits, ps, nf, restart), 24, 12), img)


def test_fast_encoder_is_the_same_codec():
    for bits, nf in ((12, 2), (16, 2), (10, 4)):
        img = smooth(20, 32, bits, bits)
        assert L.encode_fast(img, bits, nf) == L.encode(img, bits, 1, nf)


def test_tiles_with_cropped_edges():
    img = smooth(70, 100, 12, 1)
    assert np.array_equal(L.decode_tiles(L.encode_tiles(img, 12, 32, 16), 100, 70, 32, 16), img)


def test_parse_finds_segments():
    img = smooth(48, 70, 12, 2)
    strips = build_dng(width=70, height=48, bits=12, rows_per_strip=16,
                       segments=[L.encode(img[r:r + 16], 12) for r in range(0, 48, 16)])
    st, info = dng.parse(strips)
    assert st == A.OK and info.compression == 7 and not info.seg_tiled
    assert (info.seg_width, info.seg_height, info.seg_count) == (70, 16, 3)
    tiles = build_dng(width=70, height=48, bits=12, tile=(32, 16), segments=L.encode_tiles(img, 12, 32, 16))
    st, info = dng.parse(tiles)
    assert st == A.OK and info.seg_tiled and (info.seg_width, info.seg_height, info.seg_count) == (32, 16, 9)
    only_tiles = build_dng(width=70, height=48, bits=12, tile=(32, 16), strip_tags=False,
                           segments=L.encode_tiles(img, 12, 32, 16))
    assert dng.parse(only_tiles)[0] == A.FAILED
    assert od.parse(only_tiles)[0] == A.FAILED


def test_writer_segments_round_trip():
    """The package's lossless-JPEG writer (dng_synth.lj92_segment, used for
    benchmark files) decodes back exactly through the oracle decoder."""
    import numpy as np
    import oracle_lj92 as O
    from cpipe_b200.dng_synth import lj92_segment
    rng = np.random.default_rng(11)
    for h, w, bits, nf in [(16, 32, 12, 2), (7, 10, 16, 2), (9, 9, 10, 1), (40, 64, 14, 2), (12, 24, 12, 4)]:
        noise = rng.integers(0, 1 << bits, (h, w)).astype(np.uint16)
        ramp = (np.add.outer(np.arange(h), 3 * np.arange(w)) % (1 << bits)).astype(np.uint16)
        flat = np.full((h, w), 7, np.uint16)
        for img in (noise, ramp, flat):
            for tables in ("fixed", "per_component"):
                got = np.asarray(O.decode(lj92_segment(img, bits, nf, tables), w, h)).reshape(h, w)
                np.testing.assert_array_equal(got, img)


def test_writer_per_component_tables_differ():
    """Per-component tables come from each component's own statistics: a
    noisy and a flat component get different code lengths, and the scan
    selects table c for component c."""
    import numpy as np
    from cpipe_b200.dng_synth import lj92_segment
    rng = np.random.default_rng(5)
    img = np.zeros((32, 64), np.uint16)
    img[:, 0::2] = rng.integers(0, 4096, (32, 32))
    img[:, 1::2] = 100
    seg = lj92_segment(img, 12, 2, "per_component")
    dht = seg.index(b"\xff\xc4")
    n = int.from_bytes(seg[dht + 2:dht + 4], "big")
    body = seg[dht + 4:dht + 2 + n]
    t0_total = sum(body[1:17])
    t1 = body[17 + t0_total:]
    assert body[0] == 0 and t1[0] == 1 and body[1:17] != t1[1:17]
    sos = seg.index(b"\xff\xda")
    assert seg[sos + 5:sos + 9] == bytes((1, 0x00, 2, 0x10))
