"""Lossless JPEG (DNG Compression 7) decoded on the GPU (cpipe_cuda_lj92_decode
and the Compression 7 branch of cpipe_cuda_dng_decode) against the oracle
codec: every predictor, 1/2/4 components, 8-16 bits, restart intervals, tiles
cropped at the image edges, strip files, a 12 MP tiled frame; malformed
streams fail with CPIPE_FAILED."""
import ctypes as C

import numpy as np
import oracle_lj92 as L
import pytest
from cpipe_b200 import _abi as A
from cpipe_b200.dng_synth import build_dng

pytestmark = pytest.mark.gpu


def smooth(h, w, bits, seed):
    rng = np.random.default_rng(seed)
    return (np.cumsum(rng.integers(-40, 41, (h, w)), 1) % (1 << bits)).astype(np.uint16)


def gpu_decode(segs, across, sw, sh, w, h):
    Lb = A.lib()
    out = C.c_void_p()
    assert Lb.cpipe_cuda_device_alloc(w * h * 2, C.byref(out)) == 0
    keep = [C.create_string_buffer(s, len(s)) for s in segs]
    ptrs = (C.c_void_p * len(segs))(*[C.addressof(k) for k in keep])
    sizes = (C.c_size_t * len(segs))(*[len(s) for s in segs])
    st = Lb.cpipe_cuda_lj92_decode(ptrs, sizes, len(segs), across, sw, sh, w, h, out)
    img = np.zeros((h, w), np.uint16)
    if st == 0:
        assert Lb.cpipe_cuda_memcpy_d2h(img.ctypes.data, out, img.nbytes) == 0
    Lb.cpipe_cuda_device_free(out)
    return st, img


def dng_decode(data, w, h):
    Lb = A.lib()
    out = C.c_void_p()
    assert Lb.cpipe_cuda_device_alloc(w * h * 2, C.byref(out)) == 0
    st = Lb.cpipe_cuda_dng_decode(data, len(data), out, w * h * 2, None)
    img = np.zeros((h, w), np.uint16)
    assert Lb.cpipe_cuda_synchronize() == 0
    if st == 0:
        assert Lb.cpipe_cuda_memcpy_d2h(img.ctypes.data, out, img.nbytes) == 0
    Lb.cpipe_cuda_device_free(out)
    return st, img


@pytest.mark.parametrize("ps", range(1, 8))
@pytest.mark.parametrize("nf,bits,restart", [(2, 12, 0), (1, 16, 0), (4, 10, 0), (2, 14, 7), (2, 8, 5)])
def test_stream_matches_oracle(cuda_device, ps, nf, bits, restart):
    img = np.vstack([smooth(16, 48, bits, ps), np.random.default_rng(ps).integers(0, 1 << bits, (8, 48))]).astype(np.uint16)
    seg = L.encode(img, bits, ps, nf, restart)
    want = L.decode(seg, 48, 24)
    st, got = gpu_decode([seg], 1, 48, 24, 48, 24)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(got, img)


@pytest.mark.parametrize("w,h,tw,th", [(100, 70, 32, 16), (64, 64, 64, 64), (257, 129, 128, 64), (33, 17, 16, 8)])
def test_tiles_cropped(cuda_device, w, h, tw, th):
    img = smooth(h, w, 12, w + h)
    segs = L.encode_tiles(img, 12, tw, th)
    st, got = gpu_decode(segs, (w + tw - 1) // tw, tw, th, w, h)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)


def test_dng_files(cuda_device):
    img = smooth(48, 70, 12, 3)
    strips = build_dng(width=70, height=48, bits=12, rows_per_strip=16,
                       segments=[L.encode(img[r:r + 16], 12, 6) for r in range(0, 48, 16)])
    st, got = dng_decode(strips, 70, 48)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)
    tiles = build_dng(width=70, height=48, bits=12, tile=(32, 16), segments=L.encode_tiles(img, 12, 32, 16))
    st, got = dng_decode(tiles, 70, 48)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)


def test_12mp_tiled_round_trip(cuda_device):
    img = smooth(3024, 4032, 12, 12)
    data = build_dng(width=4032, height=3024, bits=12, tile=(256, 256), segments=L.encode_tiles_fast(img, 12, 256, 256))
    st, got = dng_decode(data, 4032, 3024)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)


def test_malformed_streams_fail(cuda_device):
    img = smooth(16, 32, 12, 9)
    seg = bytearray(L.encode(img, 12, 1, 2))
    sos = bytes(seg).index(b"\xff\xda")
    start = sos + 2 + int.from_bytes(seg[sos + 2:sos + 4], "big")
    # the all-ones code is never assigned: a run of stuffed 0xFF bytes cannot decode
    bad = bytes(seg[:start]) + b"\xff\x00" * 64 + b"\xff\xd9"
    assert gpu_decode([bad], 1, 32, 16, 32, 16)[0] == A.FAILED
    assert gpu_decode([bytes(seg[:start - 3])], 1, 32, 16, 32, 16)[0] == A.FAILED  # scan header cut
    assert gpu_decode([b"\x00\x01" + bytes(seg[2:])], 1, 32, 16, 32, 16)[0] == A.FAILED  # no SOI
    rst = bytearray(L.encode(img, 12, 1, 2, restart=4))
    k = bytes(rst).index(b"\xff\xd0")
    assert gpu_decode([bytes(rst[:k] + rst[k + 2:])], 1, 32, 16, 32, 16)[0] == A.FAILED  # restart marker removed
    # more samples than the segment holds
    assert gpu_decode([bytes(seg)], 1, 16, 16, 16, 16)[0] == A.FAILED


def _entropy_span(seg):
    """(start, end) of the entropy-coded bytes of a one-scan stream."""
    sos = bytes(seg).index(b"\xff\xda")
    start = sos + 2 + int.from_bytes(seg[sos + 2:sos + 4], "big")
    return start, len(seg) - 2  # EOI closes the stream


def _stats():
    """(chunks, chunks decoded again by the write walks, parallel segments,
    sequential segments) of the last decode."""
    f = (C.c_uint64 * 9)()
    assert A.lib().cpipe_cuda_lj92_last_stats(f, 9) == 0
    return f[0], f[6], f[1], f[2]


@pytest.mark.parametrize("tables", ["fixed", "per_component"])
def test_12mp_tiled_writer_tables(cuda_device, tables):
    """The benchmark layout (256x256 tiles, two components per JPEG line),
    with one table and with a table per component as DNG writers emit:
    bit-exact, every segment on the parallel path, and speculative paths
    that start at the true state of almost every chunk."""
    from cpipe_b200.dng_synth import lj92_tiles
    img = np.random.default_rng(7).integers(0, 1024, (3024, 4032)).astype(np.uint16)
    img[:1500] = smooth(1500, 4032, 10, 8)
    segs = lj92_tiles(img, 10, 256, 256, 2, tables)
    st, got = gpu_decode(segs, 16, 256, 256, 4032, 3024)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)
    chunks, redecodes, npar, nser = _stats()
    assert (npar, nser) == (len(segs), 0)
    assert chunks > 10000 and redecodes < (0.001 if tables == "fixed" else 0.05) * chunks


@pytest.mark.parametrize("tables", ["fixed", "per_component"])
def test_single_segment_frame(cuda_device, tables):
    """A whole 12 MP frame in one stream (one strip): thousands of chunk
    groups chained by one warp."""
    from cpipe_b200.dng_synth import lj92_segment
    rng = np.random.default_rng(12)
    img = smooth(3024, 4032, 14, 5)
    img[2000:] = rng.integers(0, 1 << 14, (1024, 4032))
    seg = lj92_segment(img, 14, 2, tables)
    st, got = gpu_decode([seg], 1, 4032, 3024, 4032, 3024)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)
    assert _stats()[2] == 1


@pytest.mark.parametrize("nf", [1, 2, 3, 4])
@pytest.mark.parametrize("bits", [8, 12, 16])
def test_components_and_depths_parallel(cuda_device, nf, bits):
    """Per-component tables with 1-4 components and 8-16 bits, noisy enough
    that the stream spans many chunks."""
    from cpipe_b200.dng_synth import lj92_segment
    rng = np.random.default_rng(nf * 100 + bits)
    img = rng.integers(0, 1 << bits, (96, 120 * nf)).astype(np.uint16)
    img[:40] = smooth(40, 120 * nf, bits, nf)
    seg = lj92_segment(img, bits, nf, "per_component")
    st, got = gpu_decode([seg], 1, 120 * nf, 96, 120 * nf, 96)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)


def test_short_long_and_empty_streams(cuda_device):
    """Streams that end early (zeros past the data, as a sequential decoder
    reads), carry bytes after the last sample, or hold no data at all: the
    same samples as the oracle decoder."""
    img = np.random.default_rng(3).integers(0, 4096, (64, 128)).astype(np.uint16)
    seg = bytes(L.encode(img, 12, 1, 2))
    start, end = _entropy_span(seg)
    cut = seg[:start + (end - start) // 2]
    if cut.endswith(b"\xff"):
        cut = cut[:-1]
    cases = {
        "short": cut + b"\xff\xd9",
        "long": seg[:end] + bytes(range(1, 200)) + b"\xff\xd9",
        "empty": seg[:start] + b"\xff\xd9",
        "no_eoi": seg[:end],
    }
    for name, s in cases.items():
        want = L.decode(s, 128, 64)
        st, got = gpu_decode([s], 1, 128, 64, 128, 64)
        assert st == 0, (name, A.lib().cpipe_cuda_last_error())
        np.testing.assert_array_equal(got, want, err_msg=name)


def test_invalid_code_mid_stream_fails(cuda_device):
    """64 one bits in the middle of a long stream hold no code on any path:
    the parallel decoder reports the segment as not decoding."""
    img = smooth(512, 512, 12, 4)
    seg = bytes(L.encode(img, 12, 1, 2))
    start, end = _entropy_span(seg)
    mid = start + (end - start) // 2
    while seg[mid - 1] == 0xFF:
        mid += 1
    bad = seg[:mid] + b"\xff\x00" * 8 + seg[mid:]
    assert gpu_decode([bad], 1, 512, 512, 512, 512)[0] == A.FAILED


def test_subifd_files(cuda_device):
    """Camera / converter layout (IFD0 a preview, the raw in a SubIFD), with
    an uncompressed strip and with lossless-JPEG tiles: the raw decodes."""
    from cpipe_b200.dng_synth import lj92_tiles, subifd_dng
    img = smooth(48, 70, 12, 21)
    tiled = build_dng(width=70, height=48, bits=12, tile=(32, 16),
                      segments=lj92_tiles(img, 12, 32, 16, 2, "per_component"))
    st, got = dng_decode(subifd_dng(tiled), 70, 48)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)
    flat = build_dng(width=70, height=48, pixels=img)
    st, got = dng_decode(subifd_dng(flat), 70, 48)
    assert st == 0, A.lib().cpipe_cuda_last_error()
    np.testing.assert_array_equal(got, img)
