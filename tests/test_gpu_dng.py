"""DNG ingest on the GPU: cpipe_cuda_dng_decode / cpipe_cuda_dng_unpack against
the oracle restatement of DngReader::read (bit-exact), at the reference fixture's
4x3 frame, ragged widths, every packed depth, and 12 MP frames (pack -> unpack
round trips)."""
import ctypes as C

import numpy as np
import pytest
import torch

from cpipe_b200 import _abi
from cpipe_b200.dng import DngReader

import oracle_dng as od
from dng_fixture import SHORT, build_dng

pytestmark = pytest.mark.gpu


def decode(data, out_elems=None, offset_elems=0):
    st, info = od.parse(data)
    w, h = info["width"], info["height"]
    n = w * h if out_elems is None else out_elems
    m = n + offset_elems + 8  # even: n + offset + 8 rounded below
    m += m % 2
    # 0xBEEF in every 16-bit element: untouched samples are recognisable.
    buf = torch.full((m // 2,), -1091584273, dtype=torch.int32, device="cuda").view(torch.uint16)
    L = _abi.lib()
    L.cpipe_cuda_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    dinfo = _abi.DngInfo()
    ptr = buf.data_ptr() + 2 * offset_elems
    rc = L.cpipe_cuda_dng_decode(data, len(data), C.c_void_p(ptr), 2 * n, C.byref(dinfo))
    torch.cuda.synchronize()
    host = buf.cpu().view(torch.int16).numpy().view(np.uint16)
    return rc, host[offset_elems:offset_elems + w * h].reshape(h, w) if rc == 0 else None, host


def test_reference_fixture_pixels():
    """test_dng_reader.cpp: the 4x3 frame reads back as 64, 73, ..., 163."""
    r = DngReader.read(build_dng())
    assert r.status == _abi.OK
    assert r.buffer.shape == (3, 4) and r.buffer.dtype == torch.uint16
    got = r.buffer.cpu().view(torch.int16).numpy().view(np.uint16).ravel().tolist()
    assert got == [64 + 9 * i for i in range(12)]
    md = r.metadata
    assert md["cs_role"] == "raw_camera" and md["calibration"]["linearization_table"] == [0, 128, 1024, 4095]
    assert md["capture"]["iso"] == 400 and md["capture"]["exposure_time_ns"] == 8_000_000
    assert set(md["ext_blobs"]) == {f"com.cpipe.dng.opcode_list_{i}_bytes" for i in (1, 2, 3)}
    assert md["exif_blob"] and md["xmp_blob"] and md["icc_blob"] and md["active_area"]["width"] == 4


@pytest.mark.parametrize("w,h", [(4, 3), (1, 1), (7, 5), (37, 9), (1920, 1080)])
@pytest.mark.parametrize("offset", [0, 1])
def test_words_match_oracle(w, h, offset):
    rng = np.random.default_rng(w * 31 + h)
    x = rng.integers(0, 1 << 16, (h, w), dtype=np.uint32).astype(np.uint16)
    data = build_dng(width=w, height=h, pixels=x)
    rc, got, _ = decode(data, offset_elems=offset)
    assert rc == _abi.OK
    assert np.array_equal(got, od.read(data)[1]) and np.array_equal(got, x)


@pytest.mark.parametrize("cut", [1, 2, 17, 333])
def test_short_strip_zero_fill(cut):
    """A strip shorter than the plane: its bytes, then zeros (odd cuts too)."""
    w, h = 64, 9
    x = np.random.default_rng(cut).integers(0, 65536, (h, w), dtype=np.uint32).astype(np.uint16)
    strip = x.astype("<u2").tobytes()[:-cut]
    data = build_dng(width=w, height=h, strip=strip)
    rc, got, _ = decode(data)
    assert rc == _abi.OK
    assert np.array_equal(got, od.read(data)[1])


@pytest.mark.parametrize("bits", list(range(1, 16)))
def test_packed_depths_match_oracle(bits):
    rng = np.random.default_rng(100 + bits)
    for w, h in ((37, 9), (64, 8), (1001, 3)):
        x = rng.integers(0, 1 << bits, (h, w), dtype=np.uint32).astype(np.uint16)
        strip = od.pack(x, bits)
        if len(strip) >= w * h * 2:
            continue
        data = build_dng(width=w, height=h, strip=strip, overrides={258: (SHORT, [bits])})
        for offset in (0, 1):
            rc, got, _ = decode(data, offset_elems=offset)
            assert rc == _abi.OK
            assert np.array_equal(got, od.read(data)[1]) and np.array_equal(got, x)


def test_packed_short_strip_matches_oracle():
    w, h, bits = 100, 7, 12
    x = np.random.default_rng(5).integers(0, 4096, (h, w), dtype=np.uint32).astype(np.uint16)
    strip = od.pack(x, bits)[:-61]
    data = build_dng(width=w, height=h, strip=strip, overrides={258: (SHORT, [bits])})
    rc, got, _ = decode(data)
    assert rc == _abi.OK and np.array_equal(got, od.read(data)[1])


@pytest.mark.parametrize("bits", [10, 12, 14, 16])
def test_12mp_round_trip(bits):
    """Full 4032x3024 frames: decode(pack(x)) == x, and the plane ends exactly."""
    w, h = 4032, 3024
    x = np.random.default_rng(bits).integers(0, 1 << bits, (h, w), dtype=np.uint32).astype(np.uint16)
    strip = x.astype("<u2").tobytes() if bits == 16 else od.pack(x, bits)
    data = build_dng(width=w, height=h, strip=strip, overrides={258: (SHORT, [bits])})
    rc, got, host = decode(data)
    assert rc == _abi.OK and np.array_equal(got, x)
    assert (host[w * h:] == 0xBEEF).all()  # nothing written past the plane


@pytest.mark.parametrize("w,h,bits", [(4032, 3024, 12), (1001, 7, 10), (333, 5, 14), (64, 3, 7)])
@pytest.mark.parametrize("strip_offset", [0, 1, 3])
def test_unpack_from_device_strip(w, h, bits, strip_offset):
    """Aligned strips take the word-load path, misaligned ones the byte path; both exact."""
    x = np.random.default_rng(9 + bits).integers(0, 1 << bits, (h, w), dtype=np.uint32).astype(np.uint16)
    packed = od.pack(x, bits)
    buf = torch.zeros(len(packed) + 16, dtype=torch.uint8, device="cuda")
    buf[strip_offset:strip_offset + len(packed)] = torch.from_numpy(np.frombuffer(packed, np.uint8).copy()).cuda()
    out = torch.empty((h, w), dtype=torch.uint16, device="cuda")
    L = _abi.lib()
    L.cpipe_cuda_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    rc = L.cpipe_cuda_dng_unpack(C.c_void_p(buf.data_ptr() + strip_offset), len(packed), w, h, bits,
                                 C.c_void_p(out.data_ptr()))
    torch.cuda.synchronize()
    assert rc == _abi.OK
    assert np.array_equal(out.cpu().view(torch.int16).numpy().view(np.uint16), x)


def test_error_statuses():
    L = _abi.lib()
    data = build_dng()
    rc, _, host = decode(data, out_elems=11)  # one sample short
    assert rc == _abi.BAD_INDEX and (host == 0xBEEF).all()
    # Compression 7 whose strip is not a lossless JPEG stream: the decode fails
    rc, _, _ = decode(build_dng(overrides={259: (SHORT, [7])}))
    assert rc == _abi.FAILED and L.cpipe_cuda_last_error()
    # any other compression (8 = Deflate) is left to the caller
    rc, _, _ = decode(build_dng(overrides={259: (SHORT, [8])}))
    assert rc == _abi.UNSUPPORTED and b"lossless JPEG" in L.cpipe_cuda_last_error()
    rc, _, _ = decode(build_dng(strip_byte_count=10 ** 6))  # strip past the end of the file
    assert rc == _abi.FAILED
    assert DngReader.read(build_dng(include_cfa=False)).status == _abi.FAILED
    assert DngReader.read("/nonexistent/frame.dng").status == _abi.FAILED


def test_dng_input_node(host, tmp_path):
    """com.cpipe.builtin.dng_input (dng_input.cpp:17-40): the file at "path"
    decoded on the GPU into the host's R16_UINT output, the reader's metadata
    attached; status codes for a missing path, a missing file and an output of
    the wrong extent."""
    import ctypes as C
    from cpipe_b200 import _abi as A
    from cpipe_b200.dng_synth import build_dng
    rng = np.random.default_rng(11)
    px = rng.integers(0, 4096, (48, 64)).astype(np.uint16)
    path = tmp_path / "frame.dng"
    path.write_bytes(build_dng(width=64, height=48, pixels=px))
    out = host.buffer(A.FMT_R16_UINT, 64, 48)
    st = host.run_node("com.cpipe.builtin.dng_input", [], [out], {"path": str(path)})
    assert st == 0, host.last_error()
    np.testing.assert_array_equal(out.download(), px)
    L = A.lib()
    assert L.cpipe_b200_buffer_cs_role(out._h).decode() == "raw_camera"
    has, rep, pat = C.c_int(), (C.c_uint8 * 2)(), (C.c_uint8 * 16)()
    assert L.cpipe_b200_buffer_get_cfa(out._h, C.byref(has), rep, pat) == 0
    assert has.value == 1 and list(rep) == [2, 2] and list(pat)[:4] == [0, 1, 1, 2]
    ptr, n = C.c_void_p(), C.c_size_t()
    assert L.cpipe_b200_buffer_get_blob(out._h, b"com.cpipe.dng.opcode_list_2_bytes", C.byref(ptr), C.byref(n)) == 0
    assert n.value == 8
    # the decoded frame feeds the rest of the raw path: linearize -> black level
    lin = host.buffer(A.FMT_R32_SFLOAT, 64, 48)
    assert host.run_node("com.cpipe.linearize.dng_lut", [out], [lin]) == 0, host.last_error()
    table = np.array([0, 128, 1024, 4095], np.float32)
    np.testing.assert_array_equal(lin.download(), table[np.minimum(px, 3)])
    assert host.run_node("com.cpipe.builtin.dng_input", [], [out], {}) == A.NEED_PARAM
    assert host.run_node("com.cpipe.builtin.dng_input", [], [out], {"path": str(tmp_path / "none.dng")}) == A.FAILED
    wrong = host.buffer(A.FMT_R16_UINT, 32, 48)
    assert host.run_node("com.cpipe.builtin.dng_input", [], [wrong], {"path": str(path)}) == A.BAD_INDEX
