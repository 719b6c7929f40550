"""DNG ingest, host side: the C parser (cpipe_dng_parse, no GPU) against the
oracle restatement of OpcodeListParser::parse, the reference unit test's
expectations (tests/unit/test_dng_reader.cpp), and seeded byte mutations; the
oracle's unpack against its own packer."""
import random

import numpy as np
import pytest

from cpipe_b200 import _abi
from cpipe_b200.dng import DngReader, parse
import oracle_dng as od
from dng_fixture import ASCII, LONG, SHORT, build_dng


def c_fields(info):
    rep = list(info.cfa_repeat)
    return {
        "width": info.width, "height": info.height, "bits_per_sample": info.bits_per_sample,
        "compression": info.compression, "strip_offset": info.strip_offset,
        "strip_byte_count": info.strip_byte_count, "orientation": info.orientation,
        "cfa_repeat": rep, "cfa_pattern": list(info.cfa_pattern)[:rep[0] * rep[1]],
        "black_level": [np.float32(v) for v in info.black_level], "white_level": info.white_level,
        "calibration_illuminant": list(info.calibration_illuminant), "has_matrix": list(info.has_matrix),
        "matrix": [[np.float32(v) for v in info.matrix[m]] for m in range(4)],
        "as_shot_neutral": [np.float32(v) for v in info.as_shot_neutral],
        "active_area": list(info.active_area) if info.has_active_area else None,
        "iso": info.iso, "exposure_time_ns": info.exposure_time_ns,
        "lens_aperture": np.float32(info.lens_aperture), "lens_focal_length_mm": np.float32(info.lens_focal_length_mm),
        "make": info.make.decode("latin-1"), "model": info.model.decode("latin-1"),
    }


def o_fields(info):
    out = {k: info[k] for k in ("width", "height", "bits_per_sample", "compression", "strip_offset",
                                "strip_byte_count", "orientation", "white_level", "calibration_illuminant",
                                "has_matrix", "active_area", "iso", "exposure_time_ns", "make", "model")}
    out["cfa_repeat"] = list(info["cfa_repeat"])
    out["cfa_pattern"] = list(info["cfa_pattern"])
    out["black_level"] = [np.float32(v) for v in info["black_level"]]
    out["matrix"] = [[np.float32(v) for v in m] for m in info["matrix"]]
    out["as_shot_neutral"] = [np.float32(v) for v in info["as_shot_neutral"]]
    out["lens_aperture"] = np.float32(info["lens_aperture"])
    out["lens_focal_length_mm"] = np.float32(info["lens_focal_length_mm"])
    return out


def check_same(data):
    st_c, info_c = parse(data)
    st_o, info_o = od.parse(data)
    assert st_c == st_o
    if st_c == od.OK:
        assert c_fields(info_c) == o_fields(info_o)
        lin = info_o["linearization"]
        assert info_c.linearization_count == len(lin)
        for name, i in (("opcode_list_1", 0), ("opcode_list_2", 1), ("opcode_list_3", 2)):
            off, n = info_o["blobs"].get(name, (0, 0))
            assert (info_c.opcode_list_offset[i], info_c.opcode_list_bytes[i]) == (off, n)
        assert (info_c.exif_offset, info_c.exif_bytes) == info_o["blobs"].get("exif", (0, 0))
        assert (info_c.xmp_offset, info_c.xmp_bytes) == info_o["blobs"].get("xmp", (0, 0))
        assert (info_c.icc_offset, info_c.icc_bytes) == info_o["blobs"].get("icc", (0, 0))
    return st_c, info_c


def test_reference_unit_expectations():
    """tests/unit/test_dng_reader.cpp 'decodes a synthetic Bayer DNG': fields and blobs."""
    data = build_dng()
    st, info = check_same(data)
    assert st == _abi.OK
    assert (info.width, info.height, info.bits_per_sample) == (4, 3, 16)
    assert list(info.cfa_repeat) == [2, 2] and list(info.cfa_pattern)[:4] == [0, 1, 1, 2]
    lin = np.frombuffer(data, "<u2", info.linearization_count, info.linearization_offset)
    assert lin.tolist() == [0, 128, 1024, 4095]
    assert all(info.has_matrix)
    assert info.iso == 400 and info.exposure_time_ns == 8_000_000
    assert info.lens_aperture == pytest.approx(1.7) and info.lens_focal_length_mm == pytest.approx(4.3)
    assert info.orientation == 1 and info.has_active_area and list(info.active_area) == [0, 0, 4, 3]
    assert info.exif_bytes and info.xmp_bytes and info.icc_bytes and all(info.opcode_list_bytes)
    assert list(info.black_level) == [64, 65, 66, 67] and info.white_level == 4095
    assert list(info.as_shot_neutral) == [1, 2, 3] and list(info.calibration_illuminant) == [21, 17]
    assert info.make == b"GoogleTest" and info.model == b"Pixel8UT"


def test_quad_bayer_cfa_preserved():
    """'preserves synthetic 4x4 Quad Bayer CFA metadata'."""
    pat = [0, 0, 1, 1, 0, 0, 1, 1, 1, 1, 2, 2, 1, 1, 2, 2]
    st, info = check_same(build_dng(width=8, height=8, cfa_repeat=(4, 4), cfa_pattern=pat))
    assert st == _abi.OK and list(info.cfa_repeat) == [4, 4] and list(info.cfa_pattern) == pat


@pytest.mark.parametrize("case,status", [
    (dict(include_cfa=False), _abi.UNSUPPORTED),
    (dict(cfa_repeat=(3, 3), cfa_pattern=[0] * 9), _abi.UNSUPPORTED),
    (dict(cfa_repeat=(2, 4), cfa_pattern=[0] * 8), _abi.UNSUPPORTED),
    (dict(cfa_pattern=(0, 1, 2)), _abi.UNSUPPORTED),
    (dict(overrides={262: (SHORT, [34892])}), _abi.UNSUPPORTED),
    (dict(overrides={277: (SHORT, [3])}), _abi.UNSUPPORTED),
    (dict(overrides={33421: (LONG, [2, 2])}), _abi.UNSUPPORTED),
    (dict(drop=(256,)), _abi.FAILED),
    (dict(overrides={258: (SHORT, [17])}), _abi.FAILED),
    (dict(strip_byte_count=0), _abi.FAILED),
    (dict(overrides={259: (SHORT, [7])}, drop=(273,)), _abi.FAILED),
    (dict(overrides={259: (SHORT, [7])}), _abi.OK),
    (dict(overrides={50717: (ASCII, "x")}), _abi.OK),
    (dict(include_opcode_lists=False, include_sidecars=False), _abi.OK),
])
def test_status_cases(case, status):
    st, _ = check_same(build_dng(**case))
    assert st == status


def test_bad_headers_and_tables():
    data = build_dng()
    for bad in (b"", data[:7], b"MM" + data[2:], data[:2] + b"\x2b\x00" + data[4:],
                data[:4] + (len(data) - 1).to_bytes(4, "little") + data[8:], data[:40]):
        st, _ = check_same(bad)
        assert st == _abi.FAILED


def test_non_bayer_read_fails_before_the_gpu():
    """'rejects non-Bayer DNG input': UNSUPPORTED from the parse, FAILED from the reader."""
    r = DngReader.read(build_dng(include_cfa=False))
    assert r.status == _abi.FAILED and r.buffer is None


def test_mutated_files_parse_alike():
    """Seeded single- and multi-byte mutations of the IFD and its values: the C
    parser and the oracle agree on status and every field."""
    rng = random.Random(20261204)
    base = build_dng(width=6, height=4, cfa_repeat=(2, 2))
    n_ok = 0
    for _ in range(3000):
        b = bytearray(base)
        for _ in range(rng.choice((1, 1, 2, 4))):
            pos = rng.randrange(0, min(len(b), 600))
            b[pos] = rng.randrange(256)
        st, _ = check_same(bytes(b))
        n_ok += st == _abi.OK
    assert n_ok > 100


@pytest.mark.parametrize("bits", list(range(1, 16)))
def test_oracle_pack_unpack_round_trip(bits):
    rng = np.random.default_rng(bits)
    for w, h in ((1, 1), (7, 3), (8, 2), (37, 5)):
        x = rng.integers(0, 1 << bits, (h, w), dtype=np.uint32).astype(np.uint16)
        strip = od.pack(x, bits)
        assert len(strip) == h * ((w * bits + 7) // 8)
        if len(strip) >= w * h * 2:
            continue  # as long as a 16-bit plane: read as words by rule
        assert np.array_equal(od.unpack(strip, w, h, bits), x)


def test_oracle_words_copy_semantics():
    """DngReader.cpp:145-164: min(plane, strip) bytes copied into a zeroed plane."""
    x = np.arange(12, dtype=np.uint16).reshape(3, 4) + 300
    full = x.astype("<u2").tobytes()
    assert np.array_equal(od.unpack(full, 4, 3, 16), x)
    short = od.unpack(full[:9], 4, 3, 16).ravel()
    assert short[:4].tolist() == x.ravel()[:4].tolist() and short[4] == (x.ravel()[4] & 0xFF)
    assert not short[5:].any()
    assert np.array_equal(od.unpack(full + b"\x01\x02", 4, 3, 12), x)  # >= a 16-bit plane: words


def test_subifd_raw_layout():
    """Camera / converter layout (IFD0 a preview, the raw in a SubIFD): the C
    parser and the oracle take the image tags from the SubIFD and the camera
    tags from IFD0, and agree with the same file in the reference's IFD0-only
    layout on every field but the preview-dependent offsets of inline values."""
    from cpipe_b200.dng_synth import lj92_tiles, subifd_dng
    flat = build_dng(width=70, height=48, bits=12)
    img = (np.arange(48 * 70).reshape(48, 70) * 7 % 4096).astype(np.uint16)
    tiled = build_dng(width=70, height=48, bits=12, tile=(32, 16), segments=lj92_tiles(img, 12, 32, 16))
    for base in (flat, tiled):
        st0, info0 = parse(base)
        assert st0 == od.OK
        moved = subifd_dng(base)
        st, info = check_same(moved)
        assert st == od.OK
        f0, f1 = c_fields(info0), c_fields(info)
        assert f0 == f1
        keys = ["seg_count", "seg_tiled", "seg_width", "seg_height", "linearization_offset", "exif_offset",
                "xmp_offset"]
        if base is tiled:  # out-of-line offset arrays stay put (a single strip's sits in its moved entry)
            keys += ["seg_offsets_pos", "seg_counts_pos"]
        for k in keys:
            assert getattr(info0, k) == getattr(info, k), k
        assert list(info0.opcode_list_offset) == list(info.opcode_list_offset)


def test_subifd_only_for_cfa_full_resolution():
    """IFD0 not a CFA image and no usable SubIFD: still UNSUPPORTED, as the
    reference reports it; a reduced-resolution (NewSubFileType 1) SubIFD is
    not taken."""
    import struct
    from cpipe_b200.dng_synth import subifd_dng
    moved = bytearray(subifd_dng(build_dng(width=8, height=6)))
    ifd0 = struct.unpack_from("<I", moved, 4)[0]
    n = struct.unpack_from("<H", moved, ifd0)[0]
    for k in range(n):
        e = ifd0 + 2 + 12 * k
        if struct.unpack_from("<H", moved, e)[0] == 330:
            raw_ifd = struct.unpack_from("<I", moved, e + 8)[0]
    m = struct.unpack_from("<H", moved, raw_ifd)[0]
    for k in range(m):
        e = raw_ifd + 2 + 12 * k
        if struct.unpack_from("<H", moved, e)[0] == 254:
            struct.pack_into("<I", moved, e + 8, 1)
    assert check_same(bytes(moved))[0] == od.UNSUPPORTED
    no_sub = build_dng(width=8, height=6, overrides={262: (SHORT, [2]), 277: (SHORT, [3])})
    assert check_same(no_sub)[0] == od.UNSUPPORTED
