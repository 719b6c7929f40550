"""CPU-only checks of the C-ABI library: it loads without a GPU, exports every
symbol include/*.h declares, registers the reference node ids with the
reference ABI version and manifests, and its host-side parsers / loaders
produce the reference packings.  No kernel is launched here."""
import ctypes as C
import os
import re
import struct

import numpy as np
import pytest
from conftest import ROOT
from cpipe_b200 import Registry, _abi, blobs

INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for f in os.listdir(INCLUDE):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(INCLUDE, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", src)
        names |= set(re.findall(r"\b(cpipe_(?:cuda|b200|surrogate|dng)_\w+)\s*\(", src))
        names |= set(re.findall(r"CPIPE_CUDA_PARAM_FILTER\((\w+)\)", open(os.path.join(INCLUDE, f)).read()))
    return names - {"cpipe_cuda_filter_desc", "name"}


def test_library_exports_every_declared_symbol():
    L = _abi.lib()
    declared = declared_functions()
    assert len(declared) >= 60
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert set(_abi.EXPORTS) == declared


def test_no_device_means_no_cpu_fallback():
    """Without a GPU the filters report an error instead of computing on the CPU."""
    L = _abi.lib()
    if L.cpipe_cuda_device_count() > 0:
        pytest.skip("a CUDA device is visible")
    from cpipe_b200 import call_filter, last_error
    x = np.ones((4, 4), np.float32)
    st = call_filter("blacklevel_dng_levels", [x], [np.zeros_like(x)], blobs.blacklevel([0] * 4, 10, (0, 1, 1, 2)))
    assert st == _abi.INTERNAL_ERROR
    assert "no CUDA device" in last_error()


EXPECTED_NODES = {
    # id: (input port, output port, params)
    "com.cpipe.precision_convert": ("in", "out", ["target_format"]),
    "com.cpipe.linearize.dng_lut": ("raw", "bayer", []),
    "com.cpipe.blacklevel.dng_levels": ("bayer", "bayer", []),
    "com.cpipe.lens.shading_gainmap": ("linear_bayer", "corrected_bayer", []),
    "com.cpipe.demosaic.rcd": ("bayer", "rgba", ["algorithm"]),
    "com.cpipe.demosaic.amaze": ("bayer", "rgba", ["algorithm"]),
    "com.cpipe.demosaic.bilinear": ("bayer", "rgba", []),
    "com.cpipe.demosaic.quad_bayer_remosaic": ("qbc", "bayer", []),
    "com.cpipe.wb.dual_illuminant": ("rgb", "rgb", []),
    "com.cpipe.colormatrix.dng_to_working": ("rgb", "rgb", []),
    # sigma, sigma_override as the reference; algorithm and stages select the
    # two-stage BM3D extension (default "box2x2" is the reference computation).
    "com.cpipe.denoise.bm3d": ("rgb", "rgb", ["sigma", "sigma_override", "algorithm", "stages"]),
    "com.cpipe.denoise.guided_filter": ("rgb", "rgb", ["radius", "eps", "algorithm"]),
    "com.cpipe.denoise.wavelet_bayes_shrink": ("rgb", "rgb", ["chroma_strength", "algorithm", "levels", "luma_strength", "sigma"]),
    "com.cpipe.lens.dng_opcode_list_3": ("scene_rgb", "corrected_rgb", []),
    "com.cpipe.color.3d_lut": ("rgb", "rgb", ["lut_path", "interpolation"]),
    "com.cpipe.tone.filmic_rgb": ("rgb", "rgb", ["ev", "contrast", "saturation", "highlights", "shadows"]),
    "com.cpipe.wb.greyworld_auto": ("rgb", "rgb", []),
    "com.cpipe.tone.mertens_local": (("under", "normal", "over"), "rgb",
                                     ["weight_contrast", "weight_saturation", "weight_well_exposedness"]),
    "com.cpipe.tone.aces_filmic": ("rgb", "rgb", ["toggle"]),
    "com.cpipe.tone.reinhard": ("rgb", "rgb", ["white_point"]),
    "com.cpipe.sharpen.edge_aware_usm": ("rgb", "rgb", ["strength", "radius", "threshold"]),
    "com.cpipe.color.scene_linear_to_display": ("rgb", "display", ["target"]),
    "com.cpipe.builtin.dng_input": ((), "raw", ["path"]),
}


def test_registry_and_manifests():
    reg = Registry()
    assert reg.load_builtin_nodes() == len(EXPECTED_NODES)
    assert set(reg.ids()) == set(EXPECTED_NODES)
    for node_id, (pin, pout, params) in EXPECTED_NODES.items():
        d = reg.find(node_id)
        assert d.abi == (0, 4) and d.version == "1.0.0"
        m = d.manifest
        assert m["id"] == node_id
        ins = [p["name"] for p in m["ports"] if p["kind"] == "in"]
        outs = [p["name"] for p in m["ports"] if p["kind"] == "out"]
        assert ins == (list(pin) if isinstance(pin, tuple) else [pin]) and outs == [pout], node_id
        # the reference's output layouts need a single precision per output port
        # (Pipeline.cpp:162-171), display excepted (it picks by its target)
        out_prec = [p["caps"]["precision"] for p in m["ports"] if p["kind"] == "out"][0]
        assert len(out_prec) == 1 or node_id in ("com.cpipe.precision_convert",
                                                 "com.cpipe.color.scene_linear_to_display"), node_id
        assert [p["name"] for p in m["params"]] == params, node_id
        assert m["compute"]["device"] == "CUDA"


def test_main_entry_actions_without_gpu():
    """describe / create / destroy / prepare need no device; process rejects bad contexts."""
    reg = Registry()
    reg.load_builtin_nodes()
    L = _abi.lib()
    host = L.cpipe_b200_host_abi(None)
    assert host is None
    desc = L.cpipe_b200_find_node(b"com.cpipe.denoise.bm3d").contents
    assert desc.main_entry(b"describe", None, None, None, None, None) == _abi.REPLY_DEFAULT
    inst = C.c_void_p()
    assert desc.main_entry(b"create", None, None, None, None, C.addressof(inst)) == _abi.OK
    assert inst.value
    assert desc.main_entry(b"prepare", None, None, None, None, None) == _abi.OK
    assert desc.main_entry(b"process", None, None, None, None, None) == _abi.BAD_INDEX
    assert desc.main_entry(b"destroy", None, None, None, inst, None) == _abi.OK


def test_pack_gain_maps_from_opcode_list_2():
    """OpcodeList2 parse + pack equals the dispatch layout the filter reads
    (shading_gainmap.cpp:96-137)."""
    L = _abi.lib()
    stream = blobs.opcode_list_2_with_gain_maps([blobs.gain_map_params(2, 2, 0, 1, 2.0, 2.0, [1, 2, 3, 5])])
    n = C.c_size_t(0)
    rep = (C.c_uint8 * 2)(2, 2)
    pat = (C.c_uint8 * 16)(0, 1, 1, 2)
    assert L.cpipe_b200_pack_gain_maps(stream, len(stream), rep, pat, None, C.byref(n)) == _abi.OK
    buf = C.create_string_buffer(n.value)
    assert L.cpipe_b200_pack_gain_maps(stream, len(stream), rep, pat, buf, C.byref(n)) == _abi.OK
    expect = blobs.gainmap_dispatch([dict(points_v=2, points_h=2, spacing_v=2.0, spacing_h=2.0, gains=[1, 2, 3, 5])])
    got = buf.raw
    # the header's cfa_pattern bytes 4..: same; planes carry top/left/bottom/right = 0,0,2,2
    assert got == expect
    # truncated / unsupported shapes
    bad = stream[:-4]
    assert L.cpipe_b200_pack_gain_maps(bad, len(bad), rep, pat, None, C.byref(n)) == _abi.FAILED
    three = blobs.opcode_list_2_with_gain_maps([blobs.gain_map_params(1, 1, p, 4, 1.0, 1.0, [1.0]) for p in range(3)])
    assert L.cpipe_b200_pack_gain_maps(three, len(three), rep, pat, None, C.byref(n)) == _abi.UNSUPPORTED
    planes2 = blobs.opcode_list_2_with_gain_maps([blobs.gain_map_params(1, 1, 0, 2, 1.0, 1.0, [1.0])])
    assert L.cpipe_b200_pack_gain_maps(planes2, len(planes2), rep, pat, None, C.byref(n)) == _abi.UNSUPPORTED
    other = blobs.opcode_list([(1, b"\x00" * 8)])  # non-GainMap opcodes are skipped
    assert L.cpipe_b200_pack_gain_maps(other, len(other), rep, pat, None, C.byref(n)) == _abi.NEED_METADATA


def test_pack_opcode_list_3():
    L = _abi.lib()
    stream = blobs.opcode_list([
        (1, blobs.warp_rectilinear_params([(1.0, -0.08, 0.02, 0.0, 0.0, 0.0)])),
        (3, blobs.fix_vignette_radial_params([0.5])),
        (4, blobs.fix_bad_pixels_constant_params(7)),
        (5, blobs.fix_bad_pixels_list_params(points=[(3, 4)], rects=[(0, 1, 2, 3)])),
        (6, blobs.trim_bounds_params(1, 2, 30, 40)),
    ])
    n, cnt = C.c_size_t(1 << 16), C.c_uint32()
    buf = C.create_string_buffer(n.value)
    assert L.cpipe_b200_pack_opcode_list_3(stream, len(stream), buf, C.byref(n), C.byref(cnt)) == _abi.OK
    assert cnt.value == 5
    raw = buf.raw[:n.value]
    hd = _abi.Opcode3DispatchHeader.from_buffer_copy(raw[:8])
    assert hd.opcode_count == 5
    recs = [_abi.Opcode3DispatchRecord.from_buffer_copy(raw[8 + 320 * i: 8 + 320 * (i + 1)]) for i in range(5)]
    assert [r.id for r in recs] == [1, 3, 4, 5, 6]
    assert recs[0].coefficient_count == 1 and recs[0].coefficients[0].kr1 == -0.08 and recs[0].cx_hat == 0.5
    assert recs[1].vignette_k[0] == 0.5 and recs[2].constant == 7
    assert recs[3].point_count == 1 and recs[3].rect_count == 1
    assert (recs[4].top, recs[4].left, recs[4].bottom, recs[4].right) == (1, 2, 30, 40)
    tail = raw[8 + 320 * 5:]
    assert struct.unpack("<II", tail[:8]) == (3, 4) and struct.unpack("<IIII", tail[8:24]) == (0, 1, 2, 3)
    # mandatory unknown -> UNSUPPORTED; optional unknown kept as id 0; bad sizes -> FAILED
    unk = blobs.opcode_list([(99, b"")])
    assert L.cpipe_b200_pack_opcode_list_3(unk, len(unk), None, C.byref(n), C.byref(cnt)) == _abi.UNSUPPORTED
    opt = blobs.opcode_list([(99, b"")], flags=1)
    assert L.cpipe_b200_pack_opcode_list_3(opt, len(opt), None, C.byref(n), C.byref(cnt)) == _abi.OK and cnt.value == 1
    badw = blobs.opcode_list([(3, b"\x00" * 48)])
    assert L.cpipe_b200_pack_opcode_list_3(badw, len(badw), None, C.byref(n), C.byref(cnt)) == _abi.FAILED


def test_cube_loader(tmp_path):
    L = _abi.lib()
    S = 5
    vals = np.random.default_rng(0).uniform(0, 1, size=S ** 3 * 3).astype(np.float32)
    path = str(tmp_path / "t.cube")
    blobs.write_cube(path, S, vals)
    size = C.c_uint32()
    assert L.cpipe_b200_load_lut(path.encode(), C.byref(size), None, 0) == _abi.OK and size.value == S
    out = np.zeros(S ** 3 * 3, np.float32)
    assert L.cpipe_b200_load_lut(path.encode(), C.byref(size), out.ctypes.data, out.size) == _abi.OK
    np.testing.assert_array_equal(out, vals)
    bad = str(tmp_path / "bad.cube")
    open(bad, "w").write("LUT_3D_SIZE 2\n0 0 0\n")
    assert L.cpipe_b200_load_lut(bad.encode(), C.byref(size), None, 0) == _abi.FAILED
    assert L.cpipe_b200_load_lut(str(tmp_path / "x.png").encode(), C.byref(size), None, 0) == _abi.FAILED
    spi = str(tmp_path / "t.spi3d")
    with open(spi, "w") as f:
        f.write("SPILUT 1.0\n3 3\n2 2 2\n")
        for r in range(2):
            for g in range(2):
                for b in range(2):
                    f.write(f"{r} {g} {b} {r * 0.5} {g * 0.25} {b * 0.75}\n")
    out = np.zeros(24, np.float32)
    assert L.cpipe_b200_load_lut(spi.encode(), C.byref(size), out.ctypes.data, out.size) == _abi.OK
    assert size.value == 2 and out[-3:].tolist() == [0.5, 0.25, 0.75]
