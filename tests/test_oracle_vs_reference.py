"""Pin the oracle (and the library's host-side preparation) against the
reference's own code, compiled unmodified from the reference tree by
`make -C oracle ref`: the six plain-C++ filters
(src/cpipe/nodes/{linearize,blacklevel,lens,wb,colormatrix}/*_dispatch.cpp) and
the white-balance helpers (src/cpipe/nodes/wb/WbMetadata.hpp).  Inputs are
seeded random images including odd sizes; every comparison is bit-exact."""
import ctypes as C

import numpy as np
import oracle
import pytest
from cpipe_b200 import _abi, blobs

pytestmark = pytest.mark.skipif(oracle.ref_lib() is None, reason="reference build (oracle/_ref) absent")

SIZES = [(1, 1), (3, 5), (17, 9), (64, 48)]


def rng(seed):
    return np.random.default_rng(seed)


@pytest.mark.parametrize("h,w", SIZES)
def test_linearize_matches_reference(h, w):
    r = rng(1)
    raw = r.integers(0, 1200, size=(h, w), dtype=np.uint16)
    table = np.sort(r.integers(0, 65535, size=1000)).astype(np.uint16)
    ref = np.zeros((h, w), np.float32)
    assert oracle.ref_call("linearize_dng_lut", raw, ref, blobs.linearize(table)) == 0
    st, out = oracle.linearize(raw, table)
    assert st == 0
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("cfa", [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)])
def test_blacklevel_matches_reference(h, w, cfa):
    r = rng(2)
    x = r.uniform(0, 4200, size=(h, w)).astype(np.float32)
    blob = blobs.blacklevel([64.0, 60.5, 70.25, 66.0], 4095, cfa)
    ref = np.zeros_like(x)
    assert oracle.ref_call("blacklevel_dng_levels", x, ref, blob) == 0
    st, out = oracle.blacklevel(x, blob)
    assert st == 0
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("h,w", SIZES)
def test_gainmap_matches_reference(h, w):
    r = rng(3)
    x = r.uniform(0, 1, size=(h, w)).astype(np.float32)
    one = blobs.gainmap_dispatch([dict(points_v=13, points_h=17, spacing_v=max(h, 2) / 12.0,
                                       spacing_h=max(w, 2) / 16.0, origin_v=-0.5, origin_h=0.25,
                                       gains=r.uniform(1.0, 1.8, size=13 * 17))])
    four = blobs.gainmap_dispatch([dict(plane=p, planes=4, points_v=3, points_h=4, spacing_v=2.5, spacing_h=3.0,
                                        gains=r.uniform(0.9, 1.5, size=12)) for p in range(4)],
                                  cfa_repeat=(4, 4))
    for blob in (one, four):
        ref = np.zeros_like(x)
        assert oracle.ref_call("lens_shading_gainmap", x, ref, blob) == 0
        st, out = oracle.gainmap(x, blob)
        assert st == 0
        np.testing.assert_array_equal(out, ref)


def rgba_f16(r, h, w, lo=0.0, hi=1.0):
    x = r.uniform(lo, hi, size=(h, w, 4)).astype(np.float16)
    x[..., 3] = 1.0
    return x


@pytest.mark.parametrize("h,w", SIZES)
def test_wb_and_colormatrix_match_reference(h, w):
    r = rng(4)
    x = rgba_f16(r, h, w)
    ref = np.zeros_like(x)
    assert oracle.ref_call("wb_dual_illuminant", x, ref, blobs.wb([0.5, 1.0, 0.625])) == 0
    out = oracle.wb(x.astype(np.float32), [0.5, 1.0, 0.625])
    np.testing.assert_array_equal(out, ref.astype(np.float32))
    t = r.uniform(-0.5, 1.5, size=9).astype(np.float32)
    ref = np.zeros_like(x)
    assert oracle.ref_call("colormatrix_dng_to_working", x, ref, blobs.colormatrix(t)) == 0
    out = oracle.colormatrix(x.astype(np.float32), t)
    np.testing.assert_array_equal(out, ref.astype(np.float32))


def opcode3_cases(w, h):
    warp1 = blobs.warp_record([(1.0, -0.08, 0.02, 0.0, 0.0, 0.0)])
    warp3 = blobs.warp_record([(1.0, -0.05, 0.01, 0.0, 0.001, -0.002), (0.99, 0.03, 0.0, 0.0, 0.0, 0.0),
                               (1.01, -0.1, 0.04, -0.01, 0.0, 0.0)], cx_hat=0.45, cy_hat=0.55)
    vig = blobs.vignette_record([0.4, -0.1, 0.05, 0.0, 0.01], cx_hat=0.4, cy_hat=0.6)
    bad_c = _abi.Opcode3DispatchRecord()
    bad_c.id, bad_c.constant = 4, 0
    bad_l = _abi.Opcode3DispatchRecord()
    bad_l.id, bad_l.point_offset, bad_l.point_count, bad_l.rect_offset, bad_l.rect_count = 5, 0, 2, 0, 1
    trim = _abi.Opcode3DispatchRecord()
    trim.id, trim.top, trim.left, trim.bottom, trim.right = 6, 1, 2, max(1, h - 1), max(2, w - 1)
    unknown_opt = _abi.Opcode3DispatchRecord()
    unknown_opt.id, unknown_opt.optional = 0, 1
    pts = [(min(1, h - 1), min(2, w - 1)), (0, 0)]
    rects = [(0, 0, min(2, h), min(3, w))]
    return {
        "warp1": blobs.opcode3_dispatch([warp1]),
        "warp3": blobs.opcode3_dispatch([warp3]),
        "vignette": blobs.opcode3_dispatch([vig]),
        "bad_constant": blobs.opcode3_dispatch([bad_c]),
        "bad_list": blobs.opcode3_dispatch([bad_l], points=pts, rects=rects),
        "trim": blobs.opcode3_dispatch([trim]),
        "sequence": blobs.opcode3_dispatch([unknown_opt, vig, warp1, bad_l, trim], points=pts, rects=rects),
    }


@pytest.mark.parametrize("h,w", [(1, 1), (3, 5), (24, 31)])
def test_opcode_list_3_matches_reference(h, w):
    r = rng(5)
    x = rgba_f16(r, h, w)
    x[0, 0, :3] = 0.0  # a pixel the constant bad-pixel opcode patches
    for name, blob in opcode3_cases(w, h).items():
        ref = np.zeros_like(x)
        assert oracle.ref_call("lens_dng_opcode_list_3", x, ref, blob) == 0, name
        st, out = oracle.opcode3(x.astype(np.float32), blob, f16=True)
        assert st == 0, name
        np.testing.assert_array_equal(out, ref.astype(np.float32), err_msg=name)


def test_opcode_list_3_errors_match_reference():
    x = np.zeros((4, 4, 4), np.float16)
    unknown = _abi.Opcode3DispatchRecord()
    unknown.id, unknown.optional = 0, 0
    blob = blobs.opcode3_dispatch([unknown])
    assert oracle.ref_call("lens_dng_opcode_list_3", x, np.zeros_like(x), blob) == _abi.UNSUPPORTED
    assert oracle.opcode3(x.astype(np.float32), blob)[0] == _abi.UNSUPPORTED
    assert oracle.ref_call("lens_dng_opcode_list_3", x, np.zeros_like(x), b"\x01\x00") == _abi.BAD_INDEX
    assert oracle.opcode3(x.astype(np.float32), b"\x01\x00")[0] == _abi.BAD_INDEX


WB_CASES = [
    # neutral, cm1, cm2, fm1, fm2, illum1, illum2
    ([0.5, 1.0, 0.625], [1, 0, 0, 0, 1, 0, 0, 0, 1], [1, 0, 0, 0, 1, 0, 0, 0, 1], None, None, 17, 21),
    ([0.47, 1.0, 0.71], [0.6722, -0.0635, -0.0963, -0.4287, 1.2460, 0.2028, -0.0908, 0.2162, 0.5668],
     [0.8128, -0.2218, -0.0815, -0.4148, 1.1926, 0.2469, -0.0793, 0.1797, 0.6080], None, None, 17, 21),
    ([0.61, 1.0, 0.52], [0.6722, -0.0635, -0.0963, -0.4287, 1.2460, 0.2028, -0.0908, 0.2162, 0.5668],
     [0.8128, -0.2218, -0.0815, -0.4148, 1.1926, 0.2469, -0.0793, 0.1797, 0.6080],
     [0.7, 0.1, 0.15, 0.3, 0.8, -0.1, 0.0, -0.2, 1.0], [0.72, 0.12, 0.11, 0.29, 0.82, -0.11, 0.01, -0.19, 1.02],
     23, 21),
    ([0.9, 1.0, 0.3], [1.2, -0.1, 0, -0.3, 1.1, 0.2, 0, 0.1, 0.9], [0.9, 0.05, -0.02, -0.2, 1.05, 0.1, 0.02, 0.05, 1.1],
     None, None, 24, 22),
]


@pytest.mark.parametrize("case", range(len(WB_CASES)))
def test_wb_prepare_matches_reference(case):
    neutral, cm1, cm2, fm1, fm2, i1, i2 = WB_CASES[case]
    st, ref_m, ref_cct, ref_w = oracle.ref_wb_interpolate(neutral, cm1, cm2, fm1, fm2, i1, i2)
    p = _abi.WbParams()
    cct = C.c_double()
    F9 = C.c_float * 9
    got = _abi.lib().cpipe_b200_wb_prepare((C.c_float * 3)(*neutral), F9(*cm1), F9(*cm2),
                                           F9(*fm1) if fm1 else None, F9(*fm2) if fm2 else None, i1, i2,
                                           C.byref(p), C.byref(cct))
    assert got == st == 0
    assert cct.value == ref_cct
    assert p.dual_illuminant_weight == np.float32(ref_w)
    assert list(p.camera_to_xyz_d50) == [float(np.float32(v)) for v in ref_m]


def test_wb_prepare_errors():
    F9 = C.c_float * 9
    eye = F9(1, 0, 0, 0, 1, 0, 0, 0, 1)
    p = _abi.WbParams()
    cct = C.c_double()
    L = _abi.lib()
    assert L.cpipe_b200_wb_prepare((C.c_float * 3)(0.5, 1, 0.6), eye, eye, None, None, 99, 21, C.byref(p),
                                   C.byref(cct)) == _abi.NEED_METADATA
    assert L.cpipe_b200_wb_prepare((C.c_float * 3)(0.5, 0, 0.6), eye, eye, None, None, 17, 21, C.byref(p),
                                   C.byref(cct)) == _abi.NEED_METADATA
    assert L.cpipe_b200_wb_prepare((C.c_float * 3)(0.5, 1, 0.6), None, eye, None, None, 17, 21, C.byref(p),
                                   C.byref(cct)) == _abi.NEED_METADATA
