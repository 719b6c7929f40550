"""Pin the CPU oracle to the reference's golden vectors.

The fixtures in tests/golden/ are produced by the reference's own golden
generator (tests/fixtures/gen_golden_isp_nodes.cpp, compiled unmodified by
oracle/Makefile; see tests/golden/make_golden.py).  The node parameters below
are the ones the reference golden test hands each node
(tests/unit/test_golden_isp_nodes.cpp:405-745).  The reference gate is PSNR
>= 40 dB (:72); the oracle is held to bit-exactness wherever the generator
restates the node with the same operation order, and to one f16 ulp otherwise.
"""
import numpy as np
import oracle
from conftest import golden
from cpipe_b200 import blobs
from parity import assert_f16_parity, f16_ulp_distance, psnr

RGGB = (0, 1, 1, 2)


def test_linearize_golden():
    g = golden("linearize.dng_lut")
    table = [0, 11, 23, 36, 50, 65, 81, 98, 116, 135, 155, 176, 198, 221, 245, 270]
    st, out = oracle.linearize(g["input"].astype(np.uint16), table)
    assert st == 0
    np.testing.assert_array_equal(out, g["output"])


def test_blacklevel_golden():
    g = golden("blacklevel.dng_levels")
    st, out = oracle.blacklevel(g["input"], blobs.blacklevel([64, 96, 128, 128], 1024, RGGB))
    assert st == 0
    np.testing.assert_array_equal(out, g["output"])


def test_gainmap_golden():
    # test_golden_isp_nodes.cpp:455-470: one 2x2 map, spacing 7 px on an 8x8 image.
    g = golden("lens.shading_gainmap")
    blob = blobs.gainmap_dispatch([dict(points_v=2, points_h=2, spacing_v=7.0, spacing_h=7.0,
                                        gains=[1.0, 1.2, 1.4, 1.8])])
    st, out = oracle.gainmap(g["input"], blob)
    assert st == 0
    # The generator restates the lerp weight in float (x / 7.0f) where the
    # filter uses double; results agree to float rounding.
    np.testing.assert_allclose(out, g["output"], rtol=2e-7, atol=0)
    assert psnr(out, g["output"]) > 120


def test_demosaic_goldens():
    for algo, fixture in (("bilinear", "demosaic.bilinear"), ("rcd", "demosaic.rcd"), ("amaze", "demosaic.amaze")):
        g = golden(fixture)
        out = oracle.demosaic(algo, g["input"], RGGB, f16=True)
        np.testing.assert_array_equal(out, g["output"], err_msg=algo)


def test_quad_bayer_remosaic_golden():
    g = golden("demosaic.quad_bayer_remosaic")
    out = oracle.qbc_remosaic(g["input"].astype(np.uint16))
    np.testing.assert_array_equal(out.astype(np.float32), g["output"])


def test_opcode_list_3_vignette_golden():
    # test_golden_isp_nodes.cpp:495-520: FixVignetteRadial k0 = 0.5, centre (0.5, 0.5).
    g = golden("lens.dng_opcode_list_3")
    blob = blobs.opcode3_dispatch([blobs.vignette_record([0.5])])
    st, out = oracle.opcode3(oracle.h16(g["input"]), blob, f16=True)
    assert st == 0
    # the generator evaluates the radius in float, the filter in double
    assert_f16_parity(out, g["output"], what="vignette")


def test_wb_golden():
    g = golden("wb.dual_illuminant")
    out = oracle.wb(oracle.h16(g["input"]), [0.5, 1.0, 0.25])
    np.testing.assert_array_equal(out, g["output"])


def test_colormatrix_golden():
    from cpipe_b200 import _abi
    import ctypes as C
    g = golden("colormatrix.dng_to_working")
    t = (C.c_float * 9)()
    cam = (C.c_float * 9)(0.5, 0, 0, 0, 0.25, 0, 0, 0, 2.0)
    assert _abi.lib().cpipe_b200_colormatrix_compose(cam, t) == 0
    out = oracle.colormatrix(oracle.h16(g["input"]), list(t))
    np.testing.assert_array_equal(out, g["output"])


def test_denoise_goldens():
    g = golden("denoise.bm3d")
    x = oracle.h16(g["input"])
    np.testing.assert_array_equal(oracle.bm3d_parity(x, 0.03), g["output"])
    g = golden("denoise.guided_filter")
    np.testing.assert_array_equal(oracle.guided(x, 1, 0.015), g["output"])
    g = golden("denoise.wavelet_bayes_shrink")
    np.testing.assert_array_equal(oracle.wavelet(x, 1.0), g["output"])


def test_filmic_golden():
    g = golden("tone.filmic_rgb")
    out = oracle.filmic(oracle.h16(g["input"]))
    # The generator applies the bare curve; the node also passes the default
    # saturation / highlight / shadow stages, which are identities up to float rounding.
    d = f16_ulp_distance(out, g["output"])
    assert d.max() <= 1
    assert psnr(out, g["output"]) > 60


def test_lut_golden():
    g = golden("color.3d_lut")
    out = oracle.lut3d(oracle.h16(g["input"]), g["lut"], int(g["lut_size"]), interp=0)
    np.testing.assert_array_equal(out, g["output"])
