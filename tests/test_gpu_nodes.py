"""Node-level tests on the GPU: each node driven through its plugin main_entry
by the library's host (create -> process -> destroy, metadata builder frozen
into the output), as the reference golden test drives its nodes
(tests/unit/test_golden_isp_nodes.cpp:233-269).  Covers the golden fixtures
with the metadata that test hands each node (:405-745), the known-answer cases
of the reference unit tests, and the status codes of the error paths."""
import numpy as np
import oracle
import pytest
from conftest import golden
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs
from parity import assert_f16_parity

pytestmark = pytest.mark.gpu

RGGB = (0, 1, 1, 2)
SONY_QBC = (0, 0, 1, 1, 0, 0, 1, 1, 1, 1, 2, 2, 1, 1, 2, 2)
EYE = [1, 0, 0, 0, 1, 0, 0, 0, 1]


def node(host, node_id, x, in_fmt, out_fmt, meta=None, params=None):
    h, w = x.shape[:2]
    src = host.buffer(in_fmt, w, h).upload(x)
    src.set_metadata(**(meta or {}))
    out = host.buffer(out_fmt, w, h)
    st = host.run_node(node_id, [src], [out], params)
    return st, out


def ok(host, node_id, x, in_fmt, out_fmt, meta=None, params=None):
    st, out = node(host, node_id, x, in_fmt, out_fmt, meta, params)
    assert st == 0, f"{node_id}: {A.STATUS_NAMES.get(st)} {host.last_error()}"
    return out


# ---------------------------------------------------------------- goldens
def test_golden_raw_nodes(host):
    g = golden("linearize.dng_lut")
    out = ok(host, "com.cpipe.linearize.dng_lut", g["input"].astype(np.uint16), A.FMT_R16_UINT, A.FMT_R32_SFLOAT,
             dict(linearization_table=[0, 11, 23, 36, 50, 65, 81, 98, 116, 135, 155, 176, 198, 221, 245, 270],
                  cs_role="raw_camera"))
    np.testing.assert_array_equal(out.download(), g["output"])
    assert out.has_step("linearization")

    g = golden("blacklevel.dng_levels")
    out = ok(host, "com.cpipe.blacklevel.dng_levels", g["input"], A.FMT_R32_SFLOAT, A.FMT_R32_SFLOAT,
             dict(cfa=RGGB, black_level=[64, 96, 128, 128], white_level=1024, applied_steps=["linearization"]))
    np.testing.assert_array_equal(out.download(), g["output"])
    assert out.has_step("black_white_scaling") and out.has_step("linearization")

    g = golden("lens.shading_gainmap")
    stream = blobs.opcode_list_2_with_gain_maps([blobs.gain_map_params(2, 2, 0, 1, 7.0, 7.0, [1.0, 1.2, 1.4, 1.8])])
    out = ok(host, "com.cpipe.lens.shading_gainmap", g["input"], A.FMT_R32_SFLOAT, A.FMT_R32_SFLOAT,
             dict(cfa=RGGB, blobs={"com.cpipe.dng.opcode_list_2_bytes": stream}))
    np.testing.assert_allclose(out.download(), g["output"], rtol=2e-7, atol=0)


def test_golden_demosaic_nodes(host):
    for node_id, fixture in (("com.cpipe.demosaic.bilinear", "demosaic.bilinear"),
                             ("com.cpipe.demosaic.rcd", "demosaic.rcd"),
                             ("com.cpipe.demosaic.amaze", "demosaic.amaze")):
        g = golden(fixture)
        out = ok(host, node_id, g["input"], A.FMT_R32_SFLOAT, A.FMT_R16G16B16A16_SFLOAT,
                 dict(cfa=RGGB, cs_role="raw_camera", applied_steps=["linearization", "black_white_scaling"]))
        np.testing.assert_array_equal(out.download().astype(np.float32), g["output"], err_msg=node_id)
        assert out.has_step("demosaic") and out.cfa()[0] is False  # clears_fields calibration.cfa
    g = golden("demosaic.quad_bayer_remosaic")
    out = ok(host, "com.cpipe.demosaic.quad_bayer_remosaic", g["input"].astype(np.uint16), A.FMT_R16_UINT,
             A.FMT_R16_UINT, dict(cfa=SONY_QBC, cfa_repeat=(4, 4), cs_role="raw_camera"))
    np.testing.assert_array_equal(out.download().astype(np.float32), g["output"])
    has, rep, pat = out.cfa()
    assert has and rep == (2, 2) and pat[:4] == RGGB


def test_golden_rgba_nodes(host):
    F16 = A.FMT_R16G16B16A16_SFLOAT
    g = golden("lens.dng_opcode_list_3")
    stream = blobs.opcode_list([(3, blobs.fix_vignette_radial_params([0.5]))])
    out = ok(host, "com.cpipe.lens.dng_opcode_list_3", g["input"].astype(np.float16), F16, F16,
             dict(cs_role="scene_linear_rec2020", applied_steps=["demosaic"],
                  blobs={"com.cpipe.dng.opcode_list_3_bytes": stream}))
    assert_f16_parity(out.download(), g["output"], what="opcode3 golden")

    g = golden("wb.dual_illuminant")
    out = ok(host, "com.cpipe.wb.dual_illuminant", g["input"].astype(np.float16), F16, F16,
             dict(illuminants=(17, 21), color_matrix1=EYE, color_matrix2=EYE, forward_matrix1=EYE,
                  forward_matrix2=EYE, cs_role="raw_camera", as_shot_neutral=[0.5, 1.0, 0.25],
                  applied_steps=["linearization", "black_white_scaling", "demosaic"]))
    np.testing.assert_array_equal(out.download().astype(np.float32), g["output"])
    assert out.has_step("white_balance")
    assert np.frombuffer(out.blob("com.cpipe.wb.camera_diag_f32"), np.float32).tolist() == [2.0, 1.0, 4.0]
    assert np.frombuffer(out.blob("com.cpipe.wb.camera_to_xyz_d50_f32"), np.float32).tolist() == EYE

    g = golden("colormatrix.dng_to_working")
    out = ok(host, "com.cpipe.colormatrix.dng_to_working", g["input"].astype(np.float16), F16, F16,
             dict(cs_role="raw_camera", applied_steps=["linearization", "black_white_scaling", "demosaic",
                                                       "white_balance"],
                  blobs={"com.cpipe.wb.camera_to_xyz_d50_f32":
                         np.array([0.5, 0, 0, 0, 0.25, 0, 0, 0, 2.0], np.float32).tobytes()}))
    np.testing.assert_array_equal(out.download().astype(np.float32), g["output"])
    assert out.cs_role == "scene_linear_rec2020" and out.has_step("color_matrix")

    for node_id, fixture in (("com.cpipe.denoise.bm3d", "denoise.bm3d"),
                             ("com.cpipe.denoise.guided_filter", "denoise.guided_filter"),
                             ("com.cpipe.denoise.wavelet_bayes_shrink", "denoise.wavelet_bayes_shrink")):
        g = golden(fixture)
        out = ok(host, node_id, g["input"].astype(np.float16), F16, F16,
                 dict(cs_role="scene_linear_rec2020", applied_steps=["color_matrix"]))
        np.testing.assert_array_equal(out.download().astype(np.float32), g["output"], err_msg=node_id)

    g = golden("tone.filmic_rgb")
    out = ok(host, "com.cpipe.tone.filmic_rgb", g["input"].astype(np.float16), F16, F16,
             dict(cs_role="scene_linear_rec2020", applied_steps=["denoise.bm3d", "denoise.wavelet_bayes_shrink"]))
    assert_f16_parity(out.download(), g["output"], what="filmic golden")


def test_golden_lut_node(host, tmp_path):
    g = golden("color.3d_lut")
    path = str(tmp_path / "look.cube")
    blobs.write_cube(path, int(g["lut_size"]), g["lut"])
    F16 = A.FMT_R16G16B16A16_SFLOAT
    out = ok(host, "com.cpipe.color.3d_lut", g["input"].astype(np.float16), F16, F16,
             dict(cs_role="scene_linear_rec2020", applied_steps=["tone.filmic_rgb"]), {"lut_path": path})
    np.testing.assert_array_equal(out.download().astype(np.float32), g["output"])
    assert out.has_step("color.3d_lut")


# ------------------------------------------------------------------ KATs
def test_gainmap_known_answers(host):
    """test_node_lens_shading_gainmap.cpp:136-163."""
    stream = blobs.opcode_list_2_with_gain_maps([blobs.gain_map_params(2, 2, 0, 1, 2.0, 2.0, [1, 2, 3, 5])])
    out = ok(host, "com.cpipe.lens.shading_gainmap", np.full((3, 3), 10.0, np.float32), A.FMT_R32_SFLOAT,
             A.FMT_R32_SFLOAT, dict(cfa=RGGB, blobs={"com.cpipe.dng.opcode_list_2_bytes": stream})).download().ravel()
    np.testing.assert_allclose(out[[0, 1, 2, 4, 8]], [10.0, 15.0, 20.0, 27.5, 50.0])
    stream = blobs.opcode_list_2_with_gain_maps(
        [blobs.gain_map_params(1, 1, p, 4, 1.0, 1.0, [1.0 + p]) for p in range(4)])
    out = ok(host, "com.cpipe.lens.shading_gainmap", np.ones((4, 4), np.float32), A.FMT_R32_SFLOAT,
             A.FMT_R32_SFLOAT, dict(cfa=SONY_QBC, cfa_repeat=(4, 4),
                                    blobs={"com.cpipe.dng.opcode_list_2_bytes": stream})).download().ravel()
    np.testing.assert_allclose(out[[0, 1, 2, 6, 8, 13, 10, 15]], [1, 1, 2, 2, 3, 3, 4, 4])
    # no OpcodeList2 blob -> plain copy
    x = np.random.default_rng(1).uniform(size=(5, 7)).astype(np.float32)
    out = ok(host, "com.cpipe.lens.shading_gainmap", x, A.FMT_R32_SFLOAT, A.FMT_R32_SFLOAT, dict(cfa=RGGB))
    np.testing.assert_array_equal(out.download(), x)


@pytest.mark.parametrize("node_id", ["com.cpipe.demosaic.rcd", "com.cpipe.demosaic.amaze",
                                     "com.cpipe.demosaic.bilinear"])
@pytest.mark.parametrize("cfa", [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)])
def test_demosaic_flat_field(host, node_id, cfa):
    """test_node_demosaic_rcd.cpp:8-28: a flat field stays flat (margin 1e-3) for every CFA."""
    out = ok(host, node_id, np.full((8, 8), 0.42, np.float32), A.FMT_R32_SFLOAT, A.FMT_R16G16B16A16_SFLOAT,
             dict(cfa=cfa)).download().astype(np.float32)
    np.testing.assert_allclose(out[..., :3], 0.42, atol=1e-3)
    np.testing.assert_array_equal(out[..., 3], 1.0)


def test_wb_inverse_neutral_gains(host):
    """test_node_wb.cpp:60-99: channel gains are the inverse AsShotNeutral."""
    x = np.full((2, 2, 4), 0.25, np.float16)
    x[..., 3] = 1.0
    out = ok(host, "com.cpipe.wb.dual_illuminant", x, A.FMT_R16G16B16A16_SFLOAT, A.FMT_R16G16B16A16_SFLOAT,
             dict(illuminants=(17, 21), color_matrix1=EYE, color_matrix2=EYE, as_shot_neutral=[0.5, 1.0, 0.625],
                  cs_role="raw_camera")).download().astype(np.float32)
    np.testing.assert_allclose(out[0, 0], [0.5, 0.25, 0.4, 1.0], atol=1e-3)


def test_bm3d_sigma_sources(host):
    """bm3d.cpp:21-55: `sigma`, else `sigma_override`, else NoiseProfile at 0.25, else 0.03."""
    x = np.random.default_rng(3).uniform(0.2, 0.4, size=(6, 6, 4)).astype(np.float16)
    F16 = A.FMT_R16G16B16A16_SFLOAT
    meta = dict(noise_profile=[(1e-5, 1e-3)])
    f = np.float32
    from_profile = f(np.sqrt(np.float64(f(f(1e-5) + f(1e-3) * f(0.25)))))
    for params, sigma in (({"sigma": 0.01}, f(0.01)), ({"sigma_override": 0.5}, f(0.2)), ({}, from_profile)):
        out = ok(host, "com.cpipe.denoise.bm3d", x, F16, F16, meta, params).download()
        want = oracle.bm3d_parity(x.astype(np.float32), float(sigma), True)
        np.testing.assert_array_equal(out.astype(np.float32), want)


def test_bm3d_checkerboard_rmse(host):
    """test_node_denoise_bm3d.cpp:129-181: on a 16x16 +-0.055 checkerboard the
    denoised RMSE is <= 0.2x the noisy RMSE."""
    clean = np.full((16, 16), 0.4, np.float32)
    noise = np.where((np.add.outer(np.arange(16), np.arange(16)) % 2) == 0, 0.055, -0.055).astype(np.float32)
    x = np.repeat((clean + noise)[..., None], 4, axis=2).astype(np.float16)
    x[..., 3] = 1.0
    out = ok(host, "com.cpipe.denoise.bm3d", x, A.FMT_R16G16B16A16_SFLOAT, A.FMT_R16G16B16A16_SFLOAT,
             dict(noise_profile=[(1e-3, 0.0)])).download().astype(np.float32)
    rmse = lambda a: float(np.sqrt(np.mean((a[..., :3] - 0.4) ** 2)))  # noqa: E731
    assert rmse(out) <= 0.2 * rmse(x.astype(np.float32))


def test_wavelet_preserves_luma(host):
    """test_node_denoise_wavelet_bayes_shrink.cpp:39-80."""
    x = np.random.default_rng(4).uniform(0.1, 0.6, size=(8, 8, 4)).astype(np.float16)
    x[..., 3] = 1.0
    out = ok(host, "com.cpipe.denoise.wavelet_bayes_shrink", x, A.FMT_R16G16B16A16_SFLOAT,
             A.FMT_R16G16B16A16_SFLOAT).download().astype(np.float32)
    luma = lambda a: (a[..., 0] + 2 * a[..., 1] + a[..., 2]) / 4  # noqa: E731
    np.testing.assert_allclose(luma(out), luma(x.astype(np.float32)), atol=2e-3)


def test_filmic_monotone(host):
    """test_node_tone_filmic_rgb.cpp:13-35: monotone, in [0, 1]."""
    v = np.linspace(0, 16, 64, dtype=np.float32)
    x = np.stack([v, v, v, np.ones_like(v)], -1)[None].astype(np.float16)
    out = ok(host, "com.cpipe.tone.filmic_rgb", x, A.FMT_R16G16B16A16_SFLOAT,
             A.FMT_R16G16B16A16_SFLOAT).download().astype(np.float32)[0, :, 0]
    assert np.all(np.diff(out) >= 0) and out.min() >= 0 and out.max() <= 1


def test_opcode_list_3_known_answers(host):
    """test_node_lens_dng_opcode_list_3.cpp:166-198: identity warp (kr0 = 1)
    keeps the image (eps 1e-3); vignette gains 1.0 / 2.0 / 1.5; bad pixel patched."""
    F16 = A.FMT_R16G16B16A16_SFLOAT
    x = np.random.default_rng(5).uniform(0.1, 0.9, size=(9, 9, 4)).astype(np.float16)
    stream = blobs.opcode_list([(1, blobs.warp_rectilinear_params([(1.0, 0, 0, 0, 0, 0)]))])
    out = ok(host, "com.cpipe.lens.dng_opcode_list_3", x, F16, F16,
             dict(blobs={"com.cpipe.dng.opcode_list_3_bytes": stream})).download()
    np.testing.assert_allclose(out.astype(np.float32), x.astype(np.float32), atol=1e-3)
    ones = np.ones((3, 3, 4), np.float16)
    stream = blobs.opcode_list([(3, blobs.fix_vignette_radial_params([1.0]))])
    out = ok(host, "com.cpipe.lens.dng_opcode_list_3", ones, F16, F16,
             dict(blobs={"com.cpipe.dng.opcode_list_3_bytes": stream})).download().astype(np.float32)
    assert out[1, 1, 0] == 1.0 and out[0, 0, 0] == 2.0 and out[0, 1, 0] == 1.5
    y = np.full((3, 3, 4), 0.5, np.float16)
    y[1, 1, :3] = 0.0
    stream = blobs.opcode_list([(4, blobs.fix_bad_pixels_constant_params(0))])
    out = ok(host, "com.cpipe.lens.dng_opcode_list_3", y, F16, F16,
             dict(blobs={"com.cpipe.dng.opcode_list_3_bytes": stream})).download().astype(np.float32)
    np.testing.assert_array_equal(out[1, 1, :3], 0.5)


# ------------------------------------------------------------- error paths
def test_node_status_codes(host):
    F16, F32, U16 = A.FMT_R16G16B16A16_SFLOAT, A.FMT_R32_SFLOAT, A.FMT_R16_UINT
    x = np.zeros((4, 4), np.float32)
    y = np.zeros((4, 4, 4), np.float16)
    assert node(host, "com.cpipe.blacklevel.dng_levels", x, F32, F32, {})[0] == A.NEED_METADATA
    assert node(host, "com.cpipe.blacklevel.dng_levels", x, F32, F16, dict(cfa=RGGB, white_level=10))[0] == \
        A.BAD_PRECISION
    assert node(host, "com.cpipe.linearize.dng_lut", x.astype(np.uint16), U16, F32, {})[0] == A.NEED_METADATA
    assert node(host, "com.cpipe.demosaic.rcd", x, F32, F16, dict(cfa=(0, 1, 2, 3)))[0] == A.UNSUPPORTED
    assert node(host, "com.cpipe.demosaic.quad_bayer_remosaic", x.astype(np.uint16), U16, U16,
                dict(cfa=(0,) * 16, cfa_repeat=(4, 4)))[0] == A.UNSUPPORTED
    assert node(host, "com.cpipe.wb.dual_illuminant", y, F16, F16, dict(color_matrix1=EYE))[0] == A.NEED_METADATA
    assert node(host, "com.cpipe.colormatrix.dng_to_working", y, F16, F16, dict(cs_role="raw_camera"))[0] == \
        A.NEED_METADATA
    assert node(host, "com.cpipe.color.3d_lut", y, F16, F16, {})[0] == A.NEED_PARAM
    assert node(host, "com.cpipe.precision_convert", x.astype(np.uint16), U16, F32, {}, {"target_format": "R8G8B8A8_UNORM"})[0] == \
        A.BAD_PRECISION
    bad = blobs.opcode_list([(99, b"")])
    assert node(host, "com.cpipe.lens.dng_opcode_list_3", y, F16, F16,
                dict(blobs={"com.cpipe.dng.opcode_list_3_bytes": bad}))[0] == A.UNSUPPORTED


def test_memory_cap_reports_oom(cuda_device):
    from cpipe_b200 import CpipeError, Host
    h = Host(memory_cap=1 << 20)
    with pytest.raises(CpipeError):
        h.buffer(A.FMT_R16G16B16A16_SFLOAT, 1024, 1024)  # 8 MiB > 1 MiB cap
    h.close()
