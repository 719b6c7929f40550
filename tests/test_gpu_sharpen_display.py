"""sharpen.edge_aware_usm and color.scene_linear_to_display on the GPU: the
CUDA filters against the oracles (USM: the C restatement, pinned to the
reference's golden; display: the FP64 restatement of the OCIO transforms,
within one code value for colour, exact for alpha), the nodes against the
golden fixture and the reference unit test's known answers, and the nodes'
status codes."""
import numpy as np
import oracle
import oracle_display as OD
import pytest
from conftest import golden
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs, call_filter, last_error
from parity import assert_f16_parity, assert_f32_parity

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (3, 5), (45, 67), (130, 257)]
F16 = A.FMT_R16G16B16A16_SFLOAT


def run(aot, inputs, outputs, blob):
    st = call_filter(aot, inputs, outputs, blob)
    assert st == 0, f"{aot}: status {st} {last_error()}"
    return outputs[0]


def rgba(seed, h, w, lo, hi, dtype=np.float16):
    x = np.random.default_rng(seed).uniform(lo, hi, size=(h, w, 4)).astype(dtype)
    x[..., 3] = np.random.default_rng(seed + 1).uniform(0.0, 1.0, size=(h, w)).astype(dtype)
    return x


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("strength,radius,threshold", [(0.75, 1, 0.0), (2.0, 2, 0.0), (1.3, 9, 0.02), (0.5, 1, 0.05)])
def test_usm_filter_against_oracle(cuda_device, h, w, strength, radius, threshold):
    x = rgba(80, h, w, 0.0, 1.2)
    b = blobs.usm(strength, radius, threshold)
    out = run("sharpen_edge_aware_usm", [x], [np.zeros_like(x)], b)
    assert_f16_parity(out, oracle.usm(x.astype(np.float32), strength, radius, threshold, True), what="usm f16")
    x32 = x.astype(np.float32)
    out32 = run("sharpen_edge_aware_usm", [x32], [np.zeros_like(x32)], b)
    assert_f32_parity(out32, oracle.usm(x32, strength, radius, threshold, False), what="usm f32")


def test_usm_node_golden_and_status(host):
    g = golden("sharpen.edge_aware_usm")
    x = g["input"].astype(np.float16)
    h, w = x.shape[:2]
    src = host.buffer(F16, w, h).upload(x)
    src.set_metadata(cs_role="scene_linear_rec2020", applied_steps=["color.3d_lut"])
    out = host.buffer(F16, w, h)
    assert host.run_node("com.cpipe.sharpen.edge_aware_usm", [src], [out]) == 0, host.last_error()
    assert_f16_parity(out.download(), g["output"], what="usm golden")
    assert out.has_step("sharpen.edge_aware_usm") and out.cs_role == "scene_linear_rec2020"
    # parameters are clamped as the reference node does: strength 5 -> 2, radius 0 -> 1
    out2 = host.buffer(F16, w, h)
    assert host.run_node("com.cpipe.sharpen.edge_aware_usm", [src], [out2],
                         {"strength": 5.0, "radius": 0, "threshold": 0.0}) == 0
    assert_f16_parity(out2.download(), oracle.usm(x.astype(np.float32), 2.0, 1, 0.0), what="usm clamped params")
    bad = host.buffer(A.FMT_R32G32B32A32_SFLOAT, w, h)
    assert host.run_node("com.cpipe.sharpen.edge_aware_usm", [src], [bad]) == A.BAD_PRECISION


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("target", ["sRGB", "BT2020-PQ"])
def test_display_filter_against_oracle(cuda_device, h, w, target):
    x = rgba(81, h, w, -0.2, 1.6)
    x[0, 0, :3] = 0.0
    dtype = np.uint8 if target == "sRGB" else np.uint16
    out = run("cpipe_scene_linear_to_display", [x], [np.zeros(x.shape, dtype)], blobs.display(target))
    want = OD.display(x.astype(np.float32), target)
    np.testing.assert_array_equal(out[..., 3], want[..., 3])  # alpha exact
    step = 1 if target == "sRGB" else 1 << 6
    diff = np.abs(out[..., :3].astype(np.int64) - want[..., :3].astype(np.int64))
    assert diff.max() <= step, f"{target}: max code difference {diff.max() // step}"
    if target == "BT2020-PQ":
        assert (out & 0x3F == 0).all()


def _display_node(host, x, target, out_fmt, role="scene_linear_rec2020"):
    h, w = x.shape[:2]
    src = host.buffer(F16, w, h).upload(x.astype(np.float16))
    src.set_metadata(cs_role=role)
    out = host.buffer(out_fmt, w, h)
    return host.run_node("com.cpipe.color.scene_linear_to_display", [src], [out], {"target": target}), out


def test_display_node_reference_unit_cases(host):
    """tests/unit/test_node_color_scene_linear_to_display.cpp:146-256 of the reference."""
    x = np.array([[[0.18, 0.20, 0.22, 1.0], [0.45, 0.30, 0.12, 0.5]]], np.float32)
    st, out = _display_node(host, x, "sRGB", A.FMT_R8G8B8A8_UNORM)
    assert st == 0, host.last_error()
    o = out.download().reshape(-1)
    assert (o[:6] > 0).any() and o[3] == 255 and 127 <= o[7] <= 128
    assert out.cs_role == "output_srgb" and out.has_step("color.scene_linear_to_display")
    x = np.array([[[0.05, 0.18, 0.50, 1.0], [0.90, 0.70, 0.30, 0.5]]], np.float32)
    st, out = _display_node(host, x, "BT2020-PQ", A.FMT_R16G16B16A16_UNORM)
    assert st == 0, host.last_error()
    o = out.download().reshape(-1)
    assert ((o & 0x3F) == 0).all() and o[3] == 1023 << 6 and o[7] == 512 << 6
    assert out.cs_role == "output_pq_rec2020"


def test_display_node_status_codes(host):
    x = np.full((2, 3, 4), 0.18, np.float32)
    assert _display_node(host, x, "DisplayP3", A.FMT_R8G8B8A8_UNORM)[0] == A.UNSUPPORTED
    assert _display_node(host, x, "BT2020-HLG", A.FMT_R8G8B8A8_UNORM)[0] == A.UNSUPPORTED
    assert _display_node(host, x, "AdobeRGB", A.FMT_R8G8B8A8_UNORM)[0] == A.NEED_PARAM
    assert _display_node(host, x, "sRGB", A.FMT_R16G16B16A16_UNORM)[0] == A.BAD_PRECISION
    assert _display_node(host, x, "BT2020-PQ", A.FMT_R8G8B8A8_UNORM)[0] == A.BAD_PRECISION
    assert _display_node(host, x, "sRGB", A.FMT_R8G8B8A8_UNORM, role="raw_camera")[0] == A.NEED_METADATA
