"""tone.aces_filmic and tone.reinhard on the GPU: the CUDA filters against the
C oracles (pinned to the reference goldens) on f16 and f32 frames, the nodes
against the golden fixtures and the reference nodes' parameter handling."""
import numpy as np
import oracle
import pytest
from conftest import golden
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs, call_filter, last_error
from parity import assert_f16_parity, assert_f32_parity

pytestmark = pytest.mark.gpu

F16 = A.FMT_R16G16B16A16_SFLOAT


def run(aot, x, blob):
    out = np.zeros_like(x)
    st = call_filter(aot, [x], [out], blob)
    assert st == 0, f"{aot}: status {st} {last_error()}"
    return out


@pytest.mark.parametrize("h,w", [(1, 1), (3, 5), (45, 67), (130, 257)])
def test_tone_filters_against_oracle(cuda_device, h, w):
    r = np.random.default_rng(90)
    x = r.uniform(-0.5, 12.0, size=(h, w, 4)).astype(np.float16)
    x32 = x.astype(np.float32)
    for enabled in (True, False):
        assert_f16_parity(run("tone_aces_filmic", x, blobs.aces(enabled)), oracle.aces(x32, enabled), what="aces")
        assert_f32_parity(run("tone_aces_filmic", x32, blobs.aces(enabled)), oracle.aces(x32, enabled, False),
                          what="aces f32")
    for wp in (1000000.0, 0.1, 3.7, 10.0):
        assert_f16_parity(run("tone_reinhard", x, blobs.reinhard(wp)), oracle.reinhard(x32, wp), what="reinhard")
        assert_f32_parity(run("tone_reinhard", x32, blobs.reinhard(wp)), oracle.reinhard(x32, wp, False),
                          what="reinhard f32")


def _node(host, node_id, x, params=None):
    h, w = x.shape[:2]
    src = host.buffer(F16, w, h).upload(x.astype(np.float16))
    src.set_metadata(cs_role="scene_linear_rec2020", applied_steps=["denoise.wavelet_bayes_shrink"])
    out = host.buffer(F16, w, h)
    st = host.run_node(node_id, [src], [out], params)
    assert st == 0, f"{node_id}: {A.STATUS_NAMES.get(st)} {host.last_error()}"
    return out


def test_tone_nodes_golden_and_params(host):
    g = golden("tone.aces_filmic")
    out = _node(host, "com.cpipe.tone.aces_filmic", g["input"])
    assert_f16_parity(out.download(), g["output"], what="aces golden")
    assert out.has_step("tone.aces_filmic")
    x = g["input"].astype(np.float16).astype(np.float32)
    off = _node(host, "com.cpipe.tone.aces_filmic", g["input"], {"toggle": False}).download()
    np.testing.assert_array_equal(off.astype(np.float32), x)
    g = golden("tone.reinhard")
    out = _node(host, "com.cpipe.tone.reinhard", g["input"])
    assert_f16_parity(out.download(), g["output"], what="reinhard golden")
    assert out.has_step("tone.reinhard")
    x = g["input"].astype(np.float16).astype(np.float32)
    for wp, want in ((20.0, 10.0), (0.01, 0.1), (2.5, 2.5)):  # clamped to 0.1..10 as the reference node
        got = _node(host, "com.cpipe.tone.reinhard", g["input"], {"white_point": wp}).download()
        assert_f16_parity(got, oracle.reinhard(x, want), what=f"reinhard wp {wp}")
