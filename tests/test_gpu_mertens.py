"""tone.mertens_local on the GPU: the CUDA filter against the C oracle
(pinned to the reference golden) for default and non-default weights, the
node against the golden stack, and the node's status codes."""
import numpy as np
import oracle
import pytest
from conftest import golden
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs, call_filter, last_error
from parity import assert_f16_parity

pytestmark = pytest.mark.gpu

F16 = A.FMT_R16G16B16A16_SFLOAT


@pytest.mark.parametrize("h,w", [(1, 1), (3, 5), (45, 67), (130, 257)])
@pytest.mark.parametrize("weights", [(0.0, 1.0, 1.0), (1.5, 0.5, 2.0), (0.3, 1.0, 0.0)])
def test_mertens_filter_against_oracle(cuda_device, h, w, weights):
    r = np.random.default_rng(97)
    normal = r.uniform(0.0, 1.0, size=(h, w, 4)).astype(np.float16)
    under = (normal.astype(np.float32) * 0.25).astype(np.float16)
    over = np.clip(normal.astype(np.float32) * 4.0, 0, 6).astype(np.float16)
    under[..., 3] = over[..., 3] = 1.0
    out = np.zeros_like(normal)
    st = call_filter("tone_mertens_local", [under, normal, over], [out], blobs.mertens(*weights))
    assert st == 0, last_error()
    assert_f16_parity(out, oracle.mertens(under, normal, over, *weights), what=f"mertens {weights}")


def test_mertens_node_golden_and_status(host):
    g = golden("tone.mertens_local")
    h, w = g["normal"].shape[:2]
    bufs = []
    for k in ("under", "normal", "over"):
        b = host.buffer(F16, w, h).upload(g[k].astype(np.float16))
        b.set_metadata(cs_role="scene_linear_rec2020", applied_steps=["denoise.wavelet_bayes_shrink"])
        bufs.append(b)
    out = host.buffer(F16, w, h)
    assert host.run_node("com.cpipe.tone.mertens_local", bufs, [out]) == 0, host.last_error()
    assert_f16_parity(out.download(), g["output"], what="mertens node golden")
    assert out.has_step("tone_mertens_local")
    bad = host.buffer(A.FMT_R32G32B32A32_SFLOAT, w, h)
    assert host.run_node("com.cpipe.tone.mertens_local", bufs, [bad]) == A.BAD_PRECISION
    small = host.buffer(F16, w - 1, h)
    assert host.run_node("com.cpipe.tone.mertens_local", bufs, [small]) == A.BAD_INDEX
    assert host.run_node("com.cpipe.tone.mertens_local", bufs[:2], [out]) == A.BAD_INDEX
