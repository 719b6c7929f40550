"""wb.greyworld_auto on the GPU: the exact channel sums, the neutral and the
applied gains against the oracle on frames from 1x1 to 1.5 MP (many blocks,
ragged rows), the node against the reference golden with its metadata, and
the reference node's status codes."""
import ctypes as C

import numpy as np
import oracle
import pytest
from conftest import golden
from cpipe_b200 import _abi as A
from cpipe_b200 import call_filter, last_error

pytestmark = pytest.mark.gpu

F16 = A.FMT_R16G16B16A16_SFLOAT
EYE = [1, 0, 0, 0, 1, 0, 0, 0, 1]
CAL = dict(illuminants=(17, 21), color_matrix1=EYE, color_matrix2=EYE, forward_matrix1=EYE, forward_matrix2=EYE,
           cs_role="raw_camera", applied_steps=["demosaic"])


def greyworld_filter(x):
    n = (C.c_float * 3)()
    blob = bytes(A.GreyworldParams(C.addressof(n)))
    out = np.zeros_like(x)
    st = call_filter("cpipe_wb_greyworld_auto", [x], [out], blob)
    return st, np.array(n[:], np.float32), out


@pytest.mark.parametrize("h,w", [(1, 1), (3, 5), (45, 67), (130, 257), (1000, 1500)])
def test_greyworld_filter_against_oracle(cuda_device, h, w):
    r = np.random.default_rng(95)
    x = r.uniform(0.0, 3.0, size=(h, w, 4)).astype(np.float16)
    x[..., 0] *= np.float16(0.6)
    st, n, out = greyworld_filter(x)
    assert st == 0, last_error()
    want_n, want = oracle.greyworld(x)
    np.testing.assert_array_equal(n, want_n)
    np.testing.assert_array_equal(out.astype(np.float32), want)


def test_greyworld_filter_invalid_means(cuda_device):
    x = np.full((8, 9, 4), 0.5, np.float16)
    x[..., 1] = 0.0
    assert greyworld_filter(x)[0] == A.NEED_METADATA
    x = np.full((8, 9, 4), 0.5, np.float16)
    x[3, 4, 2] = np.float16(np.inf)
    assert greyworld_filter(x)[0] == A.NEED_METADATA
    x = np.full((8, 9, 4), 0.5, np.float16)
    x[3, 4, 3] = np.float16(np.nan)  # alpha is not summed
    assert greyworld_filter(x)[0] == 0


def _node(host, x, meta, in_fmt=F16):
    h, w = x.shape[:2]
    src = host.buffer(in_fmt, w, h).upload(x)
    src.set_metadata(**meta)
    out = host.buffer(F16, w, h)
    return host.run_node("com.cpipe.wb.greyworld_auto", [src], [out]), out


def test_greyworld_node_golden_and_status(host):
    g = golden("wb.greyworld_auto")
    st, out = _node(host, g["input"].astype(np.float16), CAL)
    assert st == 0, host.last_error()
    np.testing.assert_array_equal(out.download().astype(np.float32), g["output"])
    n, _ = oracle.greyworld(g["input"])
    assert out.has_step("white_balance")
    diag = np.frombuffer(out.blob("com.cpipe.wb.camera_diag_f32"), np.float32)
    np.testing.assert_array_equal(diag, (np.float32(1.0) / n).astype(np.float32))
    assert out.blob("com.cpipe.wb.camera_to_xyz_d50_f32") is not None
    x = g["input"].astype(np.float16)
    assert _node(host, x.astype(np.float32), CAL, A.FMT_R32G32B32A32_SFLOAT)[0] == A.BAD_PRECISION
    assert _node(host, x, dict(cs_role="raw_camera"))[0] == A.NEED_METADATA
    z = x.copy()
    z[..., 1] = 0
    assert _node(host, z, CAL)[0] == A.NEED_METADATA
