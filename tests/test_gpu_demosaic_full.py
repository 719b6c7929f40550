"""Full-form RCD and AMaZE on the GPU (aot_ids demosaic_rcd_full /
demosaic_amaze_full, node parameter algorithm = "full") against the oracle.

The kernels evaluate the oracle's binary32 expressions in the same order, so
they are compared bit for bit with its binary32 instantiation (RGBA32F output)
and with its result rounded to binary16 (RGBA16F output); the error against
the FP64 instantiation is printed and bounded.  Odd and tiny sizes, all four
Bayer phases, and a 12 MP frame."""
import numpy as np
import oracle
import pytest
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs, call_filter, last_error
from cpipe_b200.scene import mosaic, scene_rgb

pytestmark = pytest.mark.gpu

CFAS = [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)]
AOT = {"rcd": "demosaic_rcd_full", "amaze": "demosaic_amaze_full"}


def bayer(h, w, seed, cfa):
    rgb = scene_rgb(w, h, seed)
    noise = np.random.default_rng(seed).normal(0.0, 0.01, (h, w)).astype(np.float32)
    return np.clip(mosaic(rgb, cfa) + noise, 0.0, 1.0).astype(np.float32)


def run_gpu(algo, x, cfa, dtype):
    out = np.zeros(x.shape + (4,), dtype)
    st = call_filter(AOT[algo], [x], [out], blobs.demosaic(cfa))
    assert st == 0, (A.STATUS_NAMES.get(st), last_error())
    return out


def expect(algo, x, cfa, dtype):
    rgb = oracle.demosaic_full(algo, x, cfa, "f32").astype(np.float32)
    want = np.ones(x.shape + (4,), np.float32)
    want[..., :3] = rgb
    return want.astype(dtype)


@pytest.mark.parametrize("algo", ["rcd", "amaze"])
@pytest.mark.parametrize("cfa", CFAS)
@pytest.mark.parametrize("h,w", [(64, 96), (63, 97), (70, 130), (17, 33), (5, 7), (2, 2), (1, 1), (200, 257)])
def test_full_demosaic_bit_exact(cuda_device, algo, cfa, h, w):
    x = bayer(h, w, h * 1000 + w, cfa)
    for dtype in (np.float16, np.float32):
        got = run_gpu(algo, x, cfa, dtype)
        want = expect(algo, x, cfa, dtype)
        bits = np.uint16 if dtype == np.float16 else np.uint32
        diff = got.view(bits) != want.view(bits)
        assert not diff.any(), f"{algo} {cfa} {h}x{w} {dtype.__name__}: {int(diff.sum())} elements differ"


@pytest.mark.parametrize("algo,min_db", [("rcd", 120.0), ("amaze", 55.0)])
def test_full_demosaic_vs_fp64(cuda_device, algo, min_db):
    x = bayer(240, 320, 7, (0, 1, 1, 2))
    got = run_gpu(algo, x, (0, 1, 1, 2), np.float32)[..., :3].astype(np.float64)
    ref = oracle.demosaic_full(algo, x, (0, 1, 1, 2), "f64")
    p = 10 * np.log10(1.0 / np.mean((got - ref) ** 2))
    print(f"{algo} full vs FP64 oracle: PSNR {p:.1f} dB, max-abs {np.abs(got - ref).max():.3g}")
    assert p >= min_db


@pytest.mark.parametrize("algo", ["rcd", "amaze"])
def test_full_demosaic_12mp(cuda_device, algo):
    x = bayer(3024, 4032, 0x5EED0002, (0, 1, 1, 2))
    got = run_gpu(algo, x, (0, 1, 1, 2), np.float16)
    want = expect(algo, x, (0, 1, 1, 2), np.float16)
    assert np.array_equal(got.view(np.uint16), want.view(np.uint16))


@pytest.mark.parametrize("node,algo", [("com.cpipe.demosaic.rcd", "rcd"), ("com.cpipe.demosaic.amaze", "amaze")])
def test_node_algorithm_full(host, node, algo):
    x = bayer(96, 128, 3, (1, 2, 0, 1))
    src = host.buffer(A.FMT_R32_SFLOAT, 128, 96).upload(x)
    src.set_metadata(cfa=(1, 2, 0, 1), cs_role="raw_camera", applied_steps=["black_white_scaling"])
    out = host.buffer(A.FMT_R16G16B16A16_SFLOAT, 128, 96)
    st = host.run_node(node, [src], [out], {"algorithm": "full"})
    assert st == 0, host.last_error()
    got = out.download()
    assert np.array_equal(got.view(np.uint16), expect(algo, x, (1, 2, 0, 1), np.float16).view(np.uint16))
    bad = host.buffer(A.FMT_R16G16B16A16_SFLOAT, 128, 96)
    assert host.run_node(node, [src], [bad], {"algorithm": "nope"}) == A.BAD_INDEX


def test_full_demosaic_refuses_non_bayer(cuda_device):
    x = np.zeros((8, 8), np.float32)
    out = np.zeros((8, 8, 4), np.float16)
    assert call_filter("demosaic_rcd_full", [x], [out], blobs.demosaic((0, 0, 1, 2))) == A.UNSUPPORTED
