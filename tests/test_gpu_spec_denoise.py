"""Spec-mode guided filter (denoise_guided_filter_spec) and a-trous wavelet
denoiser (denoise_wavelet_atrous_spec) on the GPU against the FP64 oracle
(oracle/oracle_spec_denoise.py): float32 frames within max-abs 1e-4 and PSNR
>= 60 dB, binary16 frames within one binary16 ulp and PSNR >= 60 dB; odd and
tiny sizes; every radius class and level count; the parameter refusals; and
at radius 1 and 2 the spec guided filter against the GPU's parity guided
filter (the reference's own computation)."""
import numpy as np
import oracle_spec_denoise as S
import pytest
from bm3d_scenes import clean_rgb, noisy_rgba
from cpipe_b200 import blobs, call_filter, last_error
from parity import assert_f16_parity, assert_f32_parity

pytestmark = pytest.mark.gpu


def run(aot, x, blob):
    out = np.zeros_like(x)
    st = call_filter(aot, [x], [out], blob)
    assert st == 0, f"{aot}: status {st}: {last_error()}"
    return out


def frame(h, w, sigma, seed, dtype):
    return noisy_rgba(clean_rgb(seed, h, w, rects=12), sigma, seed, dtype=dtype)


def check(got, want, dtype, what):
    if dtype == np.float16:
        assert_f16_parity(got, want, what=what)
    else:
        assert_f32_parity(got, want, max_abs=1e-4, what=what)


@pytest.mark.parametrize("dtype", [np.float32, np.float16])
@pytest.mark.parametrize("h,w,radius,eps", [(70, 53, 1, 1e-3), (129, 257, 4, 1e-3), (96, 128, 8, 1e-3),
                                            (61, 75, 16, 5e-3), (5, 9, 8, 1e-3)])
def test_guided_spec_matches_oracle(cuda_device, dtype, h, w, radius, eps):
    x = frame(h, w, 0.03, h + w, dtype)
    got = run("denoise_guided_filter_spec", x, blobs.guided(radius, eps))
    want = S.guided_spec(x.astype(np.float64), radius, eps)
    check(got, want, dtype, f"guided spec r={radius} {w}x{h} {np.dtype(dtype).name}")
    np.testing.assert_array_equal(got[..., 3], x[..., 3])


@pytest.mark.parametrize("radius", [1, 2])
def test_guided_spec_equals_parity_filter_at_small_radius(cuda_device, radius):
    x = frame(80, 96, 0.03, 4, np.float32)
    spec = run("denoise_guided_filter_spec", x, blobs.guided(radius, 1e-3))
    ref = run("denoise_guided_filter", x, blobs.guided(radius, 1e-3))
    assert_f32_parity(spec, ref, max_abs=1e-5, what=f"spec vs reference guided r={radius}")


@pytest.mark.parametrize("dtype", [np.float32, np.float16])
@pytest.mark.parametrize("h,w,levels,lumas,chromas", [(96, 64, 5, 1.0, 1.0), (201, 300, 6, 1.0, 1.0),
                                                      (17, 33, 3, 0.0, 2.0), (64, 96, 1, 1.0, 0.5)])
def test_atrous_matches_oracle(cuda_device, dtype, h, w, levels, lumas, chromas):
    sigma = 0.03
    x = frame(h, w, sigma, 7 * h + w, dtype)
    got = run("denoise_wavelet_atrous_spec", x, blobs.atrous(levels, sigma, lumas, chromas))
    want = S.atrous_spec(x.astype(np.float64), levels, sigma, lumas, chromas)
    check(got, want, dtype, f"a-trous L={levels} {w}x{h} {np.dtype(dtype).name}")
    np.testing.assert_array_equal(got[..., 3], x[..., 3])


def test_atrous_zero_levels_copies(cuda_device):
    x = frame(40, 50, 0.03, 1, np.float16)
    got = run("denoise_wavelet_atrous_spec", x, blobs.atrous(0, 0.03))
    np.testing.assert_array_equal(got.view(np.uint16), x.view(np.uint16))


def test_spec_filters_refuse_out_of_range(cuda_device):
    x = frame(16, 16, 0.03, 1, np.float32)
    out = np.zeros_like(x)
    assert call_filter("denoise_guided_filter_spec", [x], [out], blobs.guided(17, 1e-3)) != 0
    assert call_filter("denoise_guided_filter_spec", [x], [out], blobs.guided(0, 1e-3)) != 0
    assert call_filter("denoise_guided_filter_spec", [x], [out], blobs.guided(4, 0.0)) != 0
    assert call_filter("denoise_wavelet_atrous_spec", [x], [out], blobs.atrous(7, 0.03)) != 0
    assert call_filter("denoise_wavelet_atrous_spec", [x], [out], blobs.atrous(5, -1.0)) != 0


def test_spec_nodes(host):
    """com.cpipe.denoise.guided_filter with algorithm = "spec" and
    com.cpipe.denoise.wavelet_bayes_shrink with algorithm = "atrous" submit the
    spec filters (the a-trous noise sigma from the NoiseProfile, as the bm3d
    node finds it: sqrt(beta + 0.25 lambda))."""
    from cpipe_b200 import _abi as A
    x = frame(48, 64, 0.03, 12, np.float16)
    F16 = A.FMT_R16G16B16A16_SFLOAT
    src = host.buffer(F16, x.shape[1], x.shape[0]).upload(x)
    src.set_metadata(cs_role="scene_linear_rec2020", applied_steps=["color_matrix"], noise_profile=[(1e-5, 1e-3)])
    out = host.buffer(F16, x.shape[1], x.shape[0])
    st = host.run_node("com.cpipe.denoise.guided_filter", [src], [out], {"algorithm": "spec", "radius": 8, "eps": 1e-3})
    assert st == 0, host.last_error()
    want = S.guided_spec(x.astype(np.float64), 8, float(np.float32(1e-3)))
    assert_f16_parity(out.download(), want, what="guided spec node")
    assert out.has_step("denoise.guided_filter")
    st = host.run_node("com.cpipe.denoise.wavelet_bayes_shrink", [src], [out], {"algorithm": "atrous", "levels": 4})
    assert st == 0, host.last_error()
    sigma = float(np.float32(np.sqrt(np.float32(1e-5) + np.float32(1e-3) * np.float32(0.25))))
    want = S.atrous_spec(x.astype(np.float64), 4, sigma)
    assert_f16_parity(out.download(), want, what="a-trous node")
    assert host.run_node("com.cpipe.denoise.wavelet_bayes_shrink", [src], [out], {"algorithm": "nope"}) == A.BAD_INDEX
    assert host.run_node("com.cpipe.denoise.guided_filter", [src], [out], {"algorithm": "nope"}) == A.BAD_INDEX


def test_scratch_pool_is_reused_and_trimmed(cuda_device):
    """Filters with scratch (here the a-trous form, ~100 B/px) draw it from the
    library's pool: repeated calls give the same result, and trimming the pool
    between calls changes nothing but the memory held."""
    from cpipe_b200 import _abi as A
    x = frame(96, 128, 0.03, 3, np.float32)
    first = run("denoise_wavelet_atrous_spec", x, blobs.atrous(5, 0.03))
    again = run("denoise_wavelet_atrous_spec", x, blobs.atrous(5, 0.03))
    assert A.lib().cpipe_cuda_trim_scratch() == 0
    third = run("denoise_wavelet_atrous_spec", x, blobs.atrous(5, 0.03))
    np.testing.assert_array_equal(first, again)
    np.testing.assert_array_equal(first, third)
