"""The FP64 oracle of the spec-mode guided filter and a-trous wavelet denoiser
(oracle/oracle_spec_denoise.py), pinned by the properties it must have:

* the spec guided filter at radius 1 and 2 is the reference's own guided
  filter (3x3 and 5x5 boxes, guided_filter_generator.cpp:45-85), restated in
  oracle_nodes.c and pinned there against the reference's golden generator;
* constant images pass through the guided filter unchanged;
* the band gains equal the measured white-noise standard deviation of each
  a-trous band;
* zero thresholds reconstruct the input exactly (the transform is exact);
* on a noisy scene both denoise."""
import math

import numpy as np
import oracle
import oracle_spec_denoise as S
import pytest
from bm3d_scenes import clean_rgb, noisy_rgba, psnr


def scene(h, w, sigma, seed):
    clean = clean_rgb(seed, h, w)
    return clean, noisy_rgba(clean, sigma, seed, dtype=np.float32)


@pytest.mark.parametrize("radius", [1, 2])
def test_guided_spec_equals_the_reference_at_radius_1_and_2(radius):
    _, x = scene(40, 52, 0.03, 3)
    want = oracle.guided(x, radius, 1e-3, f16=False)
    got = S.guided_spec(x, radius, 1e-3)
    err = float(np.max(np.abs(got[..., :3] - want[..., :3])))
    assert err <= 2e-5, err  # FP64 against the reference's FP32 sums


def test_guided_spec_keeps_constants_and_alpha():
    x = np.full((30, 41, 4), 0.37)
    x[..., 3] = 0.6
    got = S.guided_spec(x, 8, 1e-3)
    np.testing.assert_allclose(got[..., :3], 0.37, atol=1e-12)
    np.testing.assert_array_equal(got[..., 3], x[..., 3])


@pytest.mark.parametrize("level", [1, 2, 3, 4, 5])
def test_band_gain_matches_white_noise(level):
    # deep bands are correlated over ~2^level pixels: a larger field keeps the
    # standard-deviation estimate within a few per cent
    size = 384 if level <= 3 else 1024
    rng = np.random.default_rng(level)
    n = rng.normal(0.0, 1.0, (size, size))
    bands, _ = S.decompose(n, level)
    m = 4 * (1 << level)
    std = float(np.std(bands[level - 1][m:-m, m:-m]))
    assert abs(std / S.band_gain(level) - 1.0) < 0.05, (std, S.band_gain(level))


def test_atrous_zero_strength_is_exact_reconstruction():
    _, x = scene(37, 45, 0.02, 5)
    x = np.clip(x, 0.01, None)
    got = S.atrous_spec(x, 5, 0.02, luma_strength=0.0, chroma_strength=0.0)
    np.testing.assert_allclose(got, x, atol=1e-12)


def test_spec_denoisers_denoise():
    clean, x = scene(128, 160, 0.04, 9)
    before = psnr(x[..., :3], clean)
    g = psnr(S.guided_spec(x, 8, 5e-3)[..., :3], clean)
    a = psnr(S.atrous_spec(x, 5, 0.04)[..., :3], clean)
    print(f"noisy {before:.2f} dB, guided r=8 {g:.2f} dB, a-trous 5 levels {a:.2f} dB")
    assert g > before + 1.0 and a > before + 2.0


def test_band_gains_decrease():
    g = [S.band_gain(j) for j in range(1, 7)]
    assert all(g[i] > g[i + 1] > 0.0 for i in range(5)) and math.isclose(g[0], S.band_gain(1))
