"""Comparison helpers shared by the parity tests (tolerances are stated here)."""
import numpy as np

# f16-format parity: at most one binary16 ulp per element (the reference's
# Halide lowering of float16 casts / log / pow is not reproducible here).
F16_ULPS = 1
# FP32 plain form against the FP32 restatement.
F32_MAX_ABS = 1e-4
MIN_PSNR_DB = 60.0


def f16_ulp_distance(a, b):
    """Elementwise distance in binary16 ulps between two arrays of f16 values."""
    a = np.asarray(a, dtype=np.float32).astype(np.float16).view(np.int16).astype(np.int32)
    b = np.asarray(b, dtype=np.float32).astype(np.float16).view(np.int16).astype(np.int32)
    # map sign-magnitude to a monotone integer line
    a = np.where(a < 0, -32768 - a, a)
    b = np.where(b < 0, -32768 - b, b)
    return np.abs(a - b)


def psnr(a, b, peak=1.0):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)


def assert_f16_parity(got, want, ulps=F16_ULPS, what=""):
    d = f16_ulp_distance(got, want)
    assert d.max() <= ulps, f"{what}: max {d.max()} f16 ulps at {np.unravel_index(d.argmax(), d.shape)}"
    p = psnr(got, want, peak=max(1.0, float(np.max(np.abs(want)))))
    assert p >= MIN_PSNR_DB, f"{what}: PSNR {p:.1f} dB"
    return int(d.max()), int((d > 0).sum())


def assert_f32_parity(got, want, max_abs=F32_MAX_ABS, what=""):
    err = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64))
    assert err.max() <= max_abs, f"{what}: max-abs {err.max():.3g}"
    p = psnr(got, want, peak=max(1.0, float(np.max(np.abs(want)))))
    assert p >= MIN_PSNR_DB, f"{what}: PSNR {p:.1f} dB"
