"""Seeded RGB test scenes for the two-stage BM3D tests: smooth gradients, axis
aligned rectangles of uniform reflectance and a sinusoidal zone plate (the
scene family of the benchmark's raw generator, here directly in linear RGB),
plus additive Gaussian noise of a given sigma per channel."""
import numpy as np


def clean_rgb(seed, h, w, rects=20):
    r = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    u, v = xx / max(w - 1, 1), yy / max(h - 1, 1)
    img = np.stack([0.15 + 0.5 * u, 0.2 + 0.4 * v, 0.35 + 0.25 * (1 - u) * v], -1)
    for _ in range(rects):
        x0, x1 = sorted(r.integers(0, w, 2))
        y0, y1 = sorted(r.integers(0, h, 2))
        img[y0:y1 + 1, x0:x1 + 1] = r.uniform(0.05, 0.9, 3)
    cx, cy = 0.7 * w, 0.35 * h
    rad2 = ((xx - cx) ** 2 + (yy - cy) ** 2) / (0.2 * min(h, w)) ** 2
    zone = 0.5 + 0.5 * np.cos(np.pi * rad2 * 6.0)
    m = rad2 < 1.0
    img[m] = 0.5 * img[m] + 0.4 * zone[m][:, None]
    return img


def noisy_rgba(clean, sigma, seed, dtype=np.float16):
    n = np.random.default_rng(seed + 1000).normal(0.0, sigma, clean.shape)
    h, w = clean.shape[:2]
    x = np.concatenate([clean + n, np.ones((h, w, 1))], -1)
    x[..., 3] = 0.75
    return x.astype(dtype)


def psnr(a, b, peak=1.0):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(peak * peak / mse)
