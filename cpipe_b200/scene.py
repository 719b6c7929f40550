"""Seeded synthetic raw frames for the benchmark and the tests.

The scene is linear gradients + 20 axis-aligned rectangles of uniform
reflectance in [0.05, 0.9] + a sinusoidal zone plate, mosaicked to the CFA,
then Poisson-Gaussian noise var = a*x + b in normalised units
(x_noisy = a * Poisson(x / a) + N(0, b)), scaled to the bit depth above the
black level and clamped to the white level.  A counter-based Philox generator
with a fixed seed per configuration makes every run produce the same frame.
"""
import numpy as np

RGGB = (0, 1, 1, 2)
SONY_QBC = (0, 0, 1, 1, 0, 0, 1, 1, 1, 1, 2, 2, 1, 1, 2, 2)


def scene_rgb(width, height, seed):
    """Linear RGB scene in [0, 1], float32, HxWx3."""
    rng = np.random.Generator(np.random.Philox(seed))
    y = np.linspace(0.0, 1.0, height, dtype=np.float32)[:, None]
    x = np.linspace(0.0, 1.0, width, dtype=np.float32)[None, :]
    img = np.empty((height, width, 3), np.float32)
    img[..., 0] = 0.15 + 0.55 * x + 0.1 * y
    img[..., 1] = 0.2 + 0.4 * y + 0.15 * x
    img[..., 2] = 0.1 + 0.3 * (1.0 - x) + 0.25 * y
    for _ in range(20):
        x0, x1 = np.sort(rng.integers(0, width, 2))
        y0, y1 = np.sort(rng.integers(0, height, 2))
        img[y0:y1 + 1, x0:x1 + 1] = rng.uniform(0.05, 0.9, 3).astype(np.float32)
    # zone plate in the central third
    cy, cx = height / 2.0, width / 2.0
    rr = min(height, width) / 6.0
    ys = slice(int(cy - rr), int(cy + rr))
    xs = slice(int(cx - rr), int(cx + rr))
    yy, xx = np.mgrid[ys, xs].astype(np.float32)
    d2 = ((yy - cy) ** 2 + (xx - cx) ** 2) / (rr * rr)
    zp = 0.5 + 0.4 * np.cos(np.pi * 0.5 * rr * d2)
    img[ys, xs] = (zp[..., None] * np.array([0.9, 0.85, 0.8], np.float32)).astype(np.float32)
    return np.clip(img, 0.0, 1.0)


def mosaic(rgb, cfa=RGGB, repeat=2):
    h, w, _ = rgb.shape
    out = np.empty((h, w), np.float32)
    for yy in range(repeat):
        for xx in range(repeat):
            out[yy::repeat, xx::repeat] = rgb[yy::repeat, xx::repeat, cfa[yy * repeat + xx]]
    return out


def raw_frame(width, height, seed, bits=12, black=64, a=1e-3, b=1e-5, cfa=RGGB, quad_bayer=False):
    """uint16 raw frame (HxW) with the given noise model and levels."""
    rgb = scene_rgb(width, height, seed)
    clean = mosaic(rgb, SONY_QBC if quad_bayer else cfa, 4 if quad_bayer else 2)
    rng = np.random.Generator(np.random.Philox(seed + 1))
    noisy = a * rng.poisson(clean.astype(np.float64) / a) + rng.normal(0.0, np.sqrt(b), clean.shape)
    white = (1 << bits) - 1
    v = np.rint(noisy * (white - black)) + black
    return np.clip(v, 0, white).astype(np.uint16)
