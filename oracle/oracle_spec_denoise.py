"""FP64 restatement of the spec-mode guided filter and a-trous wavelet denoiser
(filters denoise_guided_filter_spec and denoise_wavelet_atrous_spec).

TEST INFRASTRUCTURE: imported only by tests/ as the checker.  The product
library never loads it.

The reference has neither algorithm in this form.  Its guided filter
(nodes/denoise/guided_filter_generator.cpp:45-85) uses the formula below with
the box fixed at 3x3 (radius <= 1) or 5x5 (any larger radius); at radius 1 and
2 the spec filter therefore equals it, which the tests check against the
reference restatement in oracle_nodes.c.  Its wavelet node
(wavelet_bayes_shrink_generator.cpp:57-86) is one 2x2 Haar level on chroma;
the a-trous form keeps its colour space (Y = (r+2g+b)/4, Co = r-b,
Cg = g-(r+b)/2) and its inverse.  Parity with reference output is unpinned
for radius > 2 and for the a-trous form.

Published sources restated here: the guided filter of He, Sun, Tang (ECCV
2010 / TPAMI 2013) in its self-guided per-channel form; the B3-spline a-trous
transform (Starck, Murtagh, A&A 288, 1994); BayesShrink thresholds
T = sigma_n^2 / sigma_x (Chang, Yu, Vetterli, IEEE TIP 9(9), 2000).
"""
import math

import numpy as np

B3 = np.array([1.0, 4.0, 6.0, 4.0, 1.0]) / 16.0


def _box_valid(a, d):
    """Sums over every d x d window of a (valid positions), FP64."""
    c = np.zeros((a.shape[0] + 1, a.shape[1] + 1))
    c[1:, 1:] = np.cumsum(np.cumsum(a, 0), 1)
    return c[d:, d:] - c[:-d, d:] - c[d:, :-d] + c[:-d, :-d]


def guided_spec(x, radius, eps):
    """x: HxWx4.  Per channel: a, b at every position within `radius` of the
    image (outside positions included, their boxes read the clamped image),
    out = max(mean_a v + mean_b, 0); alpha copied."""
    x = np.asarray(x, np.float64)
    R = int(radius)
    d = 2 * R + 1
    n = float(d * d)
    out = x.copy()
    for c in range(3):
        v = x[..., c]
        vp = np.pad(v, 2 * R, mode="edge")
        m = _box_valid(vp, d) / n              # (h + 2R) x (w + 2R), index (i, j) <-> image (i - R, j - R)
        corr = _box_valid(vp * vp, d) / n
        var = np.maximum(corr - m * m, 0.0)
        a = var / (var + eps)
        b = m - a * m
        ma = _box_valid(a, d) / n
        mb = _box_valid(b, d) / n
        out[..., c] = np.maximum(ma * v + mb, 0.0)
    return out


def _b3(c, s):
    """Separable B3-spline smoothing with taps s apart, clamped edges."""
    h, w = c.shape
    xi = np.arange(w)
    yi = np.arange(h)
    rows = sum(B3[k] * c[:, np.clip(xi + (k - 2) * s, 0, w - 1)] for k in range(5))
    return sum(B3[k] * rows[np.clip(yi + (k - 2) * s, 0, h - 1), :] for k in range(5))


def band_gain(level):
    """2D white-noise gain of band `level` (1-based): the L2 norm of
    Phi_{level-1} - Phi_level, Phi_k = phi_k x phi_k, phi_k the 1D smoothing
    filter after k levels."""
    phis = [np.array([1.0])]
    for k in range(1, level + 1):
        s = 1 << (k - 1)
        up = np.zeros(4 * s + 1)
        up[::s] = B3
        phis.append(np.convolve(phis[-1], up))
    p, f = phis[level - 1], phis[level]
    pad = (len(f) - len(p)) // 2
    p = np.pad(p, pad)
    return math.sqrt((p @ p) ** 2 - 2.0 * (p @ f) ** 2 + (f @ f) ** 2)


def decompose(ch, levels):
    """(bands w_1..w_L, residual c_L) of one channel."""
    bands = []
    c = np.asarray(ch, np.float64)
    for j in range(levels):
        n = _b3(c, 1 << j)
        bands.append(c - n)
        c = n
    return bands, c


def atrous_thresholds(bands, noise, strength):
    out = []
    for w, sn in zip(bands, noise):
        sw2 = float(np.mean(w * w))
        sx = math.sqrt(max(sw2 - sn * sn, 0.0))
        out.append(0.0 if strength == 0.0 else (strength * sn * sn / sx if sx > 0.0 else math.inf))
    return out


def atrous_spec(x, levels, sigma, luma_strength=1.0, chroma_strength=1.0):
    x = np.asarray(x, np.float64)
    if levels == 0:
        return x.copy()
    r, g, b = x[..., 0], x[..., 1], x[..., 2]
    chans = [(r + 2.0 * g + b) * 0.25, r - b, g - (r + b) * 0.5]
    gains = [math.sqrt(6.0) / 4.0, math.sqrt(2.0), math.sqrt(1.5)]
    strengths = [luma_strength, chroma_strength, chroma_strength]
    res = []
    for c in range(3):
        bands, cl = decompose(chans[c], levels)
        noise = [sigma * gains[c] * band_gain(j + 1) for j in range(levels)]
        thr = atrous_thresholds(bands, noise, strengths[c])
        v = cl
        for j in reversed(range(levels)):
            w = bands[j]
            v = v + np.sign(w) * np.maximum(np.abs(w) - thr[j], 0.0)
        res.append(v)
    y, co, cg = res
    t = y - 0.5 * cg
    out = x.copy()
    out[..., 0] = np.maximum(t + 0.5 * co, 0.0)
    out[..., 1] = np.maximum(t + cg, 0.0)
    out[..., 2] = np.maximum(t - 0.5 * co, 0.0)
    return out
