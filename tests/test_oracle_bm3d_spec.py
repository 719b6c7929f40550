"""The FP64 two-stage BM3D oracle (oracle/oracle_bm3d.c) against properties of
the published algorithm.  No reference output exists for it (the reference's
denoise.bm3d is a 2x2 box blend), so these checks pin the restatement:
perfect reconstruction with nothing thresholded, constants preserved, grouping
by a brute-force restatement of the matching rule, copy cases, and a denoising
gain on a seeded scene."""
import numpy as np
import oracle
import pytest
from bm3d_scenes import clean_rgb, noisy_rgba, psnr
from cpipe_b200 import blobs


def rgba32(x):
    return np.asarray(x, np.float32)


def test_perfect_reconstruction_without_threshold():
    x = rgba32(noisy_rgba(clean_rgb(1, 40, 56), 0.05, 1))
    out = oracle.bm3d_spec(x, blobs.bm3d_spec(0.05, lambda3d=0.0, stages=1))
    np.testing.assert_allclose(out, x, atol=1e-12)


@pytest.mark.parametrize("stages", [1, 2])
def test_constant_image_is_preserved(stages):
    x = np.zeros((33, 45, 4), np.float32)
    x[...] = (0.4, 0.55, 0.3, 0.5)
    out = oracle.bm3d_spec(x, blobs.bm3d_spec(0.03, stages=stages))
    # Step 1 keeps the DC exactly; the Wiener gain B^2/(B^2+sigma^2) of step 2
    # shrinks it by sigma^2/B^2 (about 1e-5 relative here).
    np.testing.assert_allclose(out, x, atol=1e-12 if stages == 1 else 1e-4)


def brute_group(q, x, y, ns, n2, tau):
    R = (ns - 1) // 2
    h, w = q.shape
    ref = q[y:y + 8, x:x + 8].astype(np.int64)
    cands = []
    for yy in range(max(0, y - R), min(h - 8, y + R) + 1):
        for xx in range(max(0, x - R), min(w - 8, x + R) + 1):
            if (xx, yy) == (x, y):
                continue
            d = int(((ref - q[yy:yy + 8, xx:xx + 8]) ** 2).sum())
            if d <= int(np.floor(64.0 * tau)):
                cands.append((d, yy, xx))
    cands.sort()
    return [(x, y)] + [(xx, yy) for _, yy, xx in cands[:n2 - 1]]


@pytest.mark.parametrize("ns,n2,tau", [(39, 16, 2500.0), (11, 8, 400.0), (5, 16, 16000.0)])
def test_grouping_matches_brute_force(ns, n2, tau):
    x = rgba32(noisy_rgba(clean_rgb(2, 48, 64), 0.03, 2))
    q = oracle.bm3d_quantise_rgb(x)
    for (bx, by) in [(0, 0), (21, 12), (56, 40), (30, 3)]:
        assert oracle.bm3d_match(q, bx, by, ns, n2, tau) == brute_group(q, bx, by, ns, n2, tau)


def test_grouping_tie_break_is_raster_order():
    q = np.zeros((24, 24), np.uint8)  # every candidate ties at distance 0
    g = oracle.bm3d_match(q, 8, 8, 9, 16, 0.0)
    assert g[0] == (8, 8)
    assert g[1:] == [(4, 4), (5, 4), (6, 4), (7, 4), (8, 4), (9, 4), (10, 4), (11, 4), (12, 4),
                     (4, 5), (5, 5), (6, 5), (7, 5), (8, 5), (9, 5)]


def test_quantised_luminance():
    x = np.array([[[0.3, 0.6, 0.9, 1.0], [-1.0, 0.0, 0.0, 1.0], [2.0, 2.0, 2.0, 1.0],
                   [1.0 / 255 / 2, 0.0, 0.0, 1.0]]], np.float32)
    q = oracle.bm3d_quantise_rgb(x)
    s = np.float32(np.float32(0.3) + np.float32(0.6)) + np.float32(0.9)
    assert q[0, 0] == np.rint(np.float32(s * np.float32(1.0 / 3.0)) * np.float32(255.0))
    assert list(q[0, 1:]) == [0, 255, 0]


@pytest.mark.parametrize("h,w,sigma", [(7, 30, 0.03), (30, 5, 0.03), (20, 20, 0.0), (20, 20, -1.0)])
def test_copy_cases(h, w, sigma):
    x = rgba32(noisy_rgba(clean_rgb(3, h, w), 0.03, 3))
    out = oracle.bm3d_spec(x, blobs.bm3d_spec(sigma))
    np.testing.assert_array_equal(out, x)


def test_bad_parameters_are_refused():
    x = np.zeros((16, 16, 4), np.float32)
    for kw in (dict(n2=3), dict(n2=32), dict(ns=40), dict(ns=47), dict(nstep=0), dict(stages=3),
               dict(tau_match1=20000.0)):
        with pytest.raises(ValueError):
            oracle.bm3d_spec(x, blobs.bm3d_spec(0.03, **kw))


def test_denoising_gain_and_second_stage():
    clean = clean_rgb(4, 96, 128)
    x = rgba32(noisy_rgba(clean, 0.03, 4))
    p_noisy = psnr(x[..., :3], clean)
    s1 = oracle.bm3d_spec(x, blobs.bm3d_spec(0.03, stages=1))
    s2 = oracle.bm3d_spec(x, blobs.bm3d_spec(0.03, stages=2))
    assert np.array_equal(s2[..., 3], x[..., 3])
    p1, p2 = psnr(s1[..., :3], clean), psnr(s2[..., :3], clean)
    assert p1 > p_noisy + 6.0, (p_noisy, p1)
    assert p2 > p1, (p1, p2)
