"""GPU two-stage BM3D (aot_id denoise_bm3d_spec) against the FP64 CPU oracle.

The CUDA path computes in FP32 and, for RGBA16F buffers, rounds its output to
binary16; the oracle computes the same definition in FP64.  Groups are formed
from exact integer distances of the same FP32-quantised luminance, so step 1
groups the same blocks on both sides.  Differences come from FP32 rounding of
the transforms, from hard-threshold decisions on coefficients within rounding
of lambda*sigma, from step-2 luminance values within rounding of a quantiser
step, and from the binary16 output.  Tolerances per case: PSNR against the
oracle >= 55 dB over RGB (peak 1) and max-abs <= 5e-3; alpha bit-exact.
Measured values are printed (pytest -s).

At 4032x3024 the oracle is run on a crop whose origin lies on the reference
grid; pixels further than 2 x (2R + 8) from the crop edge depend on the same
input as in the full frame and are compared."""
import numpy as np
import oracle
import pytest
from bm3d_scenes import clean_rgb, noisy_rgba, psnr
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs, call_filter, last_error

pytestmark = pytest.mark.gpu

MIN_PSNR_DB = 55.0
MAX_ABS = 5e-3


def gpu_bm3d(x, blob):
    out = np.zeros_like(x)
    st = call_filter("denoise_bm3d_spec", [x], [out], blob)
    assert st == 0, f"status {st}: {last_error()}"
    return out


def compare(got, want, what):
    g = np.asarray(got, np.float64)[..., :3]
    w = np.asarray(want, np.float64)[..., :3]
    err = float(np.max(np.abs(g - w)))
    p = psnr(g, w)
    print(f"{what}: max-abs {err:.3g} PSNR {p:.1f} dB")
    assert p >= MIN_PSNR_DB and err <= MAX_ABS, (what, err, p)
    return err, p


CASES = [
    (96, 128, 0.03, {}),
    (77, 101, 0.03, {}),
    (64, 64, 0.05, dict(stages=1)),
    (40, 72, 0.03, dict(n2=4, ns=21, nstep=4)),
    (50, 61, 0.02, dict(n2=1)),
    (8, 8, 0.03, {}),
    (9, 300, 0.03, dict(n2=8, nstep=1, ns=15)),
    (130, 70, 0.08, dict(tau_match1=16000.0, tau_match2=3000.0, kaiser_beta=0.0)),
]


@pytest.mark.parametrize("h,w,sigma,kw", CASES)
def test_bm3d_spec_matches_fp64_oracle(cuda_device, h, w, sigma, kw):
    clean = clean_rgb(h * 7 + w, h, w)
    x = noisy_rgba(clean, sigma, h + w)
    blob = blobs.bm3d_spec(sigma, **kw)
    got = gpu_bm3d(x, blob)
    want = oracle.bm3d_spec(x.astype(np.float32), blob)
    np.testing.assert_array_equal(got[..., 3], x[..., 3])
    compare(got.astype(np.float32), want, f"{w}x{h} sigma {sigma} {kw}")


def test_bm3d_spec_f32_buffers(cuda_device):
    clean = clean_rgb(5, 72, 88)
    x = noisy_rgba(clean, 0.03, 5, dtype=np.float32)
    blob = blobs.bm3d_spec(0.03)
    got = gpu_bm3d(x, blob)
    want = oracle.bm3d_spec(x, blob)
    err, _ = compare(got, want, "f32 buffers")
    assert err <= 1e-3


@pytest.mark.parametrize("h,w,sigma", [(7, 30, 0.03), (30, 5, 0.03), (20, 20, 0.0)])
def test_bm3d_spec_copy_cases(cuda_device, h, w, sigma):
    x = noisy_rgba(clean_rgb(3, h, w), 0.03, 3)
    got = gpu_bm3d(x, blobs.bm3d_spec(sigma))
    np.testing.assert_array_equal(got.view(np.uint16), x.view(np.uint16))


def test_bm3d_spec_refuses_bad_parameters(cuda_device):
    x = noisy_rgba(clean_rgb(3, 16, 16), 0.03, 3)
    for kw in (dict(n2=3), dict(n2=32), dict(ns=40), dict(nstep=9), dict(stages=0)):
        st = call_filter("denoise_bm3d_spec", [x], [np.zeros_like(x)], blobs.bm3d_spec(0.03, **kw))
        assert st == A.BAD_INDEX, kw
    assert call_filter("denoise_bm3d_spec", [x], [np.zeros_like(x)], b"\0" * 8) == A.BAD_INDEX


def test_bm3d_spec_denoises(cuda_device):
    clean = clean_rgb(11, 160, 224)
    x = noisy_rgba(clean, 0.03, 11)
    got = gpu_bm3d(x, blobs.bm3d_spec(0.03)).astype(np.float64)
    p0, p1 = psnr(x[..., :3].astype(np.float64), clean), psnr(got[..., :3], clean)
    print(f"noisy {p0:.2f} dB -> bm3d {p1:.2f} dB")
    assert p1 > p0 + 8.0


def test_bm3d_spec_node(host):
    """com.cpipe.denoise.bm3d with algorithm = "bm3d" submits the same filter."""
    x = noisy_rgba(clean_rgb(12, 48, 64), 0.03, 12)
    F16 = A.FMT_R16G16B16A16_SFLOAT
    src = host.buffer(F16, x.shape[1], x.shape[0]).upload(x)
    src.set_metadata(cs_role="scene_linear_rec2020", applied_steps=["color_matrix"], noise_profile=[(1e-5, 1e-3)])
    out = host.buffer(F16, x.shape[1], x.shape[0])
    st = host.run_node("com.cpipe.denoise.bm3d", [src], [out], {"algorithm": "bm3d", "sigma": 0.03})
    assert st == 0, host.last_error()
    want = oracle.bm3d_spec(x.astype(np.float32), blobs.bm3d_spec(float(np.float32(0.03))))
    compare(out.download().astype(np.float32), want, "node")
    assert out.has_step("denoise.bm3d")
    assert host.run_node("com.cpipe.denoise.bm3d", [src], [out], {"algorithm": "nope"}) == A.BAD_INDEX


def test_bm3d_spec_full_frame_12mp(cuda_device):
    """4032x3024 (12 MP) frame: finite output, and the oracle on a 420x420 crop
    at a reference-grid origin agrees on the crop interior."""
    h, w, sigma = 3024, 4032, 0.032
    clean = clean_rgb(20, h, w, rects=200)
    x = noisy_rgba(clean, sigma, 20)
    blob = blobs.bm3d_spec(sigma)
    got = gpu_bm3d(x, blob)
    assert np.isfinite(got.astype(np.float32)).all()
    full = psnr(got[..., :3].astype(np.float64), clean)
    print(f"12MP: noisy {psnr(x[..., :3].astype(np.float64), clean):.2f} dB -> {full:.2f} dB")
    y0, x0, n, margin = 1503, 2499, 420, 2 * (2 * 19 + 8)
    crop = x[y0:y0 + n, x0:x0 + n].astype(np.float32)
    want = oracle.bm3d_spec(crop, blob)
    inner = slice(margin, n - margin)
    compare(got[y0:y0 + n, x0:x0 + n][inner, inner].astype(np.float32), want[inner, inner], "12MP crop interior")


@pytest.mark.parametrize("h,w,sigma,kw", [(96, 128, 0.03, {}), (77, 101, 0.05, dict(stages=1)),
                                          (50, 61, 0.02, dict(n2=4, nstep=2))])
def test_bm3d_precision_forms_against_fp64(cuda_device, h, w, sigma, kw):
    """Both transform forms against the FP64 oracle on the same input: the
    tensor-core form (FP16 hi/lo split products, FP32 accumulation) and the FP32
    CUDA-core form; binary16 and float32 frames.  The per-form error is printed."""
    clean = clean_rgb(h + 3 * w, h, w)
    for dtype in (np.float16, np.float32):
        x = noisy_rgba(clean, sigma, h * w, dtype=dtype)
        want = oracle.bm3d_spec(x.astype(np.float32), blobs.bm3d_spec(sigma, **kw))
        errs = {}
        for form in ("tensor", "fp32"):
            got = gpu_bm3d(x, blobs.bm3d_spec(sigma, transform=form, **kw)).astype(np.float32)
            errs[form] = compare(got, want, f"{form} {np.dtype(dtype).name} {w}x{h} {kw}")
        if dtype == np.float32:
            assert errs["tensor"][0] <= 2e-3 and errs["fp32"][0] <= 1e-3


@pytest.mark.parametrize("h,w,sigma", [(256, 256, 0.032), (96, 128, 0.03)])
def test_bm3d_screening_form(cuda_device, h, w, sigma):
    """The screening form (transform 2: single FP16 products on the tensor
    cores), which the surrogate's spot check runs, against the FP64 oracle and
    against the split form.  Its error is far below the spot check's 40 dB
    decision margin: >= 50 dB against both (measured values printed)."""
    clean = clean_rgb(h + 5 * w, h, w)
    x = noisy_rgba(clean, sigma, h * w + 1, dtype=np.float16)
    want = oracle.bm3d_spec(x.astype(np.float32), blobs.bm3d_spec(sigma))
    fast = gpu_bm3d(x, blobs.bm3d_spec(sigma, transform="tensor_fp16")).astype(np.float64)[..., :3]
    split = gpu_bm3d(x, blobs.bm3d_spec(sigma, transform="tensor")).astype(np.float64)[..., :3]
    p_oracle, p_split = psnr(fast, np.asarray(want, np.float64)[..., :3]), psnr(fast, split)
    print(f"screening form {w}x{h}: {p_oracle:.1f} dB against the oracle, {p_split:.1f} dB against the split form")
    assert p_oracle >= 50.0 and p_split >= 50.0
    np.testing.assert_array_equal(gpu_bm3d(x, blobs.bm3d_spec(sigma, transform="tensor_fp16"))[..., 3], x[..., 3])
