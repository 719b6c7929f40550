"""GPU parity of every filter, called through the C-ABI filter seam
(HalideParamFilterEntry with host buffers, which the library stages through the
device), against the CPU oracle on the same seeded inputs.

Tolerances (tests/parity.py): integer paths bit-exact; RGBA16F outputs within
one binary16 ulp and PSNR >= 60 dB (in practice the kernels are bit-exact for
all nodes without transcendentals); the FP32 plain form within max-abs 1e-4 and
PSNR >= 60 dB.  Sizes include 1x1, odd and non-tile-multiple shapes."""
import numpy as np
import oracle
import pytest
from cpipe_b200 import DeviceImage, _abi, blobs, call_filter, last_error
from parity import assert_f16_parity, assert_f32_parity, f16_ulp_distance

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (3, 5), (45, 67), (128, 256)]
CFAS = [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)]


def run(aot, inputs, outputs, blob=None):
    st = call_filter(aot, inputs, outputs, blob)
    assert st == 0, f"{aot}: status {st} {last_error()}"
    return outputs[0]


def bayer(seed, h, w, lo=0.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=(h, w)).astype(np.float32)


def rgba(seed, h, w, lo=0.0, hi=1.0, dtype=np.float16):
    x = np.random.default_rng(seed).uniform(lo, hi, size=(h, w, 4)).astype(dtype)
    x[..., 3] = np.random.default_rng(seed + 1).uniform(0.5, 1.0, size=(h, w)).astype(dtype)
    return x


@pytest.mark.parametrize("h,w", SIZES)
def test_raw_point_filters(cuda_device, h, w):
    r = np.random.default_rng(10)
    raw = r.integers(0, 4096, size=(h, w), dtype=np.uint16)
    out = run("precision_convert_r16u_to_f32", [raw], [np.zeros((h, w), np.float32)])
    np.testing.assert_array_equal(out, oracle.r16u_to_f32(raw))
    table = np.sort(r.integers(0, 65535, size=3000)).astype(np.uint16)
    out = run("linearize_dng_lut", [raw], [np.zeros((h, w), np.float32)], blobs.linearize(table))
    np.testing.assert_array_equal(out, oracle.linearize(raw, table)[1])
    for cfa in CFAS:
        x = bayer(11, h, w, 0, 4400)
        blob = blobs.blacklevel([64.0, 60.0, 70.5, 66.25], 4095, cfa)
        out = run("blacklevel_dng_levels", [x], [np.zeros_like(x)], blob)
        np.testing.assert_array_equal(out, oracle.blacklevel(x, blob)[1])


@pytest.mark.parametrize("h,w", SIZES)
def test_gainmap_filter(cuda_device, h, w):
    r = np.random.default_rng(12)
    x = bayer(13, h, w)
    cases = [
        blobs.gainmap_dispatch([dict(points_v=13, points_h=17, spacing_v=max(h - 1, 1) / 12.0,
                                     spacing_h=max(w - 1, 1) / 16.0, gains=r.uniform(1.0, 1.8, 13 * 17))]),
        blobs.gainmap_dispatch([dict(points_v=2, points_h=3, spacing_v=3.5, spacing_h=1.25, origin_v=-1.0,
                                     origin_h=2.0, gains=r.uniform(0.5, 2.0, 6))]),
        blobs.gainmap_dispatch([dict(plane=p, planes=4, points_v=3, points_h=4, spacing_v=2.0, spacing_h=3.0,
                                     gains=r.uniform(0.9, 1.5, 12)) for p in (2, 0, 3, 1)]),
        blobs.gainmap_dispatch([dict(plane=p, planes=4, points_v=2, points_h=2, spacing_v=4.0, spacing_h=4.0,
                                     gains=r.uniform(0.9, 1.5, 4)) for p in range(4)], cfa_repeat=(4, 4)),
    ]
    for blob in cases:
        out = run("lens_shading_gainmap", [x], [np.zeros_like(x)], blob)
        np.testing.assert_array_equal(out, oracle.gainmap(x, blob)[1])


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("algo", ["bilinear", "rcd", "amaze"])
def test_demosaic_filters(cuda_device, h, w, algo):
    for i, cfa in enumerate(CFAS):
        x = bayer(20 + i, h, w)
        x[::7, ::5] = 0.0  # zero greens exercise the RCD ratio guard
        out = run(f"demosaic_{algo}", [x], [np.zeros((h, w, 4), np.float16)], blobs.demosaic(cfa))
        want = oracle.demosaic(algo, x, cfa, f16=True)
        assert_f16_parity(out, want, what=f"{algo} {cfa}")
        out32 = run(f"demosaic_{algo}", [x], [np.zeros((h, w, 4), np.float32)], blobs.demosaic(cfa))
        assert_f32_parity(out32, oracle.demosaic(algo, x, cfa, f16=False), what=f"{algo} f32 {cfa}")


@pytest.mark.parametrize("h,w", SIZES + [(9, 4)])
def test_qbc_remosaic_filter_bit_exact(cuda_device, h, w):
    raw = np.random.default_rng(30).integers(0, 65535, size=(h, w), dtype=np.uint16)
    out = run("demosaic_quad_bayer_remosaic", [raw], [np.zeros_like(raw)])
    np.testing.assert_array_equal(out, oracle.qbc_remosaic(raw))


RGBA_CASES = [
    ("wb_dual_illuminant", lambda: blobs.wb([0.5, 1.0, 0.625]), lambda x, f: oracle.wb(x, [0.5, 1.0, 0.625], f)),
    ("colormatrix_dng_to_working", lambda: blobs.colormatrix([1.7, -0.4, -0.3, -0.2, 1.5, -0.3, 0.05, -0.3, 1.25]),
     lambda x, f: oracle.colormatrix(x, [1.7, -0.4, -0.3, -0.2, 1.5, -0.3, 0.05, -0.3, 1.25], f)),
    ("denoise_bm3d_step1", lambda: blobs.bm3d(0.0161), lambda x, f: oracle.bm3d_parity(x, 0.0161, f)),
    ("denoise_bm3d_step1", lambda: blobs.bm3d(0.05), lambda x, f: oracle.bm3d_parity(x, 0.05, f)),
    ("denoise_guided_filter", lambda: blobs.guided(1, 0.015), lambda x, f: oracle.guided(x, 1, 0.015, f)),
    ("denoise_guided_filter", lambda: blobs.guided(8, 1e-3), lambda x, f: oracle.guided(x, 8, 1e-3, f)),
    ("denoise_wavelet_bayes_shrink", lambda: blobs.wavelet(1.0), lambda x, f: oracle.wavelet(x, 1.0, f)),
    ("denoise_wavelet_bayes_shrink", lambda: blobs.wavelet(1.7), lambda x, f: oracle.wavelet(x, 1.7, f)),
    ("tone_filmic_rgb", lambda: blobs.filmic(), lambda x, f: oracle.filmic(x, f16=f)),
    ("tone_filmic_rgb", lambda: blobs.filmic(0.7, 1.4, 1.3, 0.6, 1.5),
     lambda x, f: oracle.filmic(x, 0.7, 1.4, 1.3, 0.6, 1.5, f16=f)),
]


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("case", range(len(RGBA_CASES)))
def test_rgba_filters(cuda_device, h, w, case):
    aot, blob, ref = RGBA_CASES[case]
    x = rgba(40 + case, h, w, 0.0, 1.5 if "filmic" in aot else 1.0)
    out = run(aot, [x], [np.zeros_like(x)], blob())
    assert_f16_parity(out, ref(x.astype(np.float32), True), what=aot)
    x32 = x.astype(np.float32)
    out32 = run(aot, [x32], [np.zeros_like(x32)], blob())
    assert_f32_parity(out32, ref(x32, False), what=aot + " f32")


def test_rgba_pointwise_bit_exact(cuda_device):
    """WB, colormatrix, BM3D parity form, guided and wavelet have no
    transcendentals: the CUDA kernels reproduce the oracle bit for bit."""
    x = rgba(7, 61, 93)
    for aot, blob, ref in RGBA_CASES[:8]:
        out = run(aot, [x], [np.zeros_like(x)], blob())
        assert f16_ulp_distance(out, ref(x.astype(np.float32), True)).max() == 0, aot


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("interp", [0, 1])
def test_lut_filter(cuda_device, h, w, interp):
    r = np.random.default_rng(50)
    S = 33
    grid = np.linspace(0, 1, S, dtype=np.float32)
    rr, gg, bb = np.meshgrid(grid, grid, grid, indexing="ij")
    lut = np.stack([rr ** 0.9 + 0.02 * gg, gg ** 1.1 + 0.02 * bb, bb ** 0.8 + 0.02 * rr], -1).astype(np.float32)
    x = rgba(51, h, w, -0.1, 1.1)
    x[0, 0, :3] = 1.0  # the top cell edge (r0 = S-2, dr = 1)
    out = run("color_3d_lut", [x], [np.zeros_like(x)], blobs.lut3d(S, lut, interp))
    assert_f16_parity(out, oracle.lut3d(x.astype(np.float32), lut, S, interp, True), what="lut")
    x32 = x.astype(np.float32)
    out32 = run("color_3d_lut", [x32], [np.zeros_like(x32)], blobs.lut3d(S, lut, interp))
    assert_f32_parity(out32, oracle.lut3d(x32, lut, S, interp, False), what="lut f32")


def opcode3_blobs(w, h):
    warp = blobs.warp_record([(1.0, -0.08, 0.02, 0.0, 0.0, 0.0)])
    warp3 = blobs.warp_record([(1.0, -0.05, 0.01, 0.0, 0.001, -0.002), (0.99, 0.03, 0.0, 0.0, 0.0, 0.0),
                               (1.01, -0.1, 0.04, -0.01, 0.0, 0.0)], cx_hat=0.45, cy_hat=0.55)
    vig = blobs.vignette_record([0.4, -0.1, 0.05, 0.0, 0.01], cx_hat=0.4, cy_hat=0.6)
    badc = _abi.Opcode3DispatchRecord()
    badc.id = 4
    badl = _abi.Opcode3DispatchRecord()
    badl.id, badl.point_count, badl.rect_count = 5, 2, 1
    trim = _abi.Opcode3DispatchRecord()
    trim.id, trim.top, trim.left, trim.bottom, trim.right = 6, 1, 2, max(1, h - 1), max(2, w - 1)
    pts = [(min(1, h - 1), min(2, w - 1)), (0, 0)]
    rects = [(0, 0, min(2, h), min(3, w))]
    return [blobs.opcode3_dispatch([warp]), blobs.opcode3_dispatch([warp3]), blobs.opcode3_dispatch([vig]),
            blobs.opcode3_dispatch([badc]), blobs.opcode3_dispatch([badl], pts, rects),
            blobs.opcode3_dispatch([trim]), blobs.opcode3_dispatch([vig, warp, badl, trim], pts, rects)]


@pytest.mark.parametrize("h,w", SIZES)
def test_opcode_list_3_filter(cuda_device, h, w):
    x = rgba(60, h, w)
    x[0, 0, :3] = 0.0
    for i, blob in enumerate(opcode3_blobs(w, h)):
        out = run("lens_dng_opcode_list_3", [x], [np.zeros_like(x)], blob)
        st, want = oracle.opcode3(x.astype(np.float32), blob, True)
        assert st == 0
        assert_f16_parity(out, want, what=f"opcode3 case {i}")
        x32 = x.astype(np.float32)
        out32 = run("lens_dng_opcode_list_3", [x32], [np.zeros_like(x32)], blob)
        assert_f32_parity(out32, oracle.opcode3(x32, blob, False)[1], max_abs=2e-4, what=f"opcode3 f32 case {i}")


def test_precision_convert_rgba(cuda_device):
    x = bayer(70, 37, 53, -0.5, 2.0)
    out = run("precision_convert_f32_to_rgba16f", [x], [np.zeros((37, 53, 4), np.float16)])
    np.testing.assert_array_equal(out.astype(np.float32), oracle.f32_to_rgba16f(x))
    x16 = rgba(71, 37, 53, -0.2, 1.2)
    out8 = run("precision_convert_rgba16f_to_rgba8", [x16], [np.zeros((37, 53, 4), np.uint8)])
    np.testing.assert_array_equal(out8, oracle.rgba16f_to_unorm(x16.astype(np.float32), True))
    out16 = run("precision_convert_rgba16f_to_rgba16u", [x16], [np.zeros((37, 53, 4), np.uint16)])
    np.testing.assert_array_equal(out16, oracle.rgba16f_to_unorm(x16.astype(np.float32), False))


def test_filter_error_codes(cuda_device):
    x = bayer(80, 8, 8)
    o = np.zeros_like(x)
    assert call_filter("blacklevel_dng_levels", [x], [o], None) == _abi.BAD_INDEX
    assert call_filter("blacklevel_dng_levels", [x], [o], b"\x00" * 8) == _abi.BAD_INDEX
    assert call_filter("blacklevel_dng_levels", [x], [o], blobs.blacklevel([100] * 4, 50, (0, 1, 1, 2))) == \
        _abi.NEED_METADATA
    assert call_filter("blacklevel_dng_levels", [x.astype(np.float16)], [o],
                       blobs.blacklevel([0] * 4, 10, (0, 1, 1, 2))) == _abi.BAD_PRECISION
    assert call_filter("blacklevel_dng_levels", [x], [np.zeros((4, 8), np.float32)],
                       blobs.blacklevel([0] * 4, 10, (0, 1, 1, 2))) == _abi.BAD_INDEX
    assert call_filter("linearize_dng_lut", [x.astype(np.uint16)], [o], b"\x00\x00\x00\x00") == _abi.NEED_METADATA
    assert call_filter("lens_shading_gainmap", [x], [o], blobs.gainmap_dispatch([])) == _abi.NEED_METADATA
    missing_plane = blobs.gainmap_dispatch([dict(plane=p, planes=4, points_v=1, points_h=1, spacing_v=1.0,
                                                 spacing_h=1.0, gains=[1.0]) for p in (0, 1, 2, 2)])
    assert call_filter("lens_shading_gainmap", [x], [o], missing_plane) == _abi.NEED_METADATA
    y = rgba(81, 4, 4)
    assert call_filter("color_3d_lut", [y], [np.zeros_like(y)], blobs.lut3d(1, [0, 0, 0])) == _abi.BAD_INDEX
    assert call_filter("color_3d_lut", [y], [np.zeros_like(y)], blobs.lut3d(3, np.zeros(30))) == _abi.BAD_INDEX
    unk = _abi.Opcode3DispatchRecord()
    assert call_filter("lens_dng_opcode_list_3", [y], [np.zeros_like(y)], blobs.opcode3_dispatch([unk])) == \
        _abi.UNSUPPORTED


def test_device_buffers_in_place(cuda_device, host):
    """The same filters on device pointers (halide_buffer_t.device), no staging."""
    from cpipe_b200 import _abi as A
    h, w = 96, 160
    x = rgba(90, h, w)
    src = host.buffer(A.FMT_R16G16B16A16_SFLOAT, w, h).upload(x)
    dst = host.buffer(A.FMT_R16G16B16A16_SFLOAT, w, h)
    st = call_filter("denoise_guided_filter", [DeviceImage(src.device_ptr, (h, w, 4), np.float16)],
                     [DeviceImage(dst.device_ptr, (h, w, 4), np.float16)], blobs.guided(8, 1e-3))
    assert st == 0
    assert _abi.lib().cpipe_cuda_synchronize() == 0
    assert_f16_parity(dst.download(), oracle.guided(x.astype(np.float32), 8, 1e-3, True), what="device guided")


def test_prepared_table_cache(cuda_device):
    """Linearize, GainMap and LUT tables are cached per (blob bytes, frame
    extent): alternating blobs, more distinct blobs than the cache holds (so
    entries are evicted), the same GainMap blob at two frame sizes and a trim
    in between must all give each blob's own result."""
    r = np.random.default_rng(70)
    lib = _abi.lib()
    raw = r.integers(0, 4096, size=(37, 53), dtype=np.uint16)
    tables = [np.sort(r.integers(0, 65535, size=4096)).astype(np.uint16) for _ in range(11)]
    for rep in range(2):
        for i in (0, 1, 0) + tuple(range(11)) + (3,):
            out = run("linearize_dng_lut", [raw], [np.zeros(raw.shape, np.float32)], blobs.linearize(tables[i]))
            np.testing.assert_array_equal(out, oracle.linearize(raw, tables[i])[1])
        assert lib.cpipe_cuda_trim_scratch() == 0
    gm = blobs.gainmap_dispatch([dict(points_v=5, points_h=7, spacing_v=9.0, spacing_h=11.0,
                                      gains=r.uniform(1.0, 1.8, 35))])
    for h, w in ((40, 64), (33, 90), (40, 64)):
        x = bayer(71, h, w)
        out = run("lens_shading_gainmap", [x], [np.zeros_like(x)], gm)
        np.testing.assert_array_equal(out, oracle.gainmap(x, gm)[1])
    S = 9
    x = rgba(72, 21, 19, -0.1, 1.1)
    luts = [r.uniform(0.0, 1.0, size=(S, S, S, 3)).astype(np.float32) for _ in range(3)]
    for i in (0, 1, 2, 1, 0):
        out = run("color_3d_lut", [x], [np.zeros_like(x)], blobs.lut3d(S, luts[i], 0))
        assert_f16_parity(out, oracle.lut3d(x.astype(np.float32), luts[i], S, 0, True), what=f"lut {i}")


def test_prepared_table_cache_concurrent_callers(cuda_device):
    """Two host threads call the LUT and linearize filters at once with their
    own tables (more distinct blobs than the cache holds): each result must be
    its own table's."""
    import threading
    r = np.random.default_rng(71)
    S = 9
    x = rgba(73, 17, 23, -0.1, 1.1)
    raw = r.integers(0, 4096, size=(19, 21), dtype=np.uint16)
    jobs = []
    for t in range(2):
        luts = [r.uniform(0.0, 1.0, size=(S, S, S, 3)).astype(np.float32) for _ in range(5)]
        tables = [np.sort(r.integers(0, 65535, size=4096)).astype(np.uint16) for _ in range(5)]
        jobs.append((luts, tables))
    errors = []

    def worker(luts, tables):
        try:
            for rep in range(4):
                for i in range(5):
                    out = np.zeros_like(x)
                    assert call_filter("color_3d_lut", [x], [out], blobs.lut3d(S, luts[i], 0)) == 0, last_error()
                    assert_f16_parity(out, oracle.lut3d(x.astype(np.float32), luts[i], S, 0, True), what="lut")
                    lin = np.zeros(raw.shape, np.float32)
                    assert call_filter("linearize_dng_lut", [raw], [lin], blobs.linearize(tables[i])) == 0
                    np.testing.assert_array_equal(lin, oracle.linearize(raw, tables[i])[1])
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=job) for job in jobs]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
