"""The allocation-free 3D LUT entry point (cpipe_cuda_color_3d_lut_noalloc).

It exists for callers that must not allocate device memory while they process
frames -- a frame loop with a fixed latency budget, where an allocator call can
block on the device, or a host that fixes each plugin's device memory at
start-up.  Instead of allocating per call it keeps the LUT in a fixed device
array inside the library.  This test calls it through the C ABI twice in a row,
with different LUTs (the second call must not see the first call's LUT), and
checks each result against the regular cpipe_cuda_color_3d_lut on the same
device buffers, within the f16 tolerance the other parity tests use.  It also
checks that warm calls leave the device's memory figures unchanged, and the
documented refusals: LUTs above 65 per edge and host buffers.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest
from cpipe_b200 import _abi as A
from cpipe_b200 import DeviceImage, blobs, call_entry, call_filter, last_error
from parity import assert_f16_parity

pytestmark = pytest.mark.gpu


def lut_values(size, seed):
    g = np.linspace(0.0, 1.0, size, dtype=np.float64)
    r, gg, b = np.meshgrid(g, g, g, indexing="ij")
    rng = np.random.default_rng(seed)
    gam = rng.uniform(0.7, 1.3, 3)
    out = np.stack([r ** gam[0] + 0.03 * gg, gg ** gam[1] + 0.03 * b, b ** gam[2] + 0.03 * r], -1)
    return np.clip(out, 0.0, 1.0).astype(np.float32)


class DeviceFrame:
    def __init__(self, arr):
        self.arr = np.ascontiguousarray(arr)
        self.ptr = C.c_void_p()
        L = A.lib()
        assert L.cpipe_cuda_device_alloc(self.arr.nbytes, C.byref(self.ptr)) == 0
        assert L.cpipe_cuda_memcpy_h2d(self.ptr, self.arr.ctypes.data, self.arr.nbytes) == 0

    def image(self):
        return DeviceImage(self.ptr.value, self.arr.shape, self.arr.dtype)

    def read(self):
        out = np.empty_like(self.arr)
        assert A.lib().cpipe_cuda_synchronize() == 0
        assert A.lib().cpipe_cuda_memcpy_d2h(out.ctypes.data, self.ptr, out.nbytes) == 0
        return out

    def free(self):
        A.lib().cpipe_cuda_device_free(self.ptr)


def frame(seed, h=123, w=217):
    x = np.random.default_rng(seed).uniform(-0.05, 1.05, size=(h, w, 4)).astype(np.float16)
    x[..., 3] = 1.0
    return x


def test_noalloc_lut_matches_regular_filter_twice(cuda_device):
    cases = [(33, 0, frame(1)), (17, 1, frame(2))]  # (edge, interpolation, input)
    for size, interp, x in cases:
        blob = blobs.lut3d(size, lut_values(size, size), interp)
        src = DeviceFrame(x)
        ref = DeviceFrame(np.zeros_like(x))
        got = DeviceFrame(np.zeros_like(x))
        assert call_filter("color_3d_lut", [src.image()], [ref.image()], blob) == 0, last_error()
        assert call_entry("cpipe_cuda_color_3d_lut_noalloc", [src.image()], [got.image()], blob) == 0, last_error()
        want = ref.read()
        out = got.read()
        assert_f16_parity(out, want, what=f"noalloc lut {size}^3 interp {interp}")
        assert np.array_equal(out.view(np.uint16), want.view(np.uint16))
        for f in (src, ref, got):
            f.free()


def memory_stats():
    vals = [C.c_uint64() for _ in range(4)]
    assert A.lib().cpipe_cuda_memory_stats(*[C.byref(v) for v in vals]) == 0, last_error()
    return tuple(v.value for v in vals)


def test_noalloc_lut_allocates_nothing(cuda_device):
    """Its defining property: once the device is warm, calls change neither
    the library's scratch pool, nor its prepared-table cache, nor the device's
    free memory."""
    x = frame(4, 301, 257)
    src, dst = DeviceFrame(x), DeviceFrame(np.zeros_like(x))
    blob = blobs.lut3d(33, lut_values(33, 7), 0)
    assert call_entry("cpipe_cuda_color_3d_lut_noalloc", [src.image()], [dst.image()], blob) == 0, last_error()
    assert A.lib().cpipe_cuda_synchronize() == 0
    before = memory_stats()
    for k in range(2):
        blob = blobs.lut3d(17 + 16 * k, lut_values(17 + 16 * k, 8 + k), k)
        assert call_entry("cpipe_cuda_color_3d_lut_noalloc", [src.image()], [dst.image()], blob) == 0, last_error()
    assert A.lib().cpipe_cuda_synchronize() == 0
    after = memory_stats()
    names = ("scratch reserved", "scratch used", "device free", "prepared tables")
    assert before == after, {n: (b, a) for n, b, a in zip(names, before, after) if b != a}
    src.free()
    dst.free()


def test_noalloc_lut_refusals(cuda_device):
    x = frame(3, 8, 8)
    src = DeviceFrame(x)
    dst = DeviceFrame(np.zeros_like(x))
    too_big = blobs.lut3d(66, np.zeros(66 ** 3 * 3, np.float32), 0)
    assert call_entry("cpipe_cuda_color_3d_lut_noalloc", [src.image()], [dst.image()], too_big) == A.BAD_INDEX
    assert "65" in last_error()
    ok_blob = blobs.lut3d(5, lut_values(5, 5), 0)
    assert call_entry("cpipe_cuda_color_3d_lut_noalloc", [x], [np.zeros_like(x)], ok_blob) == A.UNSUPPORTED
    src.free()
    dst.free()
