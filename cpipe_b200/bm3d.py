"""Two-stage BM3D (filter denoise_bm3d_spec) timed on a seeded synthetic frame.

The frame is the benchmark's linear-RGB scene (cpipe_b200.scene.scene_rgb)
plus additive Gaussian noise of the given sigma, binary16 RGBA, resident on the
device; the filter runs in place on the library's stream and is timed with
CUDA events over `reps` calls after three untimed ones.

    python -m cpipe_b200.bm3d [--width 4032] [--height 3024] [--stages 2]
                              [--transform tensor|fp32|tensor_fp16] [--sigma 0.032] [--reps 5]
"""
import argparse
import ctypes as C

import numpy as np

from . import _abi as A
from . import blobs
from .host import DeviceImage, call_filter, last_error
from .scene import scene_rgb


def noisy_frame(width, height, sigma, seed=0x5EED0006):
    rgb = scene_rgb(width, height, seed)
    noise = np.random.default_rng(seed + 1).normal(0.0, sigma, rgb.shape).astype(np.float32)
    x = np.empty((height, width, 4), np.float16)
    x[..., :3] = rgb + noise
    x[..., 3] = 1.0
    return x


def time_bm3d(width=4032, height=3024, stages=2, transform="tensor", sigma=0.032, reps=5):
    """Milliseconds per call of the filter on the device-resident frame."""
    L = A.lib()
    x = noisy_frame(width, height, sigma)
    pi, po = C.c_void_p(), C.c_void_p()
    assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(pi)) == 0
    assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(po)) == 0
    try:
        assert L.cpipe_cuda_memcpy_h2d(pi, x.ctypes.data, x.nbytes) == 0
        ins, outs = DeviceImage(pi.value, x.shape, x.dtype), DeviceImage(po.value, x.shape, x.dtype)
        blob = blobs.bm3d_spec(sigma, stages=stages, transform=transform)
        for _ in range(3):
            assert call_filter("denoise_bm3d_spec", [ins], [outs], blob) == 0, last_error()
        e0, e1 = C.c_void_p(), C.c_void_p()
        L.cpipe_cuda_event_create(C.byref(e0))
        L.cpipe_cuda_event_create(C.byref(e1))
        assert L.cpipe_cuda_synchronize() == 0
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(reps):
            assert call_filter("denoise_bm3d_spec", [ins], [outs], blob) == 0, last_error()
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        return ms.value / reps
    finally:
        L.cpipe_cuda_device_free(pi)
        L.cpipe_cuda_device_free(po)


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--width", type=int, default=4032)
    ap.add_argument("--height", type=int, default=3024)
    ap.add_argument("--stages", type=int, default=2)
    ap.add_argument("--transform", default="tensor", choices=("tensor", "fp32", "tensor_fp16"))
    ap.add_argument("--sigma", type=float, default=0.032)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    assert A.lib().cpipe_cuda_device_count() > 0, "no CUDA device"
    ms = time_bm3d(a.width, a.height, a.stages, a.transform, a.sigma, a.reps)
    print(f"denoise_bm3d_spec {a.transform} stages={a.stages} {a.width}x{a.height}: {ms:.3f} ms/frame")


if __name__ == "__main__":
    _main()
