"""Timing of the spec-mode denoisers on a device-resident frame: the guided
filter with the true (2r+1)^2 box (denoise_guided_filter_spec) and the
multi-level a-trous wavelet (denoise_wavelet_atrous_spec).

    python -m cpipe_b200.spec --width 4032 --height 3024 --reps 10
"""
import argparse
import ctypes as C

from . import _abi as A
from . import blobs
from .bm3d import noisy_frame
from .host import DeviceImage, call_filter, last_error

FILTERS = {
    "guided": ("denoise_guided_filter_spec", lambda a: blobs.guided(a.radius, a.eps)),
    "atrous": ("denoise_wavelet_atrous_spec", lambda a: blobs.atrous(a.levels, a.sigma)),
}


def time_filter(aot, blob, width, height, sigma=0.032, reps=10, warmup=3):
    """Milliseconds per call (CUDA events around `reps` calls after `warmup`)
    on a binary16 RGBA frame of the seeded scene plus Gaussian noise."""
    L = A.lib()
    x = noisy_frame(width, height, sigma)
    pi, po = C.c_void_p(), C.c_void_p()
    assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(pi)) == 0
    assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(po)) == 0
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    try:
        assert L.cpipe_cuda_memcpy_h2d(pi, x.ctypes.data, x.nbytes) == 0
        ins, outs = DeviceImage(pi.value, x.shape, x.dtype), DeviceImage(po.value, x.shape, x.dtype)
        for _ in range(warmup):
            assert call_filter(aot, [ins], [outs], blob) == 0, last_error()
        assert L.cpipe_cuda_synchronize() == 0
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(reps):
            assert call_filter(aot, [ins], [outs], blob) == 0, last_error()
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        return ms.value / max(reps, 1)
    finally:
        L.cpipe_cuda_event_destroy(e0)
        L.cpipe_cuda_event_destroy(e1)
        L.cpipe_cuda_device_free(pi)
        L.cpipe_cuda_device_free(po)


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--width", type=int, default=4032)
    ap.add_argument("--height", type=int, default=3024)
    ap.add_argument("--filters", default="guided,atrous")
    ap.add_argument("--radius", type=int, default=8)
    ap.add_argument("--eps", type=float, default=1e-3)
    ap.add_argument("--levels", type=int, default=5)
    ap.add_argument("--sigma", type=float, default=0.032)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    assert A.lib().cpipe_cuda_device_count() > 0, "no CUDA device"
    for name in a.filters.split(","):
        aot, make = FILTERS[name]
        ms = time_filter(aot, make(a), a.width, a.height, a.sigma, a.reps, a.warmup)
        print(f"{aot} {a.width}x{a.height}: {ms:.4f} ms/call")


if __name__ == "__main__":
    _main()
