"""Every node's filter at 12 MP on device-resident buffers, timed two ways
with CUDA events over `reps` calls (after three untimed ones):

  call_ms    the calls issued back to back: device time plus whatever host
             time a call takes beyond its kernels (blob preparation, uploads);
  device_ms  the same calls queued behind a bounded spin kernel
             (torch.cuda._sleep) on the same stream, so that the events see
             the device work alone; `queued` says whether the host finished
             issuing before the spin ended (otherwise device_ms still holds
             host gaps).

Achieved bandwidth is the node's algorithmic bytes (its input and output once,
in the reference's formats) over device_ms, against the measured HBM copy
peak.  The blobs are the 12 MP workload's
(cpipe_b200.chain.ChainConfig.full_12mp), resolved by the library's host
preparation.

    python -m cpipe_b200.roofline [--width 4032] [--height 3024] [--reps 10]
"""
import argparse
import ctypes as C
import json
import os
import time

import numpy as np
import torch

from . import _abi as A
from . import blobs as B
from .bm3d import noisy_frame
from .chain import ChainConfig
from .host import DeviceImage, call_filter, last_error

HERE = os.path.dirname(os.path.abspath(__file__))

# (node, aot_id, input kind, output kind, algorithmic B/px, blob key, bound).
# bound: "hbm" -- a point or small-stencil node whose floor is its bytes;
# "issue" -- the reference's per-pixel arithmetic (RCD/AMaZE ratios, the QBC
# 25-tap integer weights, the guided filter's exact-order box sums, the warp's
# float-float coordinates and bicubic taps, filmic's log per channel, USM's
# exact-order sums and divisions, the PQ encode's two powers per channel, the
# full-form RCD / AMaZE stages) sets the floor; "gather" -- 3D LUT cell reads through L1/L2.
NODES = [
    ("a1 precision_convert", "precision_convert_r16u_to_f32", "u16", "f32", 6, None, "hbm"),
    ("a2 linearize", "linearize_dng_lut", "u16", "f32", 6, "linearize", "hbm"),
    ("a3 blacklevel", "blacklevel_dng_levels", "f32raw", "f32", 8, "blacklevel", "hbm"),
    ("a4 GainMap", "lens_shading_gainmap", "f32", "f32", 8, "gainmap", "hbm"),
    ("a5 demosaic RCD", "demosaic_rcd", "f32", "rgba", 12, "demosaic", "issue"),
    ("a6 demosaic AMaZE", "demosaic_amaze", "f32", "rgba", 12, "demosaic", "issue"),
    ("a7 demosaic bilinear", "demosaic_bilinear", "f32", "rgba", 12, "demosaic", "hbm"),
    ("a5 demosaic RCD (full form)", "demosaic_rcd_full", "f32", "rgba", 12, "demosaic", "issue"),
    ("a6 demosaic AMaZE (full form)", "demosaic_amaze_full", "f32", "rgba", 12, "demosaic", "issue"),
    ("a8 QBC remosaic", "demosaic_quad_bayer_remosaic", "u16", "u16", 4, None, "issue"),
    ("a9 WB", "wb_dual_illuminant", "rgba", "rgba", 16, "wb", "hbm"),
    ("a10 colormatrix", "colormatrix_dng_to_working", "rgba", "rgba", 16, "colormatrix", "hbm"),
    ("a11 BM3D (reference 2x2 form)", "denoise_bm3d_step1", "rgba", "rgba", 16, "bm3d", "hbm"),
    ("a12 guided (reference, r=8 -> 5x5)", "denoise_guided_filter", "rgba", "rgba", 16, "guided", "issue"),
    ("a13 wavelet (reference 2x2 Haar)", "denoise_wavelet_bayes_shrink", "rgba", "rgba", 16, "wavelet", "hbm"),
    ("a14 OpcodeList3 warp", "lens_dng_opcode_list_3", "rgba", "rgba", 16, "opcode3", "issue"),
    ("a15 3D LUT", "color_3d_lut", "rgba", "rgba", 16, "lut", "gather"),
    ("a16 filmic", "tone_filmic_rgb", "rgba", "rgba", 16, "filmic", "issue"),
    ("wb.greyworld_auto (sum + apply)", "cpipe_wb_greyworld_auto", "rgba", "rgba", 16, "greyworld", "hbm"),
    ("tone.aces_filmic", "tone_aces_filmic", "rgba", "rgba", 16, "aces", "hbm"),
    ("tone.reinhard", "tone_reinhard", "rgba", "rgba", 16, "reinhard", "hbm"),
    ("sharpen.edge_aware_usm (3x3)", "sharpen_edge_aware_usm", "rgba", "rgba", 16, "usm", "issue"),
    ("scene_linear_to_display sRGB", "cpipe_scene_linear_to_display", "rgba", "rgba8", 12, "display_srgb", "hbm"),
    ("scene_linear_to_display PQ", "cpipe_scene_linear_to_display", "rgba", "rgba16u", 16, "display_pq", "issue"),
]


def measured_peak_gbs():
    try:
        with open(os.path.join(HERE, "..", "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def node_roofline(width=4032, height=3024, reps=10, peak_gbs=None):
    L = A.lib()
    if peak_gbs is None:
        peak_gbs, _ = measured_peak_gbs()
    cfg = ChainConfig.full_12mp(width=width, height=height)
    b = cfg.blobs()
    b["linearize"] = B.linearize(np.arange(1 << cfg.bits, dtype=np.uint16))
    b["usm"] = B.usm()
    b["aces"], b["reinhard"] = B.aces(), B.reinhard()
    b["greyworld"] = bytes(A.GreyworldParams(0))
    b["display_srgb"], b["display_pq"] = B.display("sRGB"), B.display("BT2020-PQ")
    raw = cfg.make_raw()
    frames = {"u16": raw, "f32raw": raw.astype(np.float32),
              "f32": np.clip((raw.astype(np.float32) - cfg.black) / (cfg.white - cfg.black), 0.0, 1.0),
              "rgba": noisy_frame(width, height, 0.03)}
    dev, keep = {}, []
    for kind, x in frames.items():
        p = C.c_void_p()
        assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(p)) == 0
        assert L.cpipe_cuda_memcpy_h2d(p, x.ctypes.data, x.nbytes) == 0
        dev[kind] = DeviceImage(p.value, x.shape, x.dtype)
        keep.append(p)
    outs = {}
    for kind, (shape, dtype) in {"f32": ((height, width), np.float32), "u16": ((height, width), np.uint16),
                                 "rgba": ((height, width, 4), np.float16), "rgba8": ((height, width, 4), np.uint8),
                                 "rgba16u": ((height, width, 4), np.uint16)}.items():
        p = C.c_void_p()
        assert L.cpipe_cuda_device_alloc(int(np.prod(shape)) * np.dtype(dtype).itemsize, C.byref(p)) == 0
        outs[kind] = DeviceImage(p.value, shape, dtype)
        keep.append(p)
    # the library issues on the legacy default stream, which is also torch's
    # current stream here, so the spin kernel and the calls share one queue
    assert L.cpipe_cuda_get_stream() is None and torch.cuda.current_stream().cuda_stream == 0
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))

    def timed(args, aot, spin_s):
        assert L.cpipe_cuda_synchronize() == 0
        if spin_s:
            torch.cuda._sleep(int(spin_s * 2.0e9))  # at most spin_s seconds at the 2 GHz clock
        L.cpipe_cuda_event_record(e0, None)
        t0 = time.perf_counter()
        for _ in range(reps):
            call_filter(aot, *args)
        host = time.perf_counter() - t0
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0, last_error()
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        return ms.value / reps, host

    res = {}
    try:
        for name, aot, kin, kout, bpp, key, bound in NODES:
            blob = b[key] if key else None
            args = ([dev[kin]], [outs[kout]], blob)
            for _ in range(3):
                st = call_filter(aot, *args)
                assert st == 0, f"{aot}: status {st}: {last_error()}"
            call_ms, host = timed(args, aot, 0.0)
            spin = max(0.02, 3.0 * host)
            dev_ms, host = timed(args, aot, spin)
            queued = host < 0.5 * spin
            gbs = bpp * width * height / (dev_ms * 1e-3) / 1e9
            res[name] = {"aot_id": aot, "bound": bound, "call_ms": round(call_ms, 4), "device_ms": round(dev_ms, 4),
                         "queued": bool(queued), "bytes_per_px": bpp, "achieved_gbs": round(gbs, 1),
                         "frac": round(gbs / peak_gbs, 4)}
    finally:
        for p in keep:
            L.cpipe_cuda_device_free(p)
    return res


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--width", type=int, default=4032)
    ap.add_argument("--height", type=int, default=3024)
    ap.add_argument("--reps", type=int, default=10)
    a = ap.parse_args()
    assert A.lib().cpipe_cuda_device_count() > 0, "no CUDA device"
    for k, v in node_roofline(a.width, a.height, a.reps).items():
        print(f"{k:36s} {v['bound']:6s} call {v['call_ms']:7.4f} ms  device {v['device_ms']:7.4f} ms {v['achieved_gbs']:7.1f} GB/s "
              f"{100 * v['frac']:5.1f} %{'' if v['queued'] else '  (host-bound)'}")


if __name__ == "__main__":
    _main()
