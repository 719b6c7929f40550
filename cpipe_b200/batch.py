"""Batched form: many frames of uneven size through the chain in one launch per
stage (cpipe_cuda_batch_*: persistent kernels over a (frame, tile) queue, one
CUDA graph per set of frames, an autotuner for the persistent grid sizes).

The 64-frame workload: sizes drawn log-uniform in 1-50 MP, aspect 4:3 / 3:2 /
16:9, 10 / 12 / 14-bit, RGGB / BGGR / Quad Bayer, noise a in [1e-3, 1e-2] and
b in [1e-5, 1e-4] log-uniform, each frame generated on the GPU by the seeded
scene generator.  The denoiser slot holds the reference's 2x2 blend (inside
the third stage) or, between the second and third stages, each frame's
network with its BM3D spot check (or the two-stage BM3D).  Measured: aggregate
MP/s of the batched launches, per-frame latency inside the batched launch
(device-clock completion times, p50 / p99), and each frame run alone through
its own chain.

    python -m cpipe_b200.batch [--frames 64] [--reps 5]
"""
import argparse
import ctypes as C
import json
import math

import numpy as np

from . import _abi as A
from .chain import ChainConfig
from .host import CpipeError
from .scene import RGGB, SONY_QBC

BGGR = (2, 1, 1, 0)
BLACK = {10: 16, 12: 64, 14: 256}


def workload(n=64, seed=0x5EED0004, mp_range=(1.0, 50.0), **chain_kw):
    """n frame configurations drawn as described in the module docstring;
    chain_kw go to every frame's ChainConfig (e.g. denoise="surrogate" with
    surrogate_blob)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        mp = math.exp(rng.uniform(math.log(mp_range[0]), math.log(mp_range[1])))
        aspect = (4 / 3, 3 / 2, 16 / 9)[int(rng.integers(3))]
        w = max(16, int(round(math.sqrt(mp * 1e6 * aspect) / 4)) * 4)
        h = max(16, int(round(w / aspect / 4)) * 4)
        bits = (10, 12, 14)[int(rng.integers(3))]
        kind = ("rggb", "bggr", "qbc")[int(rng.integers(3))]
        a = math.exp(rng.uniform(math.log(1e-3), math.log(1e-2)))
        b = math.exp(rng.uniform(math.log(1e-5), math.log(1e-4)))
        cfg = ChainConfig.full_12mp(width=w, height=h, bits=bits, black=float(BLACK[bits]), noise_a=a, noise_b=b,
                                    cfa=BGGR if kind == "bggr" else RGGB, quad_bayer=kind == "qbc",
                                    seed=seed + 17 * i, name=f"batch_frame_{i}_{w}x{h}_{kind}_{bits}bit",
                                    use_graph=False, **chain_kw)
        out.append((cfg, kind))
    return out


def scene_raw(d_raw, cfg, kind):
    """The frame's raw mosaic on the device (cpipe_cuda_scene_raw_cfa)."""
    pat = SONY_QBC if kind == "qbc" else (BGGR if kind == "bggr" else RGGB)
    rep = 4 if kind == "qbc" else 2
    arr = (C.c_uint8 * 16)(*pat)
    st = A.lib().cpipe_cuda_scene_raw_cfa(C.c_void_p(d_raw), cfg.width, cfg.height, C.c_uint64(cfg.seed), cfg.bits,
                                          int(cfg.black), float(cfg.noise_a), float(cfg.noise_b), arr, rep, 20, None)
    if st:
        raise CpipeError(st, "scene_raw_cfa")


class Batch:
    def __init__(self, configs):
        self.configs = list(configs)
        self._keep = []
        arr = (A.ChainConfig * len(self.configs))()
        for i, cfg in enumerate(self.configs):
            c, keep = cfg.c_config()
            self._keep.append(keep)
            arr[i] = c
        st = C.c_int32()
        self._h = A.lib().cpipe_cuda_batch_create(arr, len(self.configs), C.byref(st))
        if not self._h:
            raise CpipeError(st.value, "batch_create " + A.lib().cpipe_cuda_last_error().decode())

    def close(self):
        if self._h:
            A.lib().cpipe_cuda_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptrs(ptrs):
        return (C.c_void_p * len(ptrs))(*ptrs)

    def run(self, d_raws, d_outs, stream=None):
        st = A.lib().cpipe_cuda_batch_run(self._h, self._ptrs(d_raws), self._ptrs(d_outs), stream)
        if st:
            raise CpipeError(st, "batch_run " + A.lib().cpipe_cuda_last_error().decode())

    def autotune(self, d_raws, d_outs, stream=None):
        per_sm = (C.c_int * 3)()
        st = A.lib().cpipe_cuda_batch_autotune(self._h, self._ptrs(d_raws), self._ptrs(d_outs), stream, per_sm)
        if st:
            raise CpipeError(st, "batch_autotune " + A.lib().cpipe_cuda_last_error().decode())
        return list(per_sm)

    def frame_chain(self, i):
        return A.lib().cpipe_cuda_batch_frame_chain(self._h, i)

    def schedule(self):
        """(CTAs per SM of the three stages, rows of a stage-2 work item)."""
        per_sm, rows = (C.c_int * 3)(), C.c_int()
        A.lib().cpipe_cuda_batch_schedule(self._h, per_sm, C.byref(rows))
        return list(per_sm), rows.value

    def frame_times(self, stream=None):
        """Each frame's completion time in the last run, ms after its start."""
        ms = (C.c_float * len(self.configs))()
        st = A.lib().cpipe_cuda_batch_frame_times(self._h, stream, ms, len(self.configs))
        if st:
            raise CpipeError(st, "batch_frame_times")
        return list(ms)


def measure(n=64, reps=5, seed=0x5EED0004, **chain_kw):
    """Aggregate MP/s of the batched form; per-frame latency (p50 / p99) both
    inside the batched launch (completion times on the device clock) and for
    each frame run alone through its own chain."""
    L = A.lib()
    frames = workload(n, seed, **chain_kw)
    d_raw, d_out = [], []
    for cfg, kind in frames:
        p, q = C.c_void_p(), C.c_void_p()
        assert L.cpipe_cuda_device_alloc(cfg.width * cfg.height * 2, C.byref(p)) == 0
        assert L.cpipe_cuda_device_alloc(cfg.width * cfg.height * 8, C.byref(q)) == 0
        scene_raw(p.value, cfg, kind)
        d_raw.append(p.value)
        d_out.append(q.value)
    batch = Batch([cfg for cfg, _ in frames])
    stream = C.c_void_p()
    assert L.cpipe_cuda_stream_create(C.byref(stream)) == 0
    per_sm = batch.autotune(d_raw, d_out, stream)
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    for _ in range(2):
        batch.run(d_raw, d_out, stream)
    L.cpipe_cuda_stream_synchronize(stream)
    L.cpipe_cuda_event_record(e0, stream)
    for _ in range(reps):
        batch.run(d_raw, d_out, stream)
    L.cpipe_cuda_event_record(e1, stream)
    ms = C.c_float()
    L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
    batch_ms = ms.value / reps
    in_batch = np.array(batch.frame_times(stream))
    per_sm, rows2 = batch.schedule()
    stats = None
    if chain_kw.get("denoise") == "surrogate":
        fr, fb, worst = 0, 0, float("inf")
        for i in range(n):
            f_, fb_, w_ = C.c_uint32(), C.c_uint32(), C.c_float()
            L.cpipe_cuda_chain_denoise_stats(batch.frame_chain(i), C.byref(f_), C.byref(fb_), C.byref(w_))
            fr, fb, worst = fr + f_.value, fb + fb_.value, min(worst, w_.value)
        stats = {"frames": fr, "fallbacks_to_bm3d": fb, "worst_tile_psnr_db": round(worst, 2)}
    total_mp = sum(cfg.width * cfg.height for cfg, _ in frames) / 1e6
    lat = []
    for i, (cfg, _) in enumerate(frames):
        ch = batch.frame_chain(i)
        for r in range(3):
            if r == 2:
                L.cpipe_cuda_event_record(e0, stream)
            assert L.cpipe_cuda_chain_run(ch, C.c_void_p(d_raw[i]), C.c_void_p(d_out[i]), stream) == 0
        L.cpipe_cuda_event_record(e1, stream)
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        lat.append(ms.value)
    batch.close()
    for p in d_raw + d_out:
        L.cpipe_cuda_device_free(C.c_void_p(p))
    lat = np.array(lat)
    kinds = [k for _, k in frames]
    out = {"frames": n, "total_mp": round(total_mp, 1), "batch_ms": round(batch_ms, 3),
           "aggregate_mp_per_s": round(total_mp / (batch_ms * 1e-3), 1),
           "latency_ms_in_batch": {"p50": round(float(np.percentile(in_batch, 50)), 3),
                                   "p99": round(float(np.percentile(in_batch, 99)), 3),
                                   "max": round(float(in_batch.max()), 3),
                                   "note": "device-clock completion of each frame's last stage-3 item after the "
                                           "batched run started"},
           "latency_ms_single_frame": {"p50": round(float(np.percentile(lat, 50)), 3),
                                       "p99": round(float(np.percentile(lat, 99)), 3),
                                       "max": round(float(lat.max()), 3)},
           "single_frame_mp_per_s": round(total_mp / (lat.sum() * 1e-3), 1),
           "autotuned_ctas_per_sm": per_sm, "autotuned_stage2_rows_per_item": rows2,
           "mix": {k: kinds.count(k) for k in ("rggb", "bggr", "qbc")},
           "sizes_mp": [round(cfg.width * cfg.height / 1e6, 2) for cfg, _ in frames]}
    if stats is not None:
        out["spot_check"] = stats
    return out


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--frames", type=int, default=64)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    assert A.lib().cpipe_cuda_device_count() > 0, "no CUDA device"
    print(json.dumps(measure(args.frames, args.reps)))


if __name__ == "__main__":
    _main()
