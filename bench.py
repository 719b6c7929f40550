"""Benchmark: 12 MP ms/frame of the raw->linear chain with the learned
surrogate denoiser, against the same chain with the two-stage BM3D, on B200.

One step = the fused chain (convert, black level, GainMap, RCD, OpcodeList3
warp, WB, colormatrix, denoiser, guided, wavelet, filmic, 3D LUT) over one
4032x3024 10-bit RGGB frame already resident in HBM.  Frames rotate through a
ring of 8 raw inputs (195 MB) and 2 outputs (195 MB), so no step reads its
input from L2.  Timing: CUDA events on the chain's stream around exactly K
steps, bracketed by a barrier and a stream synchronize; max over ranks.  The
same is measured for the BM3D chain (fewer steps; it is the slow arm) and for
the chain with the reference's own denoise.bm3d computation (2x2 box blend).
Quality: PSNR of the surrogate chain's output against the BM3D chain's output
on the same frame (and of the two denoisers' outputs).  The `e2e` figure runs
the surrogate chain through the C-ABI host entry point
(cpipe_cuda_chain_run_host_frames: per frame a pinned raw frame H2D, the chain,
an RGBA16F D2H, pipelined across frames).

Multi-GPU: frames are independent, so N GPUs run N replicas on their own
frames (no collective on the data path); `value` = whole-job ms per frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "12MP ms/frame: surrogate vs plain BM3D chain on B200 at >=40 dB; % HBM roofline"
BYTES_PER_PX = {"raw_to_rgba": 10, "warp_wb_cm": 16, "denoise_tone": 16}  # algorithmic HBM bytes
KERNELS = ["raw_to_rgba", "warp_wb_cm", "denoise", "denoise_tone"]


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def chain_profile(kernel, key="dram_bytes_per_launch"):
    """A per-launch figure of a chain kernel (DRAM bytes, or warp instructions
    with key="warp_inst_per_launch") from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "traffic_full_chain_12mp.json")
    try:
        with open(path) as f:
            return json.load(f)[key].get(kernel)
    except Exception:
        return None


def traffic_per_launch(kernel):
    return chain_profile(kernel)


def issue_frac(warp_inst, ms, sm_mhz, sms=148):
    """Warp instructions per launch over the SMs' issue capacity in the launch's
    time (4 schedulers per SM, one warp instruction per clock each)."""
    if not warp_inst or not sm_mhz or ms <= 0:
        return None
    return round(warp_inst / (sms * 4 * sm_mhz * 1e6 * ms * 1e-3), 4)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) == 7:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def host_cpu():
    """CPU model, logical CPUs, and the CPUs this process may run on."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    usable = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"model": model, "nproc": os.cpu_count(), "usable": usable}


REFERENCE_ARM_BUDGET_S = 150.0  # the whole --impl reference run: warm-up and timed steps


def reference_cpu_chain(cfg):
    """The reference's CPU chain for `cfg` (oracle/chain_oracle.run_reference_chain:
    the reference's own plain-C++ filters from oracle/_ref, single-threaded as
    the reference runs them; C restatements of its Halide nodes with OpenMP over
    rows on every usable CPU).  Its blobs come from oracle/oracle_blobs, so the
    product library is never loaded.  Returns (run, threads, label)."""
    threads = host_cpu()["usable"]
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import oracle_blobs
    from chain_oracle import run_reference_chain
    if oracle.ref_lib() is None:
        raise RuntimeError("the reference build oracle/_ref is absent")
    blobs = oracle_blobs.chain_blobs(cfg)
    raw = cfg.make_raw()

    def run():
        t0 = time.perf_counter()
        run_reference_chain(cfg, raw, blobs)
        return 1000.0 * (time.perf_counter() - t0)
    label = (f"full {cfg.width}x{cfg.height} frame per step through the reference's CPU chain: its plain-C++ "
             "filters (blacklevel, GainMap, OpcodeList3 warp, WB, colormatrix) compiled from its source, "
             "single-threaded as the reference runs them; C restatements of its Halide nodes (convert, RCD, "
             "denoise.bm3d, guided, wavelet, filmic, 3D LUT; Halide is not buildable here), OpenMP over rows "
             f"on {threads} threads")
    return run, threads, label


def bm3d_cpu_crop(n=768):
    """The two-stage BM3D FP64 oracle (oracle_bm3d.c, OpenMP) on an n x n crop
    of a seeded noisy RGBA16F frame: the CPU anchor of the BM3D chain."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from cpipe_b200.scene import scene_rgb
    rng = np.random.default_rng(0x5EED0002)
    x = np.ones((n, n, 4), np.float32)
    x[..., :3] = scene_rgb(n, n, 0x5EED0002) + rng.normal(0.0, 0.032, (n, n, 3))
    x = x.astype(np.float16).astype(np.float32)
    from cpipe_b200 import blobs as B  # ctypes struct layout only; the library is not loaded
    blob = B.bm3d_spec(0.032)
    t0 = time.perf_counter()
    oracle.bm3d_spec(x, blob)
    ms = 1000.0 * (time.perf_counter() - t0)
    return {"crop": f"{n}x{n}", "crop_ms": round(ms, 1), "mp_per_s": round(n * n / 1e6 / (ms * 1e-3), 4),
            "threads": int(os.environ.get("OMP_NUM_THREADS", host_cpu()["usable"])), "kind": "port",
            "note": "FP64 oracle of the two-stage BM3D (8x8 blocks, 16-block groups, 39x39 search, step 3) on a "
                    "crop, not a 12 MP frame"}


def workload_config(cfg, world):
    """The `config` object both arms print (the reference arm computes the same
    chain with the reference's own denoise.bm3d in the denoiser slot)."""
    return {"workload": cfg.name, "frame": f"{cfg.width}x{cfg.height} RGGB 10-bit",
            "nodes": ["precision_convert", "blacklevel", "gainmap 17x13", "demosaic.rcd", "opcode_list_3 warp",
                      "wb.dual_illuminant", "colormatrix", "denoiser", "guided r8 (5x5 box, as the reference)",
                      "wavelet (2x2 Haar, as the reference)", "filmic", "3d_lut 33^3"],
            "l2": "inputs larger than L2: ring of 8 raw frames (195 MB) and 2 output frames",
            "parallelism": f"replicas x{world}"}


# ------------------------------------------------------------ rank helpers
def rank_env(default_world=1):
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", str(default_world))),
            int(os.environ.get("LOCAL_RANK", "0")))


def frame_seed(rank):
    """Replica r processes its own frames (seeded per rank): no data is shared."""
    return 0x5EED0002 + 1000 * rank


def max_over_ranks(x, dist=None, device=None):
    """Max of a per-rank scalar over the process group (CPU tensor for gloo)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_ms_per_frame(max_ms, steps, world):
    """Every rank ran `steps` frames; the job's time is the slowest rank's."""
    return max_ms / (steps * world)


def reference_arm(args):
    rank, world, _ = rank_env(args.gpus)
    if rank != 0:
        return 0
    from cpipe_b200.chain import ChainConfig
    cfg = ChainConfig.full_12mp()
    cpu = host_cpu()
    # Each step is a bounded sample: a full-width band of the frame whose rows
    # are sized so that warm-up and timed steps together take about
    # REFERENCE_ARM_BUDGET_S; the time scales to a whole frame by rows (the
    # chain's work per pixel is the same across the frame).
    try:
        probe_rows = 64
        probe, _, _ = reference_cpu_chain(ChainConfig.full_12mp(height=probe_rows, name="band"))
        probe()
        per_row_ms = probe() / probe_rows
        per_step_ms = 1000.0 * REFERENCE_ARM_BUDGET_S / max(1, args.steps + args.warmup)
        rows = int(min(cfg.height, max(16, per_step_ms / per_row_ms)) // 16 * 16)
        band = cfg if rows >= cfg.height else ChainConfig.full_12mp(height=rows, name=f"band_{cfg.width}x{rows}")
        run, threads, label = reference_cpu_chain(band)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU chain: {e}"}), flush=True)
        return 0
    if band is not cfg:
        label = (f"a {band.width}x{band.height} band of the frame (of {cfg.height} rows) per step, sized so that "
                 f"the run takes about {REFERENCE_ARM_BUDGET_S:.0f} s, step times scaled by {cfg.height}/"
                 f"{band.height}: " + label.split(" frame per step ", 1)[-1])
    scale = cfg.height / band.height
    for _ in range(args.warmup):
        run()
    t0 = time.perf_counter()
    steps = [run() * scale for _ in range(args.steps)]
    total_ms = 1000.0 * (time.perf_counter() - t0)
    v = total_ms * scale / args.steps
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ms/frame", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox scene)",
            "config": workload_config(cfg, world),
            "denoiser_slot": "denoise.bm3d as the reference computes it: a 2x2 box blend (the reference has no "
                             "block-matching BM3D and no learned denoiser)",
            "step_ms": {"min": round(min(steps), 1), "median": round(statistics.median(steps), 1),
                        "max": round(max(steps), 1)},
            "cpu": cpu,
            "cpu_baseline": {"value": round(v, 3), "unit": "ms/frame", "cores": threads, "kind": "reference",
                             "sample": label},
            "e2e": {"value": round(v, 3), "unit": "ms/frame", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


SURROGATE_FLOP_PER_PX = 2 * 9 * (4 * 32 + 6 * 32 * 32 + 32 * 3)  # real channels, 8 layers
HIDDEN_FLOP_PER_PX = 2 * 9 * 32 * 32


def measured_bf16_tflops():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops_sustained"]), "measured (sustained)"
    except Exception:
        return 1385.0, "fallback (sustained)"


def traffic_surrogate_hidden(px):
    """DRAM bytes per hidden-conv launch scaled from the committed ncu capture
    (traffic grows with the pixel count), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_surrogate_tc_conv.json")) as f:
            t = json.load(f)
        return int(t["dram_bytes_per_launch"] * px / t["pixels"])
    except Exception:
        return None


def psnr(a, b):
    import numpy as np
    d = np.asarray(a, np.float64)[..., :3] - np.asarray(b, np.float64)[..., :3]
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(1.0 / mse)


def spec_form(peak_gbs, weights):
    """The spec-mode guided filter (r = 8, eps 1e-3) and 5-level a-trous
    wavelet at 12 MP: each filter alone on a device-resident RGBA16F frame
    (CUDA events, 10 calls after 3), its achieved bandwidth at the reference
    formats' 16 B/px (RGBA16F in and out) against the measured HBM peak, and the
    full 12 MP chain with both stages in place of the reference's guided and
    wavelet nodes: once with the reference's BM3D computation and once with the
    network (and its spot check) in the denoiser slot, as the headline runs."""
    import numpy as np
    from cpipe_b200 import _abi as A
    from cpipe_b200 import blobs as BL
    from cpipe_b200.bm3d import noisy_frame
    from cpipe_b200.chain import Chain, ChainConfig
    from cpipe_b200.host import DeviceImage, call_filter, last_error
    L = A.lib()
    w, h = 4032, 3024
    x = noisy_frame(w, h, 0.032)
    pi, po = C.c_void_p(), C.c_void_p()
    assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(pi)) == 0
    assert L.cpipe_cuda_device_alloc(x.nbytes, C.byref(po)) == 0
    assert L.cpipe_cuda_memcpy_h2d(pi, x.ctypes.data, x.nbytes) == 0
    ins, outs = DeviceImage(pi.value, x.shape, x.dtype), DeviceImage(po.value, x.shape, x.dtype)
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    out = {}
    for name, aot, blob in (("guided_filter_spec_r8", "denoise_guided_filter_spec", BL.guided(8, 1e-3)),
                            ("wavelet_atrous_spec_5_levels", "denoise_wavelet_atrous_spec", BL.atrous(5, 0.032))):
        for _ in range(3):
            assert call_filter(aot, [ins], [outs], blob) == 0, last_error()
        assert L.cpipe_cuda_synchronize() == 0
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(10):
            assert call_filter(aot, [ins], [outs], blob) == 0, last_error()
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        t = ms.value / 10
        gbs = 16.0 * w * h / (t * 1e-3) / 1e9
        out[name] = {"ms": round(t, 4), "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak_gbs, 4)}
    L.cpipe_cuda_device_free(pi)
    L.cpipe_cuda_device_free(po)
    cfg = ChainConfig.full_12mp(guided_spec=True, atrous_levels=5)
    raw = cfg.make_raw()
    d_raw, d_out = C.c_void_p(), C.c_void_p()
    assert L.cpipe_cuda_device_alloc(raw.nbytes, C.byref(d_raw)) == 0
    assert L.cpipe_cuda_device_alloc(w * h * 8, C.byref(d_out)) == 0
    assert L.cpipe_cuda_memcpy_h2d(d_raw, raw.ctypes.data, raw.nbytes) == 0
    for key, c in (("chain_ms", cfg),
                   ("surrogate_chain_ms", ChainConfig.full_12mp(guided_spec=True, atrous_levels=5,
                                                                denoise="surrogate", surrogate_blob=weights))):
        ch = Chain(c)
        for _ in range(3):
            ch.run(d_raw.value, d_out.value)
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(10):
            ch.run(d_raw.value, d_out.value)
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        out[key] = round(ms.value / 10, 4)
        ch.close()
    out["chain"] = "full 12 MP chain, guided r=8 (true box), 5-level a-trous; chain_ms with the reference BM3D " \
                   "computation, surrogate_chain_ms with the network and its BM3D spot check"
    L.cpipe_cuda_device_free(d_raw)
    L.cpipe_cuda_device_free(d_out)
    return out


def config1_chain(peak_gbs, with_cpu=False):
    """The plain chain at its configured size (2016x1512 RGGB 12-bit, black 64,
    WB (2, 1, 1.6), RCD, camera matrix, denoise.bm3d with sigma from the noise
    model, wavelet, filmic, identity+gamma 33^3 LUT): CUDA events around 50
    frames after 5, inputs rotating through 8 raw frames and 4 outputs (147 MB,
    more than L2); bytes = the raw frame read and the RGBA16F frame written once
    (10 B/px).  with_cpu: also the reference's CPU chain on the same frame
    (cpu_reference_ms, on the host's cores)."""
    import numpy as np
    from cpipe_b200 import _abi as A
    from cpipe_b200.chain import Chain, ChainConfig
    L = A.lib()
    cfg = ChainConfig.small_frame()
    w, h = cfg.width, cfg.height
    base = cfg.make_raw()
    d_raw, d_out = [], []
    for k in range(8):
        fr = np.ascontiguousarray(np.roll(base, (2 * k, 4 * k), axis=(0, 1)))
        p = C.c_void_p()
        assert L.cpipe_cuda_device_alloc(fr.nbytes, C.byref(p)) == 0
        assert L.cpipe_cuda_memcpy_h2d(p, fr.ctypes.data, fr.nbytes) == 0
        d_raw.append(p)
    for _ in range(4):
        p = C.c_void_p()
        assert L.cpipe_cuda_device_alloc(w * h * 8, C.byref(p)) == 0
        d_out.append(p)
    ch = Chain(cfg)
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    for i in range(5):
        ch.run(d_raw[i % 8].value, d_out[i % 4].value)
    n = 50
    L.cpipe_cuda_event_record(e0, None)
    for i in range(n):
        ch.run(d_raw[i % 8].value, d_out[i % 4].value)
    L.cpipe_cuda_event_record(e1, None)
    assert L.cpipe_cuda_synchronize() == 0
    ms = C.c_float()
    L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
    t = ms.value / n
    ch.close()
    for p in d_raw + d_out:
        L.cpipe_cuda_device_free(p)
    gbs = 10.0 * w * h / (t * 1e-3) / 1e9
    out = {"workload": cfg.name, "frame": f"{w}x{h} RGGB 12-bit", "ms_per_frame": round(t, 4),
           "mp_per_s": round(w * h / 1e6 / (t * 1e-3), 1), "bytes_per_px": 10, "achieved_gbs": round(gbs, 1),
           "frac": round(gbs / peak_gbs, 4)}
    if with_cpu:
        # the reference's CPU chain on the same frame (one run after one untimed run)
        run, threads, _ = reference_cpu_chain(cfg)
        run()
        out["cpu_reference_ms"] = round(run(), 1)
        out["cpu_threads"] = threads
    return out


def finishing_stages():
    """The 12 MP chain (reference computation in the BM3D slot) with the
    finishing stages the reference's example pipeline runs after the LUT:
    sharpen.edge_aware_usm and the display encode, fused in one kernel
    (sRGB: RGBA8 output; BT2020-PQ: RGBA16 unorm output); CUDA events around
    10 frames on a device-resident raw frame after 3."""
    from cpipe_b200 import _abi as A
    from cpipe_b200.chain import Chain, ChainConfig
    L = A.lib()
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    out = {}
    for name, kw in (("chain_ms", {}), ("chain_sharpen_srgb_ms", dict(sharpen=True, display="sRGB")),
                     ("chain_sharpen_pq_ms", dict(sharpen=True, display="BT2020-PQ"))):
        cfg = ChainConfig.full_12mp(**kw)
        raw = cfg.make_raw()
        ch = Chain(cfg)
        d_raw, d_out = C.c_void_p(), C.c_void_p()
        assert L.cpipe_cuda_device_alloc(raw.nbytes, C.byref(d_raw)) == 0
        assert L.cpipe_cuda_device_alloc(L.cpipe_cuda_chain_output_bytes(ch._h), C.byref(d_out)) == 0
        assert L.cpipe_cuda_memcpy_h2d(d_raw, raw.ctypes.data, raw.nbytes) == 0
        for _ in range(3):
            ch.run(d_raw.value, d_out.value)
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(10):
            ch.run(d_raw.value, d_out.value)
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        out[name] = round(ms.value / 10, 4)
        ch.close()
        L.cpipe_cuda_device_free(d_raw)
        L.cpipe_cuda_device_free(d_out)
    out["note"] = ("full 12 MP chain with the reference's denoise.bm3d computation; sharpen r=1 strength 0.75 "
                   "fused with the display encode after the LUT")
    return out


def dng_ingest(peak_gbs):
    """DNG ingest of a 4032x3024 frame: the strip unpack alone from a
    device-resident strip (16-bit words; 12-bit packed), bytes = strip read +
    plane written once; cpipe_cuda_dng_decode from the file image in
    pageable host memory (parse, strip upload, unpack); and the same decode of
    a lossless-JPEG (Compression 7) file of the benchmark frame's mosaic.  CUDA events around 20
    calls after 3, the unpack over four strip / plane sets in turn (192 MB for
    16-bit, more than L2)."""
    import numpy as np
    from cpipe_b200 import _abi as A
    from cpipe_b200.dng_synth import SHORT, build_dng
    L = A.lib()
    L.cpipe_cuda_set_stream(None)
    w, h = 4032, 3024
    rng = np.random.default_rng(4032)
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    out = {"frame": f"{w}x{h}"}
    # Four strip / plane sets used in turn: 4 x (strip + plane) > the 126 MB L2.
    d_raws = [C.c_void_p() for _ in range(4)]
    for d in d_raws:
        assert L.cpipe_cuda_device_alloc(w * h * 2, C.byref(d)) == 0
    d_raw = d_raws[0]

    def timed(fn, n=20):
        for _ in range(3):
            assert fn() == 0
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(n):
            fn()
        L.cpipe_cuda_event_record(e1, None)
        assert L.cpipe_cuda_synchronize() == 0
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        return ms.value / n

    for bits in (16, 12):
        x = rng.integers(0, 1 << bits, (h, w), dtype=np.uint32).astype(np.uint16)
        if bits == 16:
            strip = x.astype("<u2").tobytes()
        else:
            rows = np.empty((h, w, bits), np.uint8)
            for i in range(bits):
                rows[..., i] = (x >> (bits - 1 - i)) & 1
            strip = np.packbits(rows.reshape(h, w * bits), axis=1).tobytes()
        d_strips = [C.c_void_p() for _ in range(4)]
        for d in d_strips:
            assert L.cpipe_cuda_device_alloc(len(strip), C.byref(d)) == 0
            assert L.cpipe_cuda_memcpy_h2d(d, strip, len(strip)) == 0
        turn = [0]

        def unpack_next():
            i = turn[0] = (turn[0] + 1) % 4
            return L.cpipe_cuda_dng_unpack(d_strips[i], len(strip), w, h, bits, d_raws[i])
        ms = timed(unpack_next)
        gbs = (len(strip) + w * h * 2) / (ms * 1e-3) / 1e9
        data = build_dng(width=w, height=h, strip=strip, overrides={258: (SHORT, [bits])})
        e2e = timed(lambda: L.cpipe_cuda_dng_decode(data, len(data), d_raw, w * h * 2, None), n=10)
        out[f"bits{bits}"] = {"unpack_ms": round(ms, 4), "achieved_gbs": round(gbs, 1),
                              "frac": round(gbs / peak_gbs, 4), "decode_from_host_ms": round(e2e, 3),
                              "file_bytes": len(data)}
        for d in d_strips:
            L.cpipe_cuda_device_free(d)
    # Compression 7: the 12 MP benchmark frame's mosaic (10-bit) as 256x256
    # lossless-JPEG tiles (predictor 1, two components per JPEG line, as DNG
    # writers store CFA data), decoded from the file image in host memory
    from cpipe_b200.chain import ChainConfig
    from cpipe_b200.dng_synth import lj92_tiles
    raw = ChainConfig.full_12mp().make_raw()
    for name, tables in (("lossless_jpeg", "per_component"), ("lossless_jpeg_one_table", "fixed")):
        data = build_dng(width=w, height=h, bits=10, tile=(256, 256),
                         segments=lj92_tiles(raw, 10, 256, 256, 2, tables))
        ms = timed(lambda: L.cpipe_cuda_dng_decode(data, len(data), d_raw, w * h * 2, None), n=10)
        got = np.empty((h, w), np.uint16)
        assert L.cpipe_cuda_memcpy_d2h(got.ctypes.data, d_raw, got.nbytes) == 0
        fig = (C.c_uint64 * 9)()
        L.cpipe_cuda_lj92_last_stats(fig, 9)
        out[name] = {"decode_from_host_ms": round(ms, 3), "mp_per_s": round(w * h / 1e6 / (ms * 1e-3), 1),
                     "file_bytes": len(data), "tiles": "256x256 (192), predictor 1",
                     "huffman_tables": "one per component, optimal" if tables != "fixed" else "one shared, fixed",
                     "stream_chunks": fig[0], "chunks_decoded_again_by_write_walks": fig[6],
                     "exact": bool(np.array_equal(got, raw))}
    for d in d_raws:
        L.cpipe_cuda_device_free(d)
    out["note"] = ("decode_from_host_ms includes the pageable host-to-device copy of the strip, "
                   "which bounds it; the unpack is the kernel's share; lossless_jpeg: each tile's stream decoded "
                   "in parallel by 1024-bit chunks (speculative paths chained by warps), predictor 1 by prefix sums")
    return out


def batched_form(weights):
    """The 64-frame uneven batch (cpipe_b200.batch): aggregate MP/s of one launch
    per stage over all frames, per-frame latency inside the batched launch and
    alone; with the reference's 2x2 blend in the denoiser slot, and with the
    network and its BM3D spot check there."""
    from cpipe_b200 import batch as B
    r = B.measure(64, 3)
    r.pop("sizes_mp", None)
    s = B.measure(64, 2, denoise="surrogate", surrogate_blob=weights)
    s.pop("sizes_mp", None)
    s.pop("mix", None)
    r["surrogate_denoiser"] = s
    return r


def qbc_50mp(weights):
    """8160x6120 Quad-Bayer frame (remosaic + chain), generated on the device:
    ms/frame of the reference-computation chain and of the surrogate chain."""
    from cpipe_b200 import _abi as A
    from cpipe_b200 import batch as B
    from cpipe_b200.chain import Chain, ChainConfig
    L = A.lib()
    out = {"frame": "8160x6120 Quad Bayer 10-bit"}
    d_raw, d_out = C.c_void_p(), C.c_void_p()
    cfg0 = ChainConfig.qbc_50mp()
    assert L.cpipe_cuda_device_alloc(cfg0.width * cfg0.height * 2, C.byref(d_raw)) == 0
    assert L.cpipe_cuda_device_alloc(cfg0.width * cfg0.height * 8, C.byref(d_out)) == 0
    B.scene_raw(d_raw.value, cfg0, "qbc")
    e0, e1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(e0))
    L.cpipe_cuda_event_create(C.byref(e1))
    for mode in ("box2x2", "surrogate"):
        ch = Chain(ChainConfig.qbc_50mp(denoise=mode, surrogate_blob=weights))
        for _ in range(2):
            ch.run(d_raw.value, d_out.value)
        L.cpipe_cuda_event_record(e0, None)
        for _ in range(3):
            ch.run(d_raw.value, d_out.value)
        L.cpipe_cuda_event_record(e1, None)
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(e0, e1, C.byref(ms))
        key = "reference_computation_chain_ms" if mode == "box2x2" else "surrogate_chain_ms"
        out[key] = round(ms.value / 3, 3)
        if mode == "surrogate":
            f, fb, worst = ch.denoise_stats()
            out["spot_check"] = {"frames": f, "fallbacks_to_bm3d": fb, "worst_tile_psnr_db": round(worst, 2)}
        ch.close()
    L.cpipe_cuda_device_free(d_raw)
    L.cpipe_cuda_device_free(d_out)
    return out


def b200_arm(args):
    import numpy as np
    rank, world, local = rank_env(args.gpus)
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from cpipe_b200 import _abi as A
    from cpipe_b200 import surrogate as S
    from cpipe_b200.chain import Chain, ChainConfig
    from cpipe_b200.roofline import node_roofline
    L = A.lib()
    assert L.cpipe_cuda_set_device(local) == 0, "no CUDA device"

    def barrier():
        if dist is not None:
            import torch
            dist.barrier(device_ids=[local])
            torch.cuda.synchronize()

    weights = S.load_weights()
    base_cfg = dict(seed=frame_seed(rank), surrogate_blob=weights)
    cfg = ChainConfig.full_12mp(denoise="surrogate", **base_cfg)
    w, h = cfg.width, cfg.height
    base = cfg.make_raw()
    ring = [np.ascontiguousarray(np.roll(base, (2 * k, 4 * k), axis=(0, 1))) for k in range(8)]
    raw_bytes = base.nbytes
    out_bytes = w * h * 8
    d_raw, d_out = [], []
    for fr in ring:
        p = C.c_void_p()
        assert L.cpipe_cuda_device_alloc(raw_bytes, C.byref(p)) == 0
        assert L.cpipe_cuda_memcpy_h2d(p, fr.ctypes.data, raw_bytes) == 0
        d_raw.append(p.value)
    for _ in range(2):
        p = C.c_void_p()
        assert L.cpipe_cuda_device_alloc(out_bytes, C.byref(p)) == 0
        d_out.append(p.value)
    stream = C.c_void_p()
    assert L.cpipe_cuda_stream_create(C.byref(stream)) == 0
    ev0, ev1 = C.c_void_p(), C.c_void_p()
    L.cpipe_cuda_event_create(C.byref(ev0))
    L.cpipe_cuda_event_create(C.byref(ev1))

    def timed(chain, frames, warmup):
        """warm-up, then exactly `frames` steps between events (stage events on)."""
        for i in range(warmup):
            chain.run(d_raw[i % 8], d_out[i % 2], stream)
        L.cpipe_cuda_stream_synchronize(stream)
        L.cpipe_cuda_chain_set_profiling(chain._h, 1)
        ms_k, nfr = (C.c_double * 4)(), C.c_int32()
        L.cpipe_cuda_chain_profile(chain._h, ms_k, C.byref(nfr))
        barrier()
        L.cpipe_cuda_stream_synchronize(stream)
        L.cpipe_cuda_event_record(ev0, stream)
        for i in range(frames):
            chain.run(d_raw[i % 8], d_out[i % 2], stream)
        L.cpipe_cuda_event_record(ev1, stream)
        L.cpipe_cuda_stream_synchronize(stream)
        barrier()
        ms = C.c_float()
        L.cpipe_cuda_event_elapsed_ms(ev0, ev1, C.byref(ms))
        L.cpipe_cuda_chain_profile(chain._h, ms_k, C.byref(nfr))
        L.cpipe_cuda_chain_set_profiling(chain._h, 0)
        stages = {k: ms_k[i] / max(1, nfr.value) for i, k in enumerate(KERNELS)}
        return max_over_ranks(float(ms.value), dist, f"cuda:{local}"), stages

    chain = Chain(cfg)
    bm3d_chain = Chain(ChainConfig.full_12mp(denoise="bm3d", **base_cfg))
    ref_chain = Chain(ChainConfig.full_12mp(**base_cfg))
    bm3d_frames = max(3, min(args.steps, 10))
    with ClockSampler(local) as clocks:
        total_ms, stages = timed(chain, args.steps, max(args.warmup, 3))
        bm3d_ms, bm3d_stages = timed(bm3d_chain, bm3d_frames, 3)
        ref_ms, ref_stages = timed(ref_chain, args.steps, 3)
        # end to end through the C-ABI host entry point for a run of frames
        # (cpipe_cuda_chain_run_host_frames): every frame's raw H2D from pinned
        # memory and its RGBA16F D2H into pinned memory happen inside the timed
        # call, overlapped with the neighbouring frames' chain
        e2e_steps = max(3, min(args.steps, 40))
        h_raw, h_outs = C.c_void_p(), [C.c_void_p(), C.c_void_p()]
        assert L.cpipe_cuda_pinned_alloc(raw_bytes, C.byref(h_raw)) == 0
        for ho in h_outs:
            assert L.cpipe_cuda_pinned_alloc(out_bytes, C.byref(ho)) == 0
        C.memmove(h_raw, ring[0].ctypes.data, raw_bytes)
        raws = (C.c_void_p * e2e_steps)(*([h_raw.value] * e2e_steps))
        outs = (C.c_void_p * e2e_steps)(*[h_outs[i % 2].value for i in range(e2e_steps)])
        assert L.cpipe_cuda_chain_run_host_frames(chain._h, raws, outs, 4, stream) == 0
        barrier()
        t0 = time.perf_counter()
        assert L.cpipe_cuda_chain_run_host_frames(chain._h, raws, outs, e2e_steps, stream) == 0
        e2e_s = time.perf_counter() - t0
        barrier()
        # one frame per call (cpipe_cuda_chain_run_host, nothing overlapped): the latency view
        sync_steps = max(3, min(args.steps, 10))
        assert L.cpipe_cuda_chain_run_host(chain._h, h_raw, h_outs[0], stream) == 0  # its graph, untimed
        t0 = time.perf_counter()
        for i in range(sync_steps):
            assert L.cpipe_cuda_chain_run_host(chain._h, h_raw, h_outs[0], stream) == 0
        sync_s = time.perf_counter() - t0
        barrier()
    clk = clocks.summary()
    spot_frames, spot_fallbacks, spot_worst = chain.denoise_stats()

    # quality: the surrogate chain against the BM3D chain on the same frame
    outs = {}
    for name, c in (("surrogate", chain), ("bm3d", bm3d_chain)):
        c.run(d_raw[0], d_out[0], stream)
        L.cpipe_cuda_stream_synchronize(stream)
        arr = np.empty((h, w, 4), np.float16)
        L.cpipe_cuda_memcpy_d2h(arr.ctypes.data, C.c_void_p(d_out[0]), out_bytes)
        outs[name] = arr.astype(np.float32)
    chain_psnr = psnr(outs["surrogate"], outs["bm3d"])
    den = {}
    for mode in ("surrogate", "bm3d"):
        c = Chain(ChainConfig.full_12mp(denoise=mode, stop_after=2, **base_cfg))
        den[mode] = c.run_host(ring[0]).astype(np.float32)
        c.close()
    den_psnr = psnr(den["surrogate"], den["bm3d"])
    # per-kernel times of the denoiser on this frame's denoiser input
    front = Chain(ChainConfig.full_12mp(stop_after=1, **base_cfg))
    front.run(d_raw[0], d_out[0], stream)
    L.cpipe_cuda_stream_synchronize(stream)
    front.close()
    sg = S.Surrogate(weights)
    sg.profile(d_out[0], d_out[1], 1, w, h, [(cfg.noise_a, cfg.noise_b)], stream=stream)
    layer_ms = sg.profile(d_out[0], d_out[1], 1, w, h, [(cfg.noise_a, cfg.noise_b)], stream=stream)
    sg.close()

    e2e_ms = max_over_ranks(e2e_s * 1000.0, dist, f"cuda:{local}")
    sync_ms = max_over_ranks(sync_s * 1000.0, dist, f"cuda:{local}")
    value = whole_job_ms_per_frame(total_ms, args.steps, world)
    bm3d_value = whole_job_ms_per_frame(bm3d_ms, bm3d_frames, world)
    ref_value = whole_job_ms_per_frame(ref_ms, args.steps, world)
    hidden_ms = sum(layer_ms[2:8]) / 6.0
    peak_tf, peak_kind = measured_bf16_tflops()
    hidden_flop = HIDDEN_FLOP_PER_PX * w * h
    achieved_tf = hidden_flop / (hidden_ms * 1e-3) / 1e12
    peak_gbs, gbs_kind = measured_peak_gbs()
    hbm = {k: {"ms": round(ref_stages[k], 4),
               "achieved_gbs": round(BYTES_PER_PX[k] * w * h / (ref_stages[k] * 1e-3) / 1e9, 1),
               "frac": round(BYTES_PER_PX[k] * w * h / (ref_stages[k] * 1e-3) / 1e9 / peak_gbs, 4),
               "traffic": traffic_per_launch(k),
               "warp_inst": chain_profile(k, "warp_inst_per_launch"),
               "issue_frac": issue_frac(chain_profile(k, "warp_inst_per_launch"), ref_stages[k],
                                        clk.get("sm_mhz"))} for k in BYTES_PER_PX}
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "ms/frame", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic (seeded Philox scene)",
        "config": workload_config(cfg, world),
        "denoiser_slot": {"denoiser": "learned surrogate: 8 3x3 conv layers, 32 channels, BF16, FP32 accumulation; "
                                      "per frame BM3D spot check on 16 256x256 tiles, BM3D fallback below 40 dB",
                          "compared_with": "the same chain with two-stage BM3D (8x8 blocks, 16-block groups, 39x39 "
                                           "search, step 3, hard threshold + Wiener); group transforms on the "
                                           "tensor cores (mma.sync) with hi/lo-split FP16 operands and FP32 "
                                           "accumulation, matching and aggregation in FP32"},
        "per_stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "bm3d_chain": {"ms_per_frame": round(bm3d_value, 3), "frames": bm3d_frames,
                       "per_stage_ms": {k: round(v, 4) for k, v in bm3d_stages.items()}},
        "speedup_vs_bm3d_chain": round(bm3d_value / value, 2),
        "psnr_vs_bm3d_chain_db": round(chain_psnr, 2),
        "psnr_denoiser_vs_bm3d_db": round(den_psnr, 2),
        "spot_check": {"tiles_per_frame": cfg.spot_tiles, "tile": "256x256", "min_psnr_db": cfg.spot_min_psnr_db,
                       "frames": spot_frames, "fallbacks_to_bm3d": spot_fallbacks,
                       "worst_tile_psnr_db": round(spot_worst, 2)},
        "reference_computation_chain": {"ms_per_frame": round(ref_value, 4),
                                        "note": "denoise.bm3d as the reference computes it (2x2 box blend)",
                                        "per_stage_ms": {k: round(v, 4) for k, v in ref_stages.items()}},
        "surrogate_layer_ms": [round(v, 4) for v in layer_ms],
        "roofline": {"bound": "tensor", "kernel": "sg_tc_conv_kernel<32,32> (tcgen05 hidden 3x3 conv layer)",
                     "achieved": round(achieved_tf, 1), "peak": peak_tf, "peak_kind": peak_kind,
                     "unit": "TFLOP/s", "frac": round(achieved_tf / peak_tf, 4),
                     "algorithmic_flop": hidden_flop, "traffic": traffic_surrogate_hidden(w * h)},
        "hbm_roofline": {"peak_gbs": peak_gbs, "peak_kind": gbs_kind, "kernels": hbm,
                         "note": "chain kernels of the reference-computation chain (CUDA events); warp_inst from "
                                 "the committed ncu summary; issue_frac = warp_inst / (148 SMs x 4 x median SM "
                                 "clock x time)"},
        "e2e": {"value": round(whole_job_ms_per_frame(e2e_ms, e2e_steps, world), 4), "unit": "ms/frame",
                "h2d_bytes_per_step": raw_bytes, "d2h_bytes_per_step": out_bytes,
                "api": "cpipe_cuda_chain_run_host_frames (copies overlapped with the neighbouring frames)",
                "single_frame_call_ms": round(sync_ms / sync_steps, 4)},
        "clocks": clk,
        "gpu_launches": 33 * args.steps,  # K1, K2, K3, 9 denoiser, 3 spot check, 2 x 9 BM3D (tiles; gated fallback)
    }
    if rank == 0 and world == 1 and not args.no_extra:
        line["batched_form"] = batched_form(weights)
        line["spec_form"] = spec_form(peak_gbs, weights)
        line["finishing_stages"] = finishing_stages()
        line["config1_chain"] = config1_chain(peak_gbs, with_cpu=not args.no_cpu_baseline)
        line["dng_ingest"] = dng_ingest(peak_gbs)
        line["node_roofline"] = {"peak_gbs": peak_gbs, "peak_kind": gbs_kind,
                                 "note": "each node's filter alone, 12 MP device buffers, bytes = its input and "
                                         "output once in the reference's formats",
                                 "nodes": node_roofline(w, h, peak_gbs=peak_gbs)}
        line["qbc_50mp"] = qbc_50mp(weights)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        run, threads, label = reference_cpu_chain(ChainConfig.full_12mp())
        v = run()
        line["cpu_baseline"] = {"value": round(v, 1), "unit": "ms/frame", "cores": threads, "kind": "reference",
                                "sample": "one " + label[len("full "):].replace(" per step", "", 1),
                                "cpu": host_cpu()}
        line["cpu_baseline_bm3d"] = bm3d_cpu_crop()
    for c in (chain, bm3d_chain, ref_chain):
        c.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batched-form and 50 MP measurements")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
