"""Learned surrogate denoiser for the BM3D slot of the raw->linear chain.

An 8-layer, 32-channel residual network of 3x3 convolutions (BF16 weights and
activations, FP32 accumulation) that stands in for the two-stage BM3D
(denoise_bm3d_spec).  Everything runs on the GPU through libcpipe_b200:

* training pairs: seeded raw frames from the device scene generator
  (cpipe_cuda_scene_raw_cfa: Bayer or Quad-Bayer mosaics, 10/12/14-bit, 1/4/20
  rectangles, noise a in [1e-3, 1e-2], b in [1e-5, 1e-4] log-uniform), the
  chain's front (Quad-Bayer frames remosaiced first) (convert, black level, GainMap, RCD,
  OpcodeList3 warp, WB, colormatrix; chain stop_after = 1) giving the
  denoiser's input, and the two-stage BM3D of that input (sigma from the noise
  profile as the denoise.bm3d node computes it) as the target;
* training: cpipe_surrogate_train_step (the project's forward, backward and Adam
  kernels) on 256x256 tiles, MSE against the BM3D output;
* serving: cpipe_surrogate_denoise, or the fused chain's denoise_mode 2.

No reference counterpart exists (the reference's AI denoise node is planned,
docs/research/08-ai-isp-algorithms.md:37, but not implemented).

    python -m cpipe_b200.surrogate train --pairs 80000 --steps 40000 --lr 1e-3 --out base.cpsn
    python -m cpipe_b200.surrogate train --init base.cpsn --pairs 80000 --steps 20000 --lr 3e-4 \
        --noise-a-max 0.015 --seed 7 --out weights.cpsn

(the committed cpipe_b200/weights/surrogate_bm3d.cpsn was made by these two
commands: the second fine-tunes on noise up to a = 0.015, past the 0.01 top of
the batched workload's mix; its report, with the base run's, is
surrogate_bm3d.report.json beside it)
"""
import argparse
import ctypes as C
import math
import os
import struct
import time

import numpy as np

from . import _abi as A
from . import blobs as B
from .host import CpipeError, DeviceImage, call_filter, last_error

LAYERS, CHANNELS = 8, 32
SHAPES = [(32, 4)] + [(32, 32)] * 6 + [(3, 32)]  # (cout, cin) per layer
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "surrogate_bm3d.cpsn")
NOISE_A = (1e-3, 1e-2)
NOISE_B = (1e-5, 1e-4)


# ------------------------------------------------------------------ weights
def init_params(seed=0):
    """He-normal initialisation; the last layer scaled by 0.1 so the network
    starts close to the identity (its output is a residual)."""
    rng = np.random.default_rng(seed)
    params = []
    for l, (co, ci) in enumerate(SHAPES):
        std = math.sqrt(2.0 / (ci * 9)) * (0.1 if l == LAYERS - 1 else 1.0)
        params.append((rng.normal(0.0, std, (co, ci, 3, 3)).astype(np.float32), np.zeros(co, np.float32)))
    return params


def to_blob(params):
    head = struct.pack("<4s5I2I", b"CPSN", 1, LAYERS, CHANNELS, 4, 3, 0, 0)
    body = b"".join(np.ascontiguousarray(W, np.float32).tobytes() + np.ascontiguousarray(b, np.float32).tobytes()
                    for W, b in params)
    return head + body


def from_blob(blob):
    magic, ver, layers, ch, cin, cout = struct.unpack("<4s5I", blob[:24])
    if magic != b"CPSN" or ver != 1 or layers != LAYERS or ch != CHANNELS or cin != 4 or cout != 3:
        raise ValueError("not a cpipe surrogate weight blob")
    flat = np.frombuffer(blob, np.float32, offset=32)
    params, o = [], 0
    for co, ci in SHAPES:
        n = co * ci * 9
        params.append((flat[o:o + n].reshape(co, ci, 3, 3).copy(), flat[o + n:o + n + co].copy()))
        o += n + co
    return params


def load_weights(path=DEFAULT_WEIGHTS):
    with open(path, "rb") as f:
        return f.read()


def noise_sigma(a, b):
    """The BM3D sigma the denoise.bm3d node derives from a one-pair noise
    profile (beta = b, lambda = a): sqrt(b + a * 0.25), in float32."""
    return float(np.sqrt(np.float64(np.float32(np.float32(b) + np.float32(a) * np.float32(0.25)))))


# ------------------------------------------------------------------ device
class DeviceArray:
    def __init__(self, nbytes):
        self.nbytes = int(nbytes)
        self._p = C.c_void_p()
        if A.lib().cpipe_cuda_device_alloc(self.nbytes, C.byref(self._p)) != 0:
            raise CpipeError(A.OOM, f"device_alloc {self.nbytes}")

    @property
    def ptr(self):
        return self._p.value

    def at(self, offset):
        return self._p.value + int(offset)

    def upload(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        assert A.lib().cpipe_cuda_memcpy_h2d(self._p, arr.ctypes.data, arr.nbytes) == 0
        return self

    def download(self, shape, dtype, offset=0):
        out = np.empty(shape, dtype)
        assert A.lib().cpipe_cuda_synchronize() == 0
        assert A.lib().cpipe_cuda_memcpy_d2h(out.ctypes.data, C.c_void_p(self.at(offset)), out.nbytes) == 0
        return out

    def free(self):
        if self._p.value:
            A.lib().cpipe_cuda_device_free(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def d2d(dst, src, nbytes, stream=None):
    st = A.lib().cpipe_cuda_memcpy_d2d_async(C.c_void_p(dst), C.c_void_p(src), int(nbytes), stream)
    if st:
        raise CpipeError(st, "d2d " + A.lib().cpipe_cuda_last_error().decode())


def _ab(noise_ab):
    flat = np.ascontiguousarray(np.asarray(noise_ab, np.float32).reshape(-1))
    return flat, flat.ctypes.data


class Surrogate:
    """The network on the current CUDA device (cpipe_surrogate_*)."""

    def __init__(self, blob):
        st = C.c_int32(0)
        raw = bytes(blob)
        self._h = A.lib().cpipe_surrogate_create(raw, len(raw), C.byref(st))
        if not self._h:
            raise CpipeError(st.value, "surrogate_create " + A.lib().cpipe_cuda_last_error().decode())

    def close(self):
        if self._h:
            A.lib().cpipe_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def denoise(self, d_in, d_out, n, width, height, noise_ab, f16=True, stream=None):
        keep, p = _ab(noise_ab)
        st = A.lib().cpipe_surrogate_denoise(self._h, d_in, d_out, n, width, height, int(f16), p, stream)
        if st:
            raise CpipeError(st, "surrogate_denoise " + A.lib().cpipe_cuda_last_error().decode())

    def set_engine(self, engine):
        """'tcgen05' (default) or 'mma' for inference."""
        st = A.lib().cpipe_surrogate_set_engine(self._h, {"mma": 0, "tcgen05": 1}[engine])
        if st:
            raise CpipeError(st, "surrogate_set_engine " + A.lib().cpipe_cuda_last_error().decode())

    def check(self):
        st = A.lib().cpipe_surrogate_check(self._h)
        if st:
            raise CpipeError(st, "surrogate_check " + A.lib().cpipe_cuda_last_error().decode())

    def profile(self, d_in, d_out, n, width, height, noise_ab, f16=True, stream=None):
        """Per-kernel times (ms) of one denoise: [input map, layer 0, ..., layer 7]."""
        keep, p = _ab(noise_ab)
        ms = (C.c_float * 9)()
        st = A.lib().cpipe_surrogate_profile(self._h, d_in, d_out, n, width, height, int(f16), p, ms, stream)
        if st:
            raise CpipeError(st, "surrogate_profile " + A.lib().cpipe_cuda_last_error().decode())
        return list(ms)

    def train_step(self, d_noisy, d_target, noise_ab, n, width, height, lr, update=True, want_loss=True,
                   stream=None):
        keep, p = _ab(noise_ab)
        loss = C.c_float(float("nan"))
        st = A.lib().cpipe_surrogate_train_step(self._h, d_noisy, d_target, p, n, width, height, float(lr),
                                                int(update), C.byref(loss) if want_loss else None, stream)
        if st:
            raise CpipeError(st, "surrogate_train_step " + A.lib().cpipe_cuda_last_error().decode())
        return loss.value if want_loss else None

    def gradients(self):
        n = sum(co * ci * 9 + co for co, ci in SHAPES)
        g = np.empty(n, np.float32)
        st = A.lib().cpipe_surrogate_gradients(self._h, g.ctypes.data, n)
        if st:
            raise CpipeError(st, "surrogate_gradients")
        return from_blob(struct.pack("<4s5I2I", b"CPSN", 1, LAYERS, CHANNELS, 4, 3, 0, 0) + g.tobytes())

    def export(self):
        size = A.lib().cpipe_surrogate_blob_size()
        buf = C.create_string_buffer(size)
        st = A.lib().cpipe_surrogate_export(self._h, buf, size)
        if st:
            raise CpipeError(st, "surrogate_export")
        return buf.raw


# ------------------------------------------------------------- training data
class PairGenerator:
    """(denoiser input, two-stage BM3D output) tile pairs made on the GPU.

    Each frame is `tile` wide and `tile * per_frame` tall, so its tiles are
    contiguous in memory; BM3D runs on the whole frame.  Frames vary at random
    between a Bayer (RGGB) and a Quad-Bayer mosaic (remosaiced by the chain's
    demosaic.quad_bayer_remosaic), between 10, 12 and 14 bits, and between 1, 4
    and 20 scene rectangles (large frames seen through 256x256 tiles are mostly
    flat)."""

    KINDS = ("rggb", "qbc")
    BITS = (10, 12, 14)
    BLACK = {10: 16, 12: 64, 14: 256}
    RECTS = (1, 4, 20)

    def __init__(self, tile=256, per_frame=8, seed=0x5EED0005, kinds=KINDS, bits=BITS, rects=RECTS):
        self.tile, self.per_frame, self.seed = tile, per_frame, seed
        self.w, self.h = tile, tile * per_frame
        self.kinds, self.bits, self.rects = tuple(kinds), tuple(bits), tuple(rects)
        self.fronts = {}
        self.raw = DeviceArray(self.w * self.h * 2)
        self.noisy = DeviceArray(self.w * self.h * 8)
        self.target = DeviceArray(self.w * self.h * 8)

    def front(self, kind, bits):
        """The chain front (stop_after = 1) for one mosaic kind and bit depth."""
        from .chain import Chain, ChainConfig
        key = (kind, bits)
        if key not in self.fronts:
            cfg = ChainConfig.full_12mp(width=self.w, height=self.h, stop_after=1, use_graph=False, bits=bits,
                                        black=float(self.BLACK[bits]), quad_bayer=kind == "qbc",
                                        name=f"surrogate_pairs_{self.w}x{self.h}_{kind}_{bits}")
            self.fronts[key] = Chain(cfg)
        return self.fronts[key]

    def nonfinite(self):
        """Non-finite values in the current frame's input and target.  The
        reference's RCD ratio c / max(g, 1e-6) (demosaic_rcd_generator.cpp:37-39)
        overflows binary16 in very dark, very noisy areas, and the colour
        matrix then turns inf - inf into NaN; such frames are not used."""
        L, n = A.lib(), C.c_uint64()
        total = 0
        for d in (self.noisy, self.target):
            assert L.cpipe_cuda_count_nonfinite(d.ptr, self.w * self.h * 4, 1, C.byref(n), None) == 0
            total += n.value
        return total

    def frame(self, index, a, b, kind="rggb", bits=10, rects=20):
        from .scene import RGGB, SONY_QBC
        L = A.lib()
        pat = (C.c_uint8 * 16)(*(SONY_QBC if kind == "qbc" else RGGB))
        st = L.cpipe_cuda_scene_raw_cfa(self.raw.ptr, self.w, self.h, C.c_uint64(self.seed + index), bits,
                                        self.BLACK[bits], float(a), float(b), pat, 4 if kind == "qbc" else 2,
                                        int(rects), None)
        if st:
            raise CpipeError(st, "scene_raw " + L.cpipe_cuda_last_error().decode())
        self.front(kind, bits).run(self.raw.ptr, self.noisy.ptr, None)
        img = lambda d: DeviceImage(d.ptr, (self.h, self.w, 4), np.float16)
        st = call_filter("denoise_bm3d_spec", [img(self.noisy)], [img(self.target)], B.bm3d_spec(noise_sigma(a, b)))
        if st:
            raise CpipeError(st, "bm3d " + last_error())

    def dataset(self, count, rng, noise_a=NOISE_A):
        """count tiles in shuffled order: (noisy, target) DeviceArrays of
        [count][tile][tile][4] binary16 and the per-tile (a, b)."""
        tb = self.tile * self.tile * 8
        noisy, target = DeviceArray(count * tb), DeviceArray(count * tb)
        ab = np.empty((count, 2), np.float32)
        slots = rng.permutation(count)
        k, f = 0, 0
        self.skipped = 0
        while k < count:
            a = float(np.exp(rng.uniform(np.log(noise_a[0]), np.log(noise_a[1]))))
            b = float(np.exp(rng.uniform(np.log(NOISE_B[0]), np.log(NOISE_B[1]))))
            kind = self.kinds[int(rng.integers(len(self.kinds)))]
            bits = self.bits[int(rng.integers(len(self.bits)))]
            rects = self.rects[int(rng.integers(len(self.rects)))]
            self.frame(f, a, b, kind, bits, rects)
            f += 1
            if self.nonfinite():
                self.skipped += 1
                continue
            for t in range(self.per_frame):
                if k == count:
                    break
                s = int(slots[k])
                d2d(noisy.at(s * tb), self.noisy.at(t * tb), tb)
                d2d(target.at(s * tb), self.target.at(t * tb), tb)
                ab[s] = (a, b)
                k += 1
        assert A.lib().cpipe_cuda_synchronize() == 0
        return noisy, target, ab

    def close(self):
        for c in self.fronts.values():
            c.close()
        self.fronts = {}
        for d in (self.raw, self.noisy, self.target):
            d.free()


def psnr(a, b, peak=1.0):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * math.log10(peak * peak / mse)


def evaluate(sg, noisy, target, ab, first, count, tile=256, batch=16):
    """Mean PSNR (RGB) of the surrogate, of the noisy input and of the
    reference's 2x2 box blend (the denoise.bm3d node's own computation), all
    against the BM3D output, over tiles [first, first + count)."""
    tb = tile * tile * 8
    out = DeviceArray(batch * tb)
    box = DeviceArray(tb)
    res = {"surrogate": [], "noisy": [], "box2x2": []}
    for s in range(first, first + count, batch):
        n = min(batch, first + count - s)
        sg.denoise(noisy.at(s * tb), out.ptr, n, tile, tile, ab[s:s + n])
        got = out.download((n, tile, tile, 4), np.float16).astype(np.float32)
        for j in range(n):
            want = target.download((tile, tile, 4), np.float16, (s + j) * tb).astype(np.float32)
            inp = noisy.download((tile, tile, 4), np.float16, (s + j) * tb).astype(np.float32)
            img = lambda d, off=0: DeviceImage(d + off, (tile, tile, 4), np.float16)
            st = call_filter("denoise_bm3d_step1", [img(noisy.ptr, (s + j) * tb)], [img(box.ptr)],
                             B.bm3d(noise_sigma(*ab[s + j])))
            assert st == 0, last_error()
            bx = box.download((tile, tile, 4), np.float16).astype(np.float32)
            res["surrogate"].append(psnr(got[j, ..., :3], want[..., :3]))
            res["noisy"].append(psnr(inp[..., :3], want[..., :3]))
            res["box2x2"].append(psnr(bx[..., :3], want[..., :3]))
    out.free()
    box.free()
    return {k: float(np.mean(v)) for k, v in res.items()}


def train(pairs=20000, steps=4000, batch=16, lr=5e-4, seed=1, tile=256, val=256, log=print, init=None,
          noise_a=NOISE_A):
    """Generate `pairs` training tiles on the GPU and train; returns (blob, report).
    init: a weights blob to start from; noise_a: the range of the noise
    model's a the tiles are drawn from (log-uniform)."""
    rng = np.random.default_rng(seed)
    t0 = time.time()
    gen = PairGenerator(tile=tile)
    noisy, target, ab = gen.dataset(pairs + val, rng, noise_a)
    gen.close()
    t_data = time.time() - t0
    skipped = gen.skipped
    log(f"pairs: {pairs} + {val} held out, {tile}x{tile}, generated in {t_data:.1f} s "
        f"({gen.skipped} frames with non-finite values skipped)")
    sg = Surrogate(init if init is not None else to_blob(init_params(seed)))
    tb = tile * tile * 8
    bn, bt = DeviceArray(batch * tb), DeviceArray(batch * tb)
    before = evaluate(sg, noisy, target, ab, pairs, val, tile)
    log(f"before: {before}")
    history = []
    t1 = time.time()
    for step in range(steps):
        idx = rng.choice(pairs, batch, replace=False)
        for j, i in enumerate(idx):
            d2d(bn.at(j * tb), noisy.at(int(i) * tb), tb)
            d2d(bt.at(j * tb), target.at(int(i) * tb), tb)
        warm = min(1.0, (step + 1) / 200.0)
        lr_t = warm * (lr * 0.5 * (1.0 + math.cos(math.pi * step / steps)) + 1e-5)
        want = step % 100 == 0 or step == steps - 1
        loss = sg.train_step(bn.ptr, bt.ptr, ab[idx], batch, tile, tile, lr_t, True, want)
        if want:
            history.append((step, loss))
            log(f"step {step:5d} lr {lr_t:.2e} loss {loss:.3e} ({10 * math.log10(1 / max(loss, 1e-30)):.2f} dB)")
    assert A.lib().cpipe_cuda_synchronize() == 0
    t_train = time.time() - t1
    after = evaluate(sg, noisy, target, ab, pairs, val, tile)
    log(f"after: {after}; training {t_train:.1f} s ({1000 * t_train / steps:.2f} ms/step)")
    blob = sg.export()
    report = dict(pairs=pairs, held_out=val, tile=tile, steps=steps, batch=batch, lr=lr, seed=seed,
                  noise_a=list(noise_a), fine_tuned=init is not None,
                  skipped_frames=skipped, data_seconds=t_data, train_seconds=t_train, before=before, after=after, history=history)
    sg.close()
    for d in (noisy, target, bn, bt):
        d.free()
    return blob, report


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--pairs", type=int, default=80000)
    t.add_argument("--steps", type=int, default=40000)
    t.add_argument("--batch", type=int, default=16)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--report", default=None)
    t.add_argument("--init", default=None, help="start from these weights (fine-tuning) instead of a random init")
    t.add_argument("--noise-a-max", type=float, default=NOISE_A[1],
                   help="upper end of the training noise model's a (log-uniform from %g)" % NOISE_A[0])
    args = ap.parse_args()
    assert A.lib().cpipe_cuda_device_count() > 0, "no CUDA device"
    init = load_weights(args.init) if args.init else None
    blob, report = train(args.pairs, args.steps, args.batch, args.lr, args.seed, init=init,
                         noise_a=(NOISE_A[0], args.noise_a_max))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with open(args.out, "wb") as f:
        f.write(blob)
    if args.report:
        import json
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    _main()
