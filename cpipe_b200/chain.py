"""The fused raw->linear chain (cpipe_cuda_chain_* in include/cpipe_b200.h) and
the workload configurations it is measured and tested on.

`ChainConfig` holds the node parameters the way the reference pipeline has
them (levels, CFA, an OpcodeList2 GainMap, the demosaic choice, an OpcodeList3
WarpRectilinear, the DNG white balance inputs, the denoise / tone / LUT
parameters).  `blobs()` resolves them with the library's own host-side
preparation -- the same code the node plugins run -- into the filter blobs,
and `Chain` runs them on the GPU.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from . import blobs as B
from .host import CpipeError
from .scene import RGGB, raw_frame

# A fixed camera -> XYZ(D50) matrix used as ForwardMatrix1 = ForwardMatrix2, so
# the dual-illuminant blend yields it exactly; the ColorMatrix pair drives the
# CCT search.
CAMERA_TO_XYZ = (0.6734, 0.2175, 0.0733, 0.2798, 0.8107, -0.0905, 0.0148, -0.1486, 0.9589)
COLOR_MATRIX1 = (0.6722, -0.0635, -0.0963, -0.4287, 1.2460, 0.2028, -0.0908, 0.2162, 0.5668)
COLOR_MATRIX2 = (0.8128, -0.2218, -0.0815, -0.4148, 1.1926, 0.2469, -0.0793, 0.1797, 0.6080)


def identity_gamma_lut(size=33, gamma=1.0 / 1.1):
    g = np.linspace(0.0, 1.0, size, dtype=np.float64)
    r, gg, b = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([r ** gamma, gg ** gamma, b ** gamma], -1).astype(np.float32)


def smooth_random_lut(size=33, seed=0x5EED0002, crosstalk=0.02):
    """Seeded monotone per-channel curves plus a small cross-talk term."""
    rng = np.random.Generator(np.random.Philox(seed))
    g = np.linspace(0.0, 1.0, size, dtype=np.float64)
    curves = []
    for _ in range(3):
        gamma = rng.uniform(0.8, 1.25)
        lift = rng.uniform(0.0, 0.04)
        knee = rng.uniform(0.2, 0.5)
        c = lift + (1.0 - lift) * g ** gamma
        c = c + 0.05 * np.sin(np.pi * g) * knee
        curves.append(np.maximum.accumulate(np.clip(c, 0.0, 1.0)))
    r, gg, b = np.meshgrid(np.arange(size), np.arange(size), np.arange(size), indexing="ij")
    cr, cg, cb = curves[0][r], curves[1][gg], curves[2][b]
    mean = (cr + cg + cb) / 3.0
    out = np.stack([cr + crosstalk * (mean - cr), cg + crosstalk * (mean - cg), cb + crosstalk * (mean - cb)], -1)
    return np.clip(out, 0.0, 1.0).astype(np.float32)


def radial_gains(points_v=13, points_h=17, lo=1.0, hi=1.8):
    yy, xx = np.mgrid[0:points_v, 0:points_h].astype(np.float64)
    dy = (yy - (points_v - 1) / 2) / ((points_v - 1) / 2)
    dx = (xx - (points_h - 1) / 2) / ((points_h - 1) / 2)
    r2 = (dx * dx + dy * dy) / 2.0
    return (lo + (hi - lo) * r2).astype(np.float32)


@dataclass
class ChainConfig:
    width: int
    height: int
    name: str = "custom"
    bits: int = 12
    black: float = 64.0
    noise_a: float = 1e-3
    noise_b: float = 1e-5
    seed: int = 0x5EED0001
    cfa: tuple = RGGB
    demosaic: str = "rcd"
    gainmap: bool = False
    warp: tuple = None             # (kr0, kr1, kr2, kr3, kt0, kt1) or None
    wb_gains: tuple = (2.0, 1.0, 1.6)
    guided_radius: int = 0         # 0: no guided node
    guided_eps: float = 1e-3
    wavelet_strength: float = -1.0  # < 0: no wavelet node
    filmic: dict = field(default_factory=dict)
    lut: str = "identity_gamma"    # identity_gamma | smooth | none
    plain_f32: bool = False
    use_graph: bool = True
    denoise: str = "box2x2"        # box2x2 (the reference's bm3d node) | bm3d (two-stage) | surrogate
    bm3d_stages: int = 2
    surrogate_blob: bytes = None   # trained network (cpipe_b200.surrogate) for denoise="surrogate"
    stop_after: int = 0            # 1: output the denoiser's input; 2: the denoiser's output
    quad_bayer: bool = False       # raw input is a Sony Quad-Bayer mosaic, remosaiced first
    spot_tiles: int = 16           # surrogate spot check: BM3D on this many 256x256 tiles per frame
    spot_min_psnr_db: float = 40.0  # ... and BM3D for the whole frame when a tile is below this
    guided_spec: bool = False      # guided filter with the true (2r+1)^2 box (radius 1..16)
    atrous_levels: int = 0         # > 0: a-trous wavelet denoiser with that many levels instead of the 2x2 Haar
    atrous_luma_strength: float = 1.0
    # finishing stages after the LUT (the reference's example pipeline continues
    # with them): sharpen.edge_aware_usm, then the display encode
    sharpen: bool = False
    sharpen_strength: float = 0.75
    sharpen_radius: int = 1
    sharpen_threshold: float = 0.0
    display: str = ""              # "" (RGBA16F output) | "sRGB" (RGBA8) | "BT2020-PQ" (RGBA16 unorm)
    tone: str = "filmic"           # tone stage: filmic | aces | reinhard
    reinhard_white_point: float = -1.0  # < 0: the reinhard node's unset value

    # ------------------------------------------------------------ workloads
    @classmethod
    def small_frame(cls, w=2016, h=1512, **kw):
        """2016x1512 RGGB 12-bit (black 64, white 4095, a=1e-3, b=1e-5):
        normalise, WB (2, 1, 1.6), RCD, camera matrix to Rec.2020, BM3D with
        sigma from the noise model, identity+gamma 33^3 LUT, filmic.  The
        wavelet node (chroma_strength 1) is kept because the reference loader
        requires it upstream of filmic."""
        base = dict(width=w, height=h, name=f"small_frame_{w}x{h}", wavelet_strength=1.0)
        base.update(kw)
        return cls(**base)

    @classmethod
    def qbc_50mp(cls, **kw):
        """8160x6120 Sony Quad-Bayer 10-bit frame (the 12 MP workload's scene,
        noise, GainMap, warp, guided, wavelet and LUT), remosaiced to RGGB by
        demosaic.quad_bayer_remosaic ahead of the chain."""
        base = dict(width=8160, height=6120, name="qbc_chain_50mp_8160x6120", quad_bayer=True)
        base.update(kw)
        return cls.full_12mp(**base)

    @classmethod
    def full_12mp(cls, **kw):
        """4032x3024 RGGB 10-bit (black 16, white 1023, a=4e-3, b=4e-5): adds a
        17x13 radial GainMap (1.0-1.8), guided r=8 eps=1e-3, the wavelet shrink,
        an OpcodeList3 WarpRectilinear (k1=-0.08, k2=0.02, k3=0) and a seeded
        smooth 33^3 LUT; RCD demosaic (AMaZE as the alternate)."""
        base = dict(width=4032, height=3024, name="full_chain_12mp_4032x3024", bits=10, black=16.0, noise_a=4e-3,
                    noise_b=4e-5, seed=0x5EED0002, gainmap=True, warp=(1.0, -0.08, 0.02, 0.0, 0.0, 0.0),
                    guided_radius=8, guided_eps=1e-3, wavelet_strength=1.0, lut="smooth")
        base.update(kw)
        return cls(**base)

    @classmethod
    def small(cls, w=96, h=64, **kw):
        return cls.full_12mp(width=w, height=h, name=f"full_chain_{w}x{h}", **kw)

    # ------------------------------------------------------------ inputs
    @property
    def white(self):
        return (1 << self.bits) - 1

    def make_raw(self, seed=None):
        return raw_frame(self.width, self.height, self.seed if seed is None else seed, bits=self.bits,
                         black=int(self.black), a=self.noise_a, b=self.noise_b, cfa=self.cfa,
                         quad_bayer=self.quad_bayer)

    @property
    def neutral(self):
        return tuple(float(np.float32(1.0) / np.float32(g)) for g in self.wb_gains)

    @property
    def bm3d_sigma(self):
        # NoiseProfile (beta = b, lambda = a) evaluated at signal 0.25 (bm3d.cpp:49-54)
        f = np.float32
        v = max(f(0.0), f(f(self.noise_b) + f(self.noise_a) * f(0.25)))
        return float(f(np.sqrt(np.float64(v))))

    def lut_values(self):
        if self.lut == "smooth":
            return smooth_random_lut(33)
        if self.lut == "identity_gamma":
            return identity_gamma_lut(33)
        return None

    # ------------------------------------------------------------ blobs
    def blobs(self):
        """Per-node filter blobs, resolved by the library's host preparation."""
        L = A.lib()
        out = {"blacklevel": B.blacklevel([self.black] * 4, self.white, self.cfa),
               "demosaic": B.demosaic(self.cfa)}
        if self.gainmap:
            stream = B.opcode_list_2_with_gain_maps([B.gain_map_params(
                17, 13, 0, 1, max(self.height - 1, 1) / 12.0, max(self.width - 1, 1) / 16.0, radial_gains())])
            n = C.c_size_t(0)
            rep, pat = (C.c_uint8 * 2)(2, 2), (C.c_uint8 * 16)(*self.cfa)
            st = L.cpipe_b200_pack_gain_maps(stream, len(stream), rep, pat, None, C.byref(n))
            buf = C.create_string_buffer(n.value)
            st = st or L.cpipe_b200_pack_gain_maps(stream, len(stream), rep, pat, buf, C.byref(n))
            if st:
                raise CpipeError(st, "pack gain maps")
            out["gainmap"] = buf.raw
            out["opcode_list_2"] = stream
        if self.warp is not None:
            stream = B.opcode_list([(1, B.warp_rectilinear_params([self.warp]))])
            n, cnt = C.c_size_t(1 << 16), C.c_uint32()
            buf = C.create_string_buffer(n.value)
            st = L.cpipe_b200_pack_opcode_list_3(stream, len(stream), buf, C.byref(n), C.byref(cnt))
            if st:
                raise CpipeError(st, "pack opcode list 3")
            out["opcode3"] = buf.raw[:n.value]
            out["opcode_list_3"] = stream
        F9 = C.c_float * 9
        wb = A.WbParams()
        cct = C.c_double()
        st = L.cpipe_b200_wb_prepare((C.c_float * 3)(*self.neutral), F9(*COLOR_MATRIX1), F9(*COLOR_MATRIX2),
                                     F9(*CAMERA_TO_XYZ), F9(*CAMERA_TO_XYZ), 17, 21, C.byref(wb), C.byref(cct))
        if st:
            raise CpipeError(st, "wb prepare")
        out["wb"] = bytes(wb)
        t = F9()
        L.cpipe_b200_colormatrix_compose(wb.camera_to_xyz_d50, t)
        out["colormatrix"] = B.colormatrix(list(t))
        out["colormatrix_t"] = list(t)
        out["bm3d"] = B.bm3d(self.bm3d_sigma)
        if self.guided_radius > 0:
            out["guided"] = B.guided(self.guided_radius, self.guided_eps)
        if self.wavelet_strength >= 0:
            out["wavelet"] = B.wavelet(self.wavelet_strength)
        out["filmic"] = B.filmic(**self.filmic)
        lut = self.lut_values()
        if lut is not None:
            out["lut"] = B.lut3d(33, lut, 0)
            out["lut_values"] = lut
        return out

    def c_config(self):
        b = self.blobs()
        cfg = A.ChainConfig()
        cfg.width, cfg.height = self.width, self.height
        C.memmove(C.addressof(cfg.black), b["blacklevel"], C.sizeof(A.BlacklevelParams))
        keep = []

        def ptr(raw):
            buf = C.create_string_buffer(raw, len(raw))
            keep.append(buf)
            return C.cast(buf, C.c_void_p), len(raw)

        if "gainmap" in b:
            cfg.gainmap_blob, cfg.gainmap_blob_size = ptr(b["gainmap"])
        cfg.demosaic = {"bilinear": 0, "rcd": 1, "amaze": 2}[self.demosaic]
        if "opcode3" in b:
            cfg.opcode3_blob, cfg.opcode3_blob_size = ptr(b["opcode3"])
        cfg.as_shot_neutral[:] = list(self.neutral)
        cfg.colormatrix[:] = b["colormatrix_t"]
        cfg.bm3d_sigma = self.bm3d_sigma
        cfg.guided_radius = self.guided_radius
        cfg.guided_eps = self.guided_eps
        cfg.wavelet_strength = self.wavelet_strength
        C.memmove(C.addressof(cfg.filmic), b["filmic"], C.sizeof(A.FilmicRgbParams))
        if "lut" in b:
            cfg.lut_blob, cfg.lut_blob_size = ptr(b["lut"])
        cfg.plain_f32 = int(self.plain_f32)
        cfg.use_graph = int(self.use_graph)
        cfg.denoise_mode = {"box2x2": 0, "bm3d": 1, "surrogate": 2}[self.denoise]
        C.memmove(C.addressof(cfg.bm3d_spec), B.bm3d_spec(self.bm3d_sigma, stages=self.bm3d_stages),
                  C.sizeof(A.Bm3dSpecParams))
        if self.surrogate_blob:
            cfg.surrogate_blob, cfg.surrogate_blob_size = ptr(bytes(self.surrogate_blob))
        cfg.noise_a, cfg.noise_b = self.noise_a, self.noise_b
        cfg.stop_after = int(self.stop_after)
        cfg.spot_tiles = int(self.spot_tiles)
        cfg.spot_min_psnr_db = float(self.spot_min_psnr_db)
        cfg.quad_bayer = int(self.quad_bayer)
        cfg.guided_spec = int(self.guided_spec)
        cfg.atrous_levels = int(self.atrous_levels)
        cfg.atrous_luma_strength = float(self.atrous_luma_strength)
        cfg.sharpen = int(self.sharpen)
        cfg.sharpen_strength = float(self.sharpen_strength)
        cfg.sharpen_radius = int(self.sharpen_radius)
        cfg.sharpen_threshold = float(self.sharpen_threshold)
        cfg.display = {"": 0, "sRGB": 1, "BT2020-PQ": 2}[self.display]
        cfg.tone = {"filmic": 0, "aces": 1, "reinhard": 2}[self.tone]
        cfg.reinhard_white_point = float(self.reinhard_white_point)
        return cfg, keep


class Chain:
    """The fused chain on the current CUDA device."""

    def __init__(self, config):
        self.config = config
        cfg, keep = config.c_config()
        st = C.c_int32(0)
        self._h = A.lib().cpipe_cuda_chain_create(C.byref(cfg), C.byref(st))
        del keep  # the library copies what it keeps
        if not self._h:
            raise CpipeError(st.value, "chain_create " + A.lib().cpipe_cuda_last_error().decode())
        self.out_dtype = {"sRGB": np.uint8, "BT2020-PQ": np.uint16}.get(
            config.display, np.float32 if config.plain_f32 else np.float16)
        self.out_shape = (config.height, config.width, 4)

    def close(self):
        if self._h:
            A.lib().cpipe_cuda_chain_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, d_raw, d_out, stream=None):
        """Device pointers (int); asynchronous on `stream` (cudaStream_t as int or None)."""
        st = A.lib().cpipe_cuda_chain_run(self._h, d_raw, d_out, stream)
        if st:
            raise CpipeError(st, "chain_run " + A.lib().cpipe_cuda_last_error().decode())

    def denoise_stats(self):
        """(frames checked, frames that fell back to BM3D, worst tile PSNR dB)."""
        f, b, p = C.c_uint32(), C.c_uint32(), C.c_float()
        st = A.lib().cpipe_cuda_chain_denoise_stats(self._h, C.byref(f), C.byref(b), C.byref(p))
        if st:
            raise CpipeError(st, "chain_denoise_stats")
        return f.value, b.value, p.value

    def run_host(self, raw, out=None, stream=None):
        raw = np.ascontiguousarray(raw, dtype=np.uint16)
        assert raw.shape == (self.config.height, self.config.width)
        if out is None:
            out = np.empty(self.out_shape, self.out_dtype)
        st = A.lib().cpipe_cuda_chain_run_host(self._h, raw.ctypes.data, out.ctypes.data, stream)
        if st:
            raise CpipeError(st, "chain_run_host " + A.lib().cpipe_cuda_last_error().decode())
        return out

    def run_host_frames(self, raws, outs=None, stream=None):
        """Several host frames through cpipe_cuda_chain_run_host_frames (uploads
        and downloads overlapped with the neighbouring frames' chain)."""
        raws = [np.ascontiguousarray(r, dtype=np.uint16) for r in raws]
        for r in raws:
            assert r.shape == (self.config.height, self.config.width)
        if outs is None:
            outs = [np.empty(self.out_shape, self.out_dtype) for _ in raws]
        n = len(raws)
        pr = (C.c_void_p * n)(*[r.ctypes.data for r in raws])
        po = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        st = A.lib().cpipe_cuda_chain_run_host_frames(self._h, pr, po, n, stream)
        if st:
            raise CpipeError(st, "chain_run_host_frames " + A.lib().cpipe_cuda_last_error().decode())
        return outs


def _main():
    """Run the 12 MP chain a few times on the GPU (used for profiler captures):
    python -m cpipe_b200.chain [--frames N] [--width W --height H] [--demosaic rcd|amaze|bilinear]
                               [--denoise box2x2|bm3d|surrogate] [--guided-spec] [--atrous-levels L]"""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--width", type=int, default=4032)
    ap.add_argument("--height", type=int, default=3024)
    ap.add_argument("--demosaic", default="rcd")
    ap.add_argument("--denoise", default="box2x2", choices=["box2x2", "bm3d", "surrogate"])
    ap.add_argument("--guided-spec", action="store_true", help="guided filter with the true (2r+1)^2 box")
    ap.add_argument("--atrous-levels", type=int, default=0, help="a-trous wavelet stages instead of the 2x2 Haar")
    args = ap.parse_args()
    L = A.lib()
    assert L.cpipe_cuda_device_count() > 0, "no CUDA device"
    blob = None
    if args.denoise == "surrogate":
        from .surrogate import load_weights
        blob = load_weights()
    cfg = ChainConfig.full_12mp(width=args.width, height=args.height, demosaic=args.demosaic, use_graph=False,
                                denoise=args.denoise, surrogate_blob=blob, guided_spec=args.guided_spec,
                                atrous_levels=args.atrous_levels)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    d_raw, d_out = C.c_void_p(), C.c_void_p()
    assert L.cpipe_cuda_device_alloc(raw.nbytes, C.byref(d_raw)) == 0
    assert L.cpipe_cuda_device_alloc(cfg.width * cfg.height * 8, C.byref(d_out)) == 0
    assert L.cpipe_cuda_memcpy_h2d(d_raw, raw.ctypes.data, raw.nbytes) == 0
    for _ in range(args.frames):
        chain.run(d_raw.value, d_out.value, None)
    assert L.cpipe_cuda_synchronize() == 0
    chain.close()
    L.cpipe_cuda_device_free(d_raw)
    L.cpipe_cuda_device_free(d_out)
    print("ran", args.frames, "frames of", cfg.name)


if __name__ == "__main__":
    _main()
