"""The raw->linear chain evaluated node by node with the CPU oracle.

TEST INFRASTRUCTURE: the checker for the fused GPU chain and the CPU baseline
of bench.py.  Node order and parameters come from cpipe_b200.chain.ChainConfig
(the reference classic pipeline order: convert, black level, GainMap, demosaic,
OpcodeList3, WB, colormatrix, BM3D, guided, wavelet, filmic, 3D LUT)."""
import numpy as np

import oracle


def run_chain_oracle(cfg, raw, blobs=None):
    b = blobs or cfg.blobs()
    f16 = not cfg.plain_f32
    if getattr(cfg, "quad_bayer", False):
        raw = oracle.qbc_remosaic(raw)
    x = oracle.r16u_to_f32(raw)
    st, x = oracle.blacklevel(x, b["blacklevel"])
    assert st == 0
    if "gainmap" in b:
        st, x = oracle.gainmap(x, b["gainmap"])
        assert st == 0
    x = oracle.demosaic(cfg.demosaic, x, cfg.cfa, f16)
    if "opcode3" in b:
        st, x = oracle.opcode3(x, b["opcode3"], f16)
        assert st == 0
    x = oracle.wb(x, cfg.neutral, f16)
    x = oracle.colormatrix(x, b["colormatrix_t"], f16)
    denoise = getattr(cfg, "denoise", "box2x2")
    if denoise == "bm3d":
        from cpipe_b200 import blobs as B
        x = oracle.bm3d_spec(x, B.bm3d_spec(cfg.bm3d_sigma, stages=cfg.bm3d_stages)).astype(np.float32)
        if f16:
            x = oracle.h16(x)
    elif denoise == "box2x2":
        x = oracle.bm3d_parity(x, cfg.bm3d_sigma, f16)
    else:
        raise ValueError(f"no oracle for denoise={denoise}")
    if cfg.guided_radius > 0:
        x = oracle.guided(x, cfg.guided_radius, cfg.guided_eps, f16)
    if cfg.wavelet_strength >= 0:
        x = oracle.wavelet(x, cfg.wavelet_strength, f16)
    x = oracle.filmic(x, f16=f16, **cfg.filmic)
    if "lut" in b:
        x = oracle.lut3d(x, b["lut_values"], 33, 0, f16)
    return x


def run_reference_chain(cfg, raw, blobs):
    """The chain as the reference computes it on the CPU, node by node: the
    reference's own plain-C++ filters compiled from its source (oracle/_ref:
    blacklevel_dng_levels, lens_shading_gainmap, lens_dng_opcode_list_3,
    wb_dual_illuminant, colormatrix_dng_to_working; single-threaded, as the
    reference runs them) and, for its Halide nodes (precision convert,
    demosaic, denoise.bm3d, guided filter, wavelet, filmic, 3D LUT), the C
    restatement above, parallel over rows with OpenMP.  The result equals
    run_chain_oracle bit for bit (the oracle is pinned to those filters).
    `blobs` comes from oracle_blobs.chain_blobs(cfg); nothing here loads the
    product library.  Supports the RGBA16F chain with the reference's 2x2
    denoise.bm3d, which is what the reference computes."""
    assert not cfg.plain_f32 and getattr(cfg, "denoise", "box2x2") == "box2x2"

    def ref(aot, x, blob):
        y = np.empty_like(x)
        st = oracle.ref_call(aot, x, y, blob)
        if st != 0:
            raise RuntimeError(f"reference filter {aot}: status {st}")
        return y

    b = blobs
    if getattr(cfg, "quad_bayer", False):
        raw = oracle.qbc_remosaic(raw)
    x = oracle.r16u_to_f32(raw)
    x = ref("blacklevel_dng_levels", x, b["blacklevel"])
    if "gainmap" in b:
        x = ref("lens_shading_gainmap", x, b["gainmap"])
    x = oracle.demosaic(cfg.demosaic, x, cfg.cfa, True).astype(np.float16)
    if "opcode3" in b:
        x = ref("lens_dng_opcode_list_3", x, b["opcode3"])
    x = ref("wb_dual_illuminant", x, b["wb"])
    x = ref("colormatrix_dng_to_working", x, b["colormatrix"]).astype(np.float32)
    x = oracle.bm3d_parity(x, cfg.bm3d_sigma, True)
    if cfg.guided_radius > 0:
        x = oracle.guided(x, cfg.guided_radius, cfg.guided_eps, True)
    if cfg.wavelet_strength >= 0:
        x = oracle.wavelet(x, cfg.wavelet_strength, True)
    x = oracle.filmic(x, f16=True, **cfg.filmic)
    if "lut_values" in b:
        x = oracle.lut3d(x, b["lut_values"], 33, 0, True)
    return x
