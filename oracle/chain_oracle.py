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
