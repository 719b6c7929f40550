"""The fused chain on the GPU against (a) the CPU oracle run node by node and
(b) the same nodes run one by one on the GPU through their plugins.  Small
frames (including odd sizes) are compared element by element; the full 12 MP
workload is compared with the oracle and checked for the size-independent
properties: fused == unfused bit for bit, deterministic, graph replay equal to
direct launch, finite and in [0, 1]."""
import os

import numpy as np
import pytest
from chain_oracle import run_chain_oracle
from cpipe_b200 import _abi as A
from cpipe_b200.chain import Chain, ChainConfig
from parity import assert_f16_parity, assert_f32_parity, f16_ulp_distance, psnr

pytestmark = pytest.mark.gpu


def run_nodes_on_gpu(host, cfg, raw):
    """The chain as a sequence of plugin nodes on device buffers (reference
    node order), returning the RGBA16F result."""
    b = cfg.blobs()
    w, h = cfg.width, cfg.height
    F32, F16, U16 = A.FMT_R32_SFLOAT, A.FMT_R16G16B16A16_SFLOAT, A.FMT_R16_UINT
    cur = host.buffer(U16, w, h).upload(raw)
    meta = dict(cfa=cfg.cfa, black_level=[cfg.black] * 4, white_level=cfg.white, cs_role="raw_camera",
                illuminants=(17, 21), as_shot_neutral=list(cfg.neutral),
                noise_profile=[(cfg.noise_b, cfg.noise_a)])
    from cpipe_b200.chain import CAMERA_TO_XYZ, COLOR_MATRIX1, COLOR_MATRIX2
    meta.update(color_matrix1=COLOR_MATRIX1, color_matrix2=COLOR_MATRIX2, forward_matrix1=CAMERA_TO_XYZ,
                forward_matrix2=CAMERA_TO_XYZ)
    blob_meta = {}
    if "opcode_list_2" in b:
        blob_meta["com.cpipe.dng.opcode_list_2_bytes"] = b["opcode_list_2"]
    if "opcode_list_3" in b:
        blob_meta["com.cpipe.dng.opcode_list_3_bytes"] = b["opcode_list_3"]
    cur.set_metadata(blobs=blob_meta, **meta)
    import tempfile, os
    from cpipe_b200 import blobs as BL
    steps = [("com.cpipe.precision_convert", F32, {"target_format": "R32_SFLOAT"}),
             ("com.cpipe.blacklevel.dng_levels", F32, {})]
    if cfg.gainmap:
        steps.append(("com.cpipe.lens.shading_gainmap", F32, {}))
    steps.append((f"com.cpipe.demosaic.{cfg.demosaic}", F16, {}))
    if cfg.warp is not None:
        steps.append(("com.cpipe.lens.dng_opcode_list_3", F16, {}))
    steps += [("com.cpipe.wb.dual_illuminant", F16, {}), ("com.cpipe.colormatrix.dng_to_working", F16, {}),
              ("com.cpipe.denoise.bm3d", F16, {"algorithm": "bm3d", "stages": cfg.bm3d_stages}
               if cfg.denoise == "bm3d" else {})]
    if cfg.guided_radius > 0:
        gp = {"radius": cfg.guided_radius, "eps": cfg.guided_eps}
        if cfg.guided_spec:
            gp["algorithm"] = "spec"
        steps.append(("com.cpipe.denoise.guided_filter", F16, gp))
    if cfg.atrous_levels > 0:
        steps.append(("com.cpipe.denoise.wavelet_bayes_shrink", F16,
                      {"algorithm": "atrous", "levels": cfg.atrous_levels, "sigma": cfg.bm3d_sigma,
                       "luma_strength": cfg.atrous_luma_strength,
                       "chroma_strength": cfg.wavelet_strength if cfg.wavelet_strength >= 0 else 1.0}))
    elif cfg.wavelet_strength >= 0:
        steps.append(("com.cpipe.denoise.wavelet_bayes_shrink", F16, {"chroma_strength": cfg.wavelet_strength}))
    if cfg.tone == "aces":
        steps.append(("com.cpipe.tone.aces_filmic", F16, {}))
    elif cfg.tone == "reinhard":
        steps.append(("com.cpipe.tone.reinhard", F16, {} if cfg.reinhard_white_point < 0 else
                      {"white_point": cfg.reinhard_white_point}))
    else:
        steps.append(("com.cpipe.tone.filmic_rgb", F16, {}))
    tmp = None
    if "lut" in b:
        tmp = tempfile.NamedTemporaryFile(suffix=".cube", delete=False)
        tmp.close()
        BL.write_cube(tmp.name, 33, b["lut_values"])
        steps.append(("com.cpipe.color.3d_lut", F16, {"lut_path": tmp.name}))
    if cfg.sharpen:
        steps.append(("com.cpipe.sharpen.edge_aware_usm", F16, {"strength": cfg.sharpen_strength,
                                                              "radius": cfg.sharpen_radius,
                                                              "threshold": cfg.sharpen_threshold}))
    if cfg.display:
        steps.append(("com.cpipe.color.scene_linear_to_display",
                      A.FMT_R8G8B8A8_UNORM if cfg.display == "sRGB" else A.FMT_R16G16B16A16_UNORM,
                      {"target": cfg.display}))
    try:
        for node_id, fmt, params in steps:
            nxt = host.buffer(fmt, w, h)
            st = host.run_node(node_id, [cur], [nxt], params)
            assert st == 0, f"{node_id}: {A.STATUS_NAMES.get(st)} {host.last_error()}"
            cur = nxt
    finally:
        if tmp:
            os.unlink(tmp.name)
    return cur.download()


SMALL = [(96, 64), (97, 63), (33, 17), (2, 2), (1, 1), (130, 70)]


@pytest.mark.parametrize("w,h", SMALL)
def test_chain_matches_oracle_small(cuda_device, w, h):
    cfg = ChainConfig.small(w, h)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    want = run_chain_oracle(cfg, raw)
    assert_f16_parity(got, want, what=f"chain {w}x{h}")
    chain.close()


@pytest.mark.parametrize("variant", [
    dict(demosaic="amaze"), dict(demosaic="bilinear"), dict(gainmap=False), dict(warp=None),
    dict(guided_radius=1, guided_eps=0.015), dict(guided_radius=0), dict(wavelet_strength=-1.0),
    dict(lut="identity_gamma"), dict(lut="none"), dict(filmic=dict(ev=0.5, contrast=1.3, saturation=1.2)),
    dict(cfa=(2, 1, 1, 0)), dict(cfa=(1, 0, 2, 1)), dict(use_graph=False),
])
def test_chain_variants_match_oracle(cuda_device, variant):
    cfg = ChainConfig.small(120, 90, **variant)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    assert_f16_parity(got, run_chain_oracle(cfg, raw), what=str(variant))
    chain.close()


def test_chain_plain_f32_form(cuda_device):
    cfg = ChainConfig.small(128, 96, plain_f32=True)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    assert got.dtype == np.float32
    assert_f32_parity(got, run_chain_oracle(cfg, raw), what="chain f32")
    chain.close()


def test_chain_equals_nodes_on_gpu(cuda_device, host):
    """Fusing the nodes changes no arithmetic: bit-identical to the plugins run one by one."""
    cfg = ChainConfig.small(160, 120)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    fused = chain.run_host(raw)
    nodes = run_nodes_on_gpu(host, cfg, raw)
    assert f16_ulp_distance(fused, nodes).max() == 0
    chain.close()


def test_chain_general_opcode_list(cuda_device):
    """OpcodeList3 lists other than a single warp take the per-node path inside the chain."""
    import ctypes as C
    from cpipe_b200 import blobs as BL
    cfg = ChainConfig.small(100, 80)
    raw = cfg.make_raw()
    b = cfg.blobs()
    vig = BL.vignette_record([0.3])
    warp = BL.warp_record([cfg.warp])
    b["opcode3"] = BL.opcode3_dispatch([vig, warp])
    c_cfg, keep = cfg.c_config()
    buf = C.create_string_buffer(b["opcode3"], len(b["opcode3"]))
    c_cfg.opcode3_blob, c_cfg.opcode3_blob_size = C.cast(buf, C.c_void_p), len(b["opcode3"])
    st = C.c_int32()
    h = A.lib().cpipe_cuda_chain_create(C.byref(c_cfg), C.byref(st))
    assert h, st.value
    out = np.empty((80, 100, 4), np.float16)
    assert A.lib().cpipe_cuda_chain_run_host(h, raw.ctypes.data, out.ctypes.data, None) == 0
    A.lib().cpipe_cuda_chain_destroy(h)
    assert_f16_parity(out, run_chain_oracle(cfg, raw, blobs=b), what="general opcode list")


def test_chain_full_12mp(cuda_device, host):
    cfg = ChainConfig.full_12mp()
    raw = cfg.make_raw()
    chain = Chain(cfg)
    a = chain.run_host(raw)
    b = chain.run_host(raw)
    assert np.array_equal(a.view(np.uint16), b.view(np.uint16)), "non-deterministic"
    af = a.astype(np.float32)
    assert np.isfinite(af).all() and af.min() >= 0.0 and af.max() <= 1.0
    cfg_ng = ChainConfig.full_12mp(use_graph=False)
    chain_ng = Chain(cfg_ng)
    c = chain_ng.run_host(raw)
    assert np.array_equal(a.view(np.uint16), c.view(np.uint16)), "graph replay differs"
    nodes = run_nodes_on_gpu(host, cfg, raw)
    assert f16_ulp_distance(a, nodes).max() == 0, "fused differs from node-by-node"
    want = run_chain_oracle(cfg, raw)
    ulps, n_off = assert_f16_parity(a, want, what="12MP chain vs oracle")
    chain.close()
    chain_ng.close()


@pytest.mark.parametrize("demosaic", ["rcd", "amaze"])
def test_chain_with_two_stage_bm3d(host, demosaic):
    """denoise_mode 1: the two-stage BM3D between colormatrix and guided.  The
    BM3D aggregation order is not fixed on the GPU (shared-memory atomics), so
    the chain is compared with the nodes one by one, and with the oracle chain
    (FP64 BM3D), within tolerances: PSNR >= 60 dB against the nodes, >= 50 dB
    against the oracle."""
    cfg = ChainConfig.full_12mp(width=200, height=136, demosaic=demosaic, denoise="bm3d")
    raw = cfg.make_raw()
    got = Chain(cfg).run_host(raw).astype(np.float32)
    nodes = run_nodes_on_gpu(host, cfg, raw).astype(np.float32)
    want = run_chain_oracle(cfg, raw)
    p_nodes, p_oracle = psnr(got[..., :3], nodes[..., :3]), psnr(got[..., :3], want[..., :3])
    print(f"bm3d chain {demosaic}: vs nodes {p_nodes:.1f} dB, vs oracle {p_oracle:.1f} dB")
    assert p_nodes >= 60.0 and p_oracle >= 50.0
    np.testing.assert_array_equal(got[..., 3], want[..., 3])


def test_chain_quad_bayer_matches_oracle(cuda_device):
    """A Quad-Bayer raw frame: demosaic.quad_bayer_remosaic (integer, bit-exact)
    then the Bayer chain, against the oracle chain."""
    cfg = ChainConfig.small(200, 148, quad_bayer=True)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    assert_f16_parity(got, run_chain_oracle(cfg, raw), what="quad bayer chain")
    chain.close()


def test_qbc_50mp_remosaic_and_bm3d_precision_forms(cuda_device):
    """The 50 MP case: an 8160x6120 Quad-Bayer frame.  The remosaic is bit-exact
    against the oracle over the whole frame; the chain runs to the end with finite
    output; and the two-stage BM3D of the chain's denoiser input, in its
    tensor-core form (FP16 hi/lo split) and its FP32 CUDA-core form, is compared
    with the FP64 oracle on the interior of a reference-grid-aligned crop (the
    error of each form is printed)."""
    import oracle as O
    from bm3d_scenes import psnr as bpsnr
    from cpipe_b200 import blobs, call_filter, last_error
    cfg = ChainConfig.qbc_50mp()
    raw = cfg.make_raw()
    bayer = np.zeros_like(raw)
    assert call_filter("demosaic_quad_bayer_remosaic", [raw], [bayer]) == 0, last_error()
    np.testing.assert_array_equal(bayer, O.qbc_remosaic(raw))
    full = Chain(cfg)
    out = full.run_host(raw)
    assert np.isfinite(out.astype(np.float32)).all()
    full.close()
    front = Chain(ChainConfig.qbc_50mp(stop_after=1))
    x = front.run_host(raw)
    front.close()
    y0, x0, n, margin = 3000, 4200, 420, 2 * (2 * 19 + 8)
    crop = x[y0:y0 + n, x0:x0 + n].astype(np.float32)
    want = O.bm3d_spec(crop, blobs.bm3d_spec(cfg.bm3d_sigma))
    inner = slice(margin, n - margin)
    for form in ("tensor", "fp32"):
        got = np.zeros_like(x)
        assert call_filter("denoise_bm3d_spec", [x], [got], blobs.bm3d_spec(cfg.bm3d_sigma, transform=form)) == 0
        g = got[y0:y0 + n, x0:x0 + n][inner, inner].astype(np.float64)[..., :3]
        w_ = want[inner, inner][..., :3]
        err, p = float(np.abs(g - w_).max()), bpsnr(g, w_)
        print(f"50 MP BM3D {form}: max-abs {err:.3g} PSNR {p:.1f} dB vs FP64 oracle")
        assert p >= 55.0 and err <= 5e-3


@pytest.mark.parametrize("mode", ["reference", "surrogate"])
def test_run_host_frames_matches_run_host(cuda_device, mode):
    """The pipelined host entry point (uploads and downloads overlapping the
    neighbouring frames' chain, two device frames each way, several graphs)
    returns for every frame what run_host returns for it alone; five distinct
    frames so both staging slots are reused."""
    from cpipe_b200 import surrogate as S
    kw = dict(width=320, height=288)
    if mode == "surrogate":
        kw.update(denoise="surrogate", surrogate_blob=S.load_weights())
    chain = Chain(ChainConfig.full_12mp(**kw))
    raw0 = chain.config.make_raw()
    raws = [np.ascontiguousarray(np.roll(raw0, (2 * k, 4 * k), axis=(0, 1))) for k in range(5)]
    want = [chain.run_host(r) for r in raws]
    got = chain.run_host_frames(raws)
    for k in range(5):
        if mode == "reference":
            np.testing.assert_array_equal(got[k].view(np.uint16), want[k].view(np.uint16), err_msg=f"frame {k}")
        else:  # a spot-check fallback would add BM3D, whose last bits vary between runs
            np.testing.assert_allclose(got[k].astype(np.float32), want[k].astype(np.float32), rtol=2e-3, atol=2e-3,
                                       err_msg=f"frame {k}")
    chain.close()


@pytest.mark.parametrize("kw", [dict(guided_spec=True, atrous_levels=5),
                                dict(guided_spec=True, guided_radius=3, atrous_levels=0, wavelet_strength=1.0),
                                dict(guided_spec=False, atrous_levels=4, denoise="bm3d")])
def test_chain_spec_denoisers_equal_nodes(host, kw):
    """The chain with the spec-mode guided filter and/or the a-trous wavelet
    stages returns, bit for bit, what the nodes with algorithm = "spec" /
    "atrous" return one by one (the stages run as their own kernels between
    the denoiser and the tone kernel)."""
    base = dict(width=160, height=112)
    base.update(kw)
    cfg = ChainConfig.full_12mp(**base)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    chain.close()
    want = run_nodes_on_gpu(host, cfg, raw)
    if cfg.denoise == "bm3d":  # BM3D's aggregation order on the GPU is not fixed
        p = psnr(got[..., :3].astype(np.float64), want[..., :3].astype(np.float64))
        assert p >= 60.0, p
    else:
        np.testing.assert_array_equal(got.view(np.uint16), want.view(np.uint16))


def test_chain_spec_stage_refusals(cuda_device):
    with pytest.raises(Exception):
        Chain(ChainConfig.full_12mp(width=64, height=64, guided_spec=True, guided_radius=17))
    with pytest.raises(Exception):
        Chain(ChainConfig.full_12mp(width=64, height=64, atrous_levels=7))


@pytest.mark.parametrize("kw", [dict(sharpen=True), dict(display="sRGB"), dict(sharpen=True, display="sRGB"),
                                dict(sharpen=True, sharpen_radius=2, sharpen_strength=1.4, sharpen_threshold=0.01,
                                     display="BT2020-PQ")])
def test_chain_finishing_stages_equal_nodes(host, kw):
    """sharpen.edge_aware_usm and the display encode as the chain's last stages
    (one fused kernel when both run) return, bit for bit, what the two nodes
    return after the LUT node."""
    cfg = ChainConfig.full_12mp(width=160, height=112, **kw)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    chain.close()
    want = run_nodes_on_gpu(host, cfg, raw)
    assert got.dtype == want.dtype and got.shape == want.shape
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))


def test_chain_finishing_stage_refusals(cuda_device):
    with pytest.raises(Exception):
        Chain(ChainConfig.full_12mp(width=64, height=64, display="sRGB", plain_f32=True))
    with pytest.raises(Exception):
        Chain(ChainConfig.full_12mp(width=64, height=64, sharpen=True, stop_after=1))


@pytest.mark.parametrize("kw", [dict(tone="aces"), dict(tone="reinhard"), dict(tone="reinhard", reinhard_white_point=2.5),
                                dict(tone="aces", sharpen=True, display="sRGB")])
def test_chain_tone_choice_equals_nodes(host, kw):
    """The tone stage with tone.aces_filmic or tone.reinhard in place of filmic
    returns, bit for bit, what those nodes return in the node-by-node chain."""
    cfg = ChainConfig.full_12mp(width=160, height=112, **kw)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    chain.close()
    want = run_nodes_on_gpu(host, cfg, raw)
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))


def test_config1_small_frame_as_configured(cuda_device, host):
    """The plain chain at its configured size: 2016x1512 RGGB 12-bit (black 64,
    white 4095, a=1e-3, b=1e-5), WB gains (2, 1, 1.6), RCD, the camera matrix
    to Rec.2020, denoise.bm3d with sigma from the noise model, filmic and the
    identity+gamma 33^3 LUT; no GainMap, warp or guided filter (the wavelet
    node stays, as the reference loader requires it upstream of filmic).
    The fused chain equals the nodes run one by one bit for bit, and the CPU
    oracle within the RGBA16F tolerance; with the reference's own plain-C++
    filters in the chain (oracle/_ref) the CPU result is the same floats."""
    import oracle_blobs
    from chain_oracle import run_reference_chain
    cfg = ChainConfig.small_frame()
    assert (cfg.width, cfg.height, cfg.bits, cfg.black, cfg.white) == (2016, 1512, 12, 64.0, 4095)
    assert not cfg.gainmap and cfg.warp is None and cfg.guided_radius == 0 and cfg.lut == "identity_gamma"
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    chain.close()
    nodes = run_nodes_on_gpu(host, cfg, raw)
    assert f16_ulp_distance(got, nodes).max() == 0, "fused differs from node-by-node"
    want = run_chain_oracle(cfg, raw)
    assert_f16_parity(got, want, what="config 1 chain vs oracle")
    import oracle as O
    if O.ref_lib() is not None:
        ref = run_reference_chain(cfg, raw, oracle_blobs.chain_blobs(cfg))
        np.testing.assert_array_equal(ref.view(np.uint32), want.view(np.uint32))


def test_config1_small_frame_plain_f32(cuda_device):
    """Config 1 in the FP32 plain form (RGBA f32 between the nodes): max-abs
    <= 1e-4 and PSNR >= 60 dB against the FP32 oracle chain."""
    cfg = ChainConfig.small_frame(plain_f32=True)
    raw = cfg.make_raw()
    chain = Chain(cfg)
    got = chain.run_host(raw)
    chain.close()
    assert got.dtype == np.float32
    assert_f32_parity(got, run_chain_oracle(cfg, raw), what="config 1 chain f32")
