"""The learned surrogate on the GPU against the CPU oracle
(oracle/oracle_surrogate.py), plus the device scene generator.

* gradients: one training step without update on a small batch (partial
  8x16 tiles included); per layer the GPU weight and bias gradients agree with
  the oracle's (which rounds to bfloat16 where the GPU stores bfloat16) within
  a relative L2 error of 2e-2, the loss within 1e-3;
* forward: the RGBA16F output against the oracle at PSNR >= 60 dB, mean
  relative error <= 2e-4 and max <= 1e-2 (relative to max(1, |value|));
* training: a short run lowers the loss and beats the untrained network;
* serving: the chain's denoise_mode 2 equals the network applied to the
  chain's own denoiser input, bit for bit;
* the committed weights, on pairs from seeds the training never saw, are
  closer to BM3D than the noisy input and the reference's 2x2 blend are.
"""
import ctypes as C
import os

import numpy as np
import oracle_surrogate as O
import pytest
from cpipe_b200 import _abi as A
from cpipe_b200 import surrogate as S
from cpipe_b200.chain import Chain, ChainConfig

pytestmark = pytest.mark.gpu


def upload_f16(x):
    return S.DeviceArray(x.nbytes).upload(np.ascontiguousarray(x, np.float16))


def test_scene_generator_matches_oracle(cuda_device):
    w, h, seed = 301, 77, 0x1234ABCD5678
    d = S.DeviceArray(w * h * 2)
    cfa = (C.c_uint8 * 4)(0, 1, 1, 2)
    for a, b in ((0.0, 0.0), (4e-3, 4e-5)):
        assert A.lib().cpipe_cuda_scene_raw(d.ptr, w, h, C.c_uint64(seed), 10, 16, a, b, cfa, 20, None) == 0
        got = d.download((h, w), np.uint16).astype(np.int64)
        want, _ = O.scene_raw(w, h, seed, 10, 16, a, b)
        diff = np.abs(got - want.astype(np.int64))
        assert diff.max() <= 1 and np.mean(diff > 0) < 1e-3, (a, b, diff.max(), np.mean(diff > 0))
    d.free()


def small_problem(seed=0, n=2, h=12, w=20):
    rng = np.random.default_rng(seed)
    rgba = rng.uniform(0.02, 0.95, (n, h, w, 4)).astype(np.float16)
    tgt = np.clip(rgba.astype(np.float32) + rng.normal(0, 0.03, rgba.shape), 0, 1).astype(np.float16)
    ab = np.array([(4e-3, 4e-5), (1e-3, 1e-5)][:n], np.float32)
    params = [(W, (b + rng.normal(0, 0.02, b.shape)).astype(np.float32)) for W, b in S.init_params(seed + 5)]
    params[-1] = (params[-1][0] * 10.0, params[-1][1])  # a last layer of full strength
    return rgba, tgt, ab, params


def test_gradients_match_oracle(cuda_device):
    rgba, tgt, ab, params = small_problem()
    n, h, w = rgba.shape[:3]
    sg = S.Surrogate(S.to_blob(params))
    dn, dt = upload_f16(rgba), upload_f16(tgt)
    loss = sg.train_step(dn.ptr, dt.ptr, ab, n, w, h, 0.0, update=False)
    grads = sg.gradients()
    want_loss, want = O.loss_and_grads(params, rgba.astype(np.float32), tgt.astype(np.float32), ab, bf=True)
    assert abs(loss - want_loss) <= 1e-3 * want_loss, (loss, want_loss)
    for l, ((gw, gb), (ow, ob)) in enumerate(zip(grads, want)):
        ew = np.linalg.norm(gw - ow) / np.linalg.norm(ow)
        eb = np.linalg.norm(gb - ob) / max(np.linalg.norm(ob), 1e-30)
        print(f"layer {l}: weight grad rel L2 {ew:.2e}, bias grad rel L2 {eb:.2e}")
        assert ew < 2e-2 and eb < 2e-2, (l, ew, eb)
    sg.close()


def test_forward_matches_oracle(cuda_device):
    rgba, _, ab, params = small_problem(1, n=2, h=19, w=35)
    n, h, w = rgba.shape[:3]
    sg = S.Surrogate(S.to_blob(params))
    din, dout = upload_f16(rgba), S.DeviceArray(rgba.nbytes)
    sg.denoise(din.ptr, dout.ptr, n, w, h, ab)
    got = dout.download(rgba.shape, np.float16).astype(np.float32)
    want, _ = O.forward(params, rgba.astype(np.float32), ab, bf=True)
    # The GPU accumulates in FP32 (mma order) and the oracle in FP64 before
    # each bfloat16 store, so an activation on a bfloat16 rounding boundary can
    # land one bfloat16 ulp apart and move the output by a few binary16 ulps.
    d = np.abs(got[..., :3] - want) / np.maximum(1.0, np.abs(want))
    p = 10.0 * np.log10(np.max(np.abs(want)) ** 2 / np.mean((got[..., :3] - want) ** 2))
    print(f"forward: max relative error {d.max():.2e}, mean {d.mean():.2e}, PSNR {p:.1f} dB")
    assert d.max() <= 1e-2 and d.mean() <= 2e-4 and p >= 60.0
    np.testing.assert_array_equal(got[..., 3], rgba[..., 3].astype(np.float32))
    sg.close()


def test_short_training_reduces_loss(cuda_device):
    rng = np.random.default_rng(2)
    gen = S.PairGenerator(tile=64, per_frame=8, seed=777)
    noisy, target, ab = gen.dataset(96, rng)
    gen.close()
    sg = S.Surrogate(S.to_blob(S.init_params(2)))
    tb = 64 * 64 * 8
    before = S.evaluate(sg, noisy, target, ab, 64, 32, tile=64)
    first = sg.train_step(noisy.ptr, target.ptr, ab[:16], 16, 64, 64, 0.0, update=False)
    for step in range(300):
        s = (step * 16) % 64
        sg.train_step(noisy.at(s * tb), target.at(s * tb), ab[s:s + 16], 16, 64, 64, 2e-3, update=True,
                      want_loss=False)
    last = sg.train_step(noisy.ptr, target.ptr, ab[:16], 16, 64, 64, 0.0, update=False)
    after = S.evaluate(sg, noisy, target, ab, 64, 32, tile=64)
    print(f"loss {first:.3e} -> {last:.3e}; held out before {before} after {after}")
    assert last < 0.5 * first
    assert after["surrogate"] > before["surrogate"] + 3.0
    sg.close()


def test_chain_surrogate_mode_equals_network_on_chain_input(cuda_device):
    blob = S.to_blob(S.init_params(4))
    base = dict(width=96, height=64, surrogate_blob=blob, spot_tiles=0)
    front = Chain(ChainConfig.full_12mp(stop_after=1, **base))
    mid = Chain(ChainConfig.full_12mp(denoise="surrogate", stop_after=2, **base))
    full = Chain(ChainConfig.full_12mp(denoise="surrogate", **base))
    cfg = front.config
    raw = cfg.make_raw()
    x = front.run_host(raw)
    y = mid.run_host(raw)
    sg = S.Surrogate(blob)
    din, dout = upload_f16(x), S.DeviceArray(x.nbytes)
    sg.denoise(din.ptr, dout.ptr, 1, 96, 64, [(cfg.noise_a, cfg.noise_b)])
    want = dout.download(x.shape, np.float16)
    np.testing.assert_array_equal(y.view(np.uint16), want.view(np.uint16))
    out = full.run_host(raw)
    assert np.isfinite(out.astype(np.float32)).all()
    for c in (front, mid, full):
        c.close()


@pytest.mark.skipif(not os.path.exists(S.DEFAULT_WEIGHTS), reason="no trained weights committed")
def test_trained_weights_gain_over_no_network(cuda_device):
    """The committed network against what the chain has without it, on fresh
    pairs (seeds the training did not use), all measured against BM3D."""
    rng = np.random.default_rng(99)
    gen = S.PairGenerator(tile=256, per_frame=8, seed=0x7E570000)
    noisy, target, ab = gen.dataset(32, rng)
    gen.close()
    sg = S.Surrogate(S.load_weights())
    r = S.evaluate(sg, noisy, target, ab, 0, 32)
    print(f"PSNR vs BM3D: surrogate {r['surrogate']:.2f} dB, noisy {r['noisy']:.2f} dB, box2x2 {r['box2x2']:.2f} dB")
    assert r["surrogate"] >= 40.0
    assert r["surrogate"] > r["noisy"] + 6.0 and r["surrogate"] > r["box2x2"] + 3.0
    sg.close()


def spot_chain(blob, min_psnr, **kw):
    return Chain(ChainConfig.full_12mp(width=320, height=288, surrogate_blob=blob, denoise="surrogate",
                                       spot_tiles=16, spot_min_psnr_db=min_psnr, **kw))


def test_spot_check_passes_and_keeps_the_network_output(cuda_device):
    """A threshold of 0 dB never falls back: the output is the network's, bit
    for bit, and the counters record one checked frame."""
    blob = S.to_blob(S.init_params(6))
    raw = ChainConfig.full_12mp(width=320, height=288).make_raw()
    plain = Chain(ChainConfig.full_12mp(width=320, height=288, surrogate_blob=blob, denoise="surrogate",
                                        spot_tiles=0, stop_after=2))
    checked = spot_chain(blob, 0.0, stop_after=2)
    a, b = plain.run_host(raw), checked.run_host(raw)
    np.testing.assert_array_equal(a.view(np.uint16), b.view(np.uint16))
    frames, fallbacks, worst = checked.denoise_stats()
    assert (frames, fallbacks) == (1, 0) and np.isfinite(worst)
    plain.close()
    checked.close()


def test_spot_check_falls_back_to_bm3d(cuda_device):
    """An unreachable threshold makes every frame fall back: the denoiser's
    output is then the two-stage BM3D of the frame (its aggregation order on
    the GPU is not fixed, hence a PSNR bound)."""
    blob = S.to_blob(S.init_params(6))
    raw = ChainConfig.full_12mp(width=320, height=288).make_raw()
    checked = spot_chain(blob, 300.0, stop_after=2)
    bm3d = Chain(ChainConfig.full_12mp(width=320, height=288, denoise="bm3d", stop_after=2))
    for _ in range(2):
        got = checked.run_host(raw).astype(np.float32)
    want = bm3d.run_host(raw).astype(np.float32)
    p = 10 * np.log10(1.0 / np.mean((got[..., :3] - want[..., :3]) ** 2))
    print(f"fallback vs BM3D chain: {p:.1f} dB")
    assert p >= 60.0
    assert checked.denoise_stats()[:2] == (2, 2)
    checked.close()
    bm3d.close()


@pytest.mark.skipif(not os.path.exists(S.DEFAULT_WEIGHTS), reason="no trained weights committed")
def test_trained_surrogate_passes_spot_check_at_12mp(cuda_device):
    """The committed network on the 4032x3024 benchmark frame: every sampled
    tile is within 40 dB of BM3D, so the chain keeps the network's output."""
    chain = Chain(ChainConfig.full_12mp(denoise="surrogate", surrogate_blob=S.load_weights()))
    raw = chain.config.make_raw()
    out = chain.run_host(raw)
    frames, fallbacks, worst = chain.denoise_stats()
    print(f"12 MP spot check: {frames} frame, {fallbacks} fallbacks, worst tile {worst:.2f} dB")
    assert frames == 1 and fallbacks == 0 and worst >= 40.0
    assert np.isfinite(out.astype(np.float32)).all()
    chain.close()


def test_trained_surrogate_passes_spot_check_at_50mp_quad_bayer(cuda_device):
    """The committed network on an 8160x6120 Sony Quad-Bayer frame (remosaiced
    ahead of the chain, scene made on the device): two frames, every sampled
    tile within 40 dB of BM3D."""
    from cpipe_b200 import batch as B
    cfg = ChainConfig.qbc_50mp(denoise="surrogate", surrogate_blob=S.load_weights())
    L = A.lib()
    d_raw, d_out = C.c_void_p(), C.c_void_p()
    assert L.cpipe_cuda_device_alloc(cfg.width * cfg.height * 2, C.byref(d_raw)) == 0
    assert L.cpipe_cuda_device_alloc(cfg.width * cfg.height * 8, C.byref(d_out)) == 0
    B.scene_raw(d_raw.value, cfg, "qbc")
    chain = Chain(cfg)
    for _ in range(2):
        chain.run(d_raw.value, d_out.value)
    assert L.cpipe_cuda_synchronize() == 0
    frames, fallbacks, worst = chain.denoise_stats()
    print(f"50 MP Quad-Bayer spot check: {frames} frames, {fallbacks} fallbacks, worst tile {worst:.2f} dB")
    assert frames == 2 and fallbacks == 0 and worst >= 40.0
    chain.close()
    L.cpipe_cuda_device_free(d_raw)
    L.cpipe_cuda_device_free(d_out)
