"""The surrogate's tcgen05 inference kernels (cpipe_b200/csrc/surrogate_tc.cu)
against its mma.sync kernels and the CPU oracle.

Both engines take the same BF16 operands and accumulate in FP32; they differ
in the order of the FP32 sums, so an activation on a bfloat16 rounding
boundary can land one bfloat16 ulp apart (in practice the two engines have
agreed bit for bit: both reduce each 16-wide K slice the same way).  Bounds:
PSNR >= 60 dB between the engines and against the oracle (rounded to binary16
like the frames), mean relative error <= 2e-4 between the engines and <= 5e-4
against the oracle (these random networks with a strong last layer amplify the
bfloat16 rounding flips), max <= 1e-2 (relative to max(1, |value|)); alpha
bit-exact; and no bounded wait inside the tcgen05
pipeline ran out (cpipe_surrogate_check)."""
import numpy as np
import oracle_surrogate as O
import os
import pytest
from cpipe_b200 import surrogate as S

pytestmark = pytest.mark.gpu


def close(got, want, what, mean_bound=2e-4):
    d = np.abs(got - want) / np.maximum(1.0, np.abs(want))
    p = 10.0 * np.log10(max(1.0, float(np.max(np.abs(want)))) ** 2 / max(float(np.mean((got - want) ** 2)), 1e-30))
    print(f"{what}: max rel {d.max():.2e}, mean {d.mean():.2e}, PSNR {p:.1f} dB")
    assert d.max() <= 1e-2 and d.mean() <= mean_bound and p >= 60.0, what


def run(sg, engine, x, ab, f16=True):
    n, h, w = x.shape[:3]
    din = S.DeviceArray(x.nbytes).upload(x)
    dout = S.DeviceArray(x.nbytes)
    sg.set_engine(engine)
    sg.denoise(din.ptr, dout.ptr, n, w, h, ab, f16=f16)
    sg.check()
    return dout.download(x.shape, x.dtype).astype(np.float32)


@pytest.mark.parametrize("n,h,w", [(2, 19, 35), (1, 64, 64), (1, 33, 130), (3, 16, 8), (1, 1, 1)])
def test_tcgen05_matches_mma_and_oracle(cuda_device, n, h, w):
    rng = np.random.default_rng(n * 1000 + h * 10 + w)
    x = rng.uniform(0.02, 0.95, (n, h, w, 4)).astype(np.float16)
    ab = np.array([(4e-3, 4e-5), (1e-3, 1e-5), (8e-3, 9e-5)][:n], np.float32)
    params = [(W, (b + rng.normal(0, 0.02, b.shape)).astype(np.float32)) for W, b in S.init_params(n + h)]
    params[-1] = (params[-1][0] * 10.0, params[-1][1])
    sg = S.Surrogate(S.to_blob(params))
    tc = run(sg, "tcgen05", x, ab)
    mma = run(sg, "mma", x, ab)
    np.testing.assert_array_equal(tc[..., 3], x[..., 3].astype(np.float32))
    close(tc[..., :3], mma[..., :3], f"tcgen05 vs mma {n}x{h}x{w}")
    want, _ = O.forward(params, x.astype(np.float32), ab, bf=True)
    want = want.astype(np.float16).astype(np.float64)  # the frames are binary16
    close(tc[..., :3], want, f"tcgen05 vs oracle {n}x{h}x{w}", mean_bound=5e-4)
    sg.close()


def test_tcgen05_float32_frames(cuda_device):
    rng = np.random.default_rng(7)
    x = rng.uniform(0.02, 0.95, (1, 24, 40, 4)).astype(np.float32)
    sg = S.Surrogate(S.to_blob(S.init_params(7)))
    tc = run(sg, "tcgen05", x, [(4e-3, 4e-5)], f16=False)
    mma = run(sg, "mma", x, [(4e-3, 4e-5)], f16=False)
    close(tc[..., :3], mma[..., :3], "f32 frames")
    np.testing.assert_array_equal(tc[..., 3], x[..., 3])
    sg.close()


@pytest.mark.skipif(not os.path.exists(S.DEFAULT_WEIGHTS), reason="no trained weights committed")
def test_tcgen05_trained_network_12mp(cuda_device):
    from cpipe_b200.chain import Chain, ChainConfig
    front = Chain(ChainConfig.full_12mp(stop_after=1))
    cfg = front.config
    x = front.run_host(cfg.make_raw())[None]
    front.close()
    sg = S.Surrogate(S.load_weights())
    ab = [(cfg.noise_a, cfg.noise_b)]
    tc = run(sg, "tcgen05", x, ab)
    mma = run(sg, "mma", x, ab)
    close(tc[..., :3], mma[..., :3], "12 MP trained network")
    sg.close()
