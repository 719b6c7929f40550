"""The batched form (cpipe_cuda_batch_*): frames of uneven size, CFA (RGGB,
BGGR, Quad Bayer), bit depth and noise in one launch per stage.  Each frame's
output must equal, bit for bit, the same frame through its own single-frame
chain (the kernels compute the same tiles with the same parameters), before and
after the autotuner changes the persistent grid sizes, and on a second run
(graph replay)."""
import ctypes as C

import numpy as np
import pytest
from chain_oracle import run_chain_oracle
from cpipe_b200 import _abi as A
from cpipe_b200 import batch as B
from cpipe_b200.chain import Chain
from parity import assert_f16_parity

pytestmark = pytest.mark.gpu


def alloc(nbytes):
    p = C.c_void_p()
    assert A.lib().cpipe_cuda_device_alloc(nbytes, C.byref(p)) == 0
    return p.value


def download(ptr, shape, dtype):
    out = np.empty(shape, dtype)
    assert A.lib().cpipe_cuda_synchronize() == 0
    assert A.lib().cpipe_cuda_memcpy_d2h(out.ctypes.data, C.c_void_p(ptr), out.nbytes) == 0
    return out


def test_batch_equals_single_frame_chains(cuda_device):
    frames = B.workload(7, seed=99, mp_range=(0.004, 0.08))
    L = A.lib()
    d_raw = [alloc(c.width * c.height * 2) for c, _ in frames]
    d_out = [alloc(c.width * c.height * 8) for c, _ in frames]
    for p, (c, k) in zip(d_raw, frames):
        B.scene_raw(p, c, k)
    batch = B.Batch([c for c, _ in frames])
    want = []
    for i, (c, _) in enumerate(frames):
        ch = Chain(c)
        ref = alloc(c.width * c.height * 8)
        ch.run(d_raw[i], ref)
        want.append(download(ref, (c.height, c.width, 4), np.float16))
        L.cpipe_cuda_device_free(C.c_void_p(ref))
        ch.close()
    for step in range(3):
        if step == 1:
            print("autotuned CTAs per SM:", batch.autotune(d_raw, d_out))
        batch.run(d_raw, d_out)
        for i, (c, k) in enumerate(frames):
            got = download(d_out[i], (c.height, c.width, 4), np.float16)
            np.testing.assert_array_equal(got.view(np.uint16), want[i].view(np.uint16), err_msg=f"{k} {c.name} run {step}")
    batch.close()
    for p in d_raw + d_out:
        L.cpipe_cuda_device_free(C.c_void_p(p))


def test_batch_frame_matches_oracle(cuda_device):
    """One Quad-Bayer and one BGGR frame of a batch against the CPU oracle chain."""
    frames = B.workload(6, seed=7, mp_range=(0.004, 0.02))
    picks = [i for i, (_, k) in enumerate(frames) if k in ("qbc", "bggr")][:2]
    d_raw = [alloc(c.width * c.height * 2) for c, _ in frames]
    d_out = [alloc(c.width * c.height * 8) for c, _ in frames]
    for p, (c, k) in zip(d_raw, frames):
        B.scene_raw(p, c, k)
    batch = B.Batch([c for c, _ in frames])
    batch.run(d_raw, d_out)
    for i in picks:
        c, k = frames[i]
        raw = download(d_raw[i], (c.height, c.width), np.uint16)
        got = download(d_out[i], (c.height, c.width, 4), np.float16)
        assert_f16_parity(got, run_chain_oracle(c, raw), what=f"batch frame {k}")
    batch.close()
    for p in d_raw + d_out:
        A.lib().cpipe_cuda_device_free(C.c_void_p(p))


def test_batch_refuses_mixed_chains(cuda_device):
    frames = B.workload(2, seed=3, mp_range=(0.004, 0.01))
    cfgs = [frames[0][0], frames[1][0]]
    cfgs[1].demosaic = "amaze"
    with pytest.raises(Exception):
        B.Batch(cfgs)


def test_batch_quad_bayer_and_14bit_frames_match_oracle(cuda_device):
    """Frames of the mix the oracle comparison above may not draw: a
    Quad-Bayer frame and a 14-bit frame, each against the CPU oracle chain."""
    frames = B.workload(24, seed=21, mp_range=(0.004, 0.02))
    picks = []
    for want in (lambda c, k: k == "qbc", lambda c, k: c.bits == 14):
        picks.append(next(i for i, (c, k) in enumerate(frames) if want(c, k) and i not in picks))
    sub = [frames[i] for i in picks]
    d_raw = [alloc(c.width * c.height * 2) for c, _ in sub]
    d_out = [alloc(c.width * c.height * 8) for c, _ in sub]
    for p, (c, k) in zip(d_raw, sub):
        B.scene_raw(p, c, k)
    batch = B.Batch([c for c, _ in sub])
    batch.run(d_raw, d_out)
    for i, (c, k) in enumerate(sub):
        raw = download(d_raw[i], (c.height, c.width), np.uint16)
        got = download(d_out[i], (c.height, c.width, 4), np.float16)
        assert_f16_parity(got, run_chain_oracle(c, raw), what=f"batch frame {k} {c.bits}-bit")
    batch.close()
    for p in d_raw + d_out:
        A.lib().cpipe_cuda_device_free(C.c_void_p(p))


def test_batch_with_the_network_in_the_denoiser_slot(cuda_device):
    """The network and its BM3D spot check between the second and third
    stages: each frame equals its own single-frame surrogate chain (within the
    tolerance of a possible BM3D fallback), before and after the autotuner; the
    frames' completion times inside the launch are ordered and within the run."""
    from cpipe_b200 import surrogate as S
    weights = S.load_weights()
    frames = B.workload(4, seed=5, mp_range=(0.07, 0.3), denoise="surrogate", surrogate_blob=weights)
    L = A.lib()
    d_raw = [alloc(c.width * c.height * 2) for c, _ in frames]
    d_out = [alloc(c.width * c.height * 8) for c, _ in frames]
    for p, (c, k) in zip(d_raw, frames):
        B.scene_raw(p, c, k)
    want = []
    for i, (c, _) in enumerate(frames):
        ch = Chain(c)
        ref = alloc(c.width * c.height * 8)
        ch.run(d_raw[i], ref)
        want.append(download(ref, (c.height, c.width, 4), np.float16).astype(np.float32))
        L.cpipe_cuda_device_free(C.c_void_p(ref))
        ch.close()
    batch = B.Batch([c for c, _ in frames])
    for step in range(2):
        if step == 1:
            per_sm, rows = batch.autotune(d_raw, d_out), batch.schedule()[1]
            assert rows in (4, 8, 16, 32)
        batch.run(d_raw, d_out)
        times = batch.frame_times()
        assert all(t > 0 for t in times)
        for i, (c, k) in enumerate(frames):
            got = download(d_out[i], (c.height, c.width, 4), np.float16).astype(np.float32)
            np.testing.assert_allclose(got, want[i], rtol=2e-3, atol=2e-3, err_msg=f"{k} {c.name} run {step}")
    batch.close()
    for p in d_raw + d_out:
        L.cpipe_cuda_device_free(C.c_void_p(p))


def test_batch_frame_times_cover_the_run(cuda_device):
    frames = B.workload(5, seed=17, mp_range=(0.01, 0.05))
    d_raw = [alloc(c.width * c.height * 2) for c, _ in frames]
    d_out = [alloc(c.width * c.height * 8) for c, _ in frames]
    for p, (c, k) in zip(d_raw, frames):
        B.scene_raw(p, c, k)
    batch = B.Batch([c for c, _ in frames])
    batch.run(d_raw, d_out)
    t = batch.frame_times()
    assert len(t) == 5 and all(0.0 < x < 1000.0 for x in t)
    batch.close()
    for p in d_raw + d_out:
        A.lib().cpipe_cuda_device_free(C.c_void_p(p))
