"""CPU checks of the surrogate's oracle (oracle/oracle_surrogate.py) and of the
weight-blob format: the oracle's backward pass against finite differences,
bfloat16 rounding against torch, the Philox4x32-10 restatement against the
published known-answer vectors (Salmon et al., SC 2011; Random123 kat_vectors),
and the blob layout against the library's size."""
import numpy as np
import oracle_surrogate as O
import pytest
import torch
from cpipe_b200 import _abi as A
from cpipe_b200 import surrogate as S


def test_blob_round_trip_and_library_size():
    p = S.init_params(3)
    blob = S.to_blob(p)
    assert len(blob) == A.lib().cpipe_surrogate_blob_size()
    for (w0, b0), (w1, b1) in zip(p, S.from_blob(blob)):
        assert np.array_equal(w0, w1) and np.array_equal(b0, b1)
    with pytest.raises(ValueError):
        S.from_blob(b"XXXX" + blob[4:])


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(0).normal(0, 3, 10000).astype(np.float32)
    x[:4] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -0.0, 65504.0]  # ties to even
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(O.bf16(x), want)


@pytest.mark.parametrize("counter,key,want", [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
])
def test_philox_known_answers(counter, key, want):
    assert tuple(int(v) for v in O.philox(*counter, *key)) == want


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    rgba = rng.uniform(0, 1, (2, 5, 7, 4)).astype(np.float32)
    tgt = rng.uniform(0, 1, (2, 5, 7, 4)).astype(np.float32)
    ab = [(4e-3, 4e-5), (1e-3, 1e-5)]
    params = [(W.astype(np.float64), b.astype(np.float64) + rng.normal(0, 0.01, b.shape)) for W, b in S.init_params(1)]
    _, grads = O.loss_and_grads(params, rgba, tgt, ab, bf=False)

    def loss_with(l, which, idx, delta):
        q = [(W.copy(), b.copy()) for W, b in params]
        q[l][which][idx] += delta
        return O.loss_and_grads(q, rgba, tgt, ab, bf=False)[0]

    for l, which, idx in [(0, 0, (3, 1, 0, 2)), (3, 0, (5, 7, 1, 1)), (7, 0, (2, 30, 2, 0)), (2, 1, (4,)),
                          (7, 1, (1,))]:
        fd = (loss_with(l, which, idx, 1e-6) - loss_with(l, which, idx, -1e-6)) / 2e-6
        np.testing.assert_allclose(grads[l][which][idx], fd, rtol=1e-5, atol=1e-12)


def test_scene_oracle_is_seeded_and_in_range():
    r1, c1 = O.scene_raw(48, 40, 7)
    r2, _ = O.scene_raw(48, 40, 7)
    r3, _ = O.scene_raw(48, 40, 8)
    assert np.array_equal(r1, r2) and not np.array_equal(r1, r3)
    assert r1.min() >= 0 and r1.max() <= 1023 and 0.0 <= c1.min() and c1.max() <= 1.0
