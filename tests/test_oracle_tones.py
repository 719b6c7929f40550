"""CPU checks of the tone.aces_filmic and tone.reinhard oracles against the
reference's golden fixtures (written by its own golden generator)."""
import numpy as np
import oracle
from conftest import golden


def test_aces_oracle_matches_reference_golden():
    g = golden("tone.aces_filmic")
    x = g["input"].astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(oracle.aces(x, True), g["output"])
    np.testing.assert_array_equal(oracle.aces(x, False), x)  # toggle off passes every channel


def test_reinhard_oracle_matches_reference_golden():
    g = golden("tone.reinhard")
    x = g["input"].astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(oracle.reinhard(x, 1000000.0), g["output"])
    y = oracle.reinhard(x, 0.1)  # a low white point saturates early
    assert (y[..., :3] >= oracle.reinhard(x, 1000000.0)[..., :3]).all() and (y <= 1.0).all()


def test_greyworld_oracle_matches_reference_golden():
    g = golden("wb.greyworld_auto")
    n, out = oracle.greyworld(g["input"])
    np.testing.assert_array_equal(out, g["output"])
    assert n[1] == 1.0
    assert oracle.greyworld(np.zeros((2, 2, 4), np.float32)) == (None, None)


def test_mertens_oracle_matches_reference_golden():
    """The golden generator multiplies the three weight factors in another
    association than the Halide generator the oracle follows: within one f16 ulp."""
    from parity import assert_f16_parity
    g = golden("tone.mertens_local")
    u, n, o = (g[k].astype(np.float16).astype(np.float32) for k in ("under", "normal", "over"))
    out = oracle.mertens(u, n, o)
    assert_f16_parity(out, g["output"], what="mertens golden")
