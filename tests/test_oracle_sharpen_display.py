"""CPU checks of the oracles for sharpen.edge_aware_usm and
color.scene_linear_to_display: the USM restatement against the reference's
golden fixture (generated by its own golden generator), the display encode
against the reference unit test's expectations and published values of the
sRGB and SMPTE ST 2084 curves."""
import numpy as np
import oracle
import oracle_display as OD
from conftest import golden


def test_usm_oracle_matches_reference_golden():
    g = golden("sharpen.edge_aware_usm")
    x = g["input"].astype(np.float16).astype(np.float32)
    out = oracle.usm(x, 0.75, 1, 0.0, f16=True)
    np.testing.assert_array_equal(out, g["output"])


def test_usm_oracle_properties():
    r = np.random.default_rng(3)
    x = r.uniform(0.0, 1.0, size=(9, 11, 4)).astype(np.float16).astype(np.float32)
    flat = np.full_like(x, 0.25)
    for radius in (1, 2):
        np.testing.assert_array_equal(oracle.usm(flat, 1.5, radius, 0.0), flat)   # no detail, no change
        np.testing.assert_array_equal(oracle.usm(x, 0.0, radius, 0.0)[..., :3], x[..., :3])  # strength 0
        np.testing.assert_array_equal(oracle.usm(x, 1.0, radius, 10.0)[..., :3], x[..., :3])  # threshold above every mask
        np.testing.assert_array_equal(oracle.usm(x, 2.0, radius, 0.0)[..., 3], x[..., 3])   # alpha passes
    assert (oracle.usm(x, 2.0, 2, 0.0) >= 0.0).all()


def test_display_oracle_reference_unit_test_values():
    srgb = OD.display(np.array([[[0.18, 0.20, 0.22, 1.0], [0.45, 0.30, 0.12, 0.5]]], np.float16).astype(np.float32),
                      "sRGB").reshape(-1)
    assert (srgb[:3] > 0).any() and srgb[3] == 255 and 127 <= srgb[7] <= 128
    pq = OD.display(np.array([[[0.05, 0.18, 0.50, 1.0], [0.90, 0.70, 0.30, 0.5]]], np.float16).astype(np.float32),
                    "BT2020-PQ").reshape(-1)
    assert ((pq & 0x3F) == 0).all() and pq[3] == 1023 << 6 and pq[7] == 512 << 6


def test_display_curves_published_values():
    # sRGB (IEC 61966-2-1 form with the moncurve breakpoint): 0.18 -> 0.4614, continuous at the break
    assert abs(OD.srgb_encode(0.18) - 0.46135) < 1e-4
    assert abs(OD.srgb_encode(OD.LIN_BREAK) - OD.ENC_BREAK) < 1e-12
    assert abs(OD.SLOPE - 1.0 / 12.923) < 1e-4
    # ST 2084: 100 cd/m^2 (linear 1.0 here) -> 0.5081; 0 -> 7.3e-7 (code 0); constants
    assert abs(OD.pq_encode(1.0) - 0.50808) < 1e-4
    assert OD.pq_encode(0.0) < 1e-6
    assert abs(OD.PQ_C1 - 3424.0 / 4096.0) < 1e-15
    # neutral grey stays neutral through the Rec.2020 -> Rec.709 matrix (rows sum to 1)
    assert np.allclose(OD.M_2020_TO_709.sum(1), 1.0, atol=1e-6)
