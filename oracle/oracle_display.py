"""FP64 restatement of the color.scene_linear_to_display encode.

TEST INFRASTRUCTURE: imported only by tests/ as the checker.  The product
library never loads it.

The reference node (src/cpipe/nodes/color/scene_linear_to_display.cpp:31-127)
runs an OpenColorIO CPU processor built from its config
(share/cpipe/ocio/v0.2/config.ocio:57-79) on the host, then quantises
(src/cpipe/runtime/HostContext.cpp:91-99, 155-185).  OpenColorIO (vcpkg
dependency `opencolorio`, absent from the reference tree) is not available
here, so its published transform definitions are restated:

  output_srgb       : MatrixTransform (the config's Rec.2020 -> Rec.709 matrix),
                      ExponentWithLinearTransform gamma 2.4 offset 0.055,
                      direction inverse (the "moncurve": e = L / slope below the
                      linear breakpoint, else (1 + o) L^(1/g) - o), then
                      RangeTransform [0, 1] -> [0, 1] (a clamp).  Alpha passes.
  output_pq_rec2020 : RangeTransform [0, 1], then FixedFunctionTransform
                      LIN_TO_PQ (SMPTE ST 2084 with linear 1.0 = 100 cd/m^2).
                      Alpha passes.

Quantisation: sRGB -> round-half-away(clamp(v, 0, 1) * 255) (R8G8B8A8_UNORM);
PQ -> round-half-away(clamp(v, 0, 1) * 1023) << 6 (R16G16B16A16_UNORM).

Pins: the reference's unit test (tests/unit/test_node_color_scene_linear_to_display.cpp:
alpha 1.0 -> 255 / 1023 << 6, alpha 0.5 -> 127..128 / 512 << 6, PQ low six
bits zero).  The colour values are unpinned against OpenColorIO itself
(whose CPU path may use fast power approximations); the tests hold the GPU
to one code value of this FP64 restatement.
"""
import numpy as np

M_2020_TO_709 = np.array([[1.6604910, -0.5876411, -0.0728499],
                          [-0.1245505, 1.1328999, -0.0083494],
                          [-0.0181508, -0.1005789, 1.1187297]])
GAMMA, OFFSET = 2.4, 0.055
ENC_BREAK = OFFSET / (GAMMA - 1.0)
LIN_BREAK = (OFFSET * GAMMA / ((GAMMA - 1.0) * (1.0 + OFFSET))) ** GAMMA
SLOPE = LIN_BREAK / ENC_BREAK
PQ_M1 = 2610.0 / 16384.0
PQ_M2 = 2523.0 / 4096.0 * 128.0
PQ_C2 = 2413.0 / 4096.0 * 32.0
PQ_C3 = 2392.0 / 4096.0 * 32.0
PQ_C1 = PQ_C3 - PQ_C2 + 1.0


def srgb_encode(lin):
    lin = np.asarray(lin, np.float64)
    hi = (1.0 + OFFSET) * np.power(np.maximum(lin, LIN_BREAK), 1.0 / GAMMA) - OFFSET
    return np.where(lin <= LIN_BREAK, lin / SLOPE, hi)


def pq_encode(v):
    v = np.clip(np.asarray(v, np.float64), 0.0, 1.0) * 0.01
    y = np.power(v, PQ_M1)
    return np.power((PQ_C1 + PQ_C2 * y) / (1.0 + PQ_C3 * y), PQ_M2)


def _round_half_away(x):
    return np.floor(x + 0.5)  # x >= 0 after the clamp


def encode_float(x, target):
    """Encoded values before quantisation: HxWx4 float64."""
    x = np.asarray(x, np.float64)
    out = np.empty_like(x)
    if target == "sRGB":
        rgb = x[..., :3] @ M_2020_TO_709.T
        out[..., :3] = np.clip(srgb_encode(rgb), 0.0, 1.0)
    elif target == "BT2020-PQ":
        out[..., :3] = pq_encode(x[..., :3])
    else:
        raise ValueError(target)
    out[..., 3] = x[..., 3]
    return out


def display(x, target):
    """uint8 HxWx4 (sRGB) or uint16 HxWx4 (BT2020-PQ, 10-bit codes << 6) from
    RGBA input values (the f16 input buffer's values)."""
    e = np.clip(encode_float(x, target), 0.0, 1.0)
    if target == "sRGB":
        return _round_half_away(e * 255.0).astype(np.uint8)
    return (_round_half_away(e * 1023.0).astype(np.uint16) << 6).astype(np.uint16)
