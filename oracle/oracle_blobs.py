"""Filter parameter blobs of the classic chain, made without the product library.

TEST INFRASTRUCTURE: used by the CPU legs of bench.py (the reference arm and
the CPU baseline), which must not load libcpipe_b200.so, and by the tests that
check these blobs against the library's own host preparation byte for byte.

Each blob restates a reference POD layout with explicit `struct` formats
(little-endian, the reference's natural alignment written out as padding):

  BlacklevelParams       detail/P1ParamDispatch.hpp:14-18
  WbParams               detail/P1ParamDispatch.hpp:24-29
  ColormatrixParams      detail/P1ParamDispatch.hpp:31-33
  GainMapDispatch*       detail/P1ParamDispatch.hpp:35-56, packed as
                         lens/shading_gainmap.cpp:96-137 packs them
  Opcode3Dispatch*       detail/P1ParamDispatch.hpp:58-94, packed as
                         lens/dng_opcode_list_3.cpp:75-168 packs a
                         WarpRectilinear

The white-balance matrix blend and CCT come from the reference's own helpers
(wb/WbMetadata.hpp interpolate_calibration) compiled into oracle/_ref; the
colour-matrix composition restates colormatrix_dng_to_working.cpp:20-28,53-65,125
in binary32 with the reference's operation order.
"""
import struct

import numpy as np

import oracle

_F = np.float32

# colormatrix_dng_to_working.cpp:20-28
D50_TO_D65 = (0.9555766, -0.0230393, 0.0631636, -0.0282895, 1.0099416, 0.0210077, 0.0122982, -0.0204830, 1.3299098)
XYZ_D65_TO_REC2020 = (1.7166512, -0.3556708, -0.2533663, -0.6666844, 1.6164812, 0.0157685, 0.0176399, -0.0427706,
                      0.9421031)


def blacklevel(black4, white, cfa4):
    return struct.pack("<4fI4B", *[float(v) for v in black4], int(white), *cfa4)


def wb(neutral, camera_to_xyz, cct, weight):
    return struct.pack("<3f9fff", *[float(v) for v in neutral], *[float(v) for v in camera_to_xyz], float(cct),
                       float(weight))


def colormatrix(t9):
    return struct.pack("<9f", *[float(v) for v in t9])


def _mul3(a, b):
    """colormatrix_dng_to_working.cpp:53-65: row-major 3x3 product in binary32,
    each element ((a0*b0 + a1*b3) + a2*b6) without fused multiply-add."""
    a = [_F(v) for v in a]
    b = [_F(v) for v in b]
    out = []
    for r in range(3):
        for c in range(3):
            out.append(_F(_F(_F(a[3 * r] * b[c]) + _F(a[3 * r + 1] * b[3 + c])) + _F(a[3 * r + 2] * b[6 + c])))
    return out


def colormatrix_compose(camera_to_xyz_d50):
    """colormatrix_dng_to_working.cpp:125: XYZ(D65)->Rec.2020 * (D50->D65 * camera->XYZ(D50))."""
    return [float(v) for v in _mul3(XYZ_D65_TO_REC2020, _mul3(D50_TO_D65, camera_to_xyz_d50))]


def gainmap_single(points_v, points_h, spacing_v, spacing_h, gains, bottom, right, cfa_repeat=(2, 2),
                   cfa_pattern=(0, 1, 1, 2), origin_v=0.0, origin_h=0.0):
    """One full-frame GainMap plane (plane 0 of 1) as the node packs it."""
    pat = list(cfa_pattern) + [0] * (16 - len(cfa_pattern))
    g = np.ascontiguousarray(gains, dtype="<f4").ravel()
    head = struct.pack("<I2B16B2x", 1, *cfa_repeat, *pat[:16])
    plane = struct.pack("<8I4d2I", 0, 0, int(bottom), int(right), 0, 1, int(points_v), int(points_h),
                        float(spacing_v), float(spacing_h), float(origin_v), float(origin_h), 0, g.size)
    return head + plane + g.tobytes()


def opcode3_warp(coefficients, cx_hat=0.5, cy_hat=0.5, optional=0):
    """One WarpRectilinear (opcode id 1) record, coefficients per plane (1..4)."""
    coeffs = [tuple(float(v) for v in k) for k in coefficients][:4]
    flat = [v for k in coeffs for v in k] + [0.0] * (6 * (4 - len(coeffs)))
    rec = struct.pack("<III4x", 1, int(optional), len(coeffs))
    rec += struct.pack("<24d", *flat) + struct.pack("<2d", float(cx_hat), float(cy_hat))
    rec += struct.pack("<5d2d", 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    rec += struct.pack("<10I", *([0] * 10))
    return struct.pack("<II", 1, 0) + rec


def wb_params(neutral, cm1, cm2, fm1, fm2, illum1=17, illum2=21):
    """WbParams from the reference's own interpolate_calibration (oracle/_ref)."""
    st, m, cct, weight = oracle.ref_wb_interpolate(neutral, cm1, cm2, fm1, fm2, illum1, illum2)
    if st != 0:
        raise RuntimeError(f"reference wb interpolation status {st}")
    return m, cct, weight


def chain_blobs(cfg):
    """The blobs cpipe_b200.chain.ChainConfig.blobs() returns (same keys and
    bytes for the chain's nodes), made from the reference's layouts and
    helpers only.  `cfg` is read for its plain parameters."""
    from cpipe_b200.chain import CAMERA_TO_XYZ, COLOR_MATRIX1, COLOR_MATRIX2, radial_gains
    out = {"blacklevel": blacklevel([cfg.black] * 4, cfg.white, cfg.cfa)}
    if cfg.gainmap:
        out["gainmap"] = gainmap_single(13, 17, max(cfg.height - 1, 1) / 12.0, max(cfg.width - 1, 1) / 16.0,
                                        radial_gains(), bottom=13, right=17, cfa_pattern=cfg.cfa)
    if cfg.warp is not None:
        out["opcode3"] = opcode3_warp([cfg.warp])
    m, cct, weight = wb_params(cfg.neutral, COLOR_MATRIX1, COLOR_MATRIX2, CAMERA_TO_XYZ, CAMERA_TO_XYZ)
    out["wb"] = wb(cfg.neutral, m, np.float32(cct), weight)
    t = colormatrix_compose(m)
    out["colormatrix"] = colormatrix(t)
    out["colormatrix_t"] = t
    lut = cfg.lut_values()
    if lut is not None:
        out["lut_values"] = lut
    return out
