"""Packers for the filter parameter blobs (the reference PODs of
include/cpipe_b200_params.h) and for the DNG OpcodeList2/OpcodeList3 byte
streams the node plugins parse.

The byte-stream builders produce the DNG 1.3 big-endian opcode-list layout
(count, then per opcode: id, dng_version, flags, param size, params), the same
layout the reference unit-test fixtures build (tests/unit/gainmap_test_fixture.hpp:34-72,
tests/unit/opcode_list_3_test_fixture.hpp:29-110)."""
import ctypes as C
import struct

import numpy as np

from . import _abi as A


def raw(struct_obj):
    return bytes(struct_obj)


# ------------------------------------------------------------------ PODs
def blacklevel(black, white, cfa4):
    p = A.BlacklevelParams()
    p.black_level[:] = list(black)
    p.white_level = int(white)
    p.cfa_pattern[:] = list(cfa4)
    return raw(p)


def demosaic(cfa4):
    p = A.DemosaicParams()
    p.cfa_pattern[:] = list(cfa4)
    return raw(p)


def wb(neutral, camera_to_xyz=(1, 0, 0, 0, 1, 0, 0, 0, 1), cct=5000.0, weight=0.5):
    p = A.WbParams()
    p.as_shot_neutral[:] = list(neutral)
    p.camera_to_xyz_d50[:] = list(camera_to_xyz)
    p.scene_cct = cct
    p.dual_illuminant_weight = weight
    return raw(p)


def colormatrix(t9):
    p = A.ColormatrixParams()
    p.transform[:] = [float(v) for v in t9]
    return raw(p)


def bm3d(sigma):
    return raw(A.Bm3dParams(sigma))


def bm3d_spec(sigma, lambda3d=2.7, tau_match1=2500.0, tau_match2=400.0, n2=16, ns=39, nstep=3,
              kaiser_beta=2.0, stages=2, transform="tensor"):
    """Two-stage BM3D parameters; defaults are the published values (8x8 blocks,
    16-block groups, 39x39 search, step 3, hard threshold then Wiener).
    transform: "tensor" (FP16 hi/lo split on the tensor cores), "fp32", or
    "tensor_fp16" (single FP16 products on the tensor cores: the screening
    form the surrogate's spot check runs)."""
    return raw(A.Bm3dSpecParams(float(sigma), float(lambda3d), float(tau_match1), float(tau_match2), int(n2),
                                int(ns), int(nstep), float(kaiser_beta), int(stages),
                                {"tensor": 0, "fp32": 1, "tensor_fp16": 2}[transform]))


def guided(radius, eps):
    return raw(A.GuidedFilterParams(int(radius), float(eps)))


def atrous(levels=5, sigma=0.03, luma_strength=1.0, chroma_strength=1.0):
    """cpipe_AtrousWaveletParams for denoise_wavelet_atrous_spec."""
    return raw(A.AtrousWaveletParams(int(levels), float(sigma), float(luma_strength), float(chroma_strength)))


def wavelet(strength):
    return raw(A.WaveletBayesShrinkParams(float(strength)))


def filmic(ev=0.0, contrast=1.0, saturation=1.0, highlights=1.0, shadows=1.0):
    return raw(A.FilmicRgbParams(ev, contrast, saturation, highlights, shadows))


def mertens(weight_contrast=0.0, weight_saturation=1.0, weight_well_exposedness=1.0):
    """cpipe_MertensLocalParams for tone_mertens_local."""
    return raw(A.MertensLocalParams(float(weight_contrast), float(weight_saturation), float(weight_well_exposedness)))


def aces(enabled=True):
    """cpipe_AcesFilmicParams for tone_aces_filmic."""
    return raw(A.AcesFilmicParams(1 if enabled else 0))


def reinhard(white_point=1000000.0):
    """cpipe_ReinhardParams for tone_reinhard (1e6: the node's value when its param is unset)."""
    return raw(A.ReinhardParams(float(white_point)))


def usm(strength=0.75, radius=1, threshold=0.0):
    """cpipe_EdgeAwareUsmParams for sharpen_edge_aware_usm."""
    return raw(A.EdgeAwareUsmParams(float(strength), int(radius), float(threshold)))


def display(target="sRGB"):
    """cpipe_DisplayParams for cpipe_scene_linear_to_display ("sRGB" or "BT2020-PQ")."""
    return raw(A.DisplayParams({"sRGB": A.DISPLAY_SRGB, "BT2020-PQ": A.DISPLAY_BT2020_PQ}[target]))


def linearize(table):
    t = np.ascontiguousarray(table, dtype=np.uint16)
    return struct.pack("<I", t.size) + t.tobytes()


def lut3d(size, values, interpolation=0):
    v = np.ascontiguousarray(values, dtype=np.float32).ravel()
    return raw(A.Lut3dParamHeader(int(size), int(v.size), int(interpolation))) + v.tobytes()


def gainmap_dispatch(maps, cfa_repeat=(2, 2), cfa_pattern=(0, 1, 1, 2)):
    """maps: list of dicts {plane, planes, points_v, points_h, spacing_v, spacing_h,
    origin_v, origin_h, gains} -> GainMapDispatchHeader + planes + gains."""
    hd = A.GainMapDispatchHeader()
    hd.map_count = len(maps)
    hd.cfa_repeat[:] = list(cfa_repeat)
    pat = list(cfa_pattern) + [0] * (16 - len(cfa_pattern))
    hd.cfa_pattern[:] = pat[:16]
    out = raw(hd)
    off = 0
    gains = b""
    for m in maps:
        g = np.ascontiguousarray(m["gains"], dtype=np.float32).ravel()
        p = A.GainMapDispatchPlane(0, 0, m["points_v"], m["points_h"], m.get("plane", 0), m.get("planes", 1),
                                   m["points_v"], m["points_h"], m["spacing_v"], m["spacing_h"],
                                   m.get("origin_v", 0.0), m.get("origin_h", 0.0), off, g.size)
        off += g.size
        out += raw(p)
        gains += g.tobytes()
    return out + gains


def opcode3_dispatch(records, points=(), rects=()):
    """records: list of Opcode3DispatchRecord; points [(row, col)]; rects [(t, l, b, r)]."""
    out = raw(A.Opcode3DispatchHeader(len(records), 0))
    for r in records:
        out += raw(r)
    for row, col in points:
        out += struct.pack("<II", row, col)
    for t, l, b, r in rects:
        out += struct.pack("<IIII", t, l, b, r)
    return out


def warp_record(coefficients, cx_hat=0.5, cy_hat=0.5):
    """coefficients: list of (kr0, kr1, kr2, kr3, kt0, kt1) per plane (1..4)."""
    r = A.Opcode3DispatchRecord()
    r.id = 1
    r.coefficient_count = len(coefficients)
    for i, k in enumerate(coefficients):
        r.coefficients[i] = A.Opcode3WarpCoefficient(*k)
    r.cx_hat, r.cy_hat = cx_hat, cy_hat
    return r


def vignette_record(k, cx_hat=0.5, cy_hat=0.5):
    r = A.Opcode3DispatchRecord()
    r.id = 3
    r.vignette_k[:] = list(k) + [0.0] * (5 - len(k))
    r.vignette_cx_hat, r.vignette_cy_hat = cx_hat, cy_hat
    return r


# ------------------------------------------------------- DNG byte streams
def _be32(v):
    return struct.pack(">I", v & 0xFFFFFFFF)


def _bed(v):
    return struct.pack(">d", v)


def gain_map_params(width, height, plane, planes, spacing_v, spacing_h, gains, origin_v=0.0, origin_h=0.0):
    """GainMap opcode parameters: a points_v x points_h = height x width grid."""
    out = _be32(0) + _be32(0) + _be32(height) + _be32(width) + _be32(plane) + _be32(planes)
    out += _be32(1) + _be32(1) + _be32(height) + _be32(width)
    out += _bed(spacing_v) + _bed(spacing_h) + _bed(origin_v) + _bed(origin_h) + _be32(1)
    for g in np.asarray(gains, dtype=np.float32).ravel():
        out += struct.pack(">f", float(g))
    return out


def opcode_list(opcodes, flags=0):
    """opcodes: list of (id, params_bytes) -> OpcodeList byte stream."""
    out = _be32(len(opcodes))
    for oid, params in opcodes:
        out += _be32(oid) + _be32(0x00010003) + _be32(flags) + _be32(len(params)) + params
    return out


def opcode_list_2_with_gain_maps(params_list):
    return opcode_list([(9, p) for p in params_list])


def warp_rectilinear_params(coefficients, cx_hat=0.5, cy_hat=0.5):
    out = _be32(len(coefficients))
    for k in coefficients:
        for v in k:
            out += _bed(v)
    return out + _bed(cx_hat) + _bed(cy_hat)


def fix_vignette_radial_params(k, cx_hat=0.5, cy_hat=0.5):
    k = list(k) + [0.0] * (5 - len(k))
    return b"".join(_bed(v) for v in k) + _bed(cx_hat) + _bed(cy_hat)


def fix_bad_pixels_constant_params(constant, bayer_phase=0):
    return _be32(constant) + _be32(bayer_phase)


def fix_bad_pixels_list_params(points=(), rects=(), bayer_phase=0):
    out = _be32(bayer_phase) + _be32(len(points)) + _be32(len(rects))
    for row, col in points:
        out += _be32(row) + _be32(col)
    for t, l, b, r in rects:
        out += _be32(t) + _be32(l) + _be32(b) + _be32(r)
    return out


def trim_bounds_params(top, left, bottom, right):
    return _be32(top) + _be32(left) + _be32(bottom) + _be32(right)


def write_cube(path, size, values, title="cpipe synthetic LUT"):
    v = np.asarray(values, dtype=np.float32).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f'TITLE "{title}"\nLUT_3D_SIZE {size}\nDOMAIN_MIN 0 0 0\nDOMAIN_MAX 1 1 1\n')
        for row in v:
            f.write("%.9g %.9g %.9g\n" % tuple(row))
