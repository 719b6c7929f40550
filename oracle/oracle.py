"""ctypes front end of the CPU oracle (oracle/_build/liboracle.so) and of the
reference build (oracle/_ref/libcpipe_ref.so).

TEST INFRASTRUCTURE: imported only by tests/, the smoke check and the CPU
baseline leg of bench.py, always as the checker.  The product library never
loads it.  All arrays are numpy; RGBA images are HxWx4 float32 (with f16=True
the outputs hold binary16 values, as the reference's RGBA16F buffers do).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcpipe_ref.so")

_o = None
_r = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        _o = C.CDLL(ORACLE_LIB)
    return _o


def ref_lib():
    """The reference's own filters (None when the reference build is absent)."""
    global _r
    if _r is None and os.path.exists(REF_LIB):
        _r = C.CDLL(REF_LIB)
        _r.cpipe_ref_call.restype = C.c_int
        _r.cpipe_ref_has.restype = C.c_int
    return _r


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _blob(b):
    buf = C.create_string_buffer(bytes(b), len(bytes(b)))
    return buf, len(bytes(b))


def h16(a):
    return np.asarray(a, dtype=np.float32).astype(np.float16).astype(np.float32)


# ------------------------------------------------------------------ nodes
def r16u_to_f32(raw):
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    out = np.empty(raw.shape, np.float32)
    lib().oracle_r16u_to_f32(_p(raw), _p(out), raw.shape[1], raw.shape[0])
    return out


def f32_to_rgba16f(x):
    x = _f32(x)
    out = np.empty(x.shape + (4,), np.float32)
    lib().oracle_f32_to_rgba16f(_p(x), _p(out), x.shape[1], x.shape[0])
    return out


def rgba16f_to_unorm(x, bits8):
    x = _f32(x)
    out = np.empty(x.shape, np.uint16)
    lib().oracle_rgba16f_to_unorm(_p(x), _p(out), x.shape[1], x.shape[0], int(bits8))
    return out.astype(np.uint8) if bits8 else out


def linearize(raw, table):
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    t = np.ascontiguousarray(table, dtype=np.uint16)
    out = np.empty(raw.shape, np.float32)
    st = lib().oracle_linearize(_p(raw), _p(out), raw.shape[1], raw.shape[0], _p(t), t.size)
    return st, out


def blacklevel(x, blob):
    x = _f32(x)
    out = np.empty_like(x)
    b, _ = _blob(blob)
    st = lib().oracle_blacklevel(_p(x), _p(out), x.shape[1], x.shape[0], b)
    return st, out


def gainmap(x, blob):
    x = _f32(x)
    out = np.empty_like(x)
    b, n = _blob(blob)
    st = lib().oracle_gainmap(_p(x), _p(out), x.shape[1], x.shape[0], b, C.c_size_t(n))
    return st, out


def demosaic(algo, x, cfa4, f16=True):
    """algo: 'bilinear' | 'rcd' | 'amaze'."""
    x = _f32(x)
    out = np.empty(x.shape + (4,), np.float32)
    cfa = (C.c_uint8 * 4)(*cfa4)
    lib().oracle_demosaic({"bilinear": 0, "rcd": 1, "amaze": 2}[algo], _p(x), _p(out), x.shape[1], x.shape[0],
                          cfa, int(f16))
    return out


def demosaic_full(algo, x, cfa4, prec="f32"):
    """Full-form RCD ('rcd') or AMaZE ('amaze') of oracle_demosaic_full.c.
    x: HxW float32 normalised mosaic.  prec 'f32': the kernels' binary32
    arithmetic; 'f64': the FP64 reference.  Returns HxWx3 float64 RGB."""
    x = _f32(x)
    h, w = x.shape
    out = np.empty((h, w, 3), np.float64)
    cfa = (C.c_uint8 * 4)(*cfa4)
    st = lib().oracle_demosaic_full({"rcd": 1, "amaze": 2}[algo], {"f32": 0, "f64": 1}[prec], _p(x), w, h, cfa,
                                    _p(out))
    if st != 0:
        raise MemoryError("oracle_demosaic_full")
    return out


def rgba_from_rgb(rgb, f16=True):
    """HxWx3 -> HxWx4 float32 with alpha 1, rounded to binary16 when f16."""
    out = np.ones(rgb.shape[:2] + (4,), np.float32)
    out[..., :3] = np.asarray(rgb, np.float32)
    return h16(out) if f16 else out


def qbc_remosaic(raw):
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    out = np.empty_like(raw)
    lib().oracle_qbc_remosaic(_p(raw), _p(out), raw.shape[1], raw.shape[0])
    return out


def wb(x, neutral, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    from cpipe_b200 import blobs  # struct layout only
    b, _ = _blob(blobs.wb(neutral))
    lib().oracle_wb(_p(x), _p(out), x.shape[1], x.shape[0], b, int(f16))
    return out


def colormatrix(x, t9, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    t = (C.c_float * 9)(*[float(v) for v in t9])
    lib().oracle_colormatrix(_p(x), _p(out), x.shape[1], x.shape[0], t, int(f16))
    return out


def bm3d_parity(x, sigma, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    lib().oracle_bm3d_parity(_p(x), _p(out), x.shape[1], x.shape[0], C.c_float(sigma), int(f16))
    return out


def bm3d_spec(x, blob, basic=False):
    """Two-stage colour BM3D in FP64 (oracle_bm3d.c).  x: HxWx4 float32 (the
    RGBA16F input as float).  Returns the HxWx4 float64 estimate, and with
    basic=True also the step-1 estimate as 3xHxW opponent (Y, U, V) planes."""
    x = _f32(x)
    h, w = x.shape[:2]
    out = np.empty((h, w, 4), np.float64)
    b3 = np.empty((3, h, w), np.float64) if basic else None
    pb, _ = _blob(blob)
    st = lib().oracle_bm3d_spec(_p(x), w, h, pb, _p(out), _p(b3) if basic else None)
    if st != 0:
        raise ValueError(f"oracle_bm3d_spec status {st}")
    return (out, b3) if basic else out


def bm3d_quantise_rgb(x):
    x = _f32(x)
    q = np.empty(x.shape[:2], np.uint8)
    lib().oracle_bm3d_quantise_rgb(_p(x), x.shape[1], x.shape[0], _p(q))
    return q


def bm3d_match(q, x, y, ns=39, n2=16, tau=2500.0):
    """Group of the reference block at (x, y): list of (x, y) block positions."""
    q = np.ascontiguousarray(q, np.uint8)
    pos = (C.c_uint32 * 16)()
    scratch = (C.c_uint64 * (ns * ns))()
    L = lib()
    L.oracle_bm3d_dthr.restype = C.c_uint32
    n = L.oracle_bm3d_match(_p(q), q.shape[1], q.shape[0], int(x), int(y), int(ns), int(n2),
                            C.c_uint32(L.oracle_bm3d_dthr(C.c_float(tau))), pos, scratch)
    return [(pos[i] & 0xFFFF, pos[i] >> 16) for i in range(n)]


def guided(x, radius, eps, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    lib().oracle_guided(_p(x), _p(out), x.shape[1], x.shape[0], int(radius), C.c_float(eps), int(f16))
    return out


def mertens(under, normal, over, wc=0.0, ws=1.0, we=1.0, f16=True):
    u, n, o = _f32(under), _f32(normal), _f32(over)
    out = np.empty_like(n)
    lib().oracle_mertens(_p(u), _p(n), _p(o), _p(out), n.shape[1], n.shape[0], C.c_float(wc), C.c_float(ws),
                         C.c_float(we), int(f16))
    return out


def aces(x, enabled=True, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    lib().oracle_aces(_p(x), _p(out), x.shape[1], x.shape[0], int(bool(enabled)), int(f16))
    return out


def reinhard(x, white_point=1000000.0, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    lib().oracle_reinhard(_p(x), _p(out), x.shape[1], x.shape[0], C.c_float(white_point), int(f16))
    return out


def usm(x, strength=0.75, radius=1, threshold=0.0, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    lib().oracle_usm(_p(x), _p(out), x.shape[1], x.shape[0], C.c_float(strength), int(radius), C.c_float(threshold),
                     int(f16))
    return out


def wavelet(x, strength, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    lib().oracle_wavelet(_p(x), _p(out), x.shape[1], x.shape[0], C.c_float(strength), int(f16))
    return out


def lut3d(x, lut_values, size, interp=0, f16=True):
    x = _f32(x)
    lut = _f32(lut_values).ravel()
    out = np.empty_like(x)
    lib().oracle_lut3d(_p(x), _p(out), x.shape[1], x.shape[0], _p(lut), int(size), int(interp), int(f16))
    return out


def filmic(x, ev=0.0, contrast=1.0, saturation=1.0, highlights=1.0, shadows=1.0, f16=True):
    from cpipe_b200 import blobs
    x = _f32(x)
    out = np.empty_like(x)
    b, _ = _blob(blobs.filmic(ev, contrast, saturation, highlights, shadows))
    lib().oracle_filmic(_p(x), _p(out), x.shape[1], x.shape[0], b, int(f16))
    return out


def opcode3(x, blob, f16=True):
    x = _f32(x)
    out = np.empty_like(x)
    w1 = np.empty_like(x)
    w2 = np.empty_like(x)
    b, n = _blob(blob)
    st = lib().oracle_opcode3(_p(x), _p(out), _p(w1), _p(w2), x.shape[1], x.shape[0], b, C.c_size_t(n), int(f16))
    return st, out


# ------------------------------------------------------- reference build
class _HDim(C.Structure):
    _fields_ = [("min", C.c_int32), ("extent", C.c_int32), ("stride", C.c_int32), ("flags", C.c_uint32)]


class _HBuf(C.Structure):
    _fields_ = [("device", C.c_uint64), ("device_interface", C.c_void_p), ("host", C.c_void_p),
                ("flags", C.c_uint64), ("code", C.c_uint8), ("bits", C.c_uint8), ("lanes", C.c_uint16),
                ("dimensions", C.c_int32), ("dim", C.POINTER(_HDim)), ("padding", C.c_void_p)]


def _hb(arr, keep):
    dims = (_HDim * 3)()
    code, bits = {np.dtype(np.uint16): (1, 16), np.dtype(np.float32): (2, 32),
                  np.dtype(np.float16): (2, 16)}[arr.dtype]
    h, w = arr.shape[:2]
    if arr.ndim == 3:
        c = arr.shape[2]
        dims[0], dims[1], dims[2] = _HDim(0, w, c, 0), _HDim(0, h, w * c, 0), _HDim(0, c, 1, 0)
        nd = 3
    else:
        dims[0], dims[1] = _HDim(0, w, 1, 0), _HDim(0, h, w, 0)
        nd = 2
    hb = _HBuf(0, None, arr.ctypes.data, 0, code, bits, 1, nd, C.cast(dims, C.POINTER(_HDim)), None)
    keep.append(dims)
    return hb


def ref_call(aot_id, inp, out, blob):
    """Run the reference's own C++ filter `aot_id` (one of the six plain-C++
    dispatch files) on numpy host buffers; returns its status."""
    r = ref_lib()
    if r is None:
        raise RuntimeError("reference build absent (make -C oracle ref)")
    keep = []
    hi, ho = _hb(inp, keep), _hb(out, keep)
    pin = (C.POINTER(_HBuf) * 1)(C.pointer(hi))
    pout = (C.POINTER(_HBuf) * 1)(C.pointer(ho))
    b, n = _blob(blob)
    return r.cpipe_ref_call(aot_id.encode(), pin, C.c_size_t(1), pout, C.c_size_t(1), b, C.c_size_t(n))


def ref_wb_interpolate(neutral, cm1, cm2, fm1=None, fm2=None, illum1=17, illum2=21):
    r = ref_lib()
    F9 = C.c_float * 9
    out = F9()
    cct = C.c_double()
    wgt = C.c_float()
    st = r.cpipe_ref_wb_interpolate((C.c_float * 3)(*neutral), F9(*cm1), F9(*cm2),
                                    F9(*fm1) if fm1 is not None else None, F9(*fm2) if fm2 is not None else None,
                                    C.c_uint(illum1), C.c_uint(illum2), out, C.byref(cct), C.byref(wgt))
    return st, list(out), cct.value, wgt.value


def greyworld(x):
    """wb.greyworld_auto (src/cpipe/nodes/wb/greyworld_auto.cpp:44-77): the
    neutral (R/G, 1, B/G) from the channel sums and v / neutral per RGB channel
    in float, rounded to binary16; alpha passes.  The sums are exact and
    rounded once (math.fsum): the reference adds sequentially in double, which
    is exact for the fixture's few values.  Returns (neutral, out) or
    (None, None) when a sum is not finite or not positive."""
    import math
    x = np.asarray(x, np.float16).astype(np.float32)
    sums = [math.fsum(x[..., c].astype(np.float64).ravel().tolist()) for c in range(3)]
    if any(not math.isfinite(v) or v <= 0.0 for v in sums):
        return None, None
    n = np.array([sums[0] / sums[1], 1.0, sums[2] / sums[1]], np.float32)
    out = x.copy()
    for c in range(3):
        out[..., c] = (x[..., c] / n[c]).astype(np.float16).astype(np.float32)
    return n, out
