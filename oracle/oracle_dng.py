"""CPU restatement of the reference's DNG ingest.

TEST INFRASTRUCTURE: imported only by tests/ as the checker.  The product
library never loads it.

parse()  follows cpipe::ingest::dng_opcode::OpcodeListParser::parse
         (src/cpipe/ingest/dng_opcode/OpcodeListParser.cpp:330-515) and its
         value readers (OpcodeListParser.cpp:84-278): little-endian TIFF only,
         IFD0 plus the Exif IFD's capture tags.  One extension for files the
         reference rejects: when IFD0 is not a CFA image, the first
         full-resolution CFA SubIFD supplies the image tags.
read()   follows cpipe::ingest::dng::DngReader::read (src/cpipe/ingest/dng/
         DngReader.cpp:190-232) on its single-strip path (DngReader.cpp:145-164):
         copy min(width * height * 2, strip bytes) into a zeroed R16 plane.
         The reference first tries LibRaw (vcpkg dependency `libraw`, absent from
         the reference tree); for strips shorter than a 16-bit plane with
         BitsPerSample < 16 this restatement unpacks the DNG 1.4 uncompressed
         packing (samples most-significant bit first, rows on byte boundaries).
         Both paths return the stored samples as they are: they equal the
         reference's single-strip fallback, not necessarily LibRaw, whose DNG
         loaders are understood (not checked here: its source is absent) to map
         samples through the file's LinearizationTable when one is present.
         Parity for the packed depths is pinned only by pack -> unpack round
         trips; the 16-bit path and the parse are pinned by the reference's own
         unit-test expectations (tests/unit/test_dng_reader.cpp).
"""
import struct

import numpy as np

OK, FAILED, UNSUPPORTED = 0, 1, 8
BYTE, ASCII, SHORT, LONG, RATIONAL, UNDEFINED, SRATIONAL = 1, 2, 3, 4, 5, 7, 10
_SIZE = {BYTE: 1, ASCII: 1, UNDEFINED: 1, SHORT: 2, LONG: 4, RATIONAL: 8, SRATIONAL: 8}
_F32 = np.float32


def _entries(b, off):
    """IFD entries {tag: (type, count, value, entry_pos)}, first occurrence kept
    (OpcodeListParser.cpp:122-150)."""
    if off + 2 > len(b):
        return None
    n = struct.unpack_from("<H", b, off)[0]
    if off + 2 + 12 * n > len(b):
        return None
    out = {}
    for i in range(n):
        p = off + 2 + 12 * i
        tag, typ, cnt, val = struct.unpack_from("<HHII", b, p)
        out.setdefault(tag, (typ, cnt, val, p))
    return out


def _data(b, e):
    """(bytes, file offset) of an entry's value (OpcodeListParser.cpp:101-119)."""
    typ, cnt, val, pos = e
    size = _SIZE.get(typ, 0) * cnt
    if size == 0 or size > len(b):
        return b"", 0
    if size <= 4:
        return struct.pack("<I", val)[:size], pos + 8
    if val > len(b) or size > len(b) - val:
        return b"", 0
    return bytes(b[val:val + size]), val


def _ints(b, e):
    d, _ = _data(b, e)
    typ, cnt = e[0], e[1]
    if not d:
        return []
    fmt = {BYTE: "B", SHORT: "H", LONG: "I"}.get(typ)
    return list(struct.unpack_from("<%d%s" % (cnt, fmt), d)) if fmt else []


def _first(b, ents, tag):
    e = ents.get(tag)
    if e is None:
        return None
    d, _ = _data(b, e)
    if not d:
        return 0
    if e[0] == SHORT and len(d) >= 2:
        return struct.unpack_from("<H", d)[0]
    if e[0] == LONG and len(d) >= 4:
        return struct.unpack_from("<I", d)[0]
    if e[0] == BYTE:
        return d[0]
    return 0


def _floats(b, ents, tag):
    """binary32 values: integers converted; rationals num / den in binary32."""
    e = ents.get(tag)
    if e is None:
        return None
    if e[0] in (BYTE, SHORT, LONG):
        return [_F32(v) for v in _ints(b, e)]
    if e[0] not in (RATIONAL, SRATIONAL):
        return []
    d, _ = _data(b, e)
    if not d:
        return []
    f = "<%d%s" % (2 * e[1], "I" if e[0] == RATIONAL else "i")
    v = struct.unpack_from(f, d)
    out = []
    for i in range(e[1]):
        num, den = _F32(v[2 * i]), _F32(v[2 * i + 1])
        out.append(_F32(0.0) if den == 0 else _F32(num / den))
    return out


def _capture(b, ents, info):
    v = _floats(b, ents, 33434)
    if v:
        info["exposure_time_ns"] = int(_F32(v[0]) * _F32(1e9))
    iso = _first(b, ents, 34855)
    if iso is not None:
        info["iso"] = iso
    v = _floats(b, ents, 33437)
    if v:
        info["lens_aperture"] = float(v[0])
    v = _floats(b, ents, 37386)
    if v:
        info["lens_focal_length_mm"] = float(v[0])


def parse(b):
    """(status, info dict) with the fields of cpipe_DngInfo."""
    b = bytes(b)
    info = {"width": 0, "height": 0, "bits_per_sample": 0, "compression": 1, "strip_offset": 0,
            "strip_byte_count": 0, "orientation": 0, "cfa_repeat": [0, 0], "cfa_pattern": [],
            "black_level": [0.0] * 4, "white_level": 0, "calibration_illuminant": [0, 0],
            "has_matrix": [0] * 4, "matrix": [[0.0] * 9 for _ in range(4)], "as_shot_neutral": [0.0] * 3,
            "active_area": None, "iso": 0, "exposure_time_ns": 0, "lens_aperture": 0.0,
            "lens_focal_length_mm": 0.0, "linearization": [], "make": "", "model": "",
            "blobs": {}}
    if len(b) < 8 or b[:2] != b"II" or struct.unpack_from("<H", b, 2)[0] != 42:
        return FAILED, info
    ents = _entries(b, struct.unpack_from("<I", b, 4)[0])
    if ents is None:
        return FAILED, info

    def cfa_image(e):
        ph, spp = _first(b, e, 262), _first(b, e, 277)
        return (32803 if ph is None else ph) == 32803 and (1 if spp is None else spp) == 1

    # Extension beyond the reference (which reads IFD0 only and rejects these
    # files): when IFD0 is not a CFA image, the first full-resolution CFA
    # SubIFD supplies the image tags; camera tags stay IFD0's.
    raw = ents
    if not cfa_image(ents) and 330 in ents and ents[330][0] in (LONG, 13) and ents[330][1] > 0:
        typ, cnt, val, pos = ents[330]
        at = pos + 8 if cnt == 1 else val
        for k in range(min(cnt, 16)):
            if at + 4 * (k + 1) > len(b):
                break
            sub = _entries(b, struct.unpack_from("<I", b, at + 4 * k)[0])
            if sub is not None and (_first(b, sub, 254) or 0) == 0 and cfa_image(sub):
                raw = sub
                break
    c = _first(b, raw, 259)
    info["compression"] = 1 if c is None else c
    if not cfa_image(raw):
        return UNSUPPORTED, info
    for key, tag in (("width", 256), ("height", 257), ("bits_per_sample", 258), ("strip_offset", 273),
                     ("strip_byte_count", 279), ("white_level", 50717)):
        v = _first(b, raw, tag)
        info[key] = 0 if v is None else v
    info["orientation"] = (_first(b, ents, 274) or 0) & 0xFF
    info["calibration_illuminant"] = [(_first(b, ents, 50778) or 0) & 0xFFFF, (_first(b, ents, 50779) or 0) & 0xFFFF]
    _capture(b, ents, info)
    for key, tag in (("make", 271), ("model", 272)):
        e = ents.get(tag)
        if e is not None and e[0] == ASCII:
            d, _ = _data(b, e)
            info[key] = d.split(b"\0")[0][:63].decode("latin-1")
    rep = raw.get(33421)
    if rep is None:
        return UNSUPPORTED, info
    r = _ints(b, rep) if rep[0] == SHORT else []
    if len(r) != 2 or r[0] != r[1] or r[0] not in (2, 4):
        return UNSUPPORTED, info
    pat = raw.get(33422)
    d = _data(b, pat)[0] if pat is not None else b""
    if not (pat is not None and len(d) == r[0] * r[1] and len(d) <= 16):
        return UNSUPPORTED, info
    info["cfa_repeat"], info["cfa_pattern"] = r, list(d)
    v = _floats(b, raw, 50714) or []
    for i in range(min(4, len(v))):
        info["black_level"][i] = float(v[i])
    e = raw.get(50712)
    if e is not None and e[0] == SHORT:
        info["linearization"] = _ints(b, e)
    for m, tag in enumerate((50721, 50722, 50964, 50965)):
        v = _floats(b, ents, tag)
        if v is not None:
            info["has_matrix"][m] = 1
            for i in range(min(9, len(v))):
                info["matrix"][m][i] = float(v[i])
    v = _floats(b, ents, 50728) or []
    for i in range(min(3, len(v))):
        info["as_shot_neutral"][i] = float(v[i])
    e = raw.get(50829)
    if e is not None:
        v = _ints(b, e)
        if len(v) == 4 and v[2] >= v[0] and v[3] >= v[1]:
            info["active_area"] = [v[1], v[0], v[3] - v[1], v[2] - v[0]]
    if 34665 in ents:
        eo = _first(b, ents, 34665)
        if eo + 2 <= len(b):
            n = 2 + struct.unpack_from("<H", b, eo)[0] * 12 + 4
            if n <= len(b) and eo <= len(b) - n:
                info["blobs"]["exif"] = (eo, n)
        ex = _entries(b, eo)
        if ex is not None:
            _capture(b, ex, info)
    for name, tag in (("xmp", 700), ("icc", 34675), ("opcode_list_1", 51008), ("opcode_list_2", 51009),
                      ("opcode_list_3", 51022)):
        e = (raw if tag > 50000 else ents).get(tag)
        if e is not None:
            d, off = _data(b, e)
            info["blobs"][name] = (off, len(d))
    if (info["width"] == 0 or info["height"] == 0 or info["bits_per_sample"] == 0
            or info["bits_per_sample"] > 16 or info["strip_byte_count"] == 0):
        return FAILED, info
    if info["compression"] != 1 and info["strip_offset"] == 0:
        return FAILED, info
    return OK, info


def unpack(strip, w, h, bits):
    """R16 plane (h, w) uint16 from the strip bytes."""
    strip = np.frombuffer(bytes(strip), np.uint8)
    plane = w * h * 2
    if bits == 16 or strip.size >= plane:
        out = np.zeros(plane, np.uint8)
        n = min(plane, strip.size)
        out[:n] = strip[:n]
        return out.view("<u2").reshape(h, w).astype(np.uint16)
    row_bytes = (w * bits + 7) // 8
    buf = np.zeros(row_bytes * h, np.uint8)
    n = min(buf.size, strip.size)
    buf[:n] = strip[:n]
    rows = np.unpackbits(buf.reshape(h, row_bytes), axis=1)[:, :w * bits].reshape(h, w, bits)
    weights = (1 << np.arange(bits - 1, -1, -1)).astype(np.uint32)
    return (rows.astype(np.uint32) @ weights).astype(np.uint16)


def pack(x, bits):
    """Inverse of unpack's packed form: (h, w) samples < 2**bits -> strip bytes."""
    x = np.asarray(x, np.uint16)
    h, w = x.shape
    rows = np.empty((h, w, bits), np.uint8)
    for i in range(bits):
        rows[..., i] = (x >> (bits - 1 - i)) & 1
    return np.packbits(rows.reshape(h, w * bits), axis=1).tobytes()


def read(b):
    """(status, plane or None, info): DngReader::read on a file image."""
    st, info = parse(b)
    if st == UNSUPPORTED:
        return FAILED, None, info
    if st != OK:
        return st, None, info
    if info["compression"] != 1:
        return UNSUPPORTED, None, info
    off, cnt = info["strip_offset"], info["strip_byte_count"]
    if off > len(b) or cnt > len(b) - off:
        return FAILED, None, info
    return OK, unpack(bytes(b)[off:off + cnt], info["width"], info["height"], info["bits_per_sample"]), info
