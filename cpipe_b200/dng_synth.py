"""Synthetic little-endian DNG files (seeded test and benchmark frames).

The tag set and values follow the reference's own synthetic fixture
(tests/unit/dng_test_fixture.hpp:199-300 in the reference: a 4x3 RGGB RAW16
frame with pixels 64 + 9 i, ISO 400, 1/125 s, f/1.7, 4.3 mm, linearization
table {0, 128, 1024, 4095}, black levels 64..67, white 4095, identity matrices,
AsShotNeutral {1, 2, 3}, illuminants 21 / 17, a full active area), so the
expectations of tests/unit/test_dng_reader.cpp apply to these files.  Layout:
header, IFD0 at offset 8 (entries sorted by tag), then the value sections.
"""
import heapq
import struct

import numpy as np

BYTE, ASCII, SHORT, LONG, RATIONAL, UNDEFINED, SRATIONAL = 1, 2, 3, 4, 5, 7, 10


def _vals(typ, values):
    if typ in (BYTE, UNDEFINED):
        return bytes(values)
    if typ == ASCII:
        return values.encode("latin-1") + b"\0"
    if typ == SHORT:
        return struct.pack("<%dH" % len(values), *values)
    if typ == LONG:
        return struct.pack("<%dI" % len(values), *values)
    if typ == RATIONAL:
        return b"".join(struct.pack("<II", n, d) for n, d in values)
    if typ == SRATIONAL:
        return b"".join(struct.pack("<ii", n, d) for n, d in values)
    raise ValueError(typ)


def default_pixels(w, h):
    return np.array([(64 + 9 * i) & 0xFFFF for i in range(w * h)], np.uint16).reshape(h, w)


def build_dng(width=4, height=3, pixels=None, strip=None, bits=16, cfa_repeat=(2, 2), cfa_pattern=(0, 1, 1, 2),
              include_cfa=True, include_opcode_lists=True, include_sidecars=True, strip_byte_count=None,
              overrides=None, drop=(), segments=None, tile=None, rows_per_strip=None, strip_tags=True):
    """bytes of a DNG.  `strip` (bytes) replaces the RAW16 little-endian words
    of `pixels`; `overrides` maps tag -> (type, values); `drop` lists tags to
    leave out.  `segments` (list of bytes) makes a Compression 7 file: tiles of
    `tile` = (width, length) when given (with StripOffsets / StripByteCounts
    also pointing at the first tile when `strip_tags`), else strips of
    `rows_per_strip` rows."""
    if segments is not None:
        return _build_segmented(width, height, segments, bits, tile, rows_per_strip, strip_tags, cfa_repeat,
                                cfa_pattern, overrides, drop)
    if strip is None:
        px = default_pixels(width, height) if pixels is None else np.asarray(pixels, np.uint16)
        strip = px.astype("<u2").tobytes()
    ident = [(1, 1), (0, 1), (0, 1), (0, 1), (1, 1), (0, 1), (0, 1), (0, 1), (1, 1)]
    tags = {
        256: (LONG, [width]), 257: (LONG, [height]), 258: (SHORT, [bits]), 259: (SHORT, [1]),
        262: (SHORT, [32803]), 271: (ASCII, "GoogleTest"), 272: (ASCII, "Pixel8UT"),
        273: (LONG, None),  # strip offset, filled in below (or by _build_segmented)
        274: (SHORT, [1]), 277: (SHORT, [1]), 278: (LONG, [height]),
        279: (LONG, [len(strip) if strip_byte_count is None else strip_byte_count]),
        33434: (RATIONAL, [(1, 125)]), 33437: (RATIONAL, [(17, 10)]),
        34665: (LONG, None),  # Exif IFD offset
        34855: (SHORT, [400]), 37386: (RATIONAL, [(43, 10)]),
        50706: (BYTE, [1, 4, 0, 0]), 50707: (BYTE, [1, 4, 0, 0]), 50708: (ASCII, "cpipe unit camera"),
        50712: (SHORT, [0, 128, 1024, 4095]),
        50714: (RATIONAL, [(64, 1), (65, 1), (66, 1), (67, 1)]), 50717: (LONG, [4095]),
        50721: (SRATIONAL, ident), 50722: (SRATIONAL, ident),
        50728: (RATIONAL, [(1, 1), (2, 1), (3, 1)]), 50778: (SHORT, [21]), 50779: (SHORT, [17]),
        50829: (LONG, [0, 0, height, width]), 50964: (SRATIONAL, ident), 50965: (SRATIONAL, ident),
    }
    if include_sidecars:
        tags[700] = (BYTE, list(b"<x:xmpmeta>unit</x:xmpmeta>\0"))
        tags[34675] = (UNDEFINED, [1, 2, 3, 4])
    if include_cfa:
        tags[33421] = (SHORT, list(cfa_repeat))
        tags[33422] = (BYTE, list(cfa_pattern))
    if include_opcode_lists:
        for tag in (51008, 51009, 51022):
            tags[tag] = (UNDEFINED, [0, 0, 0, 0, 0, 0, 0, 0])  # big-endian opcode count 0 + padding
    for t, v in (overrides or {}).items():
        tags[t] = v
    for t in drop:
        tags.pop(t, None)

    n = len(tags)
    data_start = 8 + 2 + 12 * n + 4
    sections = bytearray()
    exif = struct.pack("<H", 0) + struct.pack("<I", 0)  # an empty Exif IFD: 0 entries, no next IFD
    entries = []
    for tag in sorted(tags):
        typ, values = tags[tag]
        if tag == 273 and values is None:
            raw = None
        elif tag == 34665:
            raw = None
        else:
            raw = _vals(typ, values)
        count = 1 if raw is None else (len(raw) // {BYTE: 1, ASCII: 1, UNDEFINED: 1, SHORT: 2, LONG: 4,
                                                      RATIONAL: 8, SRATIONAL: 8}[typ])
        entries.append([tag, typ, count, raw])
    # Place out-of-line values, then the Exif IFD, then the strip (16-byte aligned).
    for e in entries:
        if e[3] is not None and len(e[3]) > 4:
            while (data_start + len(sections)) % 2:
                sections.append(0)
            off = data_start + len(sections)
            sections += e[3]
            e.append(off)
    while (data_start + len(sections)) % 2:
        sections.append(0)
    exif_off = data_start + len(sections)
    sections += exif
    while (data_start + len(sections)) % 16:
        sections.append(0)
    strip_off = data_start + len(sections)
    sections += strip

    out = bytearray(b"II" + struct.pack("<HI", 42, 8) + struct.pack("<H", n))
    for e in entries:
        tag, typ, count, raw = e[:4]
        if tag == 273 and raw is None:
            field = struct.pack("<I", strip_off)
        elif tag == 34665:
            field = struct.pack("<I", exif_off)
        elif len(raw) <= 4:
            field = raw + b"\0" * (4 - len(raw))
        else:
            field = struct.pack("<I", e[4])
        out += struct.pack("<HHI", tag, typ, count) + field
    out += struct.pack("<I", 0)
    assert len(out) == data_start
    return bytes(out + sections)


def _build_segmented(width, height, segments, bits, tile, rows_per_strip, strip_tags, cfa_repeat, cfa_pattern,
                     overrides, drop):
    """A Compression 7 file: the base tag set with the data split into
    segments, whose offset arrays are filled in once the data is placed."""
    n = len(segments)
    sizes = [len(x) for x in segments]
    ov = {259: (SHORT, [7])}
    if tile is not None:
        ov.update({322: (LONG, [tile[0]]), 323: (LONG, [tile[1]]), 324: (LONG, [0] * n), 325: (LONG, sizes)})
        if not strip_tags:
            drop = tuple(drop) + (273, 279, 278)
    else:
        ov.update({273: (LONG, [0] * n), 278: (LONG, [rows_per_strip or height]), 279: (LONG, sizes)})
    ov.update(overrides or {})
    marker = b"SEGMENTDATA!"
    base = build_dng(width, height, strip=marker, bits=bits, cfa_repeat=cfa_repeat, cfa_pattern=cfa_pattern,
                     overrides=ov, drop=drop)
    # the base file holds `marker` where the single strip would be: replace it
    # by the segments (16-byte aligned each) and patch the offsets
    at = base.index(marker)
    out = bytearray(base[:at])
    offsets = []
    for seg in segments:
        while len(out) % 16:
            out.append(0)
        offsets.append(len(out))
        out += seg
    ifd = struct.unpack_from("<I", out, 4)[0]
    count = struct.unpack_from("<H", out, ifd)[0]
    for k in range(count):
        e = ifd + 2 + 12 * k
        tag, typ, cnt = struct.unpack_from("<HHI", out, e)
        if (tile is None and tag == 273) or (tile is not None and tag == 324):
            vals = struct.pack("<%dI" % cnt, *offsets[:cnt])
        elif tile is not None and tag == 273:
            vals = struct.pack("<I", offsets[0])
        elif tile is not None and tag == 279:
            vals = struct.pack("<I", sizes[0])
        else:
            continue
        if len(vals) <= 4:
            out[e + 8:e + 12] = vals + b"\0" * (4 - len(vals))
        else:
            where = struct.unpack_from("<I", out, e + 8)[0]
            out[where:where + len(vals)] = vals
    return bytes(out)


# ------------------------------------------------------- lossless-JPEG segments
# Code lengths of difference categories 0..16 for the writer below: a fixed,
# prefix-free table (Kraft sum 0.875, so no code is all ones) that favours the
# small categories of smooth raw data.  Decoders read it from the DHT segment.
_LJ_LENGTHS = (2, 3, 3, 3, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)


def _huffman_lengths(freq):
    """Code lengths of at most 16 bits for the categories with freq > 0:
    Huffman's construction over them plus one reserved, least frequent point
    (so that no code is all ones), lengths over 16 folded back and the reserved
    point then dropped from the longest length, as T.81 Annex K.2 describes."""
    syms = [s for s in range(17) if freq[s] > 0] or [0]
    heap = [(int(freq[s]), i, (s,)) for i, s in enumerate(syms)] + [(0, len(syms), (17,))]
    heapq.heapify(heap)
    depth = dict.fromkeys(list(syms) + [17], 0)
    k = len(heap)
    while len(heap) > 1:
        fa, _, a = heapq.heappop(heap)
        fb, _, b = heapq.heappop(heap)
        for s in a + b:
            depth[s] += 1
        heapq.heappush(heap, (fa + fb, k, a + b))
        k += 1
    bits = [0] * 64
    for d in depth.values():
        bits[d] += 1
    for i in range(63, 16, -1):
        while bits[i] > 0:
            j = i - 2
            while bits[j] == 0:
                j -= 1
            bits[i] -= 2
            bits[i - 1] += 1
            bits[j + 1] += 2
            bits[j] -= 1
    longest = max(i for i in range(17) if bits[i])
    bits[longest] -= 1
    order = iter(sorted(syms, key=lambda s: (-int(freq[s]), s)))
    return {next(order): n for n in range(1, 17) for _ in range(bits[n])}


def _canonical_codes(lengths):
    """(code, length) arrays over categories 0..16 and the DHT symbol order."""
    order = sorted(lengths, key=lambda s: (lengths[s], s))
    code_of, code_len = np.zeros(17, np.int64), np.zeros(17, np.int64)
    code, prev = 0, lengths[order[0]]
    for sym in order:
        code <<= lengths[sym] - prev
        prev = lengths[sym]
        code_of[sym], code_len[sym] = code, prev
        code += 1
    counts = [0] * 16
    for sym in order:
        counts[lengths[sym] - 1] += 1
    return code_of, code_len, bytes(counts) + bytes(order)


def lj92_segment(samples, bits, components=2, tables="fixed"):
    """One lossless-JPEG stream (ITU-T T.81 process 14, DNG Compression 7) for a
    raster of uint16 samples laid out as JPEG lines of X * components samples:
    predictor 1, no restart intervals.  tables="fixed": one fixed Huffman table
    for every component; "per_component": an optimal table per component from
    its own category counts, as DNG writers emit.  For synthetic benchmark and
    test files; `samples` is (rows, X * components)."""
    a = np.asarray(samples, np.int64)
    rows, cols = a.shape
    X = cols // components
    r = a.reshape(rows, X, components)
    pred = np.empty_like(r)
    pred[0, 0] = 1 << (bits - 1)
    pred[0, 1:] = r[0, :-1]
    pred[1:, 0] = r[:-1, 0]
    pred[1:, 1:] = r[1:, :-1]
    diff = (r - pred) & 0xFFFF
    diff = np.where(diff > 0x8000, diff - 0x10000, diff).reshape(-1)
    mag = np.abs(diff)
    cat = np.where(mag == 0, 0, np.frexp(mag.astype(np.float64))[1]).astype(np.int64)
    cat[mag == 32768] = 16
    comp = np.arange(diff.size) % components
    if tables == "fixed":
        lengths = [dict(enumerate(_LJ_LENGTHS))]
    elif tables == "per_component":
        lengths = [_huffman_lengths(np.bincount(cat[comp == c], minlength=17)) for c in range(components)]
    else:
        raise ValueError("tables must be 'fixed' or 'per_component'")
    made = [_canonical_codes(ln) for ln in lengths]
    code_of = np.stack([m[0] for m in made])
    code_len = np.stack([m[1] for m in made])
    tsel = comp if len(made) > 1 else np.zeros_like(comp)
    n_extra = np.where(cat < 16, cat, 0)
    extra = np.where(diff >= 0, diff, diff + (1 << cat) - 1) & ((1 << n_extra) - 1)
    # one field per sample: the category's code followed by its extra bits
    field = (code_of[tsel, cat] << n_extra) | extra
    flen = code_len[tsel, cat] + n_extra
    end = np.cumsum(flen)
    nbits = int(end[-1]) if end.size else 0
    total = (nbits + 7) // 8 * 8
    bitbuf = np.ones(total, np.uint8)  # the tail pads with one bits
    start = end - flen
    for k in range(int(flen.max()) if flen.size else 0):
        sel = flen > k
        bitbuf[start[sel] + k] = (field[sel] >> (flen[sel] - 1 - k)) & 1
    data = np.packbits(bitbuf)
    data = np.insert(data, np.nonzero(data == 0xFF)[0] + 1, 0)  # byte stuffing
    marker = lambda m, body: bytes((0xFF, m)) + struct.pack(">H", len(body) + 2) + body
    dht = b"".join(bytes([t]) + m[2] for t, m in enumerate(made))
    sof = struct.pack(">BHHB", bits, rows, X, components) + b"".join(bytes((c + 1, 0x11, 0))
                                                                     for c in range(components))
    td = [c if len(made) > 1 else 0 for c in range(components)]
    sos = bytes([components]) + b"".join(bytes((c + 1, td[c] << 4)) for c in range(components)) + bytes((1, 0, 0))
    return (b"\xff\xd8" + marker(0xC4, dht) + marker(0xC3, sof) + marker(0xDA, sos) + data.tobytes() + b"\xff\xd9")


def lj92_tiles(img, bits, tile_w, tile_h, components=2, tables="fixed"):
    """lj92_segment of every tile_w x tile_h tile of `img`, row-major, the edge
    tiles padded by repeating the last row / column (DNG tiles are whole)."""
    img = np.asarray(img, np.uint16)
    h, w = img.shape
    across, down = -(-w // tile_w), -(-h // tile_h)
    pad = np.pad(img, ((0, down * tile_h - h), (0, across * tile_w - w)), mode="edge")
    return [lj92_segment(pad[ty * tile_h:(ty + 1) * tile_h, tx * tile_w:(tx + 1) * tile_w], bits, components,
                         tables) for ty in range(down) for tx in range(across)]


# Tags a DNG keeps in IFD0 when the raw image sits in a SubIFD: camera,
# colour and capture metadata, Exif / XMP / ICC (DNG 1.4 specification).
_CAMERA_TAGS = (271, 272, 274, 700, 33434, 33437, 34665, 34675, 34855, 37386, 50706, 50707, 50708, 50721, 50722,
                50728, 50778, 50779, 50964, 50965)


def subifd_dng(dng, thumb=(8, 6)):
    """The DNG `dng` (raw image in IFD0, as build_dng writes it) rewritten in
    the layout of camera and converter DNGs: IFD0 a small RGB preview
    (NewSubFileType 1) carrying the camera tags and a SubIFDs tag, the raw
    image's tags (NewSubFileType 0) in that SubIFD.  Data stay where they
    were; the new IFDs and the preview strip are appended."""
    b = bytearray(dng)
    ifd0 = struct.unpack_from("<I", b, 4)[0]
    n = struct.unpack_from("<H", b, ifd0)[0]
    entries = [bytes(b[ifd0 + 2 + 12 * k: ifd0 + 14 + 12 * k]) for k in range(n)]
    tag_of = lambda e: struct.unpack_from("<H", e)[0]
    camera = [e for e in entries if tag_of(e) in _CAMERA_TAGS]
    image = [e for e in entries if tag_of(e) not in _CAMERA_TAGS and tag_of(e) != 254]
    image.append(struct.pack("<HHII", 254, LONG, 1, 0))

    def append_ifd(ents):
        while len(b) % 2:
            b.append(0)
        at = len(b)
        ents = sorted(ents, key=tag_of)
        b.extend(struct.pack("<H", len(ents)) + b"".join(ents) + struct.pack("<I", 0))
        return at

    raw_ifd = append_ifd(image)
    tw, th = thumb
    while len(b) % 2:
        b.append(0)
    bits_at = len(b)
    b.extend(struct.pack("<HHH", 8, 8, 8))
    strip_at = len(b)
    b.extend(bytes((x * 37) & 0xFF for x in range(tw * th * 3)))
    preview = camera + [
        struct.pack("<HHII", 254, LONG, 1, 1), struct.pack("<HHII", 256, LONG, 1, tw),
        struct.pack("<HHII", 257, LONG, 1, th), struct.pack("<HHII", 258, SHORT, 3, bits_at),
        struct.pack("<HHIHH", 259, SHORT, 1, 1, 0), struct.pack("<HHIHH", 262, SHORT, 1, 2, 0),
        struct.pack("<HHII", 273, LONG, 1, strip_at), struct.pack("<HHIHH", 277, SHORT, 1, 3, 0),
        struct.pack("<HHII", 278, LONG, 1, th), struct.pack("<HHII", 279, LONG, 1, tw * th * 3),
        struct.pack("<HHII", 330, LONG, 1, raw_ifd),
    ]
    struct.pack_into("<I", b, 4, append_ifd(preview))
    return bytes(b)
