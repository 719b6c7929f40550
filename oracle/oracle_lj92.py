"""Lossless JPEG (ITU-T T.81 process 14, "LJ92"), the DNG Compression 7 codec.

TEST INFRASTRUCTURE: the encoder makes Compression 7 test files; the decoder
is the checker of the GPU decode.  Neither is imported by the product.

Parity unpinned: the reference decodes compressed DNGs through LibRaw (vcpkg
dependency `libraw`, absent from the reference tree; DngReader.cpp:113-124)
and holds no Compression 7 test files, so this is a restatement of the
published standard, not of a reference file, checked by round trips against
two encoders (this one and cpipe_b200.dng_synth.lj92_segment):

  * markers SOI, SOF3 (precision P, lines Y, samples per line X, Nf
    components, each H = V = 1), DHT (class 0 tables), SOS (Ns = Nf, table
    per component, Ss = predictor 1..7, Se = 0, Al = point transform Pt),
    optional DRI (restart interval Ri in MCUs), EOI (T.81 B.1-B.2);
  * entropy-coded differences: Huffman category SSSS then SSSS extra bits,
    EXTEND as T.81 F.2.2.1, SSSS = 16 meaning 32768 with no extra bits
    (H.1.2.2); 0xFF bytes stuffed with 0x00; RSTm markers between intervals;
  * prediction (T.81 H.1.2.1): the first sample of the scan and of every
    restart interval 2^(P-Pt-1); the rest of that line Ra; the first sample of
    other lines Rb; otherwise predictor Ss: 1 Ra, 2 Rb, 3 Rc, 4 Ra+Rb-Rc,
    5 Ra+((Rb-Rc)>>1), 6 Rb+((Ra-Rc)>>1), 7 (Ra+Rb)>>1; sample = (pred + diff)
    mod 2^16, shifted left by Pt;
  * DNG layout (DNG 1.4 spec, "Compression = 7"): the decoded samples, X * Nf
    per JPEG line, fill the tile (or strip) raster row after row.
"""
import heapq
import struct

import numpy as np

SOI, SOF3, DHT, SOS, DRI, EOI = 0xD8, 0xC3, 0xC4, 0xDA, 0xDD, 0xD9


# ------------------------------------------------------------------ encoder
def _category(d):
    d = int(d)
    if d == 0:
        return 0
    if d == 32768 or d == -32768:
        return 16
    return abs(d).bit_length()


def _code_lengths(freq):
    """Huffman code lengths (<= 16) for symbols with freq > 0, one code point
    reserved so that no code is all ones (T.81 K.2)."""
    syms = [s for s in range(17) if freq[s] > 0]
    if len(syms) == 1:
        return {syms[0]: 1}
    heap = [(freq[s], i, (s,)) for i, s in enumerate(syms)]
    heap.append((0, len(syms), (-1,)))  # the reserved all-ones point
    heapq.heapify(heap)
    depth = {s: 0 for s in syms + [-1]}
    k = len(syms) + 1
    while len(heap) > 1:
        fa, _, a = heapq.heappop(heap)
        fb, _, b = heapq.heappop(heap)
        for s in a + b:
            depth[s] += 1
        heapq.heappush(heap, (fa + fb, k, a + b))
        k += 1
    bits = [0] * 40
    for s, d in depth.items():
        bits[d] += 1
    # limit to 16 bits (T.81 K.3 Adjust_BITS)
    for i in range(39, 16, -1):
        while bits[i] > 0:
            j = i - 2
            while bits[j] == 0:
                j -= 1
            bits[i] -= 2
            bits[i - 1] += 1
            bits[j + 1] += 2
            bits[j] -= 1
    i = 16
    while bits[i] == 0:
        i -= 1
    bits[i] -= 1  # drop the reserved point
    order = sorted(syms, key=lambda s: (depth[s], s))
    lengths, pos = {}, 0
    for length in range(1, 17):
        for _ in range(bits[length]):
            lengths[order[pos]] = length
            pos += 1
    return lengths


def _canonical(lengths):
    """symbol -> (code, length), canonical order (T.81 C.2)."""
    codes, code, prev = {}, 0, 0
    for s in sorted(lengths, key=lambda s: (lengths[s], s)):
        code <<= lengths[s] - prev
        prev = lengths[s]
        codes[s] = (code, prev)
        code += 1
    return codes


def _predict(rows, y, x, c, nf, ps, first_line, p_bits, pt):
    if first_line and x == 0:
        return 1 << (p_bits - pt - 1)
    if first_line:
        return rows[y][(x - 1) * nf + c]
    if x == 0:
        return rows[y - 1][c]
    ra, rb, rc = rows[y][(x - 1) * nf + c], rows[y - 1][x * nf + c], rows[y - 1][(x - 1) * nf + c]
    return [0, ra, rb, rc, ra + rb - rc, ra + ((rb - rc) >> 1), rb + ((ra - rc) >> 1), (ra + rb) >> 1][ps]


def encode(tile, bits, predictor=1, components=2, restart=0):
    """LJ92 stream of `tile` (h x w uint16, values < 2**bits): JPEG lines of
    X = w / components samples per component (the tile's rows in order)."""
    tile = np.asarray(tile, np.int64)
    h, w = tile.shape
    assert w % components == 0
    X, Y, nf = w // components, h, components
    rows = tile.reshape(Y, X * nf).tolist()
    diffs, restarts_at = [], set()
    mcu, first_line_y, reset = 0, 0, True
    for y in range(Y):
        for x in range(X):
            if restart and mcu and mcu % restart == 0:
                restarts_at.add(len(diffs))
                first_line_y, reset = y, True
            for c in range(nf):
                if reset:
                    p = 1 << (bits - 1)
                else:
                    p = _predict(rows, y, x, c, nf, predictor, y == first_line_y, bits, 0)
                d = (rows[y][x * nf + c] - p) & 0xFFFF
                if d > 0x8000:
                    d -= 0x10000
                diffs.append((c, d))
            reset = False
            mcu += 1
    freq = [0] * 17
    for _, d in diffs:
        freq[_category(d)] += 1
    lengths = _code_lengths(freq)
    codes = _canonical(lengths)
    # entropy-coded segment with stuffing and restart markers
    out, acc, nacc, rst = bytearray(), 0, 0, 0

    def put(v, n):
        nonlocal acc, nacc
        acc = (acc << n) | (v & ((1 << n) - 1))
        nacc += n
        while nacc >= 8:
            b = (acc >> (nacc - 8)) & 0xFF
            out.append(b)
            if b == 0xFF:
                out.append(0)
            nacc -= 8

    def flush():
        nonlocal nacc, acc
        if nacc:
            put((1 << (8 - nacc)) - 1, 8 - nacc)
        acc = 0

    for i, (c, d) in enumerate(diffs):
        if i in restarts_at:
            flush()
            out.extend((0xFF, 0xD0 + (rst & 7)))
            rst += 1
        s = _category(d)
        code, n = codes[s]
        put(code, n)
        if 0 < s < 16:
            put(d if d >= 0 else d + (1 << s) - 1, s)
    flush()
    # headers
    counts = [0] * 16
    for s in lengths.values():
        counts[s - 1] += 1
    vals = sorted(lengths, key=lambda s: (lengths[s], s))
    dht = bytes([0x00]) + bytes(counts) + bytes(vals)
    seg = lambda m, body: bytes((0xFF, m)) + struct.pack(">H", len(body) + 2) + body
    sof = struct.pack(">BHHB", bits, Y, X, nf) + b"".join(bytes((c + 1, 0x11, 0)) for c in range(nf))
    sos = bytes([nf]) + b"".join(bytes((c + 1, 0x00)) for c in range(nf)) + bytes((predictor, 0, 0))
    stream = bytes((0xFF, SOI)) + seg(DHT, dht) + seg(SOF3, sof)
    if restart:
        stream += seg(DRI, struct.pack(">H", restart))
    return stream + seg(SOS, sos) + bytes(out) + bytes((0xFF, EOI))


# ------------------------------------------------------------------ decoder
class Lj92Error(ValueError):
    pass


def _headers(stream):
    if stream[:2] != b"\xff\xd8":
        raise Lj92Error("no SOI")
    pos, tables, frame, scan, restart = 2, {}, None, None, 0
    while pos + 4 <= len(stream):
        if stream[pos] != 0xFF:
            raise Lj92Error("marker expected")
        m = stream[pos + 1]
        n = struct.unpack_from(">H", stream, pos + 2)[0]
        body = stream[pos + 4:pos + 2 + n]
        if m == DHT:
            q = 0
            while q < len(body):
                tc_th = body[q]
                counts = list(body[q + 1:q + 17])
                vals = list(body[q + 17:q + 17 + sum(counts)])
                tables[tc_th & 0x0F] = (counts, vals)
                q += 17 + sum(counts)
        elif m == SOF3:
            p, y, x, nf = struct.unpack_from(">BHHB", body, 0)
            frame = (p, y, x, nf, [body[6 + 3 * i] for i in range(nf)])
        elif m == DRI:
            restart = struct.unpack_from(">H", body, 0)[0]
        elif m == SOS:
            ns = body[0]
            comps = [(body[1 + 2 * i], body[2 + 2 * i] >> 4) for i in range(ns)]
            ss, al = body[1 + 2 * ns], body[3 + 2 * ns] & 0x0F
            scan = (comps, ss, al)
            return tables, frame, scan, restart, pos + 2 + n
        elif m in (0xC0, 0xC1, 0xC2, 0xC5, 0xC6, 0xC7, 0xC9, 0xCA, 0xCB):
            raise Lj92Error("not a lossless Huffman frame")
        pos += 2 + n
    raise Lj92Error("no SOS")


class _Bits:
    def __init__(self, data, pos):
        self.d, self.p, self.acc, self.n = data, pos, 0, 0

    def bit(self):
        if self.n == 0:
            b = self.d[self.p] if self.p < len(self.d) else 0
            if b == 0xFF:
                nxt = self.d[self.p + 1] if self.p + 1 < len(self.d) else 0
                if nxt == 0:
                    self.p += 2
                else:
                    b = 0  # a marker: zeros past it
            else:
                self.p += 1
            self.acc, self.n = b, 8
        self.n -= 1
        return (self.acc >> self.n) & 1

    def bits(self, k):
        v = 0
        for _ in range(k):
            v = (v << 1) | self.bit()
        return v

    def restart(self):
        self.n = 0
        while self.p + 1 < len(self.d) and not (self.d[self.p] == 0xFF and 0xD0 <= self.d[self.p + 1] <= 0xD7):
            self.p += 1
        self.p += 2


def decode(stream, tile_w, tile_h):
    """Samples of one LJ92 stream laid into a tile_h x tile_w uint16 raster."""
    tables, frame, scan, restart, pos = _headers(bytes(stream))
    p_bits, Y, X, nf, ids = frame
    comps, ps, pt = scan
    tsel = {cid: t for cid, t in comps}
    dec = []
    for cid in ids:
        counts, vals = tables[tsel[cid]]
        maxcode, valptr, mincode, code, k = [-1] * 17, [0] * 17, [0] * 17, 0, 0
        for length in range(1, 17):
            if counts[length - 1]:
                valptr[length] = k
                mincode[length] = code
                code += counts[length - 1]
                k += counts[length - 1]
                maxcode[length] = code - 1
            code <<= 1
        dec.append((maxcode, valptr, mincode, vals))
    br = _Bits(bytes(stream), pos)
    rows = [[0] * (X * nf) for _ in range(Y)]
    mcu, first_line_y, reset = 0, 0, True
    for y in range(Y):
        for x in range(X):
            if restart and mcu and mcu % restart == 0:
                br.restart()
                first_line_y, reset = y, True
            for c in range(nf):
                maxcode, valptr, mincode, vals = dec[c]
                code, length = br.bit(), 1
                while code > maxcode[length]:
                    code = (code << 1) | br.bit()
                    length += 1
                    if length > 16:
                        raise Lj92Error("bad Huffman code")
                s = vals[valptr[length] + code - mincode[length]]
                if s == 0:
                    d = 0
                elif s == 16:
                    d = 32768
                else:
                    v = br.bits(s)
                    d = v if v >= (1 << (s - 1)) else v - (1 << s) + 1
                first = y == first_line_y
                if reset:
                    pred = 1 << (p_bits - pt - 1)
                else:
                    pred = _predict(rows, y, x, c, nf, ps, first, p_bits, pt)
                rows[y][x * nf + c] = (pred + d) & 0xFFFF
            reset = False
            mcu += 1
    flat = np.array(rows, np.int64).ravel()
    out = np.zeros(tile_h * tile_w, np.uint16)
    n = min(out.size, flat.size)
    out[:n] = (flat[:n] << pt) & 0xFFFF
    return out.reshape(tile_h, tile_w)


def decode_tiles(segments, width, height, tile_w, tile_h):
    """An image from its tiles (row-major tile order, each an LJ92 stream),
    the tiles past the right and bottom edges cropped."""
    across = (width + tile_w - 1) // tile_w
    img = np.zeros((height, width), np.uint16)
    for i, seg in enumerate(segments):
        ty, tx = divmod(i, across)
        t = decode(seg, tile_w, tile_h)
        y0, x0 = ty * tile_h, tx * tile_w
        hh, ww = min(tile_h, height - y0), min(tile_w, width - x0)
        if hh > 0 and ww > 0:
            img[y0:y0 + hh, x0:x0 + ww] = t[:hh, :ww]
    return img


def encode_tiles(img, bits, tile_w, tile_h, predictor=1, components=2, restart=0):
    """LJ92 streams of every tile of `img` (edge tiles padded by repeating the
    last column / row, as DNG writers pad)."""
    h, w = img.shape
    across, down = (w + tile_w - 1) // tile_w, (h + tile_h - 1) // tile_h
    pad = np.pad(np.asarray(img, np.uint16), ((0, down * tile_h - h), (0, across * tile_w - w)), mode="edge")
    return [encode(pad[ty * tile_h:(ty + 1) * tile_h, tx * tile_w:(tx + 1) * tile_w], bits, predictor, components,
                   restart) for ty in range(down) for tx in range(across)]


def encode_fast(tile, bits, components=2):
    """encode(tile, bits, predictor=1, components, restart=0), vectorised with
    numpy (the same bytes): for large test frames."""
    tile = np.asarray(tile, np.int64)
    h, w = tile.shape
    X, nf = w // components, components
    r = tile.reshape(h, X, nf)
    pred = np.empty_like(r)
    pred[0, 0, :] = 1 << (bits - 1)
    pred[0, 1:, :] = r[0, :-1, :]          # first line: Ra
    pred[1:, 0, :] = r[:-1, 0, :]          # first column: Rb
    pred[1:, 1:, :] = r[1:, :-1, :]        # predictor 1: Ra
    d = (r - pred) & 0xFFFF
    d = np.where(d > 0x8000, d - 0x10000, d).ravel()
    cat = np.zeros(d.size, np.int64)
    nz = d != 0
    cat[nz] = np.floor(np.log2(np.abs(d[nz]))).astype(np.int64) + 1
    cat[np.abs(d) == 32768] = 16
    freq = np.bincount(cat, minlength=17).tolist()
    lengths = _code_lengths(freq)
    codes = _canonical(lengths)
    code_v = np.zeros(17, np.int64)
    code_n = np.zeros(17, np.int64)
    for sym, (c, n) in codes.items():
        code_v[sym], code_n[sym] = c, n
    extra_n = np.where((cat > 0) & (cat < 16), cat, 0)
    extra_v = np.where(d >= 0, d, d + (1 << cat) - 1) & ((1 << extra_n) - 1)
    # interleave (code, extra) fields and pack MSB first
    vals = np.stack([code_v[cat], extra_v], 1).ravel()
    lens = np.stack([code_n[cat], extra_n], 1).ravel()
    total = int(lens.sum())
    pad = (-total) % 8
    vals = np.append(vals, (1 << pad) - 1)
    lens = np.append(lens, pad)
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
    nbits = total + pad
    bitarr = np.zeros(nbits, np.uint8)
    for k in range(1, 17):
        sel = lens >= k
        bitarr[(starts[sel] + lens[sel] - k)] = (vals[sel] >> (k - 1)) & 1
    data = np.packbits(bitarr)
    ff = np.nonzero(data == 0xFF)[0]
    data = np.insert(data, ff + 1, 0)
    counts = [0] * 16
    for s_ in lengths.values():
        counts[s_ - 1] += 1
    syms = sorted(lengths, key=lambda s_: (lengths[s_], s_))
    dht = bytes([0x00]) + bytes(counts) + bytes(syms)
    seg = lambda m, body: bytes((0xFF, m)) + struct.pack(">H", len(body) + 2) + body
    sof = struct.pack(">BHHB", bits, h, X, nf) + b"".join(bytes((c + 1, 0x11, 0)) for c in range(nf))
    sos = bytes([nf]) + b"".join(bytes((c + 1, 0x00)) for c in range(nf)) + bytes((1, 0, 0))
    return (bytes((0xFF, SOI)) + seg(DHT, dht) + seg(SOF3, sof) + seg(SOS, sos) + data.tobytes() +
            bytes((0xFF, EOI)))


def encode_tiles_fast(img, bits, tile_w, tile_h, components=2):
    h, w = img.shape
    across, down = (w + tile_w - 1) // tile_w, (h + tile_h - 1) // tile_h
    pad = np.pad(np.asarray(img, np.uint16), ((0, down * tile_h - h), (0, across * tile_w - w)), mode="edge")
    return [encode_fast(pad[ty * tile_h:(ty + 1) * tile_h, tx * tile_w:(tx + 1) * tile_w], bits, components)
            for ty in range(down) for tx in range(across)]
