// Host parse of a DNG's IFD0: the tags the reference's ingest reads, into
// cpipe_DngInfo.  Follows cpipe::ingest::dng_opcode::OpcodeListParser::parse
// (src/cpipe/ingest/dng_opcode/OpcodeListParser.cpp:330-515) decision for
// decision: the same header check, the same IFD bounds, the same per-type value
// reads (OpcodeListParser.cpp:84-278) and the same status for each rejection.
//
// One extension, for files the reference rejects: when IFD0 is not a
// single-plane CFA image (a camera or converter DNG whose IFD0 is the preview),
// the first SubIFD (tag 330) that is a full-resolution (NewSubFileType 0)
// single-plane CFA image supplies the image tags -- size, depth, compression,
// strips / tiles, CFA, black and white levels, linearization, active area,
// opcode lists -- while the camera tags stay IFD0's (make, model, orientation,
// illuminants, matrices, as-shot neutral, Exif, XMP, ICC), as the DNG
// specification places them.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/cpipe_b200_dng.h"
#include "../../include/cpipe_node_abi.h"

namespace cpb {
void set_error(const char* fmt, const char* detail);
}

namespace {

enum : uint16_t {
    kByte = 1, kAscii = 2, kShort = 3, kLong = 4, kRational = 5, kUndefined = 7, kSRational = 10,
};
enum : uint16_t {
    kTagWidth = 256, kTagLength = 257, kTagBits = 258, kTagCompression = 259, kTagPhotometric = 262,
    kTagNewSubFileType = 254, kTagMake = 271, kTagModel = 272, kTagStripOffsets = 273, kTagOrientation = 274, kTagSamples = 277,
    kTagRowsPerStrip = 278, kTagStripByteCounts = 279, kTagTileWidth = 322, kTagTileLength = 323,
    kTagTileOffsets = 324, kTagTileByteCounts = 325, kTagSubIfds = 330, kTagXmp = 700, kTagCfaRepeat = 33421, kTagCfaPattern = 33422,
    kTagExposure = 33434, kTagFNumber = 33437, kTagExifIfd = 34665, kTagIcc = 34675, kTagIso = 34855,
    kTagFocal = 37386, kTagLinearization = 50712, kTagBlack = 50714, kTagWhite = 50717,
    kTagColorMatrix1 = 50721, kTagColorMatrix2 = 50722, kTagAsShotNeutral = 50728,
    kTagIlluminant1 = 50778, kTagIlluminant2 = 50779, kTagActiveArea = 50829,
    kTagForwardMatrix1 = 50964, kTagForwardMatrix2 = 50965,
    kTagOpcodeList1 = 51008, kTagOpcodeList2 = 51009, kTagOpcodeList3 = 51022,
};
constexpr uint32_t kPhotometricCfa = 32803;
constexpr int kMaxEntries = 65535;

struct Tiff {
    const uint8_t* b;
    uint64_t n;
    uint32_t u16(uint64_t o) const { return (uint32_t)b[o] | ((uint32_t)b[o + 1] << 8); }
    uint32_t u32(uint64_t o) const { return u16(o) | (u16(o + 2) << 16); }
};

struct Entry {
    uint16_t tag = 0, type = 0;
    uint32_t count = 0, value = 0;
};

uint32_t type_bytes(uint16_t t) {
    switch (t) {
        case kByte: case kAscii: case kUndefined: return 1;
        case kShort: return 2;
        case kLong: return 4;
        case kRational: case kSRational: return 8;
        default: return 0;
    }
}

// A value's bytes: inline in the entry when they fit in four, else at the
// entry's offset.  `len` = 0 when the type is unknown, the count is zero or
// the bytes fall outside the file.
struct Span {
    const uint8_t* p = nullptr;
    uint64_t len = 0;
    uint64_t file_offset = 0;  // where the bytes sit in the file (inline: the entry's value field)
    uint8_t inl[4] = {0, 0, 0, 0};
};

Span value_bytes(const Tiff& t, const Entry& e, uint64_t entry_pos) {
    Span s;
    const uint64_t item = type_bytes(e.type);
    const uint64_t len = (uint64_t)e.count * item;
    if (item == 0 || len == 0 || len > t.n) return s;
    if (len <= 4) {
        for (int i = 0; i < 4; ++i) s.inl[i] = (uint8_t)((e.value >> (8 * i)) & 0xFFu);
        s.p = s.inl;
        s.len = len;
        s.file_offset = entry_pos + 8;
        return s;
    }
    if (e.value > t.n || len > t.n - e.value) return s;
    s.p = t.b + e.value;
    s.len = len;
    s.file_offset = e.value;
    return s;
}

uint32_t rd16(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
uint32_t rd32(const uint8_t* p) { return rd16(p) | (rd16(p + 2) << 16); }

struct Ifd {
    std::vector<Entry> e;
    std::vector<uint64_t> pos;  // file offset of each entry
    const Entry* find(uint16_t tag, uint64_t* where = nullptr) const {
        for (size_t i = 0; i < e.size(); ++i)
            if (e[i].tag == tag) {
                if (where) *where = pos[i];
                return &e[i];
            }
        return nullptr;
    }
};

// Reads the whole entry table at `off` (up to 65535 entries, as the count field
// allows); find() returns the first entry of a tag, as a linear search over the
// table does.
bool read_ifd(const Tiff& t, uint64_t off, Ifd* out) {
    if (off + 2 > t.n) return false;
    const uint32_t count = t.u16(off);
    if (off + 2 + (uint64_t)count * 12 > t.n) return false;
    out->e.clear();
    out->pos.clear();
    out->e.reserve(count);
    out->pos.reserve(count);
    for (uint32_t i = 0; i < count && i < (uint32_t)kMaxEntries; ++i) {
        const uint64_t o = off + 2 + (uint64_t)i * 12;
        Entry e;
        e.tag = (uint16_t)t.u16(o);
        e.type = (uint16_t)t.u16(o + 2);
        e.count = t.u32(o + 4);
        e.value = t.u32(o + 8);
        out->pos.push_back(o);
        out->e.push_back(e);
    }
    return true;
}

uint32_t first_u32(const Tiff& t, const Ifd& ifd, uint16_t tag, bool* found = nullptr) {
    uint64_t pos = 0;
    const Entry* e = ifd.find(tag, &pos);
    if (found) *found = e != nullptr;
    if (!e) return 0;
    const Span s = value_bytes(t, *e, pos);
    if (s.len == 0) return 0;
    if (e->type == kShort && s.len >= 2) return rd16(s.p);
    if (e->type == kLong && s.len >= 4) return rd32(s.p);
    if (e->type == kByte) return s.p[0];
    return 0;
}

// Integer values of a BYTE / SHORT / LONG entry (empty for other types).
int u32_values(const Tiff& t, const Entry& e, uint64_t pos, uint32_t* out, int cap) {
    const Span s = value_bytes(t, e, pos);
    if (s.len == 0) return 0;
    const uint32_t k = e.type == kByte ? 1 : e.type == kShort ? 2 : e.type == kLong ? 4 : 0;
    if (k == 0) return 0;
    int n = 0;
    for (uint32_t i = 0; i < e.count && n < cap; ++i) {
        const uint8_t* p = s.p + (uint64_t)i * k;
        out[n++] = k == 1 ? p[0] : k == 2 ? rd16(p) : rd32(p);
    }
    return n;
}

// Numeric values as binary32: integers converted, rationals as num / den in
// binary32 (0 for a zero denominator).
int float_values(const Tiff& t, const Ifd& ifd, uint16_t tag, float* out, int cap, bool* found = nullptr) {
    uint64_t pos = 0;
    const Entry* e = ifd.find(tag, &pos);
    if (found) *found = e != nullptr;
    if (!e) return 0;
    if (e->type == kByte || e->type == kShort || e->type == kLong) {
        uint32_t v[16];
        const int n = u32_values(t, *e, pos, v, cap < 16 ? cap : 16);
        for (int i = 0; i < n; ++i) out[i] = (float)v[i];
        return n;
    }
    if (e->type != kRational && e->type != kSRational) return 0;
    const Span s = value_bytes(t, *e, pos);
    if (s.len == 0) return 0;
    int n = 0;
    for (uint32_t i = 0; i < e->count && n < cap; ++i) {
        const uint8_t* p = s.p + (uint64_t)i * 8;
        const float den = e->type == kRational ? (float)rd32(p + 4) : (float)(int32_t)rd32(p + 4);
        const float num = e->type == kRational ? (float)rd32(p) : (float)(int32_t)rd32(p);
        out[n++] = den == 0.0F ? 0.0F : num / den;
    }
    return n;
}

void byte_range(const Tiff& t, const Ifd& ifd, uint16_t tag, uint32_t* off, uint32_t* len) {
    uint64_t pos = 0;
    *off = *len = 0;
    const Entry* e = ifd.find(tag, &pos);
    if (!e) return;
    const Span s = value_bytes(t, *e, pos);
    *off = (uint32_t)s.file_offset;
    *len = (uint32_t)s.len;
}

void ascii(const Tiff& t, const Ifd& ifd, uint16_t tag, char* out) {
    uint64_t pos = 0;
    const Entry* e = ifd.find(tag, &pos);
    if (!e || e->type != kAscii) return;
    const Span s = value_bytes(t, *e, pos);
    uint64_t i = 0;
    for (; i < s.len && i < 63 && s.p[i] != 0; ++i) out[i] = (char)s.p[i];
    out[i] = 0;
}

// ExposureTime, ISOSpeedRatings, FNumber, FocalLength from one IFD
// (OpcodeListParser.cpp:290-318): present tags overwrite earlier values.
void capture_tags(const Tiff& t, const Ifd& ifd, cpipe_DngInfo* d) {
    float v[1];
    bool found = false;
    if (float_values(t, ifd, kTagExposure, v, 1, &found) > 0) d->exposure_time_ns = (int64_t)(v[0] * 1000000000.0F);
    const uint32_t iso = first_u32(t, ifd, kTagIso, &found);
    if (found) d->iso = (int32_t)iso;
    if (float_values(t, ifd, kTagFNumber, v, 1) > 0) d->lens_aperture = v[0];
    if (float_values(t, ifd, kTagFocal, v, 1) > 0) d->lens_focal_length_mm = v[0];
}

int fail(int status, const char* message) {
    cpb::set_error("%s", message);
    return status;
}

}  // namespace

extern "C" int cpipe_dng_parse(const uint8_t* file, size_t file_bytes, cpipe_DngInfo* info) {
    if (info == nullptr || (file == nullptr && file_bytes != 0)) return fail(CPIPE_BAD_INDEX, "null argument");
    cpipe_DngInfo d;
    std::memset(&d, 0, sizeof(d));
    *info = d;
    const Tiff t{file, (uint64_t)file_bytes};
    if (t.n < 8 || file[0] != 'I' || file[1] != 'I' || t.u16(2) != 42)
        return fail(CPIPE_FAILED, "unsupported DNG/TIFF header");
    static thread_local Ifd ifd0, exif, sub;
    if (!read_ifd(t, t.u32(4), &ifd0)) return fail(CPIPE_FAILED, "invalid IFD table");

    bool found = false;
    auto cfa_image = [&](const Ifd& ifd) {
        uint32_t photometric = first_u32(t, ifd, kTagPhotometric, &found);
        if (!found) photometric = kPhotometricCfa;
        uint32_t samples = first_u32(t, ifd, kTagSamples, &found);
        if (!found) samples = 1;
        return photometric == kPhotometricCfa && samples == 1;
    };
    // the IFD that holds the raw image: IFD0, or (extension) a SubIFD
    const Ifd* rif = &ifd0;
    if (!cfa_image(ifd0)) {
        uint64_t where = 0;
        const Entry* subs = ifd0.find(kTagSubIfds, &where);
        if (subs && (subs->type == kLong || subs->type == 13) && subs->count > 0) {
            const uint64_t at = subs->count == 1 ? where + 8 : subs->value;
            for (uint32_t k = 0; k < subs->count && k < 16 && at + 4 * (uint64_t)(k + 1) <= t.n; ++k) {
                if (!read_ifd(t, t.u32(at + 4 * (uint64_t)k), &sub)) continue;
                if (first_u32(t, sub, kTagNewSubFileType) == 0 && cfa_image(sub)) {
                    rif = &sub;
                    break;
                }
            }
        }
    }
    const Ifd& raw = *rif;
    d.compression = first_u32(t, raw, kTagCompression, &found);
    if (!found) d.compression = 1;
    auto unsupported = [&](const char* m) {
        *info = d;
        return fail(CPIPE_UNSUPPORTED, m);
    };
    if (!cfa_image(raw)) return unsupported("only single-plane Bayer CFA DNG is supported in P1");

    d.width = first_u32(t, raw, kTagWidth);
    d.height = first_u32(t, raw, kTagLength);
    d.bits_per_sample = first_u32(t, raw, kTagBits);
    d.strip_offset = first_u32(t, raw, kTagStripOffsets);
    d.strip_byte_count = first_u32(t, raw, kTagStripByteCounts);
    d.orientation = first_u32(t, ifd0, kTagOrientation) & 0xFFu;
    d.white_level = first_u32(t, raw, kTagWhite);
    d.calibration_illuminant[0] = first_u32(t, ifd0, kTagIlluminant1) & 0xFFFFu;
    d.calibration_illuminant[1] = first_u32(t, ifd0, kTagIlluminant2) & 0xFFFFu;
    capture_tags(t, ifd0, &d);
    ascii(t, ifd0, kTagMake, d.make);
    ascii(t, ifd0, kTagModel, d.model);

    // CFA: a SHORT[2] repeat of 2x2 or 4x4, and a pattern of exactly that
    // many bytes (OpcodeListParser.cpp:413-446).
    uint64_t pos = 0;
    const Entry* rep = raw.find(kTagCfaRepeat, &pos);
    if (!rep) return unsupported("DNG is missing CFARepeatPatternDim");
    uint32_t r[4] = {0, 0, 0, 0};
    const int nr = rep->type == kShort ? u32_values(t, *rep, pos, r, 4) : 0;
    if (nr != 2 || rep->count != 2 || r[0] != r[1] || (r[0] != 2 && r[0] != 4))
        return unsupported("only 2x2 Bayer or 4x4 Quad Bayer DNG is supported");
    d.cfa_repeat[0] = r[0];
    d.cfa_repeat[1] = r[1];
    const Entry* pat = raw.find(kTagCfaPattern, &pos);
    bool cfa_ok = false;
    if (pat) {
        const Span s = value_bytes(t, *pat, pos);
        if (s.len == (uint64_t)r[0] * r[1] && s.len <= 16) {
            std::memcpy(d.cfa_pattern, s.p, s.len);
            cfa_ok = true;
        }
    }
    if (!cfa_ok) {
        d.cfa_repeat[0] = d.cfa_repeat[1] = 0;
        return unsupported("DNG is missing a supported CFA pattern");
    }

    float_values(t, raw, kTagBlack, d.black_level, 4);
    const Entry* lin = raw.find(kTagLinearization, &pos);
    if (lin && lin->type == kShort) {
        const Span s = value_bytes(t, *lin, pos);
        if (s.len) {
            d.linearization_offset = (uint32_t)s.file_offset;
            d.linearization_count = lin->count;
        }
    }
    const uint16_t mtags[4] = {kTagColorMatrix1, kTagColorMatrix2, kTagForwardMatrix1, kTagForwardMatrix2};
    for (int m = 0; m < 4; ++m) {
        bool has = false;
        float_values(t, ifd0, mtags[m], d.matrix[m], 9, &has);
        d.has_matrix[m] = has ? 1u : 0u;
    }
    float_values(t, ifd0, kTagAsShotNeutral, d.as_shot_neutral, 3);
    const Entry* aa = raw.find(kTagActiveArea, &pos);
    if (aa) {
        uint32_t v[5];
        const int n = u32_values(t, *aa, pos, v, 5);
        if (n == 4 && aa->count == 4 && v[2] >= v[0] && v[3] >= v[1]) {
            d.has_active_area = 1;
            d.active_area[0] = v[1];
            d.active_area[1] = v[0];
            d.active_area[2] = v[3] - v[1];
            d.active_area[3] = v[2] - v[0];
        }
    }
    const Entry* ex = ifd0.find(kTagExifIfd);
    if (ex) {
        const uint32_t eo = first_u32(t, ifd0, kTagExifIfd);
        if ((uint64_t)eo + 2 <= t.n) {
            const uint64_t len = 2 + (uint64_t)t.u16(eo) * 12 + 4;
            if (len <= t.n && eo <= t.n - len) {
                d.exif_offset = eo;
                d.exif_bytes = (uint32_t)len;
            }
        }
        if (read_ifd(t, eo, &exif)) capture_tags(t, exif, &d);
    }
    byte_range(t, ifd0, kTagXmp, &d.xmp_offset, &d.xmp_bytes);
    byte_range(t, ifd0, kTagIcc, &d.icc_offset, &d.icc_bytes);
    byte_range(t, raw, kTagOpcodeList1, &d.opcode_list_offset[0], &d.opcode_list_bytes[0]);
    byte_range(t, raw, kTagOpcodeList2, &d.opcode_list_offset[1], &d.opcode_list_bytes[1]);
    byte_range(t, raw, kTagOpcodeList3, &d.opcode_list_offset[2], &d.opcode_list_bytes[2]);
    // raw data segments: tiles when present, else strips
    auto array_at = [&](uint16_t tag, uint32_t* where, uint32_t* type, uint32_t* count) {
        uint64_t p = 0;
        const Entry* e = raw.find(tag, &p);
        if (!e || (e->type != kShort && e->type != kLong)) return false;
        const Span s = value_bytes(t, *e, p);
        if (s.len == 0) return false;
        *where = (uint32_t)s.file_offset;
        *type = e->type;
        *count = e->count;
        return true;
    };
    uint32_t n_off = 0, n_cnt = 0;
    if (array_at(kTagTileOffsets, &d.seg_offsets_pos, &d.seg_offsets_type, &n_off) &&
        array_at(kTagTileByteCounts, &d.seg_counts_pos, &d.seg_counts_type, &n_cnt)) {
        d.seg_tiled = 1;
        d.seg_width = first_u32(t, raw, kTagTileWidth);
        d.seg_height = first_u32(t, raw, kTagTileLength);
    } else if (array_at(kTagStripOffsets, &d.seg_offsets_pos, &d.seg_offsets_type, &n_off) &&
               array_at(kTagStripByteCounts, &d.seg_counts_pos, &d.seg_counts_type, &n_cnt)) {
        bool has_rows = false;
        const uint32_t rows = first_u32(t, raw, kTagRowsPerStrip, &has_rows);
        d.seg_width = d.width;
        d.seg_height = has_rows && rows > 0 && rows < d.height ? rows : d.height;
    }
    d.seg_count = n_off < n_cnt ? n_off : n_cnt;
    if (d.seg_width == 0 || d.seg_height == 0) d.seg_count = 0;

    *info = d;
    if (d.width == 0 || d.height == 0 || d.bits_per_sample == 0 || d.bits_per_sample > 16 ||
        d.strip_byte_count == 0)
        return fail(CPIPE_FAILED, "DNG is missing required RAW fields");
    if (d.compression != 1 && d.strip_offset == 0)
        return fail(CPIPE_FAILED, "compressed DNG is missing a raw strip offset");
    return CPIPE_OK;
}
