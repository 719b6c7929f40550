// Host-side parameter preparation done by the node plugins before a kernel
// launch: dual-illuminant white balance (CCT search and matrix blend), the
// colormatrix composition, the big-endian OpcodeList2/OpcodeList3 parsers and
// the .cube/.spi3d LUT loader.  These run once per node invocation on the CPU;
// none of them touches pixels.
#include "host_prep.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

namespace cpb::prep {

// ============================================================ white balance
// Reference: src/cpipe/nodes/wb/wb_dual_illuminant.cpp:79-282 (same helpers in
// wb/WbMetadata.hpp).  The float/double mix of the reference is kept: matrices
// are float, the CCT search and locus are double.
namespace {
constexpr double kCctLo = 1500.0, kCctHi = 10000.0;
constexpr double kGolden = 0.3819660112501051;  // (3 - sqrt 5) / 2
constexpr double kTol = 1.0E-5;

Mat3 blend(const Mat3& a, const Mat3& b, float w) {
    Mat3 o{};
    for (int i = 0; i < 9; ++i) o[i] = (w * a[i]) + ((1.0F - w) * b[i]);
    return o;
}
std::array<double, 2> locus_xy(double t) {
    // Kim et al. cubic-spline fit of the Planckian locus (as in the reference :131-147)
    const double t2 = t * t, t3 = t2 * t;
    double x = (-3.0258469E9 / t3) + (2.1070379E6 / t2) + (0.2226347E3 / t) + 0.240390;
    if (t < 4000.0) x = (-0.2661239E9 / t3) - (0.2343580E6 / t2) + (0.8776956E3 / t) + 0.179910;
    double y = (3.0817580 * x * x * x) - (5.87338670 * x * x) + (3.75112997 * x) - 0.37001483;
    if (t < 2222.0) y = (-1.1063814 * x * x * x) - (1.34811020 * x * x) + (2.18555832 * x) - 0.20219683;
    else if (t < 4000.0) y = (-0.9549476 * x * x * x) - (1.37418593 * x * x) + (2.09137015 * x) - 0.16748867;
    return {x, y};
}
double locus_distance2(const Vec3& n, const Mat3& c1, const Mat3& c2, double t1, double t2, double t) {
    const Mat3 cm = blend(c1, c2, reciprocal_cct_weight(t1, t2, t));
    Mat3 inv;
    if (!invert3(cm, &inv)) return std::numeric_limits<double>::infinity();
    const Vec3 xyz{inv[0] * n[0] + inv[1] * n[1] + inv[2] * n[2], inv[3] * n[0] + inv[4] * n[1] + inv[5] * n[2],
                   inv[6] * n[0] + inv[7] * n[1] + inv[8] * n[2]};
    const double s = (double)(xyz[0] + xyz[1] + xyz[2]);
    if (!std::isfinite(s) || s <= 0.0) return std::numeric_limits<double>::infinity();
    const auto p = locus_xy(t);
    const double dx = (double)xyz[0] / s - p[0], dy = (double)xyz[1] / s - p[1];
    return (dx * dx) + (dy * dy);
}
}  // namespace

float reciprocal_cct_weight(double cct1, double cct2, double cct) {
    const double d = (1.0 / cct1) - (1.0 / cct2);
    if (std::abs(d) <= std::numeric_limits<double>::epsilon()) return 1.0F;
    return (float)std::clamp(((1.0 / cct) - (1.0 / cct2)) / d, 0.0, 1.0);
}

bool invert3(const Mat3& m, Mat3* out) {
    const float det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                      m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (!std::isfinite(det) || std::abs(det) <= std::numeric_limits<float>::epsilon()) return false;
    const float r = 1.0F / det;
    *out = Mat3{(m[4] * m[8] - m[5] * m[7]) * r, (m[2] * m[7] - m[1] * m[8]) * r, (m[1] * m[5] - m[2] * m[4]) * r,
                (m[5] * m[6] - m[3] * m[8]) * r, (m[0] * m[8] - m[2] * m[6]) * r, (m[2] * m[3] - m[0] * m[5]) * r,
                (m[3] * m[7] - m[4] * m[6]) * r, (m[1] * m[6] - m[0] * m[7]) * r, (m[0] * m[4] - m[1] * m[3]) * r};
    return true;
}

bool illuminant_cct(uint16_t code, double* cct) {
    switch (code) {
        case 17: *cct = 2850.0; return true;  // Standard light A
        case 20: *cct = 5500.0; return true;  // D55
        case 21: *cct = 6500.0; return true;  // D65
        case 22: *cct = 7500.0; return true;  // D75
        case 23: *cct = 5000.0; return true;  // D50
        case 24: *cct = 3200.0; return true;  // ISO studio tungsten
        default: return false;
    }
}

// Brent's minimiser (golden section + parabolic interpolation) over
// [1500, 10000] K, at most 80 iterations, tolerance 1e-5*|x| + 1e-5; the
// bookkeeping follows the reference's estimate_scene_cct step for step.
double estimate_scene_cct(const Vec3& n, const Mat3& c1, const Mat3& c2, double t1, double t2) {
    double a = kCctLo, b = kCctHi;
    double x = 0.5 * (kCctLo + kCctHi), v = x, w = x;
    double fx = locus_distance2(n, c1, c2, t1, t2, x), fv = fx, fw = fx;
    double d = 0.0, e = 0.0;  // current step, step before last
    for (int it = 0; it < 80; ++it) {
        const double xm = 0.5 * (a + b);
        const double tol = (kTol * std::abs(x)) + kTol;
        if (std::abs(x - xm) <= (2.0 * tol) - (0.5 * (b - a))) break;
        bool golden = true;
        if (std::abs(e) > tol) {
            const double r = (x - w) * (fx - fv);
            const double q0 = (x - v) * (fx - fw);
            double p = ((x - v) * q0) - ((x - w) * r);
            const double q = 2.0 * (q0 - r);
            if (q > 0.0) {
                p = -p;
                const double e_old = e;
                e = d;
                if (!(std::abs(p) >= std::abs(0.5 * q * e_old) || p <= q * (a - x) || p >= q * (b - x))) {
                    double step = p / q;
                    const double u = x + step;
                    if ((u - a) < (2.0 * tol) || (b - u) < (2.0 * tol)) step = std::copysign(tol, xm - x);
                    d = step;
                    golden = false;
                }
            }
        }
        if (golden) {
            e = x < xm ? b - x : a - x;
            d = kGolden * e;
        }
        const double u = x + (std::abs(d) >= tol ? d : std::copysign(tol, d));
        const double fu = locus_distance2(n, c1, c2, t1, t2, u);
        if (fu <= fx) {
            if (u < x) b = x; else a = x;
            v = w; fv = fw;
            w = x; fw = fx;
            x = u; fx = fu;
        } else {
            if (u < x) a = u; else b = u;
            if (fu <= fw || w == x) {
                v = w; fv = fw;
                w = u; fw = fu;
            } else if (fu <= fv || v == x || v == w) {
                v = u; fv = fu;
            }
        }
    }
    return x;
}

int wb_prepare(const Vec3& neutral, const Mat3* cm1, const Mat3* cm2, const Mat3* fm1, const Mat3* fm2,
               uint16_t illum1, uint16_t illum2, cpipe_WbParams* out, double* scene_cct) {
    if (!cm1 || !cm2) return CPIPE_NEED_METADATA;
    double t1, t2;
    if (!illuminant_cct(illum1, &t1) || !illuminant_cct(illum2, &t2)) return CPIPE_NEED_METADATA;
    for (float c : neutral)
        if (!std::isfinite(c) || c <= 0.0F) return CPIPE_NEED_METADATA;
    const double cct = estimate_scene_cct(neutral, *cm1, *cm2, t1, t2);
    const float wgt = reciprocal_cct_weight(t1, t2, cct);
    Mat3 cam_to_xyz;
    if (fm1 && fm2) {
        cam_to_xyz = blend(*fm1, *fm2, wgt);
    } else if (!invert3(blend(*cm1, *cm2, wgt), &cam_to_xyz)) {
        return CPIPE_NEED_METADATA;
    }
    std::memcpy(out->as_shot_neutral, neutral.data(), sizeof(float) * 3);
    std::memcpy(out->camera_to_xyz_d50, cam_to_xyz.data(), sizeof(float) * 9);
    out->scene_cct = (float)cct;
    out->dual_illuminant_weight = wgt;
    *scene_cct = cct;
    return CPIPE_OK;
}

// ============================================================== colormatrix
// colormatrix_dng_to_working.cpp:20-28,57-70,125: XYZ(D65)->Rec.2020 * Bradford
// D50->D65 * camera->XYZ(D50), composed in float.
Mat3 mul3(const Mat3& l, const Mat3& r) {
    Mat3 o{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o[i * 3 + j] = l[i * 3 + 0] * r[0 * 3 + j] + l[i * 3 + 1] * r[1 * 3 + j] + l[i * 3 + 2] * r[2 * 3 + j];
    return o;
}
Mat3 camera_to_rec2020(const Mat3& camera_to_xyz_d50) {
    static const Mat3 kBradfordD50toD65{0.9555766F, -0.0230393F, 0.0631636F, -0.0282895F, 1.0099416F,
                                        0.0210077F, 0.0122982F, -0.0204830F, 1.3299098F};
    static const Mat3 kXyzD65toRec2020{1.7166512F, -0.3556708F, -0.2533663F, -0.6666844F, 1.6164812F,
                                       0.0157685F, 0.0176399F, -0.0427706F, 0.9421031F};
    return mul3(kXyzD65toRec2020, mul3(kBradfordD50toD65, camera_to_xyz_d50));
}

// ========================================================= OpcodeList parsers
namespace {
struct BeReader {
    const unsigned char* p;
    size_t n, off = 0;
    bool can(size_t k) const { return off <= n && k <= n - off; }
    uint32_t u32() {
        const uint32_t v = ((uint32_t)p[off] << 24) | ((uint32_t)p[off + 1] << 16) | ((uint32_t)p[off + 2] << 8) | p[off + 3];
        off += 4;
        return v;
    }
    double f64() {
        const uint64_t hi = u32(), lo = u32();
        const uint64_t bits = (hi << 32) | lo;
        double d;
        std::memcpy(&d, &bits, 8);
        return d;
    }
    float f32() {
        const uint32_t bits = u32();
        float f;
        std::memcpy(&f, &bits, 4);
        return f;
    }
};
}  // namespace

// OpcodeList2: big-endian count, then per opcode {id, dng_version, flags,
// param_bytes, params}; GainMap (id 9) params are a 76-byte header followed by
// map_points_v * map_points_h * map_planes float gains (DNG 1.3 spec; reference
// ingest/dng_opcode/OpcodeList2.cpp:94-176).
int parse_gain_maps(const void* bytes, size_t n, std::vector<GainMap>* maps, std::string* msg) {
    maps->clear();
    if (n == 0) return CPIPE_OK;
    BeReader r{static_cast<const unsigned char*>(bytes), n};
    if (!r.can(4)) { *msg = "OpcodeList2 count truncated"; return CPIPE_FAILED; }
    const uint32_t count = r.u32();
    for (uint32_t i = 0; i < count; ++i) {
        if (!r.can(16)) { *msg = "OpcodeList2 opcode header truncated"; return CPIPE_FAILED; }
        const uint32_t id = r.u32();
        r.u32();
        r.u32();
        const uint32_t size = r.u32();
        if (!r.can(size)) { *msg = "OpcodeList2 opcode params truncated"; return CPIPE_FAILED; }
        const size_t start = r.off;
        r.off += size;
        if (id != 9) continue;
        if (size < 76) { *msg = "GainMap params truncated"; return CPIPE_FAILED; }
        BeReader g{r.p + start, size};
        GainMap m;
        m.top = g.u32(); m.left = g.u32(); m.bottom = g.u32(); m.right = g.u32();
        m.plane = g.u32(); m.planes = g.u32(); m.row_pitch = g.u32(); m.col_pitch = g.u32();
        m.points_v = g.u32(); m.points_h = g.u32();
        m.spacing_v = g.f64(); m.spacing_h = g.f64(); m.origin_v = g.f64(); m.origin_h = g.f64();
        m.map_planes = g.u32();
        if (m.points_v == 0 || m.points_h == 0 || m.map_planes == 0) { *msg = "GainMap size overflows"; return CPIPE_FAILED; }
        const uint64_t total = (uint64_t)m.points_v * m.points_h * m.map_planes;
        if (total > (std::numeric_limits<uint64_t>::max() - 76) / 4 || 76 + total * 4 > size) {
            *msg = "GainMap gain table truncated";
            return CPIPE_FAILED;
        }
        const bool shape_ok = (m.planes == 1 || m.planes == 4) && m.plane < m.planes && m.map_planes == 1 &&
                              m.row_pitch > 0 && m.col_pitch > 0 && std::isfinite(m.spacing_v) &&
                              std::isfinite(m.spacing_h) && m.spacing_v > 0.0 && m.spacing_h > 0.0 &&
                              std::isfinite(m.origin_v) && std::isfinite(m.origin_h);
        if (!shape_ok) { *msg = "GainMap shape is outside cpipe v1 support"; return CPIPE_UNSUPPORTED; }
        m.gain.resize(total);
        for (uint64_t k = 0; k < total; ++k) m.gain[k] = g.f32();
        maps->push_back(std::move(m));
    }
    return CPIPE_OK;
}

// shading_gainmap.cpp:80-137: one plane-0 map, or four maps covering planes 0..3.
int validate_and_pack_gain_maps(const std::vector<GainMap>& maps, const uint8_t repeat[2], const uint8_t pattern[16],
                                std::vector<unsigned char>* blob, std::string* msg) {
    if (maps.empty()) { *msg = "GainMap opcode missing"; return CPIPE_NEED_METADATA; }
    const bool single = maps.size() == 1 && maps[0].planes == 1 && maps[0].plane == 0;
    if (!single) {
        if (maps.size() != 4) { *msg = "GainMap plane set incomplete"; return CPIPE_UNSUPPORTED; }
        bool seen[4] = {false, false, false, false};
        for (const auto& m : maps) {
            if (m.planes != 4 || m.plane >= 4 || seen[m.plane]) { *msg = "GainMap plane set invalid"; return CPIPE_UNSUPPORTED; }
            seen[m.plane] = true;
        }
    }
    cpipe_GainMapDispatchHeader hd{};
    hd.map_count = (uint32_t)maps.size();
    std::memcpy(hd.cfa_repeat, repeat, 2);
    std::memcpy(hd.cfa_pattern, pattern, 16);
    blob->assign(reinterpret_cast<const unsigned char*>(&hd), reinterpret_cast<const unsigned char*>(&hd) + sizeof(hd));
    uint32_t offset = 0;
    for (const auto& m : maps) {
        cpipe_GainMapDispatchPlane p{};
        p.top = m.top; p.left = m.left; p.bottom = m.bottom; p.right = m.right;
        p.plane = m.plane; p.planes = m.planes; p.map_points_v = m.points_v; p.map_points_h = m.points_h;
        p.map_spacing_v = m.spacing_v; p.map_spacing_h = m.spacing_h; p.map_origin_v = m.origin_v; p.map_origin_h = m.origin_h;
        p.gain_offset = offset;
        p.gain_count = (uint32_t)m.gain.size();
        offset += p.gain_count;
        const auto* c = reinterpret_cast<const unsigned char*>(&p);
        blob->insert(blob->end(), c, c + sizeof(p));
    }
    for (const auto& m : maps) {
        const auto* c = reinterpret_cast<const unsigned char*>(m.gain.data());
        blob->insert(blob->end(), c, c + m.gain.size() * sizeof(float));
    }
    return CPIPE_OK;
}

// OpcodeList3 (reference ingest/dng_opcode/OpcodeList3.cpp:83-296 parse,
// nodes/lens/dng_opcode_list_3.cpp:75-168 pack): known opcodes must have exactly
// the DNG parameter sizes; unknown mandatory opcodes are unsupported, unknown
// optional ones are kept as id 0 records.
int parse_and_pack_opcode3(const void* bytes, size_t n, std::vector<unsigned char>* blob, uint32_t* count,
                           std::string* msg) {
    *count = 0;
    blob->clear();
    if (n == 0) return CPIPE_OK;
    BeReader r{static_cast<const unsigned char*>(bytes), n};
    if (!r.can(4)) { *msg = "OpcodeList3 count truncated"; return CPIPE_FAILED; }
    const uint32_t total = r.u32();
    std::vector<cpipe_Opcode3DispatchRecord> recs;
    std::vector<cpipe_Opcode3BadPoint> pts;
    std::vector<cpipe_Opcode3BadRect> rects;
    for (uint32_t i = 0; i < total; ++i) {
        if (!r.can(16)) { *msg = "OpcodeList3 opcode header truncated"; return CPIPE_FAILED; }
        const uint32_t raw = r.u32();
        r.u32();
        const uint32_t flags = r.u32();
        const uint32_t size = r.u32();
        if (!r.can(size)) { *msg = "OpcodeList3 opcode params truncated"; return CPIPE_FAILED; }
        BeReader q{r.p + r.off, size};
        r.off += size;
        cpipe_Opcode3DispatchRecord rec{};
        rec.optional = (flags & 1U) ? 1U : 0U;
        const bool known = raw == 1 || raw == 3 || raw == 4 || raw == 5 || raw == 6;
        rec.id = known ? raw : 0U;
        if (!known) {
            if (!rec.optional) { *msg = "OpcodeList3 mandatory unknown opcode"; return CPIPE_UNSUPPORTED; }
            recs.push_back(rec);
            continue;
        }
        bool ok = false;
        if (raw == 1) {  // WarpRectilinear: N, N x {kr0..kr3, kt0, kt1}, cx, cy
            if (size >= 4) {
                const uint32_t planes = q.u32();
                ok = planes >= 1 && planes <= 4 && size == 4 + (size_t)planes * 48 + 16;
                if (ok) {
                    rec.coefficient_count = planes;
                    for (uint32_t k = 0; k < planes; ++k) {
                        auto& c = rec.coefficients[k];
                        c.kr0 = q.f64(); c.kr1 = q.f64(); c.kr2 = q.f64(); c.kr3 = q.f64(); c.kt0 = q.f64(); c.kt1 = q.f64();
                    }
                    rec.cx_hat = q.f64();
                    rec.cy_hat = q.f64();
                }
            }
        } else if (raw == 3) {  // FixVignetteRadial: k0..k4, cx, cy
            ok = size == 56;
            if (ok) {
                for (double& k : rec.vignette_k) k = q.f64();
                rec.vignette_cx_hat = q.f64();
                rec.vignette_cy_hat = q.f64();
            }
        } else if (raw == 4) {  // FixBadPixelsConstant: constant, bayer phase
            ok = size == 8;
            if (ok) {
                rec.constant = q.u32();
                rec.bayer_phase = q.u32();
            }
        } else if (raw == 5) {  // FixBadPixelsList: phase, #points, #rects, points, rects
            if (size >= 12) {
                rec.bayer_phase = q.u32();
                const uint64_t np = q.u32(), nr = q.u32();
                ok = (uint64_t)size == 12 + np * 8 + nr * 16;
                if (ok) {
                    rec.point_offset = (uint32_t)pts.size();
                    rec.point_count = (uint32_t)np;
                    for (uint64_t k = 0; k < np; ++k) {
                        cpipe_Opcode3BadPoint p;
                        p.row = q.u32();
                        p.column = q.u32();
                        pts.push_back(p);
                    }
                    rec.rect_offset = (uint32_t)rects.size();
                    rec.rect_count = (uint32_t)nr;
                    for (uint64_t k = 0; k < nr; ++k) {
                        cpipe_Opcode3BadRect b;
                        b.top = q.u32(); b.left = q.u32(); b.bottom = q.u32(); b.right = q.u32();
                        rects.push_back(b);
                    }
                }
            }
        } else {  // TrimBounds: top, left, bottom, right
            ok = size == 16;
            if (ok) {
                rec.top = q.u32(); rec.left = q.u32(); rec.bottom = q.u32(); rec.right = q.u32();
            }
        }
        if (!ok) { *msg = "OpcodeList3 known opcode params invalid"; return CPIPE_FAILED; }
        recs.push_back(rec);
    }
    cpipe_Opcode3DispatchHeader hd{(uint32_t)recs.size(), 0};
    auto put = [&](const void* p, size_t k) {
        const auto* c = static_cast<const unsigned char*>(p);
        blob->insert(blob->end(), c, c + k);
    };
    put(&hd, sizeof(hd));
    if (!recs.empty()) put(recs.data(), recs.size() * sizeof(recs[0]));
    if (!pts.empty()) put(pts.data(), pts.size() * sizeof(pts[0]));
    if (!rects.empty()) put(rects.data(), rects.size() * sizeof(rects[0]));
    *count = (uint32_t)recs.size();
    return CPIPE_OK;
}

// =========================================================== 3D LUT loader
// .cube: TITLE/DOMAIN_* ignored, LUT_3D_SIZE S (2..256), then S^3 RGB rows in
// file order (blue fastest); .spi3d: "SPILUT", 3 3, S S S, indexed rows.
// Reference color/Cube3dLutLoader.cpp:57-204.
int load_lut(const std::string& path, uint32_t* size, std::vector<float>* values, std::string* msg) {
    std::ifstream in(path);
    if (!in) { *msg = "failed to open 3D LUT file"; return CPIPE_FAILED; }
    std::string ext;
    const auto dot = path.find_last_of('.');
    if (dot != std::string::npos) ext = path.substr(dot);
    std::transform(ext.begin(), ext.end(), ext.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    values->clear();
    *size = 0;
    auto valid = [&](long s) {
        if (s < 2) { *msg = "3D LUT size must be at least 2"; return false; }
        if (s > 256) { *msg = "3D LUT size above P2 loader limit"; return false; }
        return true;
    };
    if (ext == ".cube") {
        std::string line;
        while (std::getline(in, line)) {
            const auto hash = line.find('#');
            if (hash != std::string::npos) line.resize(hash);
            std::istringstream row(line);
            std::string head;
            if (!(row >> head)) continue;
            if (head == "TITLE" || head == "DOMAIN_MIN" || head == "DOMAIN_MAX") continue;
            if (head == "LUT_3D_SIZE") {
                long s = 0;
                if (!(row >> s) || s < 0) { *msg = "invalid LUT_3D_SIZE"; return CPIPE_FAILED; }
                if (!valid(s)) return CPIPE_FAILED;
                *size = (uint32_t)s;
                values->reserve((size_t)s * s * s * 3);
                continue;
            }
            std::istringstream vals(line);
            float r, g, b;
            if (!(vals >> r >> g >> b)) { *msg = "invalid .cube RGB row"; return CPIPE_FAILED; }
            values->push_back(r);
            values->push_back(g);
            values->push_back(b);
        }
        if (*size == 0) { *msg = "missing LUT_3D_SIZE"; return CPIPE_FAILED; }
        if (values->size() != (size_t)*size * *size * *size * 3) { *msg = "wrong number of .cube RGB rows"; return CPIPE_FAILED; }
        return CPIPE_OK;
    }
    if (ext == ".spi3d") {
        std::string magic;
        double version;
        int di, dout, rs, gs, bs;
        if (!(in >> magic >> version) || magic != "SPILUT") { *msg = "missing SPILUT header"; return CPIPE_FAILED; }
        if (!(in >> di >> dout) || di != 3 || dout != 3) { *msg = "unsupported .spi3d component count"; return CPIPE_FAILED; }
        if (!(in >> rs >> gs >> bs) || rs != gs || gs != bs || rs < 0) { *msg = "unsupported .spi3d grid dimensions"; return CPIPE_FAILED; }
        if (!valid(rs)) return CPIPE_FAILED;
        const size_t S = (size_t)rs;
        values->assign(S * S * S * 3, 0.0F);
        std::vector<char> seen(S * S * S, 0);
        int r, g, b;
        float orr, og, ob;
        while (in >> r >> g >> b >> orr >> og >> ob) {
            if (r < 0 || g < 0 || b < 0 || r >= rs || g >= rs || b >= rs) { *msg = ".spi3d index out of range"; return CPIPE_FAILED; }
            const size_t idx = ((size_t)r * S + g) * S + b;
            (*values)[idx * 3] = orr;
            (*values)[idx * 3 + 1] = og;
            (*values)[idx * 3 + 2] = ob;
            seen[idx] = 1;
        }
        if (!std::all_of(seen.begin(), seen.end(), [](char c) { return c != 0; })) { *msg = "missing .spi3d sample rows"; return CPIPE_FAILED; }
        *size = (uint32_t)S;
        return CPIPE_OK;
    }
    *msg = "unsupported 3D LUT extension";
    return CPIPE_UNSUPPORTED;
}

}  // namespace cpb::prep

// ======================================================= C entry points
// Host-logic entry points (no device work), so a reference integration and the
// CPU test suite can call the parameter preparation on its own.
extern "C" {

int cpipe_b200_wb_prepare(const float neutral[3], const float cm1[9], const float cm2[9], const float* fm1,
                          const float* fm2, uint16_t illum1, uint16_t illum2, cpipe_WbParams* out, double* scene_cct) {
    if (!neutral || !out || !scene_cct) return CPIPE_BAD_INDEX;
    try {
        cpb::prep::Vec3 n{neutral[0], neutral[1], neutral[2]};
        cpb::prep::Mat3 a{}, b{}, f1{}, f2{};
        if (cm1) std::memcpy(a.data(), cm1, sizeof(a));
        if (cm2) std::memcpy(b.data(), cm2, sizeof(b));
        if (fm1) std::memcpy(f1.data(), fm1, sizeof(f1));
        if (fm2) std::memcpy(f2.data(), fm2, sizeof(f2));
        return cpb::prep::wb_prepare(n, cm1 ? &a : nullptr, cm2 ? &b : nullptr, fm1 ? &f1 : nullptr,
                                     fm2 ? &f2 : nullptr, illum1, illum2, out, scene_cct);
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}

int cpipe_b200_colormatrix_compose(const float camera_to_xyz_d50[9], float out[9]) {
    if (!camera_to_xyz_d50 || !out) return CPIPE_BAD_INDEX;
    cpb::prep::Mat3 m;
    std::memcpy(m.data(), camera_to_xyz_d50, sizeof(m));
    const cpb::prep::Mat3 t = cpb::prep::camera_to_rec2020(m);
    std::memcpy(out, t.data(), sizeof(t));
    return CPIPE_OK;
}

// Parse an OpcodeList2 stream and pack the GainMap dispatch blob the
// lens_shading_gainmap filter takes.  *blob_size in: capacity, out: bytes needed.
int cpipe_b200_pack_gain_maps(const void* opcode_list_2, size_t n, const uint8_t cfa_repeat[2],
                              const uint8_t cfa_pattern[16], void* blob, size_t* blob_size) {
    if (!blob_size || !cfa_repeat || !cfa_pattern) return CPIPE_BAD_INDEX;
    try {
        std::vector<cpb::prep::GainMap> maps;
        std::string msg;
        int st = cpb::prep::parse_gain_maps(opcode_list_2, n, &maps, &msg);
        if (st != CPIPE_OK) return st;
        std::vector<unsigned char> out;
        st = cpb::prep::validate_and_pack_gain_maps(maps, cfa_repeat, cfa_pattern, &out, &msg);
        if (st != CPIPE_OK) return st;
        const size_t cap = *blob_size;
        *blob_size = out.size();
        if (blob && cap >= out.size()) std::memcpy(blob, out.data(), out.size());
        return (blob && cap < out.size()) ? CPIPE_BAD_INDEX : CPIPE_OK;
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}

// Parse an OpcodeList3 stream into the lens_dng_opcode_list_3 dispatch blob.
int cpipe_b200_pack_opcode_list_3(const void* opcode_list_3, size_t n, void* blob, size_t* blob_size,
                                  uint32_t* opcode_count) {
    if (!blob_size || !opcode_count) return CPIPE_BAD_INDEX;
    try {
        std::vector<unsigned char> out;
        std::string msg;
        const int st = cpb::prep::parse_and_pack_opcode3(opcode_list_3, n, &out, opcode_count, &msg);
        if (st != CPIPE_OK) return st;
        const size_t cap = *blob_size;
        *blob_size = out.size();
        if (blob && cap >= out.size()) std::memcpy(blob, out.data(), out.size());
        return (blob && cap < out.size()) ? CPIPE_BAD_INDEX : CPIPE_OK;
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}

// Load a .cube / .spi3d file; values may be null to query the size.
int cpipe_b200_load_lut(const char* path, uint32_t* size, float* values, size_t capacity) {
    if (!path || !size) return CPIPE_BAD_INDEX;
    try {
        std::vector<float> v;
        std::string msg;
        const int st = cpb::prep::load_lut(path, size, &v, &msg);
        if (st != CPIPE_OK) return st;
        if (values) {
            if (capacity < v.size()) return CPIPE_BAD_INDEX;
            std::memcpy(values, v.data(), v.size() * sizeof(float));
        }
        return CPIPE_OK;
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}

}  // extern "C"
