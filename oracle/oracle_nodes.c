/* CPU oracle for the cpipe raw->linear node chain.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests, the smoke check
 * and the CPU-baseline leg of the benchmark load it; the product path never
 * does.  Each function restates one reference node, keeping the reference's
 * floating-point operation order so results are bit-identical where the
 * reference is plain C++ and within one f16 ulp where it is Halide-generated
 * (Halide v21 lowering of float16 casts / log / pow is not available here).
 *
 * Storage modes: every RGBA function takes dense interleaved RGBA float arrays.
 * With f16 != 0 the outputs are rounded to IEEE binary16 after each node, as
 * the reference does when it writes an R16G16B16A16_SFLOAT buffer; with
 * f16 == 0 the node is evaluated in plain FP32 with no inter-node rounding.
 *
 * Build: gcc -O2 -fPIC -shared -fopenmp -ffp-contract=off (no FMA contraction;
 * the reference Halide target x86-64-linux has no FMA feature,
 * reference src/cpipe/nodes/CMakeLists.txt:33).
 */
#include <math.h>
#include <stdlib.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "../include/cpipe_b200_params.h"

#define OK 0
#define ST_BAD_INDEX 5
#define ST_NEED_METADATA 9
#define ST_UNSUPPORTED 8

/* ---- f16 helpers (reference src/cpipe/nodes/detail/Float16.hpp:11-24) ---- */
static inline float h16(float v) { return (float)(_Float16)v; }
static inline float rnd(float v, int f16) { return f16 ? h16(v) : v; }
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
static inline float maxf(float a, float b) { return a < b ? b : a; } /* std::max */

uint16_t oracle_float_to_half(float v) {
    _Float16 h = (_Float16)v;
    uint16_t bits;
    memcpy(&bits, &h, 2);
    return bits;
}
float oracle_half_to_float(uint16_t bits) {
    _Float16 h;
    memcpy(&h, &bits, 2);
    return (float)h;
}

/* ---- a1: precision_convert (src/cpipe/nodes/precision/precision_convert_generator.cpp:31-124) ---- */
void oracle_r16u_to_f32(const uint16_t* in, float* out, int w, int h) {
    for (long i = 0; i < (long)w * h; ++i) out[i] = (float)in[i];
}
void oracle_f32_to_rgba16f(const float* in, float* out, int w, int h) {
    for (long i = 0; i < (long)w * h; ++i) {
        const float v = h16(in[i]);
        out[4 * i + 0] = v;
        out[4 * i + 1] = v;
        out[4 * i + 2] = v;
        out[4 * i + 3] = 1.0F;
    }
}
void oracle_rgba16f_to_unorm(const float* in, uint16_t* out, int w, int h, int bits8) {
    for (long i = 0; i < (long)w * h * 4; ++i) {
        const float scale = bits8 ? 255.0F : 65535.0F;
        const float s = (clampf(in[i], 0.0F, 1.0F) * scale) + 0.5F;
        out[i] = (uint16_t)s;
    }
}

/* ---- a2: linearize (src/cpipe/nodes/linearize/linearize_dng_lut_dispatch.cpp:17-51) ---- */
int oracle_linearize(const uint16_t* in, float* out, int w, int h, const uint16_t* table, int n) {
    if (n <= 0) return ST_NEED_METADATA;
    const int last = n - 1;
    for (long i = 0; i < (long)w * h; ++i) {
        const int idx = in[i] < last ? in[i] : last;
        out[i] = (float)table[idx];
    }
    return OK;
}

/* ---- a3: blacklevel (src/cpipe/nodes/blacklevel/blacklevel_dng_levels_dispatch.cpp:16-47) ---- */
int oracle_blacklevel(const float* in, float* out, int w, int h, const cpipe_BlacklevelParams* p) {
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const unsigned cfa_index = ((unsigned)(y & 1) * 2U) + (unsigned)(x & 1);
            const unsigned ch = p->cfa_pattern[cfa_index] < 3 ? p->cfa_pattern[cfa_index] : 3;
            const float black = p->black_level[ch];
            const float denom = (float)p->white_level - black;
            if (denom <= 0.0F) return ST_NEED_METADATA;
            out[(long)y * w + x] = clampf((in[(long)y * w + x] - black) / denom, 0.0F, 1.0F);
        }
    }
    return OK;
}

/* ---- a4: gainmap (src/cpipe/nodes/lens/shading_gainmap_dispatch.cpp:23-133) ---- */
typedef struct { uint32_t low, high; float weight; } axis_t;
static axis_t sample_axis(double coord, uint32_t points) {
    axis_t a = {0, 0, 0.0F};
    if (points <= 1U || coord <= 0.0) return a;
    const double last = (double)(points - 1U);
    if (coord >= last) { a.low = a.high = points - 1U; return a; }
    a.low = (uint32_t)floor(coord);
    a.high = a.low + 1U;
    a.weight = (float)(coord - (double)a.low);
    return a;
}
static inline float lerpf(float a, float b, float t) { return a + ((b - a) * t); }

int oracle_gainmap(const float* in, float* out, int w, int h, const void* blob, size_t blob_size) {
    if (blob == NULL || blob_size < sizeof(cpipe_GainMapDispatchHeader)) return ST_BAD_INDEX;
    const cpipe_GainMapDispatchHeader* hd = (const cpipe_GainMapDispatchHeader*)blob;
    if (hd->map_count == 0U || hd->map_count > 4U) return ST_NEED_METADATA;
    const size_t map_bytes = hd->map_count * sizeof(cpipe_GainMapDispatchPlane);
    if (blob_size < sizeof(*hd) + map_bytes) return ST_BAD_INDEX;
    const cpipe_GainMapDispatchPlane* maps =
        (const cpipe_GainMapDispatchPlane*)((const char*)blob + sizeof(*hd));
    const float* gains = (const float*)((const char*)blob + sizeof(*hd) + map_bytes);
    const size_t gain_bytes = blob_size - sizeof(*hd) - map_bytes;
    for (uint32_t i = 0; i < hd->map_count; ++i) {
        const uint64_t req = ((uint64_t)maps[i].gain_offset + maps[i].gain_count) * sizeof(float);
        if (maps[i].map_points_v == 0U || maps[i].map_points_h == 0U || maps[i].gain_count == 0U ||
            req > gain_bytes)
            return ST_BAD_INDEX;
    }
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const cpipe_GainMapDispatchPlane* m = NULL;
            if (hd->map_count == 1U) {
                m = &maps[0];
            } else {
                uint32_t plane = ((uint32_t)(y & 1) * 2U) + (uint32_t)(x & 1);
                if (hd->cfa_repeat[0] == 4U && hd->cfa_repeat[1] == 4U)
                    plane = ((((uint32_t)y % 4U) / 2U) * 2U) + (((uint32_t)x % 4U) / 2U);
                for (uint32_t i = 0; i < hd->map_count; ++i)
                    if (maps[i].plane == plane) { m = &maps[i]; break; }
            }
            if (m == NULL) return ST_NEED_METADATA;
            const float* g = gains + m->gain_offset;
            const double gy = ((double)y - m->map_origin_v) / m->map_spacing_v;
            const double gx = ((double)x - m->map_origin_h) / m->map_spacing_h;
            const axis_t sy = sample_axis(gy, m->map_points_v);
            const axis_t sx = sample_axis(gx, m->map_points_h);
            const uint32_t rs = m->map_points_h;
            const float g00 = g[sy.low * rs + sx.low], g10 = g[sy.low * rs + sx.high];
            const float g01 = g[sy.high * rs + sx.low], g11 = g[sy.high * rs + sx.high];
            const float gain = lerpf(lerpf(g00, g10, sx.weight), lerpf(g01, g11, sx.weight), sy.weight);
            out[(long)y * w + x] = in[(long)y * w + x] * gain;
        }
    }
    return OK;
}

/* ---- a5-a7: demosaic (demosaic_{rcd,amaze,bilinear}_generator.cpp) ---- */
typedef struct { const float* p; int w, h; const int* cfa; } bayer_t;
static inline float bs(const bayer_t* b, int x, int y) {
    return b->p[(long)clampi(y, 0, b->h - 1) * b->w + clampi(x, 0, b->w - 1)];
}
static inline int cfa_at(const bayer_t* b, int x, int y) { return b->cfa[((y & 1) * 2) + (x & 1)]; }

/* RCD green, demosaic_rcd_generator.cpp:28-35 */
static float rcd_green(const bayer_t* b, int x, int y) {
    const float c = bs(b, x, y);
    if (cfa_at(b, x, y) == 1) return c;
    const float gh = 0.5F * (bs(b, x - 1, y) + bs(b, x + 1, y));
    const float gv = 0.5F * (bs(b, x, y - 1) + bs(b, x, y + 1));
    const float dh = fabsf(bs(b, x - 2, y) - bs(b, x + 2, y));
    const float dv = fabsf(bs(b, x, y - 2) - bs(b, x, y + 2));
    if (dh < dv) return gh;
    if (dv < dh) return gv;
    return 0.5F * (gh + gv);
}
static inline float rcd_ratio(const bayer_t* b, int x, int y) {
    return bs(b, x, y) / maxf(rcd_green(b, x, y), 0.000001F);
}
/* AMaZE green, demosaic_amaze_generator.cpp:24-46 */
static float amaze_green(const bayer_t* b, int x, int y) {
    const float c = bs(b, x, y);
    if (cfa_at(b, x, y) == 1) return c;
    const float ct = 2.0F * c;
    const float ghn = bs(b, x - 1, y) + bs(b, x + 1, y);
    const float gvn = bs(b, x, y - 1) + bs(b, x, y + 1);
    const float ghs = ct - bs(b, x - 2, y) - bs(b, x + 2, y);
    const float gvs = ct - bs(b, x, y - 2) - bs(b, x, y + 2);
    const float gh = (0.5F * ghn) + (0.25F * ghs);
    const float gv = (0.5F * gvn) + (0.25F * gvs);
    const float grh = fabsf(bs(b, x - 1, y) - bs(b, x + 1, y)) + fabsf(bs(b, x - 2, y) - c) +
                      fabsf(bs(b, x + 2, y) - c);
    const float grv = fabsf(bs(b, x, y - 1) - bs(b, x, y + 1)) + fabsf(bs(b, x, y - 2) - c) +
                      fabsf(bs(b, x, y + 2) - c);
    if (grh < grv) return gh;
    if (grv < grh) return gv;
    return 0.5F * (gh + gv);
}
static inline float amaze_chroma(const bayer_t* b, int x, int y) {
    return bs(b, x, y) - amaze_green(b, x, y);
}

/* algo: 0 bilinear, 1 rcd, 2 amaze.  out: RGBA. */
int oracle_demosaic(int algo, const float* in, float* out, int w, int h, const uint8_t cfa8[4], int f16) {
    int cfa[4] = {cfa8[0], cfa8[1], cfa8[2], cfa8[3]};
    bayer_t B = {in, w, h, cfa};
    const bayer_t* b = &B;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const float c = bs(b, x, y);
            const int site = cfa_at(b, x, y);
            const int red = site == 0, blue = site == 2;
            const int hred = cfa_at(b, x - 1, y) == 0, hblue = cfa_at(b, x - 1, y) == 2;
            float r, g, bl;
            if (algo == 0) { /* demosaic_bilinear_generator.cpp:23-41 */
                const float hz = 0.5F * (bs(b, x - 1, y) + bs(b, x + 1, y));
                const float vt = 0.5F * (bs(b, x, y - 1) + bs(b, x, y + 1));
                const float cross = 0.25F * (bs(b, x - 1, y) + bs(b, x + 1, y) + bs(b, x, y - 1) + bs(b, x, y + 1));
                const float diag = 0.25F * (bs(b, x - 1, y - 1) + bs(b, x + 1, y - 1) + bs(b, x - 1, y + 1) + bs(b, x + 1, y + 1));
                r = red ? c : blue ? diag : hred ? hz : vt;
                g = (red || blue) ? cross : c;
                bl = blue ? c : red ? diag : hred ? vt : hz;
            } else if (algo == 1) { /* demosaic_rcd_generator.cpp:37-63 */
                const float gc = rcd_green(b, x, y);
                const float rh = gc * 0.5F * (rcd_ratio(b, x - 1, y) + rcd_ratio(b, x + 1, y));
                const float rv = gc * 0.5F * (rcd_ratio(b, x, y - 1) + rcd_ratio(b, x, y + 1));
                const float rd = gc * 0.25F * (rcd_ratio(b, x - 1, y - 1) + rcd_ratio(b, x + 1, y - 1) +
                                               rcd_ratio(b, x - 1, y + 1) + rcd_ratio(b, x + 1, y + 1));
                r = maxf(0.0F, red ? c : blue ? rd : hred ? rh : rv);
                g = maxf(0.0F, gc);
                bl = maxf(0.0F, blue ? c : red ? rd : hblue ? rh : rv);
            } else { /* demosaic_amaze_generator.cpp:48-66 */
                const float gc = amaze_green(b, x, y);
                const float chh = 0.5F * (amaze_chroma(b, x - 1, y) + amaze_chroma(b, x + 1, y));
                const float chv = 0.5F * (amaze_chroma(b, x, y - 1) + amaze_chroma(b, x, y + 1));
                const float chd = 0.25F * (amaze_chroma(b, x - 1, y - 1) + amaze_chroma(b, x + 1, y - 1) +
                                           amaze_chroma(b, x - 1, y + 1) + amaze_chroma(b, x + 1, y + 1));
                const float rh = gc + chh, rv = gc + chv, rd = gc + chd;
                const float ri = blue ? rd : hred ? rh : rv;
                const float bi = red ? rd : hblue ? rh : rv;
                r = maxf(0.0F, red ? c : ri);
                g = maxf(0.0F, gc);
                bl = maxf(0.0F, blue ? c : bi);
            }
            float* o = out + 4 * ((long)y * w + x);
            o[0] = rnd(r, f16);
            o[1] = rnd(g, f16);
            o[2] = rnd(bl, f16);
            o[3] = 1.0F;
        }
    }
    return OK;
}

/* ---- a8: Quad Bayer remosaic (demosaic_quad_bayer_remosaic_generator.cpp:17-58), integer ---- */
static inline int qbc_color(int x, int y) {
    const int mx = ((x % 4) + 4) % 4, my = ((y % 4) + 4) % 4;
    if (my < 2 && mx < 2) return 0;
    if (my >= 2 && mx >= 2) return 2;
    return 1;
}
void oracle_qbc_remosaic(const uint16_t* in, uint16_t* out, int w, int h) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int target = ((y & 1) == 0 && (x & 1) == 0) ? 0 : (((y & 1) != 0 && (x & 1) != 0) ? 2 : 1);
            uint32_t ws = 0, wsum = 0;
            for (int dy = -2; dy <= 2; ++dy) {
                for (int dx = -2; dx <= 2; ++dx) {
                    const int sx = clampi(x + dx, 0, w - 1), sy = clampi(y + dy, 0, h - 1);
#define Q(X, Y) ((int)in[(long)clampi((Y), 0, h - 1) * w + clampi((X), 0, w - 1)])
                    const int gx = abs(Q(sx - 1, sy) - Q(sx + 1, sy));
                    const int gy = abs(Q(sx, sy - 1) - Q(sx, sy + 1));
                    const int pen = 64 + gx + gy + ((abs(dx) + abs(dy)) * 16);
                    int cw = 65536 / pen;
                    if (cw < 1) cw = 1;
                    const uint32_t wt = qbc_color(sx, sy) == target ? (uint32_t)cw : 0U;
                    ws += wt * (uint32_t)Q(sx, sy);
                    wsum += wt;
#undef Q
                }
            }
            out[(long)y * w + x] = wsum == 0 ? 0 : (uint16_t)((ws + (wsum / 2U)) / wsum);
        }
    }
}

/* ---- RGBA helpers ---- */
typedef struct { const float* p; int w, h; } rgba_t;
static inline float rs(const rgba_t* im, int x, int y, int c) {
    return im->p[4 * ((long)clampi(y, 0, im->h - 1) * im->w + clampi(x, 0, im->w - 1)) + c];
}

/* ---- tone.aces_filmic (src/cpipe/nodes/tone/aces_filmic_generator.cpp:22-52) and
 * tone.reinhard (reinhard_generator.cpp:20-48): per RGB channel, alpha passes. */
static float aces_fit(float v) {
    v = maxf(0.0F, v);
    return clampf((v * ((2.51F * v) + 0.03F)) / ((v * ((2.43F * v) + 0.59F)) + 0.14F), 0.0F, 1.0F);
}
void oracle_aces(const float* in, float* out, int w, int h, int enabled, int f16) {
    const long n = (long)w * h;
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 4; ++c) {
            const float v = in[4 * i + c];
            out[4 * i + c] = rnd(c == 3 || enabled == 0 ? v : aces_fit(v), f16);
        }
}
void oracle_reinhard(const float* in, float* out, int w, int h, float white_point, int f16) {
    const long n = (long)w * h;
    const float wp2 = white_point * white_point;
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 4; ++c) {
            const float x = in[4 * i + c];
            float o = x;
            if (c != 3) {
                const float v = maxf(0.0F, x);
                o = clampf((v * (1.0F + (v / wp2))) / (1.0F + v), 0.0F, 1.0F);
            }
            out[4 * i + c] = rnd(o, f16);
        }
}

/* ---- tone.mertens_local (src/cpipe/nodes/tone/mertens_local_generator.cpp:22-115):
 * the Halide generator's expression order, libm exp / sqrt / pow. */
static float mertens_cew(float v) {
    const float k = 2.0F * 0.20F * 0.20F;
    const float d = v - 0.5F;
    return expf(-(d * d) / k);
}
static float mertens_w(const float* f, float wc, float ws, float we) {
    const float red = maxf(0.0F, f[0]), green = maxf(0.0F, f[1]), blue = maxf(0.0F, f[2]);
    const float mean = ((f[0] + f[1]) + f[2]) / 3.0F;
    const float sat = sqrtf(((((red - mean) * (red - mean)) + ((green - mean) * (green - mean))) +
                             ((blue - mean) * (blue - mean))) / 3.0F + 0.0001F);
    const float well = (mertens_cew(red) * mertens_cew(green)) * mertens_cew(blue);
    const float contrast = fabsf(mean - 0.5F);
    const float cf = wc == 0.0F ? 1.0F : powf(contrast + 0.01F, wc);
    const float sf = ws == 1.0F ? sat + 0.01F : powf(sat + 0.01F, ws);
    const float ef = we == 1.0F ? well : powf(well + 0.0001F, we);
    return (cf * sf) * ef;
}
void oracle_mertens(const float* u, const float* n, const float* o, float* out, int w, int h, float wc, float ws,
                    float we, int f16) {
    const long count = (long)w * h;
    for (long i = 0; i < count; ++i) {
        const float* U = u + 4 * i;
        const float* N = n + 4 * i;
        const float* O = o + 4 * i;
        const float wu = mertens_w(U, wc, ws, we), wn = mertens_w(N, wc, ws, we), wo = mertens_w(O, wc, ws, we);
        const float total = maxf((wu + wn) + wo, 0.000001F);
        for (int c = 0; c < 3; ++c)
            out[4 * i + c] = rnd(clampf((((wu * U[c]) + (wn * N[c])) + (wo * O[c])) / total, 0.0F, 1.0F), f16);
        out[4 * i + 3] = rnd(N[3], f16);
    }
}

/* ---- sharpen.edge_aware_usm (src/cpipe/nodes/sharpen/edge_aware_usm_generator.cpp:11-75) ----
 * blur = mean3x3 (radius <= 1, explicit 9-term left-associated sum) or mean5x5
 * (0 + the 25 terms in row-major order), both over the clamped input;
 * mask = v - blur; RGB = max(0, |mask| >= threshold ? v + strength * mask : v);
 * alpha = v. */
void oracle_usm(const float* in, float* out, int w, int h, float strength, int radius, float threshold, int f16) {
    rgba_t I = {in, w, h};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            for (int c = 0; c < 4; ++c) {
                const float v = rs(&I, x, y, c);
                float o = v;
                if (c != 3) {
                    float blur;
                    if (radius <= 1) {
                        float s = rs(&I, x - 1, y - 1, c);
                        s = s + rs(&I, x, y - 1, c);
                        s = s + rs(&I, x + 1, y - 1, c);
                        s = s + rs(&I, x - 1, y, c);
                        s = s + rs(&I, x, y, c);
                        s = s + rs(&I, x + 1, y, c);
                        s = s + rs(&I, x - 1, y + 1, c);
                        s = s + rs(&I, x, y + 1, c);
                        s = s + rs(&I, x + 1, y + 1, c);
                        blur = s / 9.0F;
                    } else {
                        float s = 0.0F;
                        for (int dy = -2; dy <= 2; ++dy)
                            for (int dx = -2; dx <= 2; ++dx) s += rs(&I, x + dx, y + dy, c);
                        blur = s / 25.0F;
                    }
                    const float mask = v - blur;
                    const float sh = fabsf(mask) >= threshold ? v + (strength * mask) : v;
                    o = maxf(0.0F, sh);
                }
                out[4 * ((long)y * w + x) + c] = rnd(o, f16);
            }
        }
    }
}

/* ---- a9: white balance pixel op (wb/wb_dual_illuminant_dispatch.cpp:16-48) ---- */
void oracle_wb(const float* in, float* out, int w, int h, const cpipe_WbParams* p, int f16) {
    for (long i = 0; i < (long)w * h; ++i) {
        for (int c = 0; c < 3; ++c) out[4 * i + c] = rnd(in[4 * i + c] / p->as_shot_neutral[c], f16);
        out[4 * i + 3] = in[4 * i + 3];
    }
}

/* ---- a10: colormatrix pixel op (colormatrix/colormatrix_dng_to_working_dispatch.cpp:17-62) ---- */
void oracle_colormatrix(const float* in, float* out, int w, int h, const float t[9], int f16) {
    for (long i = 0; i < (long)w * h; ++i) {
        const float r = in[4 * i], g = in[4 * i + 1], b = in[4 * i + 2];
        out[4 * i + 0] = rnd(t[0] * r + t[1] * g + t[2] * b, f16);
        out[4 * i + 1] = rnd(t[3] * r + t[4] * g + t[5] * b, f16);
        out[4 * i + 2] = rnd(t[6] * r + t[7] * g + t[8] * b, f16);
        out[4 * i + 3] = in[4 * i + 3];
    }
}

/* ---- a11: BM3D parity form (denoise/bm3d_step1_generator.cpp:9-16,42-56) ---- */
void oracle_bm3d_parity(const float* in, float* out, int w, int h, float sigma, int f16) {
    rgba_t I = {in, w, h};
    const float s = fminf(1.0F, fmaxf(0.0F, sigma / 0.03F));
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int bx = (x / 2) * 2, by = (y / 2) * 2;
            for (int c = 0; c < 4; ++c) {
                const float v = rs(&I, x, y, c);
                float o;
                if (c == 3) {
                    o = v;
                } else {
                    const float basic = (rs(&I, bx, by, c) + rs(&I, bx + 1, by, c) + rs(&I, bx, by + 1, c) +
                                         rs(&I, bx + 1, by + 1, c)) * 0.25F;
                    const float d = (v * (1.0F - s)) + (basic * s);
                    o = maxf(0.0F, d);
                }
                out[4 * ((long)y * w + x) + c] = rnd(o, f16);
            }
        }
    }
}

/* ---- a12: guided filter (denoise/guided_filter_generator.cpp:11-28,45-85) ---- */
static float gf_box(const rgba_t* I, int x, int y, int c, int r, int sq) {
    float sum = 0.0F;
    if (r == 1) {
        /* mean3x3: explicit 9-term left-associated sum, :11-17 */
        const float v[9] = {rs(I, x - 1, y - 1, c), rs(I, x, y - 1, c), rs(I, x + 1, y - 1, c),
                            rs(I, x - 1, y, c),     rs(I, x, y, c),     rs(I, x + 1, y, c),
                            rs(I, x - 1, y + 1, c), rs(I, x, y + 1, c), rs(I, x + 1, y + 1, c)};
        sum = sq ? v[0] * v[0] : v[0];
        for (int i = 1; i < 9; ++i) sum = sum + (sq ? v[i] * v[i] : v[i]);
        return sum / 9.0F;
    }
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            const float v = rs(I, x + dx, y + dy, c);
            sum += sq ? v * v : v;
        }
    return sum / 25.0F;
}
static void gf_ab(const rgba_t* I, int x, int y, int c, int r, float eps, float* a, float* b) {
    const float m = gf_box(I, x, y, c, r, 0);
    const float corr = gf_box(I, x, y, c, r, 1);
    const float var = maxf(0.0F, corr - (m * m));
    *a = var / (var + eps);
    *b = m - (*a * m);
}
/* The generator inlines a and b at every use (25 or 9 evaluations per output);
 * here each is evaluated once per position of the extended domain
 * [-r, w + r) x [-r, h + r) that the output boxes read, on the same clamped
 * input, so the box sums add the same floats in the same order. */
void oracle_guided(const float* in, float* out, int w, int h, int radius, float eps, int f16) {
    rgba_t I = {in, w, h};
    const int r = radius <= 1 ? 1 : 2;
    const long ew = w + 2 * r, eh = h + 2 * r;
    float* ab = (float*)malloc(sizeof(float) * 6 * (size_t)ew * (size_t)eh);
    if (ab == NULL) return;
#pragma omp parallel for schedule(static)
    for (long yy = 0; yy < eh; ++yy)
        for (long xx = 0; xx < ew; ++xx)
            for (int c = 0; c < 3; ++c) {
                float* d = ab + 6 * (yy * ew + xx) + 2 * c;
                gf_ab(&I, (int)xx - r, (int)yy - r, c, r, eps, &d[0], &d[1]);
            }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            for (int c = 0; c < 4; ++c) {
                const float v = rs(&I, x, y, c);
                float o;
                if (c == 3) {
                    o = v;
                } else {
                    float sa = 0.0F, sb = 0.0F;
                    int first = 1;
                    for (int dy = -r; dy <= r; ++dy)
                        for (int dx = -r; dx <= r; ++dx) {
                            const float* d = ab + 6 * ((long)(y + dy + r) * ew + (x + dx + r)) + 2 * c;
                            if (r == 1 && first) {
                                sa = d[0];
                                sb = d[1];
                                first = 0;
                            } else {
                                sa = sa + d[0];
                                sb = sb + d[1];
                            }
                        }
                    sa = r == 1 ? sa / 9.0F : sa / 25.0F;
                    sb = r == 1 ? sb / 9.0F : sb / 25.0F;
                    o = maxf(0.0F, (sa * v) + sb);
                }
                out[4 * ((long)y * w + x) + c] = rnd(o, f16);
            }
        }
    }
    free(ab);
}

/* ---- a13: wavelet Bayes shrink (denoise/wavelet_bayes_shrink_generator.cpp:9-31,57-86) ---- */
static inline float soft_th(float v, float t) { return v > t ? v - t : (v < -t ? v + t : 0.0F); }
static inline float wv_comp(const rgba_t* I, int x, int y, int comp) {
    const float r = rs(I, x, y, 0), g = rs(I, x, y, 1), b = rs(I, x, y, 2);
    return comp == 1 ? r - b : g - ((r + b) * 0.5F);
}
static float wv_block(const rgba_t* I, int x, int y, int comp, float th) {
    const int bx = (x / 2) * 2, by = (y / 2) * 2;
    const float p00 = wv_comp(I, bx, by, comp), p10 = wv_comp(I, bx + 1, by, comp);
    const float p01 = wv_comp(I, bx, by + 1, comp), p11 = wv_comp(I, bx + 1, by + 1, comp);
    const float ll = 0.25F * (p00 + p10 + p01 + p11);
    const float hh = soft_th(0.25F * (p00 - p10 + p01 - p11), th);
    const float vv = soft_th(0.25F * (p00 + p10 - p01 - p11), th);
    const float dd = soft_th(0.25F * (p00 - p10 - p01 + p11), th);
    const int ox = x & 1, oy = y & 1;
    if (ox == 0 && oy == 0) return ll + hh + vv + dd;
    if (ox == 1 && oy == 0) return ll - hh + vv - dd;
    if (ox == 0 && oy == 1) return ll + hh - vv - dd;
    return ll - hh - vv + dd;
}
void oracle_wavelet(const float* in, float* out, int w, int h, float strength, int f16) {
    rgba_t I = {in, w, h};
    const float th = 0.035F * strength;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const float r = rs(&I, x, y, 0), g = rs(&I, x, y, 1), b = rs(&I, x, y, 2);
            const float luma = (r + (2.0F * g) + b) * 0.25F;
            const float co = wv_block(&I, x, y, 1, th), cg = wv_block(&I, x, y, 2, th);
            const float t = luma - (0.5F * cg);
            float* o = out + 4 * ((long)y * w + x);
            o[0] = rnd(maxf(0.0F, t + (0.5F * co)), f16);
            o[1] = rnd(maxf(0.0F, t + cg), f16);
            o[2] = rnd(maxf(0.0F, t - (0.5F * co)), f16);
            o[3] = rnd(maxf(0.0F, rs(&I, x, y, 3)), f16);
        }
    }
}

/* ---- a15: 3D LUT (color/lut3d_generator.cpp:35-138) ---- */
static inline float lut_s(const float* lut, int S, int ch, int r, int g, int b) {
    return lut[(((long)r * S + g) * S + b) * 3 + ch];
}
static inline float add_delta(float base, float from, float to, float w) { return base + ((to - from) * w); }
void oracle_lut3d(const float* in, float* out, int w, int h, const float* lut, int S, int interp, int f16) {
    const int mi = S - 1;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)w * h; ++i) {
        const float rsc = clampf(in[4 * i + 0], 0.0F, 1.0F) * (float)mi;
        const float gsc = clampf(in[4 * i + 1], 0.0F, 1.0F) * (float)mi;
        const float bsc = clampf(in[4 * i + 2], 0.0F, 1.0F) * (float)mi;
        const int r0 = clampi((int)floorf(rsc), 0, S - 2);
        const int g0 = clampi((int)floorf(gsc), 0, S - 2);
        const int b0 = clampi((int)floorf(bsc), 0, S - 2);
        const float dr = rsc - (float)r0, dg = gsc - (float)g0, db = bsc - (float)b0;
        for (int c = 0; c < 3; ++c) {
            const float c000 = lut_s(lut, S, c, r0, g0, b0), c100 = lut_s(lut, S, c, r0 + 1, g0, b0);
            const float c010 = lut_s(lut, S, c, r0, g0 + 1, b0), c001 = lut_s(lut, S, c, r0, g0, b0 + 1);
            const float c110 = lut_s(lut, S, c, r0 + 1, g0 + 1, b0), c101 = lut_s(lut, S, c, r0 + 1, g0, b0 + 1);
            const float c011 = lut_s(lut, S, c, r0, g0 + 1, b0 + 1), c111 = lut_s(lut, S, c, r0 + 1, g0 + 1, b0 + 1);
            float v;
            if (interp == 1) {
                const float c00 = c000 + ((c100 - c000) * dr), c10 = c010 + ((c110 - c010) * dr);
                const float c01 = c001 + ((c101 - c001) * dr), c11 = c011 + ((c111 - c011) * dr);
                const float c0 = c00 + ((c10 - c00) * dg), c1 = c01 + ((c11 - c01) * dg);
                v = c0 + ((c1 - c0) * db);
            } else if (dr >= dg && dg >= db) {
                v = add_delta(add_delta(add_delta(c000, c000, c100, dr), c100, c110, dg), c110, c111, db);
            } else if (dr >= db && db >= dg) {
                v = add_delta(add_delta(add_delta(c000, c000, c100, dr), c100, c101, db), c101, c111, dg);
            } else if (db >= dr && dr >= dg) {
                v = add_delta(add_delta(add_delta(c000, c000, c001, db), c001, c101, dr), c101, c111, dg);
            } else if (dg >= dr && dr >= db) {
                v = add_delta(add_delta(add_delta(c000, c000, c010, dg), c010, c110, dr), c110, c111, db);
            } else if (dg >= db && db >= dr) {
                v = add_delta(add_delta(add_delta(c000, c000, c010, dg), c010, c011, db), c011, c111, dr);
            } else {
                v = add_delta(add_delta(add_delta(c000, c000, c001, db), c001, c011, dg), c011, c111, dr);
            }
            out[4 * i + c] = rnd(clampf(v, 0.0F, 1.0F), f16);
        }
        out[4 * i + 3] = in[4 * i + 3];
    }
}

/* ---- a16: filmic RGB (tone/filmic_rgb_generator.cpp:22-70) ---- */
void oracle_filmic(const float* in, float* out, int w, int h, const cpipe_FilmicRgbParams* p, int f16) {
    const float exposure = powf(2.0F, p->ev);
    const float inv_contrast = 1.0F / p->contrast;
    /* log(1 + 6*18) is a compile-time constant in the generator; folded in double. */
    const float log_white = (float)log(109.0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)w * h; ++i) {
        float t[3];
        for (int c = 0; c < 3; ++c) {
            const float e = maxf(0.0F, in[4 * i + c] * exposure);
            const float curved = clampf(logf(1.0F + (6.0F * e)) / log_white, 0.0F, 1.0F);
            const float v = powf(maxf(0.0F, curved), inv_contrast);
            const float sd = (p->shadows - 1.0F) * 0.08F * (1.0F - v) * (1.0F - v);
            const float hd = (p->highlights - 1.0F) * 0.08F * v * v;
            t[c] = clampf(v + sd + hd, 0.0F, 1.0F);
        }
        const float luma = (0.2126F * t[0]) + (0.7152F * t[1]) + (0.0722F * t[2]);
        for (int c = 0; c < 3; ++c)
            out[4 * i + c] = rnd(clampf(luma + ((t[c] - luma) * p->saturation), 0.0F, 1.0F), f16);
        out[4 * i + 3] = in[4 * i + 3];
    }
}

/* ---- a14: OpcodeList3 (lens/dng_opcode_list_3_dispatch.cpp:33-398) ---- */
static inline long po(int w, int x, int y, int c) { return ((long)y * w + x) * 4 + c; }
static inline float op_px(const float* im, int w, int h, int x, int y, int c) {
    return im[po(w, clampi(x, 0, w - 1), clampi(y, 0, h - 1), c)];
}
static inline float cubicf(float p0, float p1, float p2, float p3, float t) {
    const float a0 = (-0.5F * p0) + (1.5F * p1) - (1.5F * p2) + (0.5F * p3);
    const float a1 = p0 - (2.5F * p1) + (2.0F * p2) - (0.5F * p3);
    const float a2 = (-0.5F * p0) + (0.5F * p2);
    return (((a0 * t) + a1) * t + a2) * t + p1;
}
static float bicubic(const float* im, int w, int h, double x, double y, int c) {
    x = x < 0.0 ? 0.0 : (x > (double)(w - 1) ? (double)(w - 1) : x);
    y = y < 0.0 ? 0.0 : (y > (double)(h - 1) ? (double)(h - 1) : y);
    const int ix = (int)floor(x), iy = (int)floor(y);
    const float tx = (float)(x - (double)ix), ty = (float)(y - (double)iy);
    float rows[4];
    for (int r = 0; r < 4; ++r) {
        const int sy = iy + r - 1;
        rows[r] = cubicf(op_px(im, w, h, ix - 1, sy, c), op_px(im, w, h, ix, sy, c),
                         op_px(im, w, h, ix + 1, sy, c), op_px(im, w, h, ix + 2, sy, c), tx);
    }
    return cubicf(rows[0], rows[1], rows[2], rows[3], ty);
}
static double max_corner(double cx, double cy, int w, int h) {
    const double x1 = (double)(w - 1), y1 = (double)(h - 1);
    const double d00 = (cx * cx) + (cy * cy), d10 = ((x1 - cx) * (x1 - cx)) + (cy * cy);
    const double d01 = (cx * cx) + ((y1 - cy) * (y1 - cy));
    const double d11 = ((x1 - cx) * (x1 - cx)) + ((y1 - cy) * (y1 - cy));
    double m = d00;
    if (d10 > m) m = d10;
    if (d01 > m) m = d01;
    if (d11 > m) m = d11;
    return sqrt(m);
}
static float patched(const float* src, int w, int h, int x, int y, int c) {
    static const int kdx[4] = {-1, 1, 0, 0}, kdy[4] = {0, 0, -1, 1};
    float sum = 0.0F;
    int n = 0;
    for (int i = 0; i < 4; ++i) {
        const int nx = x + kdx[i], ny = y + kdy[i];
        if (nx < 0 || nx >= w || ny < 0 || ny >= h) continue;
        sum += op_px(src, w, h, nx, ny, c);
        ++n;
    }
    if (n == 0) return op_px(src, w, h, x, y, c);
    return sum / (float)n;
}
static void patch_px(const float* src, float* dst, int w, int h, int x, int y, int f16) {
    if (x < 0 || x >= w || y < 0 || y >= h) return;
    for (int c = 0; c < 3; ++c) dst[po(w, x, y, c)] = rnd(patched(src, w, h, x, y, c), f16);
}

/* `work` and `next` are caller-provided w*h*4 scratch arrays; result ends in out. */
int oracle_opcode3(const float* in, float* out, float* work, float* next, int w, int h,
                   const void* blob, size_t blob_size, int f16) {
    if (blob == NULL || blob_size < sizeof(cpipe_Opcode3DispatchHeader)) return ST_BAD_INDEX;
    const cpipe_Opcode3DispatchHeader* hd = (const cpipe_Opcode3DispatchHeader*)blob;
    const size_t rec_bytes = (size_t)hd->opcode_count * sizeof(cpipe_Opcode3DispatchRecord);
    if (blob_size < sizeof(*hd) + rec_bytes) return ST_BAD_INDEX;
    const cpipe_Opcode3DispatchRecord* recs = (const cpipe_Opcode3DispatchRecord*)((const char*)blob + sizeof(*hd));
    size_t npt = 0, nrc = 0;
    for (uint32_t i = 0; i < hd->opcode_count; ++i) {
        if ((size_t)recs[i].point_offset + recs[i].point_count > npt) npt = (size_t)recs[i].point_offset + recs[i].point_count;
        if ((size_t)recs[i].rect_offset + recs[i].rect_count > nrc) nrc = (size_t)recs[i].rect_offset + recs[i].rect_count;
    }
    const size_t pts_off = sizeof(*hd) + rec_bytes;
    const size_t rc_off = pts_off + npt * sizeof(cpipe_Opcode3BadPoint);
    if (blob_size < rc_off + nrc * sizeof(cpipe_Opcode3BadRect)) return ST_BAD_INDEX;
    const cpipe_Opcode3BadPoint* pts = (const cpipe_Opcode3BadPoint*)((const char*)blob + pts_off);
    const cpipe_Opcode3BadRect* rcs = (const cpipe_Opcode3BadRect*)((const char*)blob + rc_off);
    if (w <= 0 || h <= 0) return ST_BAD_INDEX;
    const long n = (long)w * h * 4;
    memcpy(work, in, (size_t)n * sizeof(float));
    for (uint32_t k = 0; k < hd->opcode_count; ++k) {
        const cpipe_Opcode3DispatchRecord* r = &recs[k];
        memcpy(next, work, (size_t)n * sizeof(float));
        switch (r->id) {
            case CPIPE_OPCODE3_UNKNOWN:
                if (r->optional == 0U) return ST_UNSUPPORTED;
                continue;
            case CPIPE_OPCODE3_WARP_RECTILINEAR: { /* apply_warp :89-124 */
                if (r->coefficient_count == 0U || w <= 1 || h <= 1) break;
                const double cx = r->cx_hat * (double)(w - 1), cy = r->cy_hat * (double)(h - 1);
                const double m = max_corner(cx, cy, w, h);
                if (m <= 2.220446049250313e-16) break;
                /* single-threaded, as the reference's plain-C++ filter */
                for (int y = 0; y < h; ++y)
                    for (int x = 0; x < w; ++x) {
                        const double dx = ((double)x - cx) / m, dy = ((double)y - cy) / m;
                        const double r2 = (dx * dx) + (dy * dy), r4 = r2 * r2, r6 = r4 * r2;
                        for (int c = 0; c < 4; ++c) {
                            const uint32_t ci = (uint32_t)c < r->coefficient_count - 1U ? (uint32_t)c : r->coefficient_count - 1U;
                            const cpipe_Opcode3WarpCoefficient* q = &r->coefficients[ci];
                            const double f = q->kr0 + (q->kr1 * r2) + (q->kr2 * r4) + (q->kr3 * r6);
                            const double tx = (2.0 * q->kt0 * dx * dy) + (q->kt1 * (r2 + 2.0 * dx * dx));
                            const double ty = (q->kt0 * (r2 + 2.0 * dy * dy)) + (2.0 * q->kt1 * dx * dy);
                            const double sx = cx + (m * ((f * dx) + tx));
                            const double sy = cy + (m * ((f * dy) + ty));
                            next[po(w, x, y, c)] = rnd(bicubic(work, w, h, sx, sy, c), f16);
                        }
                    }
                break;
            }
            case CPIPE_OPCODE3_FIX_VIGNETTE_RADIAL: { /* apply_vignette :126-158 */
                if (w <= 1 || h <= 1) break;
                const double cx = r->vignette_cx_hat * (double)(w - 1), cy = r->vignette_cy_hat * (double)(h - 1);
                const double m = max_corner(cx, cy, w, h);
                if (m <= 2.220446049250313e-16) break;
                for (int y = 0; y < h; ++y)
                    for (int x = 0; x < w; ++x) {
                        const double dx = ((double)x - cx) / m, dy = ((double)y - cy) / m;
                        const double r2 = (dx * dx) + (dy * dy), r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4, r10 = r8 * r2;
                        const double gain = 1.0 + (r->vignette_k[0] * r2) + (r->vignette_k[1] * r4) +
                                            (r->vignette_k[2] * r6) + (r->vignette_k[3] * r8) + (r->vignette_k[4] * r10);
                        for (int c = 0; c < 3; ++c)
                            next[po(w, x, y, c)] = rnd((float)((double)work[po(w, x, y, c)] * gain), f16);
                    }
                break;
            }
            case CPIPE_OPCODE3_FIX_BAD_PIXELS_CONSTANT: { /* :160-203 */
                const float k = (float)r->constant;
                for (int y = 0; y < h; ++y)
                    for (int x = 0; x < w; ++x) {
                        int p = 0;
                        for (int c = 0; c < 3; ++c) p = p || fabsf(op_px(work, w, h, x, y, c) - k) <= 0.0001F;
                        if (p) patch_px(work, next, w, h, x, y, f16);
                    }
                break;
            }
            case CPIPE_OPCODE3_FIX_BAD_PIXELS_LIST: { /* :205-233 */
                for (uint32_t i = 0; i < r->point_count; ++i) {
                    const cpipe_Opcode3BadPoint* q = &pts[(size_t)r->point_offset + i];
                    patch_px(work, next, w, h, (int)q->column, (int)q->row, f16);
                }
                for (uint32_t i = 0; i < r->rect_count; ++i) {
                    const cpipe_Opcode3BadRect* q = &rcs[(size_t)r->rect_offset + i];
                    const int top = (int)q->top < h ? (int)q->top : h, bottom = (int)q->bottom < h ? (int)q->bottom : h;
                    const int left = (int)q->left < w ? (int)q->left : w, right = (int)q->right < w ? (int)q->right : w;
                    for (int y = top > 0 ? top : 0; y < (bottom > 0 ? bottom : 0); ++y)
                        for (int x = left > 0 ? left : 0; x < (right > 0 ? right : 0); ++x) patch_px(work, next, w, h, x, y, f16);
                }
                break;
            }
            case CPIPE_OPCODE3_TRIM_BOUNDS: { /* :235-252 */
                for (int y = 0; y < h; ++y)
                    for (int x = 0; x < w; ++x) {
                        const int inside = (uint32_t)y >= r->top && (uint32_t)y < r->bottom &&
                                           (uint32_t)x >= r->left && (uint32_t)x < r->right;
                        if (inside) continue;
                        for (int c = 0; c < 4; ++c) next[po(w, x, y, c)] = 0.0F;
                    }
                break;
            }
            default:
                return ST_UNSUPPORTED;
        }
        float* t = work;
        work = next;
        next = t;
    }
    memcpy(out, work, (size_t)n * sizeof(float));
    return OK;
}
