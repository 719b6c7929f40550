// Device-side math for every node of the raw->linear chain.  Each function
// keeps the reference's floating-point operation order (cited per function) so
// that, with -fmad=false, a kernel built from it reproduces the reference
// arithmetic; the per-node kernels (kernels_nodes.cu) and the fused chain
// kernels (chain.cu) share these definitions.
#pragma once

#include "common.cuh"

namespace cpb {

// ---------------------------------------------------------------- raw domain
// Black/white scaling with the per-CFA-index constants precomputed on the host
// exactly as the reference does per pixel (blacklevel_dng_levels_dispatch.cpp:31-45).
struct BlackDev {
    float black[4];  // indexed by (y&1)*2 + (x&1)
    float denom[4];  // float(white_level) - black
};
__device__ __forceinline__ float blacklevel_px(float v, int x, int y, const BlackDev& p) {
    const int i = ((y & 1) * 2) + (x & 1);
    return clampf((v - p.black[i]) / p.denom[i], 0.0F, 1.0F);
}

// GainMap: axis samples are evaluated on the host in double, exactly as
// sample_axis (shading_gainmap_dispatch.cpp:23-36), and stored per column / row.
struct AxisSample {
    uint32_t low, high;
    float weight;
};
struct GainMapDev {
    int map_count;
    int qbc;                   // 4x4 CFA repeat: plane from (y%4)/2, (x%4)/2
    int plane_to_map[4];       // -1 when no map covers that plane
    const float* gains[4];     // per map, row-major map_points_v x map_points_h
    int points_h[4], points_v[4];
    const AxisSample* cols[4]; // per map, w entries
    const AxisSample* rows[4]; // per map, h entries
    // per map, points_v x hw: the horizontal interpolation of each grid row at
    // every image column (gainmap_hrows_kernel), shared by all image rows
    const float* hrow[4];
    int hw;
};
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + ((b - a) * t); }
__device__ __forceinline__ int gain_map_index(int x, int y, const GainMapDev& g) {
    if (g.map_count == 1) return 0;
    int plane = ((y & 1) * 2) + (x & 1);
    if (g.qbc) plane = (((y % 4) / 2) * 2) + ((x % 4) / 2);
    return g.plane_to_map[plane];
}
// The reference's bilinear gain (shading_gainmap_dispatch.cpp:38-72):
// lerp(lerp(g00, g10, wx), lerp(g01, g11, wx), wy).  The inner lerps depend
// on the grid row and the column only, so they are evaluated once per (grid
// row, column) into hrow (gain_hrow, same operands and order) and the pixel
// reads the two it needs.
__device__ __forceinline__ float gain_hrow(int m, int r, int x, const GainMapDev& g) {
    const AxisSample sx = g.cols[m][x];
    const float* gm = g.gains[m] + r * g.points_h[m];
    return lerpf(__ldg(gm + sx.low), __ldg(gm + sx.high), sx.weight);
}
__device__ __forceinline__ float gain_px(int m, int x, int y, const GainMapDev& g) {
    const AxisSample sy = g.rows[m][y];
    const float* h = g.hrow[m];
    return lerpf(__ldg(h + (size_t)sy.low * g.hw + x), __ldg(h + (size_t)sy.high * g.hw + x), sy.weight);
}

// ----------------------------------------------------------------- demosaic
// The three demosaics read a shared-memory tile `t` holding the clamped input
// (repeat_edge) with a fixed halo; `T(dx,dy)` addresses it relative to the
// pixel being evaluated.  cfa_at uses unclamped coordinates, as the generator's
// cfa_at(x, y) = cfa_pattern((y & 1) * 2 + (x & 1)) does.
struct Cfa {
    int p[4];
    __device__ __forceinline__ int at(int x, int y) const { return p[((y & 1) * 2) + (x & 1)]; }
};

// demosaic_rcd_generator.cpp:28-35
template <class Tap>
__device__ __forceinline__ float rcd_green(const Tap& T, int x, int y, const Cfa& cfa) {
    const float c = T(0, 0);
    const float gh = 0.5F * (T(-1, 0) + T(1, 0));
    const float gv = 0.5F * (T(0, -1) + T(0, 1));
    const float dh = fabsf(T(-2, 0) - T(2, 0));
    const float dv = fabsf(T(0, -2) - T(0, 2));
    if (cfa.at(x, y) == 1) return c;
    if (dh < dv) return gh;
    if (dv < dh) return gv;
    return 0.5F * (gh + gv);
}
// demosaic_amaze_generator.cpp:24-46
template <class Tap>
__device__ __forceinline__ float amaze_green(const Tap& T, int x, int y, const Cfa& cfa) {
    const float c = T(0, 0);
    if (cfa.at(x, y) == 1) return c;
    const float ct = 2.0F * c;
    const float ghn = T(-1, 0) + T(1, 0);
    const float gvn = T(0, -1) + T(0, 1);
    const float ghs = ct - T(-2, 0) - T(2, 0);
    const float gvs = ct - T(0, -2) - T(0, 2);
    const float gh = (0.5F * ghn) + (0.25F * ghs);
    const float gv = (0.5F * gvn) + (0.25F * gvs);
    const float grh = fabsf(T(-1, 0) - T(1, 0)) + fabsf(T(-2, 0) - c) + fabsf(T(2, 0) - c);
    const float grv = fabsf(T(0, -1) - T(0, 1)) + fabsf(T(0, -2) - c) + fabsf(T(0, 2) - c);
    if (grh < grv) return gh;
    if (grv < grh) return gv;
    return 0.5F * (gh + gv);
}

// ------------------------------------------------------------ RGBA pixel ops
// wb_dual_illuminant_dispatch.cpp:31-45: rgb / AsShotNeutral, alpha copied.
__device__ __forceinline__ Rgba wb_px(Rgba v, const float n[3]) {
    return Rgba{v.r / n[0], v.g / n[1], v.b / n[2], v.a};
}
// colormatrix_dng_to_working_dispatch.cpp:33-50
__device__ __forceinline__ Rgba cm_px(Rgba v, const float t[9]) {
    return Rgba{t[0] * v.r + t[1] * v.g + t[2] * v.b, t[3] * v.r + t[4] * v.g + t[5] * v.b,
                t[6] * v.r + t[7] * v.g + t[8] * v.b, v.a};
}

// x / d for a divisor fixed per launch, by Markstein's method (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): with inv = RN(1/d), q0 = RN(x inv),
// the exact remainder r = x - q0 d (one FMA) and q = RN(q0 + r inv) (one FMA).
// Used only where |x| lies in [2^-90, 2^126] (ConstDiv::ok); the library's
// self-test (cpipe_cuda_selftest_const_division) compares it with IEEE
// division on every binary32 in that range for each divisor the kernels use
// (the box sizes 9 and 25).
struct ConstDiv {
    float d, inv;  // inv = 1/d rounded to nearest (computed on the host in double)
};
__device__ __forceinline__ bool const_div_ok(float x) {
    const float a = fabsf(x);
    return a >= 0x1p-90F && a <= 0x1p126F;
}
__device__ __forceinline__ float const_div(float x, const ConstDiv& c) {
    if (!const_div_ok(x)) return x / c.d;
    const float q0 = __fmul_rn(x, c.inv);
    const float r = __fmaf_rn(-q0, c.d, x);
    return __fmaf_rn(r, c.inv, q0);
}

// filmic_rgb_generator.cpp:22-36,57-70.  exposure = pow(2, ev) and
// inv_contrast = 1/contrast are computed once per launch on the host with the
// same float operations; log_white = log(109) is the generator's constant.
struct FilmicDev {
    float exposure, inv_contrast, saturation, highlights, shadows, log_white;
};
// Two exact shortcuts for the default parameters: pow(x, 1) == x for x >= 0
// (the reference's libm powf returns x exactly), and with shadows == highlights
// == 1 both range terms are +0, so v + sd + hd == v.
__device__ __forceinline__ float filmic_tone(float value, const FilmicDev& p) {
    const float e = max0(value * p.exposure);
    const float curved = clampf(logf(1.0F + (6.0F * e)) / p.log_white, 0.0F, 1.0F);
    const float v = p.inv_contrast == 1.0F ? max0(curved) : powf(max0(curved), p.inv_contrast);
    if (p.shadows == 1.0F && p.highlights == 1.0F) return clampf(v, 0.0F, 1.0F);
    const float sd = (p.shadows - 1.0F) * 0.08F * (1.0F - v) * (1.0F - v);
    const float hd = (p.highlights - 1.0F) * 0.08F * v * v;
    return clampf(v + sd + hd, 0.0F, 1.0F);
}
__device__ __forceinline__ Rgba filmic_px(Rgba v, const FilmicDev& p) {
    const float t0 = filmic_tone(v.r, p), t1 = filmic_tone(v.g, p), t2 = filmic_tone(v.b, p);
    const float luma = (0.2126F * t0) + (0.7152F * t1) + (0.0722F * t2);
    return Rgba{clampf(luma + ((t0 - luma) * p.saturation), 0.0F, 1.0F),
                clampf(luma + ((t1 - luma) * p.saturation), 0.0F, 1.0F),
                clampf(luma + ((t2 - luma) * p.saturation), 0.0F, 1.0F), v.a};
}

// tone.aces_filmic (aces_filmic_generator.cpp:22-31): the Narkowicz 2016 fit.
__device__ __forceinline__ float aces_fit(float v) {
    v = max0(v);
    return clampf((v * ((2.51F * v) + 0.03F)) / ((v * ((2.43F * v) + 0.59F)) + 0.14F), 0.0F, 1.0F);
}
// tone.reinhard (reinhard_generator.cpp:22-28): clamp(v (1 + v / wp^2) / (1 + v), 0, 1), v = max(0, x).
__device__ __forceinline__ float reinhard_px(float x, float wp2) {
    const float v = max0(x);
    return clampf((v * (1.0F + (v / wp2))) / (1.0F + v), 0.0F, 1.0F);
}

// lut3d_generator.cpp:49-138.  The LUT is stored as float4 (r,g,b,0) per cell,
// cell index ((r*S + g)*S + b), blue fastest (reference color/lut3d_generator.cpp:83-86).
__device__ __forceinline__ float add_delta(float base, float from, float to, float w) {
    return base + ((to - from) * w);
}
__device__ __forceinline__ float4 add_delta4(float4 base, float4 from, float4 to, float w) {
    return make_float4(add_delta(base.x, from.x, to.x, w), add_delta(base.y, from.y, to.y, w),
                       add_delta(base.z, from.z, to.z, w), 0.0F);
}
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(a.x + ((b.x - a.x) * t), a.y + ((b.y - a.y) * t), a.z + ((b.z - a.z) * t), 0.0F);
}
__device__ __forceinline__ Rgba lut_px(Rgba v, const float4* __restrict__ lut, int S, int interp) {
    const float mi = (float)(S - 1);
    const float rs = clampf(v.r, 0.0F, 1.0F) * mi;
    const float gs = clampf(v.g, 0.0F, 1.0F) * mi;
    const float bs = clampf(v.b, 0.0F, 1.0F) * mi;
    const int r0 = clampi((int)floorf(rs), 0, S - 2);
    const int g0 = clampi((int)floorf(gs), 0, S - 2);
    const int b0 = clampi((int)floorf(bs), 0, S - 2);
    const float dr = rs - (float)r0, dg = gs - (float)g0, db = bs - (float)b0;
    const int base = (r0 * S + g0) * S + b0;
    const int sr = S * S, sg = S;
    const float4 c000 = __ldg(lut + base);
    const float4 c111 = __ldg(lut + base + sr + sg + 1);
    float4 o;
    if (interp == 1) {
        const float4 c100 = __ldg(lut + base + sr), c010 = __ldg(lut + base + sg);
        const float4 c001 = __ldg(lut + base + 1), c110 = __ldg(lut + base + sr + sg);
        const float4 c101 = __ldg(lut + base + sr + 1), c011 = __ldg(lut + base + sg + 1);
        const float4 c00 = lerp4(c000, c100, dr), c10 = lerp4(c010, c110, dr);
        const float4 c01 = lerp4(c001, c101, dr), c11 = lerp4(c011, c111, dr);
        const float4 c0 = lerp4(c00, c10, dg), c1 = lerp4(c01, c11, dg);
        o = lerp4(c0, c1, db);
    } else {
        // Tetrahedral: the first matching branch of the generator's select chain;
        // each branch reads only the two intermediate corners it walks through.
        int s1, s2;
        float w1, w2, w3;
        if (dr >= dg && dg >= db) { s1 = sr; s2 = sr + sg; w1 = dr; w2 = dg; w3 = db; }
        else if (dr >= db && db >= dg) { s1 = sr; s2 = sr + 1; w1 = dr; w2 = db; w3 = dg; }
        else if (db >= dr && dr >= dg) { s1 = 1; s2 = sr + 1; w1 = db; w2 = dr; w3 = dg; }
        else if (dg >= dr && dr >= db) { s1 = sg; s2 = sr + sg; w1 = dg; w2 = dr; w3 = db; }
        else if (dg >= db && db >= dr) { s1 = sg; s2 = sg + 1; w1 = dg; w2 = db; w3 = dr; }
        else { s1 = 1; s2 = sg + 1; w1 = db; w2 = dg; w3 = dr; }
        const float4 ca = __ldg(lut + base + s1), cb = __ldg(lut + base + s2);
        o = add_delta4(add_delta4(add_delta4(c000, c000, ca, w1), ca, cb, w2), cb, c111, w3);
    }
    return Rgba{clampf(o.x, 0.0F, 1.0F), clampf(o.y, 0.0F, 1.0F), clampf(o.z, 0.0F, 1.0F), v.a};
}

// The same interpolation as lut_px with the cells read through `fetch(i)`
// (cell i as float4 r, g, b, -), for LUTs stored in another layout.
template <class Fetch>
__device__ __forceinline__ Rgba lut_px_cells(Rgba v, const Fetch& fetch, int S, int interp) {
    const float mi = (float)(S - 1);
    const float rs = clampf(v.r, 0.0F, 1.0F) * mi;
    const float gs = clampf(v.g, 0.0F, 1.0F) * mi;
    const float bs = clampf(v.b, 0.0F, 1.0F) * mi;
    const int r0 = clampi((int)floorf(rs), 0, S - 2);
    const int g0 = clampi((int)floorf(gs), 0, S - 2);
    const int b0 = clampi((int)floorf(bs), 0, S - 2);
    const float dr = rs - (float)r0, dg = gs - (float)g0, db = bs - (float)b0;
    const int base = (r0 * S + g0) * S + b0;
    const int sr = S * S, sg = S;
    const float4 c000 = fetch(base);
    const float4 c111 = fetch(base + sr + sg + 1);
    float4 o;
    if (interp == 1) {
        const float4 c100 = fetch(base + sr), c010 = fetch(base + sg);
        const float4 c001 = fetch(base + 1), c110 = fetch(base + sr + sg);
        const float4 c101 = fetch(base + sr + 1), c011 = fetch(base + sg + 1);
        const float4 c00 = lerp4(c000, c100, dr), c10 = lerp4(c010, c110, dr);
        const float4 c01 = lerp4(c001, c101, dr), c11 = lerp4(c011, c111, dr);
        const float4 c0 = lerp4(c00, c10, dg), c1 = lerp4(c01, c11, dg);
        o = lerp4(c0, c1, db);
    } else {
        // Tetrahedral: the first matching branch of the generator's select chain;
        // each branch reads only the two intermediate corners it walks through.
        int s1, s2;
        float w1, w2, w3;
        if (dr >= dg && dg >= db) { s1 = sr; s2 = sr + sg; w1 = dr; w2 = dg; w3 = db; }
        else if (dr >= db && db >= dg) { s1 = sr; s2 = sr + 1; w1 = dr; w2 = db; w3 = dg; }
        else if (db >= dr && dr >= dg) { s1 = 1; s2 = sr + 1; w1 = db; w2 = dr; w3 = dg; }
        else if (dg >= dr && dr >= db) { s1 = sg; s2 = sr + sg; w1 = dg; w2 = dr; w3 = db; }
        else if (dg >= db && db >= dr) { s1 = sg; s2 = sg + 1; w1 = dg; w2 = db; w3 = dr; }
        else { s1 = 1; s2 = sg + 1; w1 = db; w2 = dg; w3 = dr; }
        const float4 ca = fetch(base + s1), cb = fetch(base + s2);
        o = add_delta4(add_delta4(add_delta4(c000, c000, ca, w1), ca, cb, w2), cb, c111, w3);
    }
    return Rgba{clampf(o.x, 0.0F, 1.0F), clampf(o.y, 0.0F, 1.0F), clampf(o.z, 0.0F, 1.0F), v.a};
}
// bm3d_step1_generator.cpp:42-56 (parity form): blend toward the aligned 2x2 mean.
__device__ __forceinline__ float bm3d_blend(float v, float p00, float p10, float p01, float p11, float s) {
    const float basic = (p00 + p10 + p01 + p11) * 0.25F;
    return max0((v * (1.0F - s)) + (basic * s));
}

// wavelet_bayes_shrink_generator.cpp:9-31,63-85
__device__ __forceinline__ float soft_th(float v, float t) {
    return v > t ? v - t : (v < -t ? v + t : 0.0F);
}
struct HaarBand { float ll, h, v, d; };
__device__ __forceinline__ HaarBand haar_shrink(float p00, float p10, float p01, float p11, float th) {
    HaarBand b;
    b.ll = 0.25F * (p00 + p10 + p01 + p11);
    b.h = soft_th(0.25F * (p00 - p10 + p01 - p11), th);
    b.v = soft_th(0.25F * (p00 + p10 - p01 - p11), th);
    b.d = soft_th(0.25F * (p00 - p10 - p01 + p11), th);
    return b;
}
__device__ __forceinline__ float haar_pick(const HaarBand& b, int ox, int oy) {
    if (ox == 0 && oy == 0) return b.ll + b.h + b.v + b.d;
    if (ox == 1 && oy == 0) return b.ll - b.h + b.v - b.d;
    if (ox == 0 && oy == 1) return b.ll + b.h - b.v - b.d;
    return b.ll - b.h - b.v + b.d;
}
__device__ __forceinline__ float wv_co(Rgba p) { return p.r - p.b; }
__device__ __forceinline__ float wv_cg(Rgba p) { return p.g - ((p.r + p.b) * 0.5F); }
// Output for pixel (ox, oy) of the aligned 2x2 block q[0..3] = (0,0),(1,0),(0,1),(1,1);
// `p` is that pixel (q[oy*2+ox], passed separately so q is never indexed at run time).
__device__ __forceinline__ Rgba wavelet_px(const Rgba q[4], const Rgba& p, int ox, int oy, float th) {
    const HaarBand bco = haar_shrink(wv_co(q[0]), wv_co(q[1]), wv_co(q[2]), wv_co(q[3]), th);
    const HaarBand bcg = haar_shrink(wv_cg(q[0]), wv_cg(q[1]), wv_cg(q[2]), wv_cg(q[3]), th);
    const float luma = (p.r + (2.0F * p.g) + p.b) * 0.25F;
    const float co = haar_pick(bco, ox, oy), cg = haar_pick(bcg, ox, oy);
    const float t = luma - (0.5F * cg);
    return Rgba{max0(t + (0.5F * co)), max0(t + cg), max0(t - (0.5F * co)), max0(p.a)};
}

// --------------------------------------------------------------- OpcodeList3
// Catmull-Rom cubic (dng_opcode_list_3_dispatch.cpp:48-53).
__device__ __forceinline__ float cubic(float p0, float p1, float p2, float p3, float t) {
    const float a0 = (-0.5F * p0) + (1.5F * p1) - (1.5F * p2) + (0.5F * p3);
    const float a1 = p0 - (2.5F * p1) + (2.0F * p2) - (0.5F * p3);
    const float a2 = (-0.5F * p0) + (0.5F * p2);
    return (((a0 * t) + a1) * t + a2) * t + p1;
}
__device__ __forceinline__ Rgba cubic4(Rgba p0, Rgba p1, Rgba p2, Rgba p3, float t) {
    return Rgba{cubic(p0.r, p1.r, p2.r, p3.r, t), cubic(p0.g, p1.g, p2.g, p3.g, t),
                cubic(p0.b, p1.b, p2.b, p3.b, t), cubic(p0.a, p1.a, p2.a, p3.a, t)};
}

// Warp coefficients converted to float-float on the host, in pixel units.
// The reference evaluates, in double (dng_opcode_list_3_dispatch.cpp:103-115),
//   dx = X/m, dy = Y/m, r2 = dx^2 + dy^2, f = kr0 + kr1 r2 + kr2 r2^2 + kr3 r2^3
//   sx = cx + m (f dx + 2 kt0 dx dy + kt1 (r2 + 2 dx^2))           (sy alike)
// with X = x - cx, Y = y - cy.  Multiplying the m through gives the same real
// number as
//   sx = x + (f - 1) X + 2 t0 X Y + t1 (q + 2 X^2),  q = X^2 + Y^2, r2 = q / m^2,
//   t0 = kt0 / m, t1 = kt1 / m,
// which needs far fewer float-float operations; its float-float error (~1e-12 px)
// is far below the binary32 spacing of the bicubic weight it feeds.
struct WarpCoefDev {
    ff kr0m1, kr1, kr2, kr3, t0, t1;  // kr0 - 1, kr1..kr3, kt0 / m, kt1 / m
    int has_kr3, has_tan;
};
struct WarpDev {
    int count;  // 1..4 coefficient sets; channel c uses min(c, count-1)
    WarpCoefDev k[4];
    ff cx, cy, inv_m2;  // inv_m2 = 1 / m^2
    float xmax, ymax;   // w-1, h-1
};
__device__ __forceinline__ ff ff_add_f(ff a, float b) {
    ff s = two_sum(a.hi, b);
    s.lo = __fadd_rn(s.lo, a.lo);
    return quick_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ ff ff_scale2(ff a) { return ff{a.hi * 2.0F, a.lo * 2.0F}; }
// Source coordinate of output pixel (x, y) for coefficient set k.
__device__ __forceinline__ void warp_src(const WarpCoefDev& k, float x, float y, ff X, ff Y, ff q, ff r2, ff* sx,
                                         ff* sy) {
    // (f - 1) by Horner in r2
    ff p = k.has_kr3 ? ff_add(k.kr2, ff_mul(r2, k.kr3)) : k.kr2;
    p = ff_add(k.kr1, ff_mul(r2, p));
    const ff fm1 = ff_add(k.kr0m1, ff_mul(r2, p));
    ff dx = ff_mul(fm1, X), dy = ff_mul(fm1, Y);
    if (k.has_tan) {
        const ff xy2 = ff_scale2(ff_mul(X, Y));
        dx = ff_add(dx, ff_add(ff_mul(k.t0, xy2), ff_mul(k.t1, ff_add(q, ff_scale2(ff_mul(X, X))))));
        dy = ff_add(dy, ff_add(ff_mul(k.t0, ff_add(q, ff_scale2(ff_mul(Y, Y)))), ff_mul(k.t1, xy2)));
    }
    *sx = ff_add_f(dx, x);
    *sy = ff_add_f(dy, y);
}
// Bicubic sample (all four channels) of the warp output pixel (x, y) for
// coefficient set k: source coordinate clamped to the frame, Catmull-Rom taps
// with clamped reads (sample_bicubic :55-73).
template <class T>
__device__ __forceinline__ Rgba warp_sample(const Img& in, const WarpDev& w, const WarpCoefDev& k, float x, float y,
                                            ff X, ff Y, ff q, ff r2);
// Clamp a float-float coordinate to [0, maxv] (sample_bicubic :57-58).
__device__ __forceinline__ ff ff_clamp0(ff v, float maxv) {
    if (v.hi < 0.0F || (v.hi == 0.0F && v.lo < 0.0F)) return ff_from(0.0F);
    if (v.hi > maxv || (v.hi == maxv && v.lo > 0.0F)) return ff_from(maxv);
    return v;
}

// Bicubic source position of an output pixel: the 4x4 footprint's origin + 1
// and the two fractions.
struct WarpTap {
    int ix, iy;
    float tx, ty;
};
__device__ __forceinline__ WarpTap warp_tap(const WarpDev& w, const WarpCoefDev& k, float x, float y, ff X, ff Y, ff q,
                                            ff r2) {
    ff sx, sy;
    warp_src(k, x, y, X, Y, q, r2, &sx, &sy);
    sx = ff_clamp0(sx, w.xmax);
    sy = ff_clamp0(sy, w.ymax);
    const int ix = ff_floor(sx), iy = ff_floor(sy);
    return WarpTap{ix, iy, ff_frac(sx, ix), ff_frac(sy, iy)};
}
// Catmull-Rom sample (all four channels) at a tap, clamped reads (sample_bicubic :55-73).
template <class T>
__device__ __forceinline__ Rgba bicubic_at(const Img& in, const WarpTap& t) {
    const int ix = t.ix, iy = t.iy;
    const float tx = t.tx, ty = t.ty;
    Rgba rows[4];
    if (ix >= 1 && ix + 2 < in.w && iy >= 1 && iy + 2 < in.h) {
        // the 4x4 footprint lies inside the frame: the same taps without clamping
        const T* base = px<const T>(in, ix - 1, iy - 1);
        const long long ps = in.pix_stride;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const T* row = base + (long long)r * in.row_stride;
            rows[r] = cubic4(load_rgba(row), load_rgba(row + ps), load_rgba(row + 2 * ps), load_rgba(row + 3 * ps), tx);
        }
        return cubic4(rows[0], rows[1], rows[2], rows[3], ty);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int yy = iy + r - 1;
        rows[r] = cubic4(load_clamped<T>(in, ix - 1, yy), load_clamped<T>(in, ix, yy), load_clamped<T>(in, ix + 1, yy),
                         load_clamped<T>(in, ix + 2, yy), tx);
    }
    return cubic4(rows[0], rows[1], rows[2], rows[3], ty);
}
template <class T>
__device__ __forceinline__ Rgba warp_sample(const Img& in, const WarpDev& w, const WarpCoefDev& k, float x, float y,
                                            ff X, ff Y, ff q, ff r2) {
    return bicubic_at<T>(in, warp_tap(w, k, x, y, X, Y, q, r2));
}
// The tap of output pixel (x, y) for coefficient set 0 (the whole pixel when count == 1).
__device__ __forceinline__ WarpTap warp_tap_px(const WarpDev& w, int x, int y) {
    const float fx = (float)x, fy = (float)y;
    const ff X = ff_add_f(ff_neg(w.cx), fx), Y = ff_add_f(ff_neg(w.cy), fy);
    const ff q = ff_add(ff_mul(X, X), ff_mul(Y, Y));
    const ff r2 = ff_mul(q, w.inv_m2);
    return warp_tap(w, w.k[0], fx, fy, X, Y, q, r2);
}

// Warp output pixel (x, y), all channels (channel c uses coefficient set min(c, count-1)).
template <class T>
__device__ __forceinline__ Rgba warp_px(const Img& in, const WarpDev& w, int x, int y) {
    const float fx = (float)x, fy = (float)y;
    const ff X = ff_add_f(ff_neg(w.cx), fx), Y = ff_add_f(ff_neg(w.cy), fy);
    const ff q = ff_add(ff_mul(X, X), ff_mul(Y, Y));
    const ff r2 = ff_mul(q, w.inv_m2);
    Rgba v = warp_sample<T>(in, w, w.k[0], fx, fy, X, Y, q, r2);
    if (w.count > 1) {
        const Rgba g = warp_sample<T>(in, w, w.k[1], fx, fy, X, Y, q, r2);
        v.g = g.g;
        v.b = g.b;
        v.a = g.a;
        if (w.count > 2) {
            const Rgba b = warp_sample<T>(in, w, w.k[2], fx, fy, X, Y, q, r2);
            v.b = b.b;
            v.a = b.a;
            if (w.count > 3) v.a = warp_sample<T>(in, w, w.k[3], fx, fy, X, Y, q, r2).a;
        }
    }
    return v;
}

// Guided-filter box sum: the D x D window of rows k..k+D-1 of `win`, added in
// the generator's row-major left-associated order (guided_filter_generator.cpp:60-76).
template <int D, int ROWS>
__device__ __forceinline__ float box_chain(const float (&win)[ROWS][D], int k) {
    float s = win[k][0];
#pragma unroll
    for (int dy = 0; dy < D; ++dy)
#pragma unroll
        for (int dx = 0; dx < D; ++dx)
            if (dy != 0 || dx != 0) s = s + win[k + dy][dx];
    return s;
}
// Two box sums in the same order at once, one per float2 component, with the
// sm_100 packed add (each component rounds exactly as __fadd_rn).
template <int D, int ROWS>
__device__ __forceinline__ float2 box_chain2(const float2 (&win)[ROWS][D], int k) {
    float2 s = win[k][0];
#pragma unroll
    for (int dy = 0; dy < D; ++dy)
#pragma unroll
        for (int dx = 0; dx < D; ++dx)
            if (dy != 0 || dx != 0) s = __fadd2_rn(s, win[k + dy][dx]);
    return s;
}

}  // namespace cpb
