// Spec-mode guided filter (aot_id denoise_guided_filter_spec) and multi-level
// a-trous wavelet denoiser (aot_id denoise_wavelet_atrous_spec) on sm_100a.
//
// The reference's denoise.guided_filter boxes with 3x3 when radius <= 1 and
// 5x5 for any larger radius (nodes/denoise/guided_filter_generator.cpp:11-28,
// 66-70); its denoise.wavelet_bayes_shrink is one 2x2 Haar level on chroma
// (wavelet_bayes_shrink_generator.cpp:57-86).  These are the forms the nodes
// are named after.  Definitions shared with the FP64 CPU oracle
// (oracle/oracle_spec_denoise.py):
//
// guided   per RGB channel, self-guided, the reference's formula with a true
//          (2r+1)^2 box: m = S/N, corr = Q/N, var = max(corr - m^2, 0),
//          a = var/(var + eps), b = m - a m at every position within r of the
//          output (positions outside the image included; every box reads the
//          clamped image), out = max(mean_a v + mean_b, 0); alpha copied.
// a-trous  the reference wavelet node's colour space, Y = (r+2g+b)/4,
//          Co = r-b, Cg = g-(r+b)/2; per channel c_0 = the channel,
//          c_{j+1} = h_j * c_j (separable B3 spline [1 4 6 4 1]/16 with taps
//          2^j apart, clamped edges), w_{j+1} = c_j - c_{j+1}; per band
//          sigma_n = sigma g_c n_j (g_Y = sqrt6/4, g_Co = sqrt2, g_Cg = sqrt1.5;
//          n_j the 2D white-noise gain of band j, atrous_band_gain),
//          sigma_w^2 = mean of w^2 over the frame, sigma_x = sqrt(max(sigma_w^2 -
//          sigma_n^2, 0)), T = strength sigma_n^2 / sigma_x (T = 0 when the
//          strength is 0, else infinite when sigma_x = 0); soft threshold;
//          c = c_L + sum of the shrunk bands (level L first); inverse colour
//          transform t = Y - Cg/2, (t + Co/2, t + Cg, t - Co/2) clamped at 0;
//          alpha copied.
//
// Kernels
//   gsp_ab / gsp_out     the guided filter as two tile kernels with sliding
//                        binary32 box sums along rows and columns (see below).
//   atrous_walk_kernel   one level: per block 256 columns and one residue class
//                        of rows (y = phi + k 2^j), each thread walking its
//                        column with the five vertical taps of each channel in
//                        registers (one new row per step), the horizontal taps
//                        through shared memory; c_{j+1} written, the block's
//                        sum of w_{j+1}^2 per channel; the first level reads
//                        c_0 (Y, Co, Cg) from the input frame.
//   atrous_thresh_kernel per (level, channel): the tiles' sums added in a fixed
//                        order (compensated binary32), the BayesShrink
//                        threshold.
//   atrous_recon_kernel  c_0 from the input, the bands c_j - c_{j+1} from the
//                        stored levels, shrink, sum, inverse colour transform.
#include "spec_denoise.h"

#include <math.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "../../include/cpipe_node_abi.h"
#include "kernels.h"

namespace cpb {
namespace {

// ------------------------------------------------------------------ guided
// Two tile kernels in binary32 with sliding box sums along both axes; the
// paired sums (sum v, sum v^2) and (sum a, sum b) run as sm_100 packed adds.
//   ab   per channel (grid z), a 64x32 tile of the extended domain
//        [-R, w+R) x [-R, h+R): the clamped image tile with its 2R halo staged
//        in shared memory by asynchronous copies; row sums of (v, v^2) over 2R+1 columns (one sliding
//        window per 16 outputs, restarted at each window); column sums of
//        those over 2R+1 rows (one window per 8 outputs); m = S/N, corr = Q/N
//        (products with the binary32 reciprocal of N), var = max(corr - m^2, 0),
//        a = var/(var+eps) (__fdividef: within 2 ulp), b = m - a m into the a
//        and b planes (extended domain, row pitch w + 2R).
//   out  per 64x32 output tile, the three channels in turn: the (a, b) pairs
//        with their 2R halo staged by asynchronous copies and box-summed the
//        same way; per pixel
//        out = max(mean_a v + mean_b, 0) (means as products with 1/N) held in
//        registers, then written with the input's alpha.
// Each running sum adds at most 2R+1 + 2 * 15 terms, so binary16 frames stay
// within one binary16 ulp of the FP64 definition and binary32 frames within
// 1e-5.  Shared-memory pitches are odd (in elements of the stored type), so
// the lanes of a warp (rows in the row pass, columns in the column pass) hit
// distinct banks.
constexpr int kGsTW = 64, kGsTH = 32, kGsRunX = 16, kGsRunY = 8, kGsThreads = 256;
static_assert(kGsTW * (kGsTH / kGsRunY) == kGsThreads, "one column window per thread");
static_assert((kGsTW / kGsRunX) * 64 == kGsThreads && kGsTH + 2 * kGuidedSpecMaxRadius <= 64,
              "one row window per thread: the staged rows fit 64 lanes");
struct GsPlanes {
    int w, h, R, Wa, Ha;
    float* a;  // [3][Ha][Wa]
    float* b;
};
GsPlanes gs_planes(int w, int h, int R, void* scratch) {
    GsPlanes p{w, h, R, w + 2 * R, h + 2 * R, nullptr, nullptr};
    p.a = static_cast<float*>(scratch);
    p.b = p.a + 3 * (size_t)p.Ha * p.Wa;
    return p;
}
__host__ __device__ constexpr int gs_pitch(int R) { return (kGsTW + 2 * R) | 1; }  // staged pitch (elements)
constexpr int kGsPH = kGsTW + 1;                                                  // row-sum pitch (float2)
// ab: scalar staged tile + float2 row sums; out: float2 staged tile + float2 row sums
__host__ __device__ constexpr size_t gs_ab_smem(int R) {
    return (size_t)(kGsTH + 2 * R) * gs_pitch(R) * 4 + (size_t)(kGsTH + 2 * R) * kGsPH * 8;
}
__host__ __device__ constexpr size_t gs_out_smem(int R) {
    return (size_t)(kGsTH + 2 * R) * gs_pitch(R) * 8 + (size_t)(kGsTH + 2 * R) * kGsPH * 8;
}
__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }
// 4-byte asynchronous global -> shared copies: a warp's whole staging is in
// flight at once instead of one dependent load per iteration.
__device__ __forceinline__ void gs_cp4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void gs_cp_wait() { asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory"); }
// A staged 32-bit word -> the channel's value: binary32 frames stage the value,
// binary16 frames the word holding channels (c & ~1, c | 1).
template <class T>
__device__ __forceinline__ float gs_val(uint32_t word, int c);
template <>
__device__ __forceinline__ float gs_val<float>(uint32_t word, int) { return __uint_as_float(word); }
template <>
__device__ __forceinline__ float gs_val<__half>(uint32_t word, int c) {
    return __half2float(__ushort_as_half((unsigned short)((c & 1) ? (word >> 16) : (word & 0xFFFFU))));
}

template <class T>
__global__ void __launch_bounds__(kGsThreads) gsp_ab_kernel(Img in, GsPlanes p, float eps) {
    extern __shared__ float4 gsm4[];
    float* gsm = reinterpret_cast<float*>(gsm4);
    const int R = p.R, D = 2 * R + 1, SR = kGsTH + 2 * R, SC = kGsTW + 2 * R, PV = gs_pitch(R);
    float* sv = gsm;
    float2* hs = reinterpret_cast<float2*>(gsm + ((SR * PV + 1) & ~1));
    const int c = blockIdx.z, X0 = blockIdx.x * kGsTW, Y0 = blockIdx.y * kGsTH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // plane column X0 + q's box starts at image column X0 - 2R + q
    const int cw = std::is_same<T, float>::value ? c : (c & ~1);  // element of the staged word
    for (int r = warp; r < SR; r += kGsThreads / 32) {
        const T* row = px<const T>(in, 0, clampi(Y0 - 2 * R + r, 0, in.h - 1)) + cw;
        float* dst = sv + r * PV;
        for (int q = lane; q < SC; q += 32) gs_cp4(dst + q, row + 4 * clampi(X0 - 2 * R + q, 0, in.w - 1));
    }
    gs_cp_wait();
    __syncthreads();
    // row pass: one window per thread, rows on the lanes (SR <= 64 rows)
    {
        const int r = threadIdx.x & 63, x0 = (threadIdx.x >> 6) * kGsRunX;
        if (r < SR) {
        const uint32_t* row = reinterpret_cast<const uint32_t*>(sv) + r * PV + x0;
        float2 s = make_float2(0.0F, 0.0F);
#pragma unroll 4
        for (int k = 0; k < D; ++k) {
            const float v = gs_val<T>(row[k], c);
            s = __fadd2_rn(s, make_float2(v, v * v));
        }
        float2* o = hs + r * kGsPH + x0;
        o[0] = s;
#pragma unroll
        for (int x = 1; x < kGsRunX; ++x) {
            const float vi = gs_val<T>(row[x + D - 1], c), vo = gs_val<T>(row[x - 1], c);
            s = __fadd2_rn(__fadd2_rn(s, make_float2(vi, vi * vi)), make_float2(-vo, -(vo * vo)));
            o[x] = s;
        }
        }
    }
    __syncthreads();
    const float invN = 1.0F / (float)(D * D);
    const int x = threadIdx.x % kGsTW, y0 = (threadIdx.x / kGsTW) * kGsRunY;
    const int xa = X0 + x;
    float2 S = make_float2(0.0F, 0.0F);
#pragma unroll 4
    for (int k = 0; k < D; ++k) S = __fadd2_rn(S, hs[(y0 + k) * kGsPH + x]);
    const size_t plane = (size_t)p.Ha * p.Wa;
    // plane offsets fit 32 bits (Ha * Wa < 2^31 is checked on the host)
    float* pa = p.a + (size_t)c * plane + (unsigned)((Y0 + y0) * p.Wa + xa);
    float* pb = p.b + (size_t)c * plane + (unsigned)((Y0 + y0) * p.Wa + xa);
    const float2* hin = hs + (y0 + D) * kGsPH + x;
    const float2* hout = hs + y0 * kGsPH + x;
    const int nrow = min(kGsRunY, p.Ha - (Y0 + y0));
    const bool col = xa < p.Wa;
#pragma unroll
    for (int y = 0; y < kGsRunY; ++y) {
        if (y > 0) S = __fadd2_rn(__fadd2_rn(S, hin[(y - 1) * kGsPH]), neg2(hout[(y - 1) * kGsPH]));
        if (col && y < nrow) {
            const float2 mc = __fmul2_rn(S, make_float2(invN, invN));  // (m, corr)
            const float var = maxf(mc.y - mc.x * mc.x, 0.0F);
            const float a = __fdividef(var, var + eps);
            pa[y * p.Wa] = a;
            pb[y * p.Wa] = mc.x - a * mc.x;
        }
    }
}

template <class T>
__global__ void __launch_bounds__(kGsThreads, 4) gsp_out_kernel(Img in, Img out, GsPlanes p) {
    extern __shared__ float4 gsm4[];
    const int R = p.R, D = 2 * R + 1, SR = kGsTH + 2 * R, SC = kGsTW + 2 * R, PV = gs_pitch(R);
    float2* sab = reinterpret_cast<float2*>(gsm4);
    float2* hs = sab + SR * PV;
    const int X0 = blockIdx.x * kGsTW, Y0 = blockIdx.y * kGsTH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float invN = 1.0F / (float)(D * D);
    const size_t plane = (size_t)p.Ha * p.Wa;
    const int x = threadIdx.x % kGsTW, y0 = (threadIdx.x / kGsTW) * kGsRunY;
    const int gx = X0 + x;
    // output x reads plane columns x .. x + 2R (extended x - R .. x + R)
    auto stage = [&](int c) {
        const float* ca = p.a + (size_t)c * plane;
        const float* cb = p.b + (size_t)c * plane;
        for (int r = warp; r < SR; r += kGsThreads / 32) {
            const unsigned ro = (unsigned)min(Y0 + r, p.Ha - 1) * (unsigned)p.Wa;
            const float* ra = ca + ro;
            const float* rb = cb + ro;
            float2* dst = sab + r * PV;
            for (int q = lane; q < SC; q += 32) {
                const int xq = min(X0 + q, p.Wa - 1);
                gs_cp4(&dst[q].x, ra + xq);
                gs_cp4(&dst[q].y, rb + xq);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    stage(0);
    // the thread's eight input pixels (alpha and v), loaded once
    Rgba vin[kGsRunY];
#pragma unroll
    for (int y = 0; y < kGsRunY; ++y) {
        const int gy = Y0 + y0 + y;
        vin[y] = (gx < p.w && gy < p.h) ? load_rgba(px<const T>(in, gx, gy)) : Rgba{0.0F, 0.0F, 0.0F, 0.0F};
    }
    float res[3][kGsRunY];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (c > 0) stage(c);  // the previous channel's passes are done with sab
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        {
            const int r = threadIdx.x & 63, x0 = (threadIdx.x >> 6) * kGsRunX;
            if (r < SR) {
            const float2* row = sab + r * PV + x0;
            float2 s = make_float2(0.0F, 0.0F);
#pragma unroll 4
            for (int k = 0; k < D; ++k) s = __fadd2_rn(s, row[k]);
            float2* o = hs + r * kGsPH + x0;
            o[0] = s;
#pragma unroll
            for (int xx = 1; xx < kGsRunX; ++xx) {
                s = __fadd2_rn(__fadd2_rn(s, row[xx + D - 1]), neg2(row[xx - 1]));
                o[xx] = s;
            }
            }
        }
        __syncthreads();
        float2 S = make_float2(0.0F, 0.0F);
#pragma unroll 4
        for (int k = 0; k < D; ++k) S = __fadd2_rn(S, hs[(y0 + k) * kGsPH + x]);
        const float2* hin = hs + (y0 + D) * kGsPH + x;
        const float2* hout = hs + y0 * kGsPH + x;
#pragma unroll
        for (int y = 0; y < kGsRunY; ++y) {
            if (y > 0) S = __fadd2_rn(__fadd2_rn(S, hin[(y - 1) * kGsPH]), neg2(hout[(y - 1) * kGsPH]));
            const float2 mab = __fmul2_rn(S, make_float2(invN, invN));  // (mean_a, mean_b)
            const float v = c == 0 ? vin[y].r : (c == 1 ? vin[y].g : vin[y].b);
            res[c][y] = max0(mab.x * v + mab.y);
        }
        __syncthreads();  // the next channel restages sab and rewrites hs
    }
    if (gx >= p.w) return;
#pragma unroll
    for (int y = 0; y < kGsRunY; ++y) {
        const int gy = Y0 + y0 + y;
        if (gy < p.h) store_rgb_keep_alpha(px<T>(out, gx, gy), Rgba{res[0][y], res[1][y], res[2][y], 0.0F},
                                           px<const T>(in, gx, gy));
    }
}

// ----------------------------------------------------------------- a-trous
// Scratch holds c_1 .. c_L (three FP32 planes each); the bands are never
// stored: w_{j+1} = c_j - c_{j+1} is formed again where it is needed (the
// same binary32 subtraction of the same stored values), and c_0 comes from the
// input frame each time (the same colour transform).
constexpr int kAtThreads = 256;  // level block: 256 columns

template <class T>
__device__ __forceinline__ void atrous_c0(const Img& in, int x, int y, float& Y, float& Co, float& Cg) {
    const Rgba p = load_rgba(px<const T>(in, x, y));
    Y = (p.r + 2.0F * p.g + p.b) * 0.25F;
    Co = p.r - p.b;
    Cg = p.g - (p.r + p.b) * 0.5F;
}

__device__ __forceinline__ float b3(float a, float b, float c, float d, float e) {
    return 0.0625F * (a + e) + 0.25F * (b + d) + 0.375F * c;
}

// The tile's sums of w^2 per channel: warp shuffles, then the warps in order.
__device__ __forceinline__ void atrous_tile_sums(const float (&acc)[3], float* __restrict__ part) {
    __shared__ float red[kAtThreads / 32][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float a = acc[c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xFFFFFFFFU, a, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][c] = a;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        float a = 0.0F;
        for (int k = 0; k < kAtThreads / 32; ++k) a += red[k][threadIdx.x];
        part[(size_t)(blockIdx.y * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = a;
    }
}

// One tap row's raw words for one column: the three level planes, or the
// input pixel (converted to c_0 by value()).
template <class T, bool FIRST>
struct AtrousRaw {
    float v[3];
    __device__ __forceinline__ void fetch(const Img&, const float* __restrict__ cin, long long npx, int w, int x, int y) {
        const float* p = cin + (unsigned)(y * w + x);
        v[0] = __ldg(p);
        v[1] = __ldg(p + npx);
        v[2] = __ldg(p + 2 * npx);
    }
    __device__ __forceinline__ void value(float (&o)[3]) const {
        o[0] = v[0];
        o[1] = v[1];
        o[2] = v[2];
    }
};
template <class T>
struct AtrousRaw<T, true> {
    typename std::conditional<std::is_same<T, float>::value, float4, uint2>::type u;
    __device__ __forceinline__ void fetch(const Img& in, const float*, long long, int, int x, int y) {
        u = *reinterpret_cast<const decltype(u)*>(px<const T>(in, x, y));
    }
    __device__ __forceinline__ void value(float (&o)[3]) const {
        const Rgba p = load_rgba(reinterpret_cast<const T*>(&u));
        o[0] = (p.r + 2.0F * p.g + p.b) * 0.25F;
        o[1] = p.r - p.b;
        o[2] = p.g - (p.r + p.b) * 0.5F;
    }
};
template <class T, bool FIRST>
__device__ __forceinline__ void atrous_tap(const Img& in, const float* __restrict__ cin, long long npx, int w, int x,
                                           int y, float (&v)[3]) {
    if (FIRST) {
        atrous_c0<T>(in, x, y, v[0], v[1], v[2]);
    } else {
        const float* p = cin + (long long)y * w + x;
        v[0] = __ldg(p);
        v[1] = __ldg(p + npx);
        v[2] = __ldg(p + 2 * npx);
    }
}
// One level as a polyphase walk: the taps of
// output row y lie in rows y + m s, so the rows of one residue class phi
// (y = phi + k s) form a dense 5-tap filter.  A block covers 256 columns
// (256 - 4s outputs and their 2s halo each side); each thread keeps one
// column's five vertical taps per channel in registers and walks kAtSeg steps
// of one residue class, loading one new row per step; per step the block's
// vertical results go through shared memory for the horizontal taps.  Every
// c_j value is read about once (plus the 4s/(256 - 4s) column halo and the four
// warm-up rows per walk).  Per output: the vertical B3 taps first, then the
// horizontal ones, each b3(t[-2s], t[-s], t[0], t[s], t[2s]); the first level
// (s = 1) reads c_0 = (Y, Co, Cg) from the input frame.
constexpr int kAtSeg = 32;  // steps per walk
__host__ __device__ constexpr int atrous_walk_cols(int s) { return kAtThreads - 4 * s; }
template <class T, bool FIRST>
__global__ void __launch_bounds__(kAtThreads) atrous_walk_kernel(Img in, const float* __restrict__ cin,
                                                                 float* __restrict__ cout, float* __restrict__ part,
                                                                 int w, int h, long long npx, int s) {
    __shared__ float vrow[3][kAtThreads];
    const int t = threadIdx.x, OW = atrous_walk_cols(s);
    const int x0 = blockIdx.x * OW;                      // first output column
    const int xc = clampi(x0 - 2 * s + t, 0, w - 1);      // this thread's (clamped) column
    const int phi = blockIdx.y % s, k0 = (blockIdx.y / s) * kAtSeg;
    // steps with phi + s k < h (block-uniform)
    const int nk = phi < h ? min(kAtSeg, (h - 1 - phi) / s + 1 - k0) : 0;
    float acc[3] = {0.0F, 0.0F, 0.0F};
    if (nk > 0) {
        const int x = x0 + t - 2 * s;
        const bool out = t >= 2 * s && t < 2 * s + OW && x < w;
        float ring[5][3];  // c_j at rows y - 2s .. y + 2s (clamped) of this column
        const int yb = phi + s * k0;
#pragma unroll
        for (int m = 0; m < 5; ++m) atrous_tap<T, FIRST>(in, cin, npx, w, xc, clampi(yb + (m - 2) * s, 0, h - 1), ring[m]);
        for (int k = 0; k < nk; ++k) {
            const int y = yb + s * k;
#pragma unroll
            for (int c = 0; c < 3; ++c) vrow[c][t] = b3(ring[0][c], ring[1][c], ring[2][c], ring[3][c], ring[4][c]);
            // the next step's new row, in flight across this step's barriers
            // (raw words; converted after them)
            AtrousRaw<T, FIRST> nxt;
            nxt.fetch(in, cin, npx, w, xc, min(y + 3 * s, h - 1));
            __syncthreads();
            if (out) {
                float* dst = cout + (unsigned)(y * w + x);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float* v = vrow[c] + t;
                    const float hv = b3(v[-2 * s], v[-s], v[0], v[s], v[2 * s]);
                    const float d = ring[2][c] - hv;
                    dst[c * npx] = hv;
                    acc[c] += d * d;
                }
            }
            __syncthreads();  // vrow is rewritten by the next step
#pragma unroll
            for (int m = 0; m < 4; ++m)
#pragma unroll
                for (int c = 0; c < 3; ++c) ring[m][c] = ring[m + 1][c];
            nxt.value(ring[4]);
        }
    }
    atrous_tile_sums(acc, part);
}

struct AtrousThrArgs {
    float noise[kAtrousMaxLevels][3];
    float strength[3];
};

// block (level, channel): the tiles' sums of w^2 in a fixed order -> threshold;
// level j's sums start at part + j * stride (3 per tile), nb[j] tiles
struct AtrousTiles {
    int nb[kAtrousMaxLevels];
    int stride;
};
// Compensated binary32 addition (Knuth's TwoSum): hi + lo carries the sum
// to about 48 significant bits, so the fixed-order reduction below needs no
// FP64.
struct Ff2 {
    float hi, lo;
};
__device__ __forceinline__ Ff2 ff_add(Ff2 a, float b) {
    const float s = __fadd_rn(a.hi, b);
    const float bp = __fsub_rn(s, a.hi);
    const float e = __fadd_rn(__fsub_rn(a.hi, __fsub_rn(s, bp)), __fsub_rn(b, bp));
    return Ff2{s, __fadd_rn(a.lo, e)};
}
__device__ __forceinline__ Ff2 ff_add(Ff2 a, Ff2 b) {
    Ff2 r = ff_add(a, b.hi);
    r.lo = __fadd_rn(r.lo, b.lo);
    return r;
}
__global__ void __launch_bounds__(256) atrous_thresh_kernel(const float* __restrict__ part, AtrousTiles tl, long long npx,
                                                            AtrousThrArgs a, float* __restrict__ thr) {
    const int j = blockIdx.x / 3, c = blockIdx.x % 3, nblocks = tl.nb[j];
    __shared__ Ff2 red[256];
    Ff2 s{0.0F, 0.0F};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s = ff_add(s, part[(size_t)j * tl.stride + (size_t)b * 3 + c]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) red[threadIdx.x] = ff_add(red[threadIdx.x], red[threadIdx.x + k]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // mean of w^2: (hi + lo) / npx, npx exact in binary32 up to 2^24 and
        // rounded once above it
        const float sw2 = __fdiv_rn(__fadd_rn(red[0].hi, red[0].lo), (float)npx), sn = a.noise[j][c];
        const float sx = sqrtf(fmaxf(__fsub_rn(sw2, __fmul_rn(sn, sn)), 0.0F));
        const float st = a.strength[c];
        thr[j * 3 + c] = st == 0.0F ? 0.0F : (sx > 0.0F ? __fdiv_rn(__fmul_rn(__fmul_rn(st, sn), sn), sx) : INFINITY);
    }
}

__device__ __forceinline__ float soft(float w, float t) {
    const float m = fabsf(w) - t;
    return m > 0.0F ? copysignf(m, w) : 0.0F;
}

// c = c_L + sum over j = L-1 .. 0 of soft(c_j - c_{j+1}, T_j), c_0 from the
// input; inverse colour transform; alpha copied.  c_j (j >= 1) sits at
// cl + (j - 1) * 3 * npx.
template <class T>
__global__ void atrous_recon_kernel(Img in, Img out, const float* __restrict__ cl, const float* __restrict__ thr,
                                    int levels, long long npx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= in.w) return;
    const long long o = (long long)y * in.w + x;
    float c0[3];
    atrous_c0<T>(in, x, y, c0[0], c0[1], c0[2]);
    float v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* p = cl + c * npx + o;
        float hi = __ldg(p + (long long)(levels - 1) * 3 * npx);  // c_L
        float r = hi;
        for (int j = levels - 1; j >= 0; --j) {
            const float lo = j == 0 ? c0[c] : __ldg(p + (long long)(j - 1) * 3 * npx);  // c_j
            r = r + soft(lo - hi, thr[j * 3 + c]);
            hi = lo;
        }
        v[c] = r;
    }
    const float t = v[0] - 0.5F * v[2];
    store_rgb_keep_alpha(px<T>(out, x, y), Rgba{max0(t + 0.5F * v[1]), max0(t + v[2]), max0(t - 0.5F * v[1]), 0.0F},
                         px<const T>(in, x, y));
}

// The same per pixel for four pixels per thread (frames whose width is a
// multiple of 4): 16-byte loads from each level plane.
template <class T>
__global__ void atrous_recon4_kernel(Img in, Img out, const float* __restrict__ cl, const float* __restrict__ thr,
                                     int levels, long long npx) {
    const int x = 4 * (blockIdx.x * blockDim.x + threadIdx.x), y = blockIdx.y;
    if (x >= in.w) return;
    const unsigned o = (unsigned)(y * in.w + x);
    Rgba px4[4];
    float c0[4][3];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        px4[i] = load_rgba(px<const T>(in, x + i, y));
        c0[i][0] = (px4[i].r + 2.0F * px4[i].g + px4[i].b) * 0.25F;
        c0[i][1] = px4[i].r - px4[i].b;
        c0[i][2] = px4[i].g - (px4[i].r + px4[i].b) * 0.5F;
    }
    float v[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* p = cl + c * npx + o;
        float4 hi4 = __ldg(reinterpret_cast<const float4*>(p + (long long)(levels - 1) * 3 * npx));  // c_L
        float hi[4] = {hi4.x, hi4.y, hi4.z, hi4.w};
        float r[4] = {hi4.x, hi4.y, hi4.z, hi4.w};
        for (int j = levels - 1; j >= 0; --j) {
            float lo[4];
            if (j == 0) {
#pragma unroll
                for (int i = 0; i < 4; ++i) lo[i] = c0[i][c];
            } else {
                const float4 l4 = __ldg(reinterpret_cast<const float4*>(p + (long long)(j - 1) * 3 * npx));  // c_j
                lo[0] = l4.x;
                lo[1] = l4.y;
                lo[2] = l4.z;
                lo[3] = l4.w;
            }
            const float t = thr[j * 3 + c];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                r[i] = r[i] + soft(lo[i] - hi[i], t);
                hi[i] = lo[i];
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i][c] = r[i];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float t = v[i][0] - 0.5F * v[i][2];
        store_rgb_keep_alpha(px<T>(out, x + i, y),
                             Rgba{max0(t + 0.5F * v[i][1]), max0(t + v[i][2]), max0(t - 0.5F * v[i][1]), 0.0F},
                             px<const T>(in, x + i, y));
    }
}

size_t align256(size_t v) { return (v + 255U) & ~(size_t)255U; }

dim3 atrous_walk_grid(int w, int h, int s) {
    const int rows = (h + s - 1) / s;  // steps of the longest residue class
    return dim3((unsigned)((w + atrous_walk_cols(s) - 1) / atrous_walk_cols(s)),
                (unsigned)(s * ((rows + kAtSeg - 1) / kAtSeg)));
}

}  // namespace

cudaError_t guided_spec_setup() {
    const int ab = (int)gs_ab_smem(kGuidedSpecMaxRadius), ob = (int)gs_out_smem(kGuidedSpecMaxRadius);
    cudaError_t e = cudaSuccess;
    for (const void* f : {(const void*)gsp_ab_kernel<__half>, (const void*)gsp_ab_kernel<float>})
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, ab);
    for (const void* f : {(const void*)gsp_out_kernel<__half>, (const void*)gsp_out_kernel<float>})
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, ob);
    return e;
}

size_t guided_spec_scratch_bytes(int w, int h, int radius) {
    const size_t Wa = (size_t)w + 2 * radius, Ha = (size_t)h + 2 * radius;
    return 2 * 3 * Ha * Wa * sizeof(float);
}

cudaError_t guided_spec_run(const Img& in, const Img& out, bool f16, int radius, float eps, void* scratch,
                            cudaStream_t st) {
    if (radius < 1 || radius > kGuidedSpecMaxRadius) return cudaErrorInvalidValue;
    const GsPlanes p = gs_planes(in.w, in.h, radius, scratch);
    if ((size_t)p.Ha * p.Wa >= ((size_t)1 << 31)) return cudaErrorInvalidValue;  // 32-bit plane offsets
    // the staging copies move aligned 32-bit words of interleaved RGBA pixels
    const size_t elem = f16 ? 2 : 4;
    if (in.pix_stride != 4 || (reinterpret_cast<uintptr_t>(in.data) & 3U) != 0 || (in.row_stride * elem) % 4 != 0)
        return cudaErrorInvalidValue;
    const dim3 ga((unsigned)((p.Wa + kGsTW - 1) / kGsTW), (unsigned)((p.Ha + kGsTH - 1) / kGsTH), 3);
    const size_t sa = gs_ab_smem(radius), so = gs_out_smem(radius);
    if (f16) gsp_ab_kernel<__half><<<ga, kGsThreads, sa, st>>>(in, p, eps);
    else gsp_ab_kernel<float><<<ga, kGsThreads, sa, st>>>(in, p, eps);
    const dim3 go((unsigned)((in.w + kGsTW - 1) / kGsTW), (unsigned)((in.h + kGsTH - 1) / kGsTH));
    if (f16) gsp_out_kernel<__half><<<go, kGsThreads, so, st>>>(in, out, p);
    else gsp_out_kernel<float><<<go, kGsThreads, so, st>>>(in, out, p);
    return cudaGetLastError();
}

double atrous_band_gain(int level) {
    // phi_0 = delta, phi_k = phi_{k-1} * h_{k-1}; band j = Phi_{j-1} - Phi_j in 2D
    // (Phi = phi x phi), so |band|^2 = (sum p^2)^2 - 2 (sum p f)^2 + (sum f^2)^2.
    std::vector<double> prev(1, 1.0), cur;
    const double h[5] = {1.0 / 16, 4.0 / 16, 6.0 / 16, 4.0 / 16, 1.0 / 16};
    for (int k = 1; k <= level; ++k) {
        const int s = 1 << (k - 1), half = (int)prev.size() / 2;
        cur.assign(prev.size() + 4 * s, 0.0);
        const int ch = (int)cur.size() / 2;
        for (int i = 0; i < (int)prev.size(); ++i)
            for (int t = 0; t < 5; ++t) cur[ch + (i - half) + (t - 2) * s] += prev[i] * h[t];
        if (k < level) prev.swap(cur);
    }
    // prev = phi_{level-1}, cur = phi_level, both centred
    const int off = ((int)cur.size() - (int)prev.size()) / 2;
    double pp = 0.0, pf = 0.0, ff = 0.0;
    for (int i = 0; i < (int)cur.size(); ++i) {
        const double p = (i >= off && i < off + (int)prev.size()) ? prev[i - off] : 0.0;
        pp += p * p;
        pf += p * cur[i];
        ff += cur[i] * cur[i];
    }
    return sqrt(pp * pp - 2.0 * pf * pf + ff * ff);
}

int atrous_plan(const cpipe_AtrousWaveletParams* p, int w, int h, AtrousPlan* out) {
    if (!p || !out || w <= 0 || h <= 0) return CPIPE_BAD_INDEX;
    if (p->levels < 0 || p->levels > kAtrousMaxLevels) return CPIPE_BAD_INDEX;
    if (!(p->sigma >= 0.0F) || !std::isfinite(p->sigma)) return CPIPE_BAD_INDEX;
    if (!(p->luma_strength >= 0.0F) || !std::isfinite(p->luma_strength)) return CPIPE_BAD_INDEX;
    if (!(p->chroma_strength >= 0.0F) || !std::isfinite(p->chroma_strength)) return CPIPE_BAD_INDEX;
    AtrousPlan& q = *out;
    q = AtrousPlan{};
    q.w = w;
    q.h = h;
    q.levels = p->levels;
    q.copy = p->levels == 0;
    if (q.copy) return CPIPE_OK;
    const double g[3] = {sqrt(6.0) / 4.0, sqrt(2.0), sqrt(1.5)};
    for (int j = 0; j < q.levels; ++j) {
        const double n = atrous_band_gain(j + 1);
        for (int c = 0; c < 3; ++c) q.noise[j][c] = (float)((double)p->sigma * g[c] * n);
    }
    q.strength[0] = p->luma_strength;
    q.strength[1] = q.strength[2] = p->chroma_strength;
    const size_t npx = (size_t)w * h, plane3 = 3 * npx * sizeof(float);
    size_t o = 0;
    q.off_c = o;  // c_1 .. c_L
    o = align256(o + (size_t)q.levels * plane3);
    q.off_part = o;
    size_t tiles = 0;
    for (int j = 0; j < q.levels; ++j) {
        const dim3 g = atrous_walk_grid(w, h, 1 << j);
        tiles = std::max(tiles, (size_t)g.x * g.y);
    }
    q.tiles = (int)tiles;
    o = align256(o + (size_t)q.levels * tiles * 3 * sizeof(float));
    q.off_thr = o;
    o = align256(o + (size_t)q.levels * 3 * sizeof(float));
    q.bytes = o;
    return CPIPE_OK;
}

cudaError_t atrous_setup() { return cudaSuccess; }  // the level kernels use static shared memory only

cudaError_t atrous_run(const AtrousPlan& p, const Img& in, const Img& out, bool f16, void* scratch, cudaStream_t st) {
    if (p.copy) {
        const int elem = f16 ? 2 : 4;
        return launch_copy(in.data, in.row_stride * elem, out.data, out.row_stride * elem, (long long)in.w * 4 * elem,
                           in.h, st);
    }
    char* base = static_cast<char*>(scratch);
    const long long npx = (long long)p.w * p.h;
    if (npx >= ((long long)1 << 31)) return cudaErrorInvalidValue;  // 32-bit plane offsets
    float* cl = reinterpret_cast<float*>(base + p.off_c);  // c_{j+1} at cl + j * 3 * npx
    float* part = reinterpret_cast<float*>(base + p.off_part);
    float* thr = reinterpret_cast<float*>(base + p.off_thr);
    AtrousTiles tl{};
    tl.stride = p.tiles * 3;
    for (int j = 0; j < p.levels; ++j) {
        const int s = 1 << j;
        float* cout = cl + (size_t)j * 3 * npx;
        float* pj = part + (size_t)j * tl.stride;
        const dim3 wg = atrous_walk_grid(p.w, p.h, s);
        tl.nb[j] = (int)(wg.x * wg.y);
        if (j == 0) {
            if (f16) atrous_walk_kernel<__half, true><<<wg, kAtThreads, 0, st>>>(in, nullptr, cout, pj, p.w, p.h, npx, s);
            else atrous_walk_kernel<float, true><<<wg, kAtThreads, 0, st>>>(in, nullptr, cout, pj, p.w, p.h, npx, s);
        } else {
            // past the first level the input frame is not read (T is immaterial)
            atrous_walk_kernel<float, false><<<wg, kAtThreads, 0, st>>>(in, cl + (size_t)(j - 1) * 3 * npx, cout, pj,
                                                                        p.w, p.h, npx, s);
        }
    }
    AtrousThrArgs ta{};
    for (int j = 0; j < p.levels; ++j)
        for (int k = 0; k < 3; ++k) ta.noise[j][k] = p.noise[j][k];
    for (int k = 0; k < 3; ++k) ta.strength[k] = p.strength[k];
    atrous_thresh_kernel<<<p.levels * 3, 256, 0, st>>>(part, tl, npx, ta, thr);
    if (p.w % 4 == 0) {
        const dim3 pg((unsigned)((p.w / 4 + 127) / 128), (unsigned)p.h);
        if (f16) atrous_recon4_kernel<__half><<<pg, 128, 0, st>>>(in, out, cl, thr, p.levels, npx);
        else atrous_recon4_kernel<float><<<pg, 128, 0, st>>>(in, out, cl, thr, p.levels, npx);
    } else {
        const dim3 pg((unsigned)((p.w + 255) / 256), (unsigned)p.h);
        if (f16) atrous_recon_kernel<__half><<<pg, 256, 0, st>>>(in, out, cl, thr, p.levels, npx);
        else atrous_recon_kernel<float><<<pg, 256, 0, st>>>(in, out, cl, thr, p.levels, npx);
    }
    return cudaGetLastError();
}

}  // namespace cpb
