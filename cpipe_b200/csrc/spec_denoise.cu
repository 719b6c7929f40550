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
//   gsp_ab / gsp_out     the guided filter as two column-strip kernels with
//                        running binary32 box sums (see below).
//   atrous_prep_kernel   RGBA -> Y, Co, Cg planes (FP32).
//   atrous_h_kernel      one level's horizontal B3 pass of all three planes
//                        into a scratch plane set (taps 2^j apart, clamped).
//   atrous_v_kernel      per 64x32 tile: the vertical pass from the scratch
//                        planes, c_{j+1} and w_{j+1}, the tile's sum of w^2
//                        per channel (no halo staging: the taps come through
//                        L1 / L2).
//   atrous_thresh_kernel per (level, channel): the tiles' sums added in a fixed
//                        order (compensated binary32), the BayesShrink
//                        threshold.
//   atrous_recon_kernel  shrink, sum, inverse colour transform.
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
// Two kernels over column strips, per RGB channel, in binary32:
//   ab    a thread per column xa of the extended domain [-R, w+R) walks a
//         segment of kGsSeg rows ya: the horizontal sums of v and v^2 of the
//         clamped image row entering the vertical box (staged in shared
//         memory) are added to running column sums, a and b are written, and
//         the sums of the row leaving the box are subtracted;
//   out   a thread per output column walks kGsSeg rows the same way over the
//         a and b planes of all three channels (horizontal sums of the entering
//         and leaving rows), out = max(mean_a v + mean_b, 0), alpha copied.
// Each segment starts its running sums afresh (2R rows of warm-up), so no sum
// runs over more than kGsSeg + 2R rows.  Binary16 values square exactly in
// binary32; against the FP64 definition the results are within one binary16
// ulp (binary16 frames) or 1e-5 (binary32 frames).
constexpr int kGsThreads = 128, kGsSeg = 64;
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
// block: extended columns [xs, xs + 128) of channel blockIdx.z, extended rows
// ya in [blockIdx.y * kGsSeg - R, + kGsSeg)
template <class T>
__global__ void __launch_bounds__(kGsThreads) gsp_ab_kernel(Img in, GsPlanes p, float eps) {
    __shared__ float s_new[kGsThreads + 2 * kGuidedSpecMaxRadius], s_old[kGsThreads + 2 * kGuidedSpecMaxRadius];
    const int c = blockIdx.z, xs = blockIdx.x * kGsThreads, t = threadIdx.x, R = p.R, D = 2 * R + 1;
    const int ya0 = (int)blockIdx.y * kGsSeg - R, ya1 = min(ya0 + kGsSeg, p.h + R);
    const float N = (float)(D * D);
    // extended column xi = xs + t is image column xi - R; its box reads image
    // columns xi - 2R .. xi, staged at s[t .. t + 2R]
    auto stage = [&](float* buf, int row) {
        const int y = clampi(row, 0, in.h - 1);
        for (int i = t; i < kGsThreads + 2 * R; i += kGsThreads)
            buf[i] = (float)px<const T>(in, clampi(xs - 2 * R + i, 0, in.w - 1), y)[c];
    };
    auto hsum = [&](const float* buf, float& h1, float& h2) {
        h1 = 0.0F;
        h2 = 0.0F;
        for (int k = 0; k < D; ++k) {
            const float v = buf[t + k];
            h1 = h1 + v;
            h2 = h2 + v * v;
        }
    };
    float s1 = 0.0F, s2 = 0.0F, h1, h2;
    for (int r = ya0 - R; r < ya0 + R; ++r) {
        stage(s_new, r);
        __syncthreads();
        hsum(s_new, h1, h2);
        s1 = s1 + h1;
        s2 = s2 + h2;
        __syncthreads();
    }
    const int xi = xs + t;
    for (int ya = ya0; ya < ya1; ++ya) {
        stage(s_new, ya + R);
        stage(s_old, ya - R);
        __syncthreads();
        hsum(s_new, h1, h2);
        s1 = s1 + h1;
        s2 = s2 + h2;
        const float m = s1 / N, corr = s2 / N;
        const float var = maxf(corr - m * m, 0.0F);
        const float a = var / (var + eps);
        if (xi < p.Wa) {
            const size_t o = ((size_t)c * p.Ha + (ya + R)) * p.Wa + xi;
            p.a[o] = a;
            p.b[o] = m - a * m;
        }
        hsum(s_old, h1, h2);
        s1 = s1 - h1;
        s2 = s2 - h2;
        __syncthreads();
    }
}
// block: output columns [xs, xs + 128), rows [blockIdx.y * kGsSeg, + kGsSeg)
template <class T>
__global__ void __launch_bounds__(kGsThreads) gsp_out_kernel(Img in, Img out, GsPlanes p) {
    constexpr int kS = kGsThreads + 2 * kGuidedSpecMaxRadius;
    __shared__ float s_new[6][kS], s_old[6][kS];
    const int xs = blockIdx.x * kGsThreads, t = threadIdx.x, R = p.R, D = 2 * R + 1;
    const int y0 = (int)blockIdx.y * kGsSeg, y1 = min(y0 + kGsSeg, p.h);
    const float N = (float)(D * D);
    const size_t plane = (size_t)p.Ha * p.Wa;
    // output column x reads extended columns x .. x + 2R (image x - R .. x + R)
    auto stage = [&](float (*buf)[kS], int ya) {
        const size_t row = (size_t)(ya + R) * p.Wa;
        for (int i = t; i < kGsThreads + 2 * R; i += kGsThreads) {
            const size_t xi = row + (size_t)min(xs + i, p.Wa - 1);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                buf[2 * c][i] = p.a[c * plane + xi];
                buf[2 * c + 1][i] = p.b[c * plane + xi];
            }
        }
    };
    float sa[3] = {0.0F, 0.0F, 0.0F}, sb[3] = {0.0F, 0.0F, 0.0F};
    auto add = [&](float (*buf)[kS], float sign) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float ha = 0.0F, hb = 0.0F;
            for (int k = 0; k < D; ++k) {
                ha = ha + buf[2 * c][t + k];
                hb = hb + buf[2 * c + 1][t + k];
            }
            if (sign > 0.0F) {
                sa[c] = sa[c] + ha;
                sb[c] = sb[c] + hb;
            } else {
                sa[c] = sa[c] - ha;
                sb[c] = sb[c] - hb;
            }
        }
    };
    for (int ya = y0 - R; ya < y0 + R; ++ya) {
        stage(s_new, ya);
        __syncthreads();
        add(s_new, 1.0F);
        __syncthreads();
    }
    const int x = xs + t;
    for (int y = y0; y < y1; ++y) {
        stage(s_new, y + R);
        stage(s_old, y - R);
        __syncthreads();
        add(s_new, 1.0F);
        if (x < p.w) {
            const T* src = px<const T>(in, x, y);
            const Rgba v = load_rgba(src);
            store_rgb_keep_alpha(px<T>(out, x, y),
                                 Rgba{max0((sa[0] / N) * v.r + sb[0] / N), max0((sa[1] / N) * v.g + sb[1] / N),
                                      max0((sa[2] / N) * v.b + sb[2] / N), 0.0F},
                                 src);
        }
        add(s_old, -1.0F);
        __syncthreads();
    }
}

// ----------------------------------------------------------------- a-trous
constexpr int kAtTW = 64, kAtTH = 32, kAtThreads = 256;

template <class T>
__global__ void atrous_prep_kernel(Img in, float* __restrict__ c0, long long npx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= in.w) return;
    const Rgba p = load_rgba(px<const T>(in, x, y));
    const long long o = (long long)y * in.w + x;
    c0[o] = (p.r + 2.0F * p.g + p.b) * 0.25F;
    c0[npx + o] = p.r - p.b;
    c0[2 * npx + o] = p.g - (p.r + p.b) * 0.5F;
}

__device__ __forceinline__ float b3(float a, float b, float c, float d, float e) {
    return 0.0625F * (a + e) + 0.25F * (b + d) + 0.375F * c;
}

// One level in two passes over frame-wide planes (no halo staging): the
// horizontal B3 pass of each channel's rows into tmp, then, per 64x32 tile,
// the vertical pass, c_{j+1}, w_{j+1} = c_j - c_{j+1} and the tile's sum of
// w^2 per channel.  Taps clamp at the frame edges; the pixel-to-thread mapping
// of the vertical pass fixes the order of each tile's sum.
__global__ void __launch_bounds__(kAtThreads) atrous_h_kernel(const float* __restrict__ cin, float* __restrict__ tmp,
                                                              int w, long long npx, int s) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, c = blockIdx.z;
    if (x >= w) return;
    const float* row = cin + c * npx + (long long)y * w;
    tmp[c * npx + (long long)y * w + x] = b3(__ldg(row + clampi(x - 2 * s, 0, w - 1)), __ldg(row + clampi(x - s, 0, w - 1)),
                                             __ldg(row + x), __ldg(row + clampi(x + s, 0, w - 1)),
                                             __ldg(row + clampi(x + 2 * s, 0, w - 1)));
}
__global__ void __launch_bounds__(kAtThreads) atrous_v_kernel(const float* __restrict__ cin, const float* __restrict__ tmp,
                                                              float* __restrict__ cout, float* __restrict__ wout,
                                                              float* __restrict__ part, int w, int h, long long npx,
                                                              int s) {
    const int x0 = blockIdx.x * kAtTW, y0 = blockIdx.y * kAtTH;
    float acc[3] = {0.0F, 0.0F, 0.0F};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* t = tmp + c * npx;
        for (int i = threadIdx.x; i < kAtTH * kAtTW; i += kAtThreads) {
            const int r = i / kAtTW, xx = i - r * kAtTW;
            const int x = x0 + xx, y = y0 + r;
            if (x >= w || y >= h) continue;
            const float v = b3(__ldg(t + (long long)clampi(y - 2 * s, 0, h - 1) * w + x),
                               __ldg(t + (long long)clampi(y - s, 0, h - 1) * w + x), __ldg(t + (long long)y * w + x),
                               __ldg(t + (long long)clampi(y + s, 0, h - 1) * w + x),
                               __ldg(t + (long long)clampi(y + 2 * s, 0, h - 1) * w + x));
            const long long o = c * npx + (long long)y * w + x;
            const float d = __ldg(cin + o) - v;
            cout[o] = v;
            wout[o] = d;
            acc[c] += d * d;
        }
    }
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

// One level in one pass per 64x32 tile for taps up to 16 apart: the tile's
// rows [y0 - 2s, y0 + 32 + 2s) of c_j over columns [x0 - 2s, x0 + 64 + 2s)
// (clamped) staged in shared memory, the horizontal B3 pass of those rows into
// shared memory, then the vertical pass, c_{j+1}, w_{j+1} and the tile's sum of
// w^2 per channel -- the same operands, taps and pixel-to-thread mapping as the
// two-pass form above, so the same floats, without the frame-wide scratch
// planes of the horizontal pass.
constexpr int kAtFuseMaxStep = 16;
size_t atrous_level_smem(int s) {
    return ((size_t)(kAtTH + 4 * s) * (kAtTW + 4 * s) + (size_t)(kAtTH + 4 * s) * kAtTW) * sizeof(float);
}
__global__ void __launch_bounds__(kAtThreads) atrous_level_kernel(const float* __restrict__ cin, float* __restrict__ cout,
                                                                  float* __restrict__ wout, float* __restrict__ part,
                                                                  int w, int h, long long npx, int s) {
    extern __shared__ float sm[];
    const int x0 = blockIdx.x * kAtTW, y0 = blockIdx.y * kAtTH;
    const int SR = kAtTH + 4 * s, SC = kAtTW + 4 * s;
    float* st = sm;            // staged c_j: SR x SC
    float* hp = sm + SR * SC;  // horizontal pass: SR x kAtTW
    float acc[3] = {0.0F, 0.0F, 0.0F};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* src = cin + c * npx;
        __syncthreads();
        for (int i = threadIdx.x; i < SR * SC; i += kAtThreads) {
            const int r = i / SC, q = i - r * SC;
            st[i] = __ldg(src + (long long)clampi(y0 - 2 * s + r, 0, h - 1) * w + clampi(x0 - 2 * s + q, 0, w - 1));
        }
        __syncthreads();
        for (int i = threadIdx.x; i < SR * kAtTW; i += kAtThreads) {
            const int r = i / kAtTW, tx = i - r * kAtTW;
            const float* row = st + r * SC + tx + 2 * s;
            hp[i] = b3(row[-2 * s], row[-s], row[0], row[s], row[2 * s]);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kAtTH * kAtTW; i += kAtThreads) {
            const int r = i / kAtTW, xx = i - r * kAtTW;
            const int x = x0 + xx, y = y0 + r;
            if (x >= w || y >= h) continue;
            const float* col = hp + (r + 2 * s) * kAtTW + xx;
            const float v = b3(col[-2 * s * kAtTW], col[-s * kAtTW], col[0], col[s * kAtTW], col[2 * s * kAtTW]);
            const long long o = c * npx + (long long)y * w + x;
            const float d = st[(r + 2 * s) * SC + xx + 2 * s] - v;
            cout[o] = v;
            wout[o] = d;
            acc[c] += d * d;
        }
    }
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

template <class T>
__global__ void atrous_recon_kernel(Img in, Img out, const float* __restrict__ cl, const float* __restrict__ wv,
                                    const float* __restrict__ thr, int levels, long long npx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= in.w) return;
    const long long o = (long long)y * in.w + x;
    float v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float r = cl[c * npx + o];
        for (int j = levels - 1; j >= 0; --j) r = r + soft(wv[((long long)j * 3 + c) * npx + o], thr[j * 3 + c]);
        v[c] = r;
    }
    const float t = v[0] - 0.5F * v[2];
    store_rgb_keep_alpha(px<T>(out, x, y), Rgba{max0(t + 0.5F * v[1]), max0(t + v[2]), max0(t - 0.5F * v[1]), 0.0F},
                         px<const T>(in, x, y));
}

size_t align256(size_t v) { return (v + 255U) & ~(size_t)255U; }

}  // namespace

cudaError_t guided_spec_setup() { return cudaSuccess; }  // the pass kernels use no dynamic shared memory

size_t guided_spec_scratch_bytes(int w, int h, int radius) {
    const size_t Wa = (size_t)w + 2 * radius, Ha = (size_t)h + 2 * radius;
    return 2 * 3 * Ha * Wa * sizeof(float);
}

cudaError_t guided_spec_run(const Img& in, const Img& out, bool f16, int radius, float eps, void* scratch,
                            cudaStream_t st) {
    if (radius < 1 || radius > kGuidedSpecMaxRadius) return cudaErrorInvalidValue;
    const GsPlanes p = gs_planes(in.w, in.h, radius, scratch);
    const dim3 ga((unsigned)((p.Wa + kGsThreads - 1) / kGsThreads), (unsigned)((p.Ha + kGsSeg - 1) / kGsSeg), 3);
    if (f16) gsp_ab_kernel<__half><<<ga, kGsThreads, 0, st>>>(in, p, eps);
    else gsp_ab_kernel<float><<<ga, kGsThreads, 0, st>>>(in, p, eps);
    const dim3 go((unsigned)((in.w + kGsThreads - 1) / kGsThreads), (unsigned)((in.h + kGsSeg - 1) / kGsSeg));
    if (f16) gsp_out_kernel<__half><<<go, kGsThreads, 0, st>>>(in, out, p);
    else gsp_out_kernel<float><<<go, kGsThreads, 0, st>>>(in, out, p);
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
    q.gx = (w + kAtTW - 1) / kAtTW;
    q.gy = (h + kAtTH - 1) / kAtTH;
    const size_t npx = (size_t)w * h, plane3 = 3 * npx * sizeof(float);
    size_t o = 0;
    q.off_c0 = o;
    o = align256(o + plane3);
    q.off_c1 = o;
    o = align256(o + plane3);
    q.off_tmp = o;
    o = align256(o + plane3);
    q.off_w = o;
    o = align256(o + (size_t)q.levels * plane3);
    q.off_part = o;
    o = align256(o + (size_t)q.levels * q.gx * q.gy * 3 * sizeof(float));
    q.off_thr = o;
    o = align256(o + (size_t)q.levels * 3 * sizeof(float));
    q.bytes = o;
    return CPIPE_OK;
}

cudaError_t atrous_setup() {
    return cudaFuncSetAttribute(atrous_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)atrous_level_smem(kAtFuseMaxStep));
}

cudaError_t atrous_run(const AtrousPlan& p, const Img& in, const Img& out, bool f16, void* scratch, cudaStream_t st) {
    if (p.copy) {
        const int elem = f16 ? 2 : 4;
        return launch_copy(in.data, in.row_stride * elem, out.data, out.row_stride * elem, (long long)in.w * 4 * elem,
                           in.h, st);
    }
    char* base = static_cast<char*>(scratch);
    float* c[2] = {reinterpret_cast<float*>(base + p.off_c0), reinterpret_cast<float*>(base + p.off_c1)};
    float* wv = reinterpret_cast<float*>(base + p.off_w);
    float* tmp = reinterpret_cast<float*>(base + p.off_tmp);
    float* part = reinterpret_cast<float*>(base + p.off_part);
    float* thr = reinterpret_cast<float*>(base + p.off_thr);
    const long long npx = (long long)p.w * p.h;
    const dim3 pg((unsigned)((p.w + 255) / 256), (unsigned)p.h);
    if (f16) atrous_prep_kernel<__half><<<pg, 256, 0, st>>>(in, c[0], npx);
    else atrous_prep_kernel<float><<<pg, 256, 0, st>>>(in, c[0], npx);
    AtrousTiles tl{};
    tl.stride = p.gx * p.gy * 3;
    for (int j = 0; j < p.levels; ++j) {
        const int s = 1 << j;
        const dim3 lg((unsigned)p.gx, (unsigned)p.gy);
        tl.nb[j] = (int)(lg.x * lg.y);
        if (s <= kAtFuseMaxStep) {
            atrous_level_kernel<<<lg, kAtThreads, atrous_level_smem(s), st>>>(
                c[j & 1], c[(j + 1) & 1], wv + (size_t)j * 3 * npx, part + (size_t)j * tl.stride, p.w, p.h, npx, s);
            continue;
        }
        const dim3 hg((unsigned)((p.w + kAtThreads - 1) / kAtThreads), (unsigned)p.h, 3);
        atrous_h_kernel<<<hg, kAtThreads, 0, st>>>(c[j & 1], tmp, p.w, npx, s);
        atrous_v_kernel<<<lg, kAtThreads, 0, st>>>(c[j & 1], tmp, c[(j + 1) & 1], wv + (size_t)j * 3 * npx,
                                                   part + (size_t)j * tl.stride, p.w, p.h, npx, s);
    }
    AtrousThrArgs ta{};
    for (int j = 0; j < p.levels; ++j)
        for (int k = 0; k < 3; ++k) ta.noise[j][k] = p.noise[j][k];
    for (int k = 0; k < 3; ++k) ta.strength[k] = p.strength[k];
    atrous_thresh_kernel<<<p.levels * 3, 256, 0, st>>>(part, tl, npx, ta, thr);
    if (f16) atrous_recon_kernel<__half><<<pg, 256, 0, st>>>(in, out, c[p.levels & 1], wv, thr, p.levels, npx);
    else atrous_recon_kernel<float><<<pg, 256, 0, st>>>(in, out, c[p.levels & 1], wv, thr, p.levels, npx);
    return cudaGetLastError();
}

}  // namespace cpb
