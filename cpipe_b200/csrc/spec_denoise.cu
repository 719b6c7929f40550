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
//   guided_spec_kernel   32x32 output tile, the clamped input with a 2r halo
//                        for all three channels in shared memory; per channel
//                        separable box sums (rows, then columns) of v - k and
//                        (v - k)^2 (k: the tile's centre sample, so the
//                        variance does not cancel), a and b on the tile plus r,
//                        separable box sums of a and b, the output.
//   atrous_prep_kernel   RGBA -> Y, Co, Cg planes (FP32).
//   atrous_h_kernel      one level's horizontal B3 pass of all three planes
//                        into a scratch plane set (taps 2^j apart, clamped).
//   atrous_v_kernel      per 64x32 tile: the vertical pass from the scratch
//                        planes, c_{j+1} and w_{j+1}, the tile's sum of w^2
//                        per channel (no halo staging: the taps come through
//                        L1 / L2).
//   atrous_thresh_kernel per (level, channel): the tiles' sums added in a fixed
//                        order (FP64), the BayesShrink threshold.
//   atrous_recon_kernel  shrink, sum, inverse colour transform.
#include "spec_denoise.h"

#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/cpipe_node_abi.h"
#include "kernels.h"

namespace cpb {
namespace {

// ------------------------------------------------------------------ guided
constexpr int kGsTW = 32, kGsTH = 32, kGsThreads = 256;

// Row-major shared buffers use odd pitches: the row passes give consecutive
// threads consecutive rows, which then fall in different banks.
__host__ __device__ inline int odd(int v) { return v | 1; }
__host__ __device__ inline size_t gs_floats(int R) {
    const size_t IW = odd(kGsTW + 4 * R), IH = kGsTH + 4 * R, AW = odd(kGsTW + 2 * R), AH = kGsTH + 2 * R;
    return 3 * IW * IH + 2 * AW * IH + 2 * AW * AH + 2 * (size_t)odd(kGsTW) * AH;
}

template <class T>
__global__ void __launch_bounds__(kGsThreads) guided_spec_kernel(Img in, Img out, int R, float eps) {
    extern __shared__ float sm[];
    // extents (IWn x IH input, AWn x AH for a / b) and odd row pitches
    const int IWn = kGsTW + 4 * R, IH = kGsTH + 4 * R, AWn = kGsTW + 2 * R, AH = kGsTH + 2 * R, D = 2 * R + 1;
    const int IW = odd(IWn), AW = odd(AWn), TP = odd(kGsTW);
    const float N = (float)(D * D);
    float* s_v = sm;                  // [3][IH][IW] clamped input
    float* s_r1 = s_v + 3 * IW * IH;  // [IH][AW] row sums of v - k
    float* s_r2 = s_r1 + IH * AW;     // [IH][AW] row sums of (v - k)^2
    float* s_a = s_r2 + IH * AW;      // [AH][AW]
    float* s_b = s_a + AH * AW;
    float* s_ra = s_b + AH * AW;      // [AH][TP] row sums of a
    float* s_rb = s_ra + AH * TP;
    const int x0 = blockIdx.x * kGsTW, y0 = blockIdx.y * kGsTH;
    for (int i = threadIdx.x; i < IWn * IH; i += blockDim.x) {
        const int ty = i / IWn, tx = i - ty * IWn;
        const Rgba v = load_clamped<T>(in, x0 - 2 * R + tx, y0 - 2 * R + ty);
        s_v[ty * IW + tx] = v.r;
        s_v[IW * IH + ty * IW + tx] = v.g;
        s_v[2 * IW * IH + ty * IW + tx] = v.b;
    }
    __syncthreads();
    // Box sums along rows or columns: each item is a run of up to kGsSeg
    // consecutive outputs, its first window summed directly and the rest slid
    // (one add and one subtract per output; the slide restarts every run).
    constexpr int kGsSeg = 8;
    static_assert(kGsTW * (kGsTH / kGsSeg) <= kGsThreads && kGsTW % kGsSeg == 0 && kGsTH % kGsSeg == 0, "runs");
    float res[kGsSeg][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* v = s_v + c * IW * IH;
        const float k = v[(2 * R + kGsTH / 2) * IW + 2 * R + kGsTW / 2];
        const int rseg = (AWn + kGsSeg - 1) / kGsSeg;
        for (int it = threadIdx.x; it < IH * rseg; it += blockDim.x) {  // rows of v: (v - k), (v - k)^2
            const int y = it % IH, x0s = (it / IH) * kGsSeg, n = min(kGsSeg, AWn - x0s);
            const float* row = v + y * IW + x0s;
            float s1 = 0.0F, s2 = 0.0F;
            for (int d = 0; d < D; ++d) {
                const float t = row[d] - k;
                s1 = s1 + t;
                s2 = s2 + t * t;
            }
            s_r1[y * AW + x0s] = s1;
            s_r2[y * AW + x0s] = s2;
            for (int i = 1; i < n; ++i) {
                const float ti = row[i + D - 1] - k, to = row[i - 1] - k;
                s1 = (s1 + ti) - to;
                s2 = (s2 + ti * ti) - to * to;
                s_r1[y * AW + x0s + i] = s1;
                s_r2[y * AW + x0s + i] = s2;
            }
        }
        __syncthreads();
        const int cseg = (AH + kGsSeg - 1) / kGsSeg;
        for (int it = threadIdx.x; it < AWn * cseg; it += blockDim.x) {  // columns -> a, b
            const int x = it % AWn, y0s = (it / AWn) * kGsSeg, n = min(kGsSeg, AH - y0s);
            float s1 = 0.0F, s2 = 0.0F;
            for (int d = 0; d < D; ++d) {
                s1 = s1 + s_r1[(y0s + d) * AW + x];
                s2 = s2 + s_r2[(y0s + d) * AW + x];
            }
            for (int i = 0; i < n; ++i) {
                if (i > 0) {
                    s1 = (s1 + s_r1[(y0s + i + D - 1) * AW + x]) - s_r1[(y0s + i - 1) * AW + x];
                    s2 = (s2 + s_r2[(y0s + i + D - 1) * AW + x]) - s_r2[(y0s + i - 1) * AW + x];
                }
                const float mk = s1 / N, corr = s2 / N;
                const float var = max0(corr - mk * mk);
                const float m = mk + k;
                const float a = var / (var + eps);
                s_a[(y0s + i) * AW + x] = a;
                s_b[(y0s + i) * AW + x] = m - a * m;
            }
        }
        __syncthreads();
        const int tseg = kGsTW / kGsSeg;
        for (int it = threadIdx.x; it < AH * tseg; it += blockDim.x) {  // rows of a, b
            const int y = it % AH, x0s = (it / AH) * kGsSeg;
            const float* ra = s_a + y * AW + x0s;
            const float* rb = s_b + y * AW + x0s;
            float sa = 0.0F, sb = 0.0F;
            for (int d = 0; d < D; ++d) {
                sa = sa + ra[d];
                sb = sb + rb[d];
            }
            s_ra[y * TP + x0s] = sa;
            s_rb[y * TP + x0s] = sb;
            for (int i = 1; i < kGsSeg; ++i) {
                sa = (sa + ra[i + D - 1]) - ra[i - 1];
                sb = (sb + rb[i + D - 1]) - rb[i - 1];
                s_ra[y * TP + x0s + i] = sa;
                s_rb[y * TP + x0s + i] = sb;
            }
        }
        __syncthreads();
        // columns of the row-summed a, b -> the output: thread t < kGsTW * kGsTH / kGsSeg
        // owns the run of rows 8 (t / kGsTW).. of column t % kGsTW, kept in registers
        if ((int)threadIdx.x < kGsTW * (kGsTH / kGsSeg)) {
            const int it = threadIdx.x;
            const int x = it % kGsTW, y0s = (it / kGsTW) * kGsSeg;
            float sa = 0.0F, sb = 0.0F;
            for (int d = 0; d < D; ++d) {
                sa = sa + s_ra[(y0s + d) * TP + x];
                sb = sb + s_rb[(y0s + d) * TP + x];
            }
#pragma unroll
            for (int i = 0; i < kGsSeg; ++i) {
                if (i > 0) {
                    sa = (sa + s_ra[(y0s + i + D - 1) * TP + x]) - s_ra[(y0s + i - 1) * TP + x];
                    sb = (sb + s_rb[(y0s + i + D - 1) * TP + x]) - s_rb[(y0s + i - 1) * TP + x];
                }
                const int y = y0s + i;
                res[i][c] = max0((sa / N) * v[(y + 2 * R) * IW + x + 2 * R] + (sb / N));
            }
        }
        __syncthreads();
    }
    if ((int)threadIdx.x < kGsTW * (kGsTH / kGsSeg)) {
        const int x = x0 + (int)threadIdx.x % kGsTW, yb = y0 + ((int)threadIdx.x / kGsTW) * kGsSeg;
#pragma unroll
        for (int i = 0; i < kGsSeg; ++i) {
            const int y = yb + i;
            if (x < out.w && y < out.h)
                store_rgb_keep_alpha(px<T>(out, x, y), Rgba{res[i][0], res[i][1], res[i][2], 0.0F}, px<const T>(in, x, y));
        }
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
__global__ void __launch_bounds__(256) atrous_thresh_kernel(const float* __restrict__ part, AtrousTiles tl, long long npx,
                                                            AtrousThrArgs a, float* __restrict__ thr) {
    const int j = blockIdx.x / 3, c = blockIdx.x % 3, nblocks = tl.nb[j];
    __shared__ double red[256];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += (double)part[(size_t)j * tl.stride + (size_t)b * 3 + c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double sw2 = red[0] / (double)npx, sn = (double)a.noise[j][c];
        const double sx = sqrt(fmax(sw2 - sn * sn, 0.0));
        const float st = a.strength[c];
        thr[j * 3 + c] = st == 0.0F ? 0.0F : (sx > 0.0 ? (float)((double)st * sn * sn / sx) : INFINITY);
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

cudaError_t guided_spec_setup() {
    const int bytes = (int)(gs_floats(kGuidedSpecMaxRadius) * sizeof(float));
    cudaError_t e = cudaFuncSetAttribute(guided_spec_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(guided_spec_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

cudaError_t guided_spec_run(const Img& in, const Img& out, bool f16, int radius, float eps, cudaStream_t st) {
    if (radius < 1 || radius > kGuidedSpecMaxRadius) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)((in.w + kGsTW - 1) / kGsTW), (unsigned)((in.h + kGsTH - 1) / kGsTH));
    const size_t bytes = gs_floats(radius) * sizeof(float);
    if (f16) guided_spec_kernel<__half><<<grid, kGsThreads, bytes, st>>>(in, out, radius, eps);
    else guided_spec_kernel<float><<<grid, kGsThreads, bytes, st>>>(in, out, radius, eps);
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

cudaError_t atrous_setup() { return cudaSuccess; }  // the two-pass level kernels use no dynamic shared memory

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
