// Per-node sm_100a kernels: one launch per reference filter (aot_id), reading
// and writing the reference's own buffer formats (R16_UINT / R32_SFLOAT Bayer
// planes, interleaved RGBA f16, plus an RGBA f32 "plain form").  All kernels
// are HBM-bandwidth kernels: coalesced vector loads along rows, grids sized to
// the image (at 12 MP every launch covers >= 148 SMs many times over), and
// shared-memory halo tiles for the stencil nodes.
#include <type_traits>

#include "demosaic.cuh"
#include "kernels.h"
#include "nodes.cuh"

namespace cpb {

namespace {

constexpr int kPtThreads = 256;

inline dim3 row_grid(int w, int h, int px_per_thread) {
    const int per_block = kPtThreads * px_per_thread;
    return dim3((unsigned)((w + per_block - 1) / per_block), (unsigned)h, 1);
}

// ------------------------------------------------------------- raw point ops
// Each thread handles 4 consecutive pixels of one row.
template <class Op>
__global__ void __launch_bounds__(kPtThreads) raw_point_kernel(Img in, Img out, Op op) {
    const int y = blockIdx.y;
    const int x0 = (blockIdx.x * kPtThreads + threadIdx.x) * 4;
    if (x0 >= in.w) return;
    op(in, out, x0, y);
}

struct R16ToF32 {
    __device__ void operator()(const Img& in, const Img& out, int x0, int y) const {
        const uint16_t* s = px<const uint16_t>(in, x0, y);
        float* d = px<float>(out, x0, y);
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) d[i] = (float)s[i];
    }
};
struct Linearize {
    const uint16_t* table;
    int last;
    __device__ void operator()(const Img& in, const Img& out, int x0, int y) const {
        const uint16_t* s = px<const uint16_t>(in, x0, y);
        float* d = px<float>(out, x0, y);
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) {
            const int v = s[i];
            d[i] = (float)__ldg(table + (v < last ? v : last));
        }
    }
};
struct Blacklevel {
    BlackDev p;
    __device__ void operator()(const Img& in, const Img& out, int x0, int y) const {
        const float* s = px<const float>(in, x0, y);
        float* d = px<float>(out, x0, y);
        if (x0 + 4 <= in.w && ((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d)) & 15) == 0) {
            const float4 v = *reinterpret_cast<const float4*>(s);
            *reinterpret_cast<float4*>(d) =
                make_float4(blacklevel_px(v.x, x0, y, p), blacklevel_px(v.y, x0 + 1, y, p),
                            blacklevel_px(v.z, x0 + 2, y, p), blacklevel_px(v.w, x0 + 3, y, p));
            return;
        }
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) d[i] = blacklevel_px(s[i], x0 + i, y, p);
    }
};
struct GainMap {
    GainMapDev g;
    __device__ void operator()(const Img& in, const Img& out, int x0, int y) const {
        const float* s = px<const float>(in, x0, y);
        float* d = px<float>(out, x0, y);
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) {
            const int m = gain_map_index(x0 + i, y, g);
            d[i] = s[i] * gain_px(m, x0 + i, y, g);
        }
    }
};

// Plain copy of one row segment, any element size (used by the pass-through cases).
__global__ void copy_rows_kernel(const char* src, long long src_pitch, char* dst, long long dst_pitch,
                                 long long row_bytes) {
    const char* s = src + (long long)blockIdx.y * src_pitch;
    char* d = dst + (long long)blockIdx.y * dst_pitch;
    for (long long i = (long long)(blockIdx.x * blockDim.x + threadIdx.x) * 16; i < row_bytes;
         i += (long long)gridDim.x * blockDim.x * 16) {
        if (i + 16 <= row_bytes && ((reinterpret_cast<uintptr_t>(s + i) | reinterpret_cast<uintptr_t>(d + i)) & 15) == 0) {
            *reinterpret_cast<uint4*>(d + i) = *reinterpret_cast<const uint4*>(s + i);
        } else {
            for (long long j = i; j < i + 16 && j < row_bytes; ++j) d[j] = s[j];
        }
    }
}

// ---------------------------------------------------------------- demosaic
struct F32Loader {
    Img in;
    __device__ __forceinline__ float operator()(int gx, int gy) const { return *px<const float>(in, gx, gy); }
};
template <int ALGO, class TOut>
__global__ void __launch_bounds__(256) demosaic_kernel(Img in, Img out, Cfa cfa) {
    demosaic_tile<ALGO, TOut>(F32Loader{in}, in.w, in.h, out, cfa);
}

// ---------------------------------------------------------------- QBC remosaic
// demosaic_quad_bayer_remosaic_generator.cpp:17-58, integer arithmetic.  Tile
// with halo 3 (5x5 gather of pixels whose gradients reach one further).
constexpr int kQbTW = 64, kQbTH = 16, kQbHalo = 3;
constexpr int kQbIW = kQbTW + 2 * kQbHalo, kQbIH = kQbTH + 2 * kQbHalo;
__device__ __forceinline__ int qbc_color(int x, int y) {
    const int mx = ((x % 4) + 4) % 4, my = ((y % 4) + 4) % 4;
    return (my < 2 && mx < 2) ? 0 : ((my >= 2 && mx >= 2) ? 2 : 1);
}
__global__ void __launch_bounds__(256) qbc_kernel(Img in, Img out) {
    __shared__ int s[kQbIH * kQbIW];
    const int x0 = blockIdx.x * kQbTW, y0 = blockIdx.y * kQbTH;
    for (int i = threadIdx.x; i < kQbIH * kQbIW; i += blockDim.x) {
        const int ty = i / kQbIW, tx = i - ty * kQbIW;
        s[i] = *px<const uint16_t>(in, clampi(x0 - kQbHalo + tx, 0, in.w - 1), clampi(y0 - kQbHalo + ty, 0, in.h - 1));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kQbTH * kQbTW; i += blockDim.x) {
        const int ty = i / kQbTW, tx = i - ty * kQbTW;
        const int x = x0 + tx, y = y0 + ty;
        if (x >= out.w || y >= out.h) continue;
        const int target = ((y & 1) == 0 && (x & 1) == 0) ? 0 : (((y & 1) != 0 && (x & 1) != 0) ? 2 : 1);
        uint32_t ws = 0, wsum = 0;
#pragma unroll
        for (int dy = -2; dy <= 2; ++dy) {
#pragma unroll
            for (int dx = -2; dx <= 2; ++dx) {
                const int sx = clampi(x + dx, 0, in.w - 1), sy = clampi(y + dy, 0, in.h - 1);
                // tile coordinates of (sx, sy); clamped neighbours of sx stay inside the halo
                const int lx = sx - (x0 - kQbHalo), ly = sy - (y0 - kQbHalo);
                const int lxm = clampi(sx - 1, 0, in.w - 1) - (x0 - kQbHalo), lxp = clampi(sx + 1, 0, in.w - 1) - (x0 - kQbHalo);
                const int lym = clampi(sy - 1, 0, in.h - 1) - (y0 - kQbHalo), lyp = clampi(sy + 1, 0, in.h - 1) - (y0 - kQbHalo);
                const int gx = abs(s[ly * kQbIW + lxm] - s[ly * kQbIW + lxp]);
                const int gy = abs(s[lym * kQbIW + lx] - s[lyp * kQbIW + lx]);
                const int pen = 64 + gx + gy + ((abs(dx) + abs(dy)) * 16);
                int cw = 65536 / pen;
                cw = cw < 1 ? 1 : cw;
                const uint32_t wt = qbc_color(sx, sy) == target ? (uint32_t)cw : 0U;
                ws += wt * (uint32_t)s[ly * kQbIW + lx];
                wsum += wt;
            }
        }
        *px<uint16_t>(out, x, y) = wsum == 0 ? 0 : (uint16_t)((ws + (wsum / 2U)) / wsum);
    }
}

// ------------------------------------------------------------ RGBA point ops
template <class T, class Op>
__global__ void __launch_bounds__(kPtThreads) rgba_point_kernel(Img in, Img out, Op op) {
    const int y = blockIdx.y;
    const int x = blockIdx.x * kPtThreads + threadIdx.x;
    if (x >= in.w) return;
    const T* s = px<const T>(in, x, y);
    op(s, px<T>(out, x, y));
}

template <bool F16>
struct RgbaRound {
    __device__ static Rgba apply(Rgba v) { return Rgba{rnd<F16>(v.r), rnd<F16>(v.g), rnd<F16>(v.b), v.a}; }
};

template <class T>
struct WbOp {
    float n[3];
    __device__ void operator()(const T* s, T* d) const { store_rgb_keep_alpha(d, wb_px(load_rgba(s), n), s); }
};
template <class T>
struct CmOp {
    float t[9];
    __device__ void operator()(const T* s, T* d) const { store_rgb_keep_alpha(d, cm_px(load_rgba(s), t), s); }
};
template <class T>
struct FilmicOp {
    FilmicDev p;
    __device__ void operator()(const T* s, T* d) const { store_rgb_keep_alpha(d, filmic_px(load_rgba(s), p), s); }
};
template <class T>
struct LutOp {
    const float4* lut;
    int S, interp;
    __device__ void operator()(const T* s, T* d) const { store_rgb_keep_alpha(d, lut_px(load_rgba(s), lut, S, interp), s); }
};
// f32 -> RGBA f16 (precision_convert_generator.cpp:48-56): grey replicated, alpha 1.
struct F32ToRgba16f {
    __device__ void operator()(const Img& in, const Img& out, int x0, int y) const {
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) {
            const float v = *px<const float>(in, x0 + i, y);
            store_rgba(px<__half>(out, x0 + i, y), Rgba{v, v, v, 1.0F});
        }
    }
};
// RGBA f16 -> RGBA unorm8/16 (precision_convert_generator.cpp:66-117).
template <class TU, int SCALE>
struct Rgba16fToUnorm {
    __device__ void operator()(const Img& in, const Img& out, int x0, int y) const {
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) {
            const Rgba v = load_rgba(px<const __half>(in, x0 + i, y));
            TU* d = px<TU>(out, x0 + i, y);
            const float c[4] = {v.r, v.g, v.b, v.a};
            for (int k = 0; k < 4; ++k) d[k] = (TU)((clampf(c[k], 0.0F, 1.0F) * (float)SCALE) + 0.5F);
        }
    }
};

// ------------------------------------------------------------- 2x2 block ops
// One thread per aligned 2x2 block; clamped reads at odd right/bottom edges.
template <class T, bool F16>
__global__ void __launch_bounds__(256) bm3d_parity_kernel(Img in, Img out, float s) {
    const int bx = (blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const int by = blockIdx.y * 2;
    if (bx >= in.w) return;
    Rgba q[4];
    q[0] = load_clamped<T>(in, bx, by);
    q[1] = load_clamped<T>(in, bx + 1, by);
    q[2] = load_clamped<T>(in, bx, by + 1);
    q[3] = load_clamped<T>(in, bx + 1, by + 1);
    for (int k = 0; k < 4; ++k) {
        const int x = bx + (k & 1), y = by + (k >> 1);
        if (x >= out.w || y >= out.h) continue;
        const Rgba v = q[k];
        const Rgba o{bm3d_blend(v.r, q[0].r, q[1].r, q[2].r, q[3].r, s),
                     bm3d_blend(v.g, q[0].g, q[1].g, q[2].g, q[3].g, s),
                     bm3d_blend(v.b, q[0].b, q[1].b, q[2].b, q[3].b, s), v.a};
        store_rgba(px<T>(out, x, y), o);
    }
}
template <class T>
__global__ void __launch_bounds__(256) wavelet_kernel(Img in, Img out, float th) {
    const int bx = (blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const int by = blockIdx.y * 2;
    if (bx >= in.w) return;
    Rgba q[4];
    q[0] = load_clamped<T>(in, bx, by);
    q[1] = load_clamped<T>(in, bx + 1, by);
    q[2] = load_clamped<T>(in, bx, by + 1);
    q[3] = load_clamped<T>(in, bx + 1, by + 1);
    for (int k = 0; k < 4; ++k) {
        const int x = bx + (k & 1), y = by + (k >> 1);
        if (x >= out.w || y >= out.h) continue;
        store_rgba(px<T>(out, x, y), wavelet_px(q, q[k], k & 1, k >> 1, th));
    }
}

// ------------------------------------------------------------ guided filter
// guided_filter_generator.cpp:45-85.  R = 1 (3x3 box) or 2 (5x5 box).  The
// tile holds the clamped input with halo 2R; a and b are evaluated for the tile
// plus halo R at unclamped coordinates (their inner reads are clamped), then
// boxed again.  Sums keep the generator's row-major, left-associated order.
constexpr int kGfTW = 32, kGfTH = 16;
template <class T, bool F16, int R>
__global__ void __launch_bounds__(256) guided_kernel(Img in, Img out, float eps) {
    constexpr int IW = kGfTW + 4 * R, IH = kGfTH + 4 * R;
    constexpr int AW = kGfTW + 2 * R, AH = kGfTH + 2 * R;
    __shared__ float s_v[3][IH * IW];
    __shared__ float s_a[3][AH * AW];
    __shared__ float s_b[3][AH * AW];
    const int x0 = blockIdx.x * kGfTW, y0 = blockIdx.y * kGfTH;
    for (int i = threadIdx.x; i < IH * IW; i += blockDim.x) {
        const int ty = i / IW, tx = i - ty * IW;
        const Rgba v = load_clamped<T>(in, x0 - 2 * R + tx, y0 - 2 * R + ty);
        s_v[0][i] = v.r;
        s_v[1][i] = v.g;
        s_v[2][i] = v.b;
    }
    __syncthreads();
    constexpr float N = (float)((2 * R + 1) * (2 * R + 1));
    for (int i = threadIdx.x; i < 3 * AH * AW; i += blockDim.x) {
        const int c = i / (AH * AW);
        const int j = i - c * AH * AW;
        const int ty = j / AW, tx = j - ty * AW;
        // centre of this a/b sample in s_v coordinates
        const float* v = s_v[c] + (ty + R) * IW + (tx + R);
        float sm = 0.0F, sq = 0.0F;
        bool first = true;
#pragma unroll
        for (int dy = -R; dy <= R; ++dy)
#pragma unroll
            for (int dx = -R; dx <= R; ++dx) {
                const float t = v[dy * IW + dx];
                if (R == 1 && first) { sm = t; sq = t * t; first = false; }
                else { sm = sm + t; sq = sq + (t * t); }
            }
        const float m = sm / N, corr = sq / N;
        const float var = max0(corr - (m * m));
        const float a = var / (var + eps);
        s_a[c][j] = a;
        s_b[c][j] = m - (a * m);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kGfTH * kGfTW; i += blockDim.x) {
        const int ty = i / kGfTW, tx = i - ty * kGfTW;
        const int x = x0 + tx, y = y0 + ty;
        if (x >= out.w || y >= out.h) continue;
        const Rgba src = load_rgba(px<const T>(in, x, y));
        float o[3];
        for (int c = 0; c < 3; ++c) {
            const float* A = s_a[c] + (ty + R) * AW + (tx + R);
            const float* B = s_b[c] + (ty + R) * AW + (tx + R);
            float sa = 0.0F, sb = 0.0F;
            bool first = true;
#pragma unroll
            for (int dy = -R; dy <= R; ++dy)
#pragma unroll
                for (int dx = -R; dx <= R; ++dx) {
                    if (R == 1 && first) { sa = A[dy * AW + dx]; sb = B[dy * AW + dx]; first = false; }
                    else { sa = sa + A[dy * AW + dx]; sb = sb + B[dy * AW + dx]; }
                }
            const float v = s_v[c][(ty + 2 * R) * IW + (tx + 2 * R)];
            o[c] = max0(((sa / N) * v) + (sb / N));
        }
        store_rgba(px<T>(out, x, y), Rgba{o[0], o[1], o[2], src.a});
    }
}

// --------------------------------------------------------------- OpcodeList3
template <class T, bool F16>
__global__ void __launch_bounds__(128) warp_kernel(Img in, Img out, WarpDev w) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= out.w) return;
    store_rgba(px<T>(out, x, y), warp_px<T>(in, w, x, y));
}

// FixVignetteRadial (:126-158): gain evaluated in float-float, value*gain rounded to float.
struct VignetteDev {
    ff cx, cy, inv_m, k[5];
};
template <class T, bool F16>
__global__ void __launch_bounds__(256) vignette_kernel(Img in, Img out, VignetteDev v) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= out.w) return;
    const ff dx = ff_mul(ff_sub(ff_from((float)x), v.cx), v.inv_m);
    const ff dy = ff_mul(ff_sub(ff_from((float)y), v.cy), v.inv_m);
    const ff r2 = ff_add(ff_mul(dx, dx), ff_mul(dy, dy));
    const ff r4 = ff_mul(r2, r2), r6 = ff_mul(r4, r2), r8 = ff_mul(r4, r4), r10 = ff_mul(r8, r2);
    ff g = ff_add(ff_from(1.0F), ff_mul(v.k[0], r2));
    g = ff_add(g, ff_mul(v.k[1], r4));
    g = ff_add(g, ff_mul(v.k[2], r6));
    g = ff_add(g, ff_mul(v.k[3], r8));
    g = ff_add(g, ff_mul(v.k[4], r10));
    const T* s = px<const T>(in, x, y);
    const Rgba p = load_rgba(s);
    auto mulr = [&](float a) {
        const ff prod = ff_mul(ff_from(a), g);
        return __fadd_rn(prod.hi, prod.lo);
    };
    store_rgb_keep_alpha(px<T>(out, x, y), Rgba{mulr(p.r), mulr(p.g), mulr(p.b), p.a}, s);
}

// Average of the in-bounds 4-neighbours (patched_channel :160-179).
template <class T>
__device__ __forceinline__ Rgba patched_px(const Img& in, int x, int y) {
    float sr = 0.0F, sg = 0.0F, sb = 0.0F;
    int n = 0;
    const int kdx[4] = {-1, 1, 0, 0}, kdy[4] = {0, 0, -1, 1};
    for (int i = 0; i < 4; ++i) {
        const int nx = x + kdx[i], ny = y + kdy[i];
        if (nx < 0 || nx >= in.w || ny < 0 || ny >= in.h) continue;
        const Rgba q = load_rgba(px<const T>(in, nx, ny));
        sr += q.r;
        sg += q.g;
        sb += q.b;
        ++n;
    }
    const Rgba c = load_rgba(px<const T>(in, x, y));
    if (n == 0) return c;
    return Rgba{sr / (float)n, sg / (float)n, sb / (float)n, c.a};
}
template <class T>
__global__ void __launch_bounds__(256) bad_constant_kernel(Img in, Img out, float k) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= out.w) return;
    const T* s = px<const T>(in, x, y);
    const Rgba p = load_rgba(s);
    const bool patch = fabsf(p.r - k) <= 0.0001F || fabsf(p.g - k) <= 0.0001F || fabsf(p.b - k) <= 0.0001F;
    if (patch) store_rgb_keep_alpha(px<T>(out, x, y), patched_px<T>(in, x, y), s);
    else *reinterpret_cast<typename std::conditional<sizeof(T) == 2, uint2, float4>::type*>(px<T>(out, x, y)) =
             *reinterpret_cast<const typename std::conditional<sizeof(T) == 2, uint2, float4>::type*>(s);
}
// Bad pixel list: out already holds a copy of in; patch listed points and rects.
template <class T>
__global__ void bad_list_kernel(Img in, Img out, const uint32_t* pts, int npts, const uint32_t* rects, int nrects) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
        const int y = (int)pts[2 * i], x = (int)pts[2 * i + 1];
        if (x < 0 || x >= in.w || y < 0 || y >= in.h) continue;
        const T* s = px<const T>(in, x, y);
        store_rgb_keep_alpha(px<T>(out, x, y), patched_px<T>(in, x, y), s);
    }
    // Rect bounds as the reference clamps them: min(bound, extent), then max(0, .)
    // (dng_opcode_list_3_dispatch.cpp:219-229); bounds are compared as unsigned so
    // values >= 2^31 clamp to the extent instead of going negative.
    for (int r = 0; r < nrects; ++r) {
        const int top = (int)min(rects[4 * r], (uint32_t)in.h), left = (int)min(rects[4 * r + 1], (uint32_t)in.w);
        const int bottom = (int)min(rects[4 * r + 2], (uint32_t)in.h), right = (int)min(rects[4 * r + 3], (uint32_t)in.w);
        const int rw = right - left, rh = bottom - top;
        if (rw <= 0 || rh <= 0) continue;
        for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < (long long)rw * rh; i += gridDim.x * blockDim.x) {
            const int x = left + (int)(i % rw), y = top + (int)(i / rw);
            const T* s = px<const T>(in, x, y);
            store_rgb_keep_alpha(px<T>(out, x, y), patched_px<T>(in, x, y), s);
        }
    }
}
template <class T>
__global__ void __launch_bounds__(256) trim_kernel(Img in, Img out, uint32_t top, uint32_t left, uint32_t bottom, uint32_t right) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= out.w) return;
    const bool inside = (uint32_t)y >= top && (uint32_t)y < bottom && (uint32_t)x >= left && (uint32_t)x < right;
    const Rgba p = inside ? load_rgba(px<const T>(in, x, y)) : Rgba{0.0F, 0.0F, 0.0F, 0.0F};
    store_rgba(px<T>(out, x, y), p);
}

}  // namespace

// ============================================================ host launchers
cudaError_t launch_r16u_to_f32(const Img& in, const Img& out, cudaStream_t st) {
    raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, R16ToF32{});
    return cudaGetLastError();
}
cudaError_t launch_linearize(const Img& in, const Img& out, const uint16_t* d_table, int n, cudaStream_t st) {
    raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, Linearize{d_table, n - 1});
    return cudaGetLastError();
}
cudaError_t launch_blacklevel(const Img& in, const Img& out, const BlackDev& p, cudaStream_t st) {
    raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, Blacklevel{p});
    return cudaGetLastError();
}
cudaError_t launch_gainmap(const Img& in, const Img& out, const GainMapDev& g, cudaStream_t st) {
    raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, GainMap{g});
    return cudaGetLastError();
}
cudaError_t launch_copy(const void* src, long long src_pitch, void* dst, long long dst_pitch, long long row_bytes,
                        int rows, cudaStream_t st) {
    const long long chunks = (row_bytes + 16 * 256 - 1) / (16 * 256);
    copy_rows_kernel<<<dim3((unsigned)(chunks < 64 ? chunks : 64), (unsigned)rows), 256, 0, st>>>(
        static_cast<const char*>(src), src_pitch, static_cast<char*>(dst), dst_pitch, row_bytes);
    return cudaGetLastError();
}
cudaError_t launch_demosaic(int algo, const Img& in, const Img& out, bool out_f16, const int cfa[4], cudaStream_t st) {
    const dim3 grid((unsigned)((in.w + kDmTW - 1) / kDmTW), (unsigned)((in.h + kDmTH - 1) / kDmTH));
    const Cfa c{{cfa[0], cfa[1], cfa[2], cfa[3]}};
#define DM(A)                                                                         \
    if (out_f16) demosaic_kernel<A, __half><<<grid, 256, 0, st>>>(in, out, c);        \
    else demosaic_kernel<A, float><<<grid, 256, 0, st>>>(in, out, c);
    if (algo == 0) { DM(0) } else if (algo == 1) { DM(1) } else { DM(2) }
#undef DM
    return cudaGetLastError();
}
cudaError_t launch_qbc_remosaic(const Img& in, const Img& out, cudaStream_t st) {
    const dim3 grid((unsigned)((in.w + kQbTW - 1) / kQbTW), (unsigned)((in.h + kQbTH - 1) / kQbTH));
    qbc_kernel<<<grid, 256, 0, st>>>(in, out);
    return cudaGetLastError();
}
cudaError_t launch_f32_to_rgba16f(const Img& in, const Img& out, cudaStream_t st) {
    raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, F32ToRgba16f{});
    return cudaGetLastError();
}
cudaError_t launch_rgba16f_to_unorm(const Img& in, const Img& out, int bits8, cudaStream_t st) {
    if (bits8) raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, Rgba16fToUnorm<uint8_t, 255>{});
    else raw_point_kernel<<<row_grid(in.w, in.h, 4), kPtThreads, 0, st>>>(in, out, Rgba16fToUnorm<uint16_t, 65535>{});
    return cudaGetLastError();
}

#define RGBA_DISPATCH(F16, KERNEL_F16, KERNEL_F32) \
    if (F16) { KERNEL_F16; } else { KERNEL_F32; }

cudaError_t launch_wb(const Img& in, const Img& out, bool f16, const float n[3], cudaStream_t st) {
    const dim3 g = row_grid(in.w, in.h, 1);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, WbOp<__half>{{n[0], n[1], n[2]}})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, WbOp<float>{{n[0], n[1], n[2]}})));
    return cudaGetLastError();
}
cudaError_t launch_colormatrix(const Img& in, const Img& out, bool f16, const float t[9], cudaStream_t st) {
    const dim3 g = row_grid(in.w, in.h, 1);
    CmOp<__half> oh;
    CmOp<float> of;
    for (int i = 0; i < 9; ++i) oh.t[i] = of.t[i] = t[i];
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, oh)),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, of)));
    return cudaGetLastError();
}
cudaError_t launch_filmic(const Img& in, const Img& out, bool f16, const FilmicDev& p, cudaStream_t st) {
    const dim3 g = row_grid(in.w, in.h, 1);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, FilmicOp<__half>{p})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, FilmicOp<float>{p})));
    return cudaGetLastError();
}
cudaError_t launch_lut3d(const Img& in, const Img& out, bool f16, const float4* d_lut, int S, int interp, cudaStream_t st) {
    const dim3 g = row_grid(in.w, in.h, 1);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, LutOp<__half>{d_lut, S, interp})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, LutOp<float>{d_lut, S, interp})));
    return cudaGetLastError();
}
cudaError_t launch_bm3d_parity(const Img& in, const Img& out, bool f16, float sigma, cudaStream_t st) {
    // strength = min(1, max(0, sigma / 0.03)) (bm3d_step1_generator.cpp:50)
    const float s = fminf(1.0F, fmaxf(0.0F, sigma / 0.03F));
    const dim3 g((unsigned)(((in.w + 1) / 2 + 255) / 256), (unsigned)((in.h + 1) / 2));
    RGBA_DISPATCH(f16, (bm3d_parity_kernel<__half, true><<<g, 256, 0, st>>>(in, out, s)),
                  (bm3d_parity_kernel<float, false><<<g, 256, 0, st>>>(in, out, s)));
    return cudaGetLastError();
}
cudaError_t launch_wavelet(const Img& in, const Img& out, bool f16, float strength, cudaStream_t st) {
    const float th = 0.035F * strength;
    const dim3 g((unsigned)(((in.w + 1) / 2 + 255) / 256), (unsigned)((in.h + 1) / 2));
    RGBA_DISPATCH(f16, (wavelet_kernel<__half><<<g, 256, 0, st>>>(in, out, th)),
                  (wavelet_kernel<float><<<g, 256, 0, st>>>(in, out, th)));
    return cudaGetLastError();
}
cudaError_t launch_guided(const Img& in, const Img& out, bool f16, int radius, float eps, cudaStream_t st) {
    const dim3 g((unsigned)((in.w + kGfTW - 1) / kGfTW), (unsigned)((in.h + kGfTH - 1) / kGfTH));
    if (radius <= 1) {
        RGBA_DISPATCH(f16, (guided_kernel<__half, true, 1><<<g, 256, 0, st>>>(in, out, eps)),
                      (guided_kernel<float, false, 1><<<g, 256, 0, st>>>(in, out, eps)));
    } else {
        RGBA_DISPATCH(f16, (guided_kernel<__half, true, 2><<<g, 256, 0, st>>>(in, out, eps)),
                      (guided_kernel<float, false, 2><<<g, 256, 0, st>>>(in, out, eps)));
    }
    return cudaGetLastError();
}
cudaError_t launch_warp(const Img& in, const Img& out, bool f16, const WarpDev& w, cudaStream_t st) {
    const dim3 g((unsigned)((out.w + 127) / 128), (unsigned)out.h);
    RGBA_DISPATCH(f16, (warp_kernel<__half, true><<<g, 128, 0, st>>>(in, out, w)),
                  (warp_kernel<float, false><<<g, 128, 0, st>>>(in, out, w)));
    return cudaGetLastError();
}
cudaError_t launch_vignette(const Img& in, const Img& out, bool f16, const VignetteParams& p, cudaStream_t st) {
    VignetteDev v;
    v.cx = p.cx;
    v.cy = p.cy;
    v.inv_m = p.inv_m;
    for (int i = 0; i < 5; ++i) v.k[i] = p.k[i];
    const dim3 g((unsigned)((out.w + 255) / 256), (unsigned)out.h);
    RGBA_DISPATCH(f16, (vignette_kernel<__half, true><<<g, 256, 0, st>>>(in, out, v)),
                  (vignette_kernel<float, false><<<g, 256, 0, st>>>(in, out, v)));
    return cudaGetLastError();
}
cudaError_t launch_bad_constant(const Img& in, const Img& out, bool f16, float k, cudaStream_t st) {
    const dim3 g((unsigned)((out.w + 255) / 256), (unsigned)out.h);
    RGBA_DISPATCH(f16, (bad_constant_kernel<__half><<<g, 256, 0, st>>>(in, out, k)),
                  (bad_constant_kernel<float><<<g, 256, 0, st>>>(in, out, k)));
    return cudaGetLastError();
}
cudaError_t launch_bad_list(const Img& in, const Img& out, bool f16, const uint32_t* d_pts, int npts,
                            const uint32_t* d_rects, int nrects, cudaStream_t st) {
    RGBA_DISPATCH(f16, (bad_list_kernel<__half><<<kSmCount, 256, 0, st>>>(in, out, d_pts, npts, d_rects, nrects)),
                  (bad_list_kernel<float><<<kSmCount, 256, 0, st>>>(in, out, d_pts, npts, d_rects, nrects)));
    return cudaGetLastError();
}
cudaError_t launch_trim(const Img& in, const Img& out, bool f16, uint32_t top, uint32_t left, uint32_t bottom,
                        uint32_t right, cudaStream_t st) {
    const dim3 g((unsigned)((out.w + 255) / 256), (unsigned)out.h);
    RGBA_DISPATCH(f16, (trim_kernel<__half><<<g, 256, 0, st>>>(in, out, top, left, bottom, right)),
                  (trim_kernel<float><<<g, 256, 0, st>>>(in, out, top, left, bottom, right)));
    return cudaGetLastError();
}

}  // namespace cpb
