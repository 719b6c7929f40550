// Per-node sm_100a kernels: one launch per reference filter (aot_id), reading
// and writing the reference's own buffer formats (R16_UINT / R32_SFLOAT Bayer
// planes, interleaved RGBA f16, plus an RGBA f32 "plain form").  All kernels
// are HBM-bandwidth kernels: coalesced vector loads along rows, grids sized to
// the image (at 12 MP every launch covers >= 148 SMs many times over), and
// shared-memory halo tiles for the stencil nodes.
#include <cmath>
#include <cstring>
#include <type_traits>

#include "../../include/cpipe_b200_params.h"
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

// Bayer-plane point ops with vector access: each thread handles N consecutive
// pixels of one row (N = 16 for u16 input, 8 for f32: 32 bytes read per
// thread), loading and storing in 16-byte pieces when the segment is whole,
// unit-strided and aligned; other segments (row tails, strided or unaligned
// buffers) take the per-pixel path.  Op maps (input value, x, y) -> float.
__device__ __forceinline__ bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <class TI, class Op>
__device__ __forceinline__ void raw_vec_row(const Img& in, const Img& out, const Op& op, int y) {
    constexpr int N = 32 / (int)sizeof(TI);
    const int x0 = (blockIdx.x * kPtThreads + threadIdx.x) * N;
    if (x0 >= in.w) return;
    const TI* s = px<const TI>(in, x0, y);
    float* d = px<float>(out, x0, y);
    if (x0 + N <= in.w && in.pix_stride == 1 && out.pix_stride == 1 && al16(s) && al16(d)) {
        alignas(16) TI v[N];
        alignas(16) float o[N];
#pragma unroll
        for (int i = 0; i < 2; ++i) reinterpret_cast<uint4*>(v)[i] = __ldcs(reinterpret_cast<const uint4*>(s) + i);
#pragma unroll
        for (int i = 0; i < N; ++i) o[i] = op(v[i], x0 + i, y);
#pragma unroll
        for (int i = 0; i < N / 4; ++i) __stcs(reinterpret_cast<float4*>(d) + i, reinterpret_cast<const float4*>(o)[i]);
        return;
    }
    for (int i = 0; i < N && x0 + i < in.w; ++i)
        *px<float>(out, x0 + i, y) = op(*px<const TI>(in, x0 + i, y), x0 + i, y);
}
template <class TI, class Op>
__global__ void __launch_bounds__(kPtThreads) raw_vec_kernel(Img in, Img out, Op op) {
    raw_vec_row<TI>(in, out, op, (int)blockIdx.y);
}

struct R16ToF32 {
    __device__ float operator()(uint16_t v, int, int) const { return (float)v; }
};
struct Linearize {
    const uint16_t* table;
    int last;
    __device__ float operator()(uint16_t v, int, int) const { return (float)__ldg(table + (v < last ? v : last)); }
};
// Linearize with the table copied to shared memory first (tables of up to
// kLinSmemMax entries, which covers every 10..14-bit sensor): the per-pixel
// lookups then read shared memory instead of gathering through L1.
constexpr int kLinSmemMax = 16384;
struct LinearizeShared {
    const uint16_t* table;  // shared memory
    int last;
    __device__ float operator()(uint16_t v, int, int) const { return (float)table[v < last ? v : last]; }
};
// Each block covers rows blockIdx.y, blockIdx.y + gridDim.y, ... so that the
// table is copied once per block, not once per row.
constexpr int kLinRowBlocks = 148 * 8;
__global__ void __launch_bounds__(kPtThreads) linearize_smem_kernel(Img in, Img out, const uint16_t* table, int n) {
    extern __shared__ __align__(16) uint16_t s_tab[];
    for (int i = threadIdx.x; i < n; i += kPtThreads) s_tab[i] = __ldg(table + i);
    __syncthreads();
    const LinearizeShared op{s_tab, n - 1};
    for (int y = blockIdx.y; y < in.h; y += gridDim.y) raw_vec_row<uint16_t>(in, out, op, y);
}
struct Blacklevel {
    BlackDev p;
    __device__ float operator()(float v, int x, int y) const { return blacklevel_px(v, x, y, p); }
};
// hrow[m][r * hw + x] = gain_hrow(m, r, x) for every map, grid row and column.
__global__ void __launch_bounds__(kPtThreads) gainmap_hrows_kernel(GainMapDev g) {
    const int m = blockIdx.z, r = blockIdx.y;
    const int x = blockIdx.x * kPtThreads + threadIdx.x;
    if (m >= g.map_count || r >= g.points_v[m] || x >= g.hw) return;
    const_cast<float*>(g.hrow[m])[(size_t)r * g.hw + x] = gain_hrow(m, r, x, g);
}

// One map for every plane (the common case): 8 consecutive pixels per thread
// with 16-byte loads of the pixels and of both grid-row tables, and 16-byte
// stores; whole, unit-strided, aligned segments only (others per pixel).
constexpr int kGmPx = 8;
__global__ void __launch_bounds__(kPtThreads) gainmap_one_map_kernel(Img in, Img out, GainMapDev g) {
    const int y = blockIdx.y;
    const int x0 = (blockIdx.x * kPtThreads + threadIdx.x) * kGmPx;
    if (x0 >= in.w) return;
    const AxisSample sy = g.rows[0][y];
    const float* hl = g.hrow[0] + (size_t)sy.low * g.hw + x0;
    const float* hh = g.hrow[0] + (size_t)sy.high * g.hw + x0;
    const float* s = px<const float>(in, x0, y);
    float* d = px<float>(out, x0, y);
    if (x0 + kGmPx <= in.w && in.pix_stride == 1 && out.pix_stride == 1 && al16(s) && al16(d) && al16(hl) && al16(hh)) {
#pragma unroll
        for (int i = 0; i < kGmPx / 4; ++i) {
            const float4 v = __ldcs(reinterpret_cast<const float4*>(s) + i);
            const float4 a = __ldg(reinterpret_cast<const float4*>(hl) + i), b = __ldg(reinterpret_cast<const float4*>(hh) + i);
            __stcs(reinterpret_cast<float4*>(d) + i,
                   make_float4(v.x * lerpf(a.x, b.x, sy.weight), v.y * lerpf(a.y, b.y, sy.weight),
                               v.z * lerpf(a.z, b.z, sy.weight), v.w * lerpf(a.w, b.w, sy.weight)));
        }
        return;
    }
    for (int i = 0; i < kGmPx && x0 + i < in.w; ++i)
        *px<float>(out, x0 + i, y) = *px<const float>(in, x0 + i, y) * lerpf(__ldg(hl + i), __ldg(hh + i), sy.weight);
}

// GainMap: lanes take interleaved pixels (x0 + lane + 32 j) so that a warp's
// per-column axis samples (12 bytes each) and its pixels are read as
// contiguous runs; 8 pixels per thread (maps per plane).
__global__ void __launch_bounds__(kPtThreads) gainmap_kernel(Img in, Img out, GainMapDev g) {
    const int y = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int x0 = (blockIdx.x * kPtThreads + (threadIdx.x & ~31)) * kGmPx + lane;
    float v[kGmPx];
#pragma unroll
    for (int j = 0; j < kGmPx; ++j) {
        const int x = x0 + 32 * j;
        v[j] = x < in.w ? __ldcs(px<const float>(in, x, y)) : 0.0F;
    }
#pragma unroll
    for (int j = 0; j < kGmPx; ++j) {
        const int x = x0 + 32 * j;
        if (x < in.w) __stcs(px<float>(out, x, y), v[j] * gain_px(gain_map_index(x, y, g), x, y, g));
    }
}

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
// demosaic_quad_bayer_remosaic_generator.cpp:17-58, integer arithmetic.  A tap
// (dx, dy) of output (x, y) reads source s = (clamp(x+dx), clamp(y+dy)); its
// weight is 65536 / (64 + G(s) + 16 (|dx| + |dy|)), G(s) the source's clamped
// horizontal plus vertical gradient, when the source's colour is the output's
// Bayer target, else 0.  The weight depends on the tap only through the
// source and the distance class d = |dx| + |dy| (0..4), so each tile first
// computes, for every cell of its halo-2 ring, the clamped source's value,
// colour and five class weights (5 divisions per cell instead of 25 per
// output), addressed by the cell's unclamped position: the 25-tap sum then
// reads cells with fixed offsets and no clamps.  Tile 64x16, input halo 3.
constexpr int kQbTW = 64, kQbTH = 16, kQbHalo = 3;
constexpr int kQbIW = kQbTW + 2 * kQbHalo, kQbIH = kQbTH + 2 * kQbHalo;
constexpr int kQbCW = kQbTW + 4, kQbCH = kQbTH + 4;  // cells: tile + halo 2
__device__ __forceinline__ int qbc_color(int x, int y) {
    const int mx = ((x % 4) + 4) % 4, my = ((y % 4) + 4) % 4;
    return (my < 2 && mx < 2) ? 0 : ((my >= 2 && mx >= 2) ? 2 : 1);
}
// floor(65536 / p) for 64 <= p < 2^18, by reciprocal estimate and one
// remainder correction (division by multiplication with an approximate
// reciprocal, Warren, Hacker's Delight 2nd ed., ch. 10).  rcp.approx has
// relative error <= 2^-23, so 65536 * rcp(p) is within 1024 * 2^-22 < 1 of
// the true quotient q <= 1024: the truncated estimate is q or one off either
// way, and the sign of the remainder 65536 - q0 p picks the exact floor.
__device__ __forceinline__ int div65536(int p) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"((float)p));
    int q = (int)(65536.0F * r);
    const int rem = 65536 - q * p;
    q += rem < 0 ? -1 : (rem >= p ? 1 : 0);
    return q;
}
__global__ void __launch_bounds__(256) qbc_kernel(Img in, Img out) {
    __shared__ int s[kQbIH * kQbIW];
    __shared__ uint32_t s_vc[kQbCH * kQbCW];        // value | colour << 16
    __shared__ uint16_t s_cw[5][kQbCH * kQbCW];     // class weights, d = 0..4
    const int x0 = blockIdx.x * kQbTW, y0 = blockIdx.y * kQbTH;
    constexpr int kLoads = (kQbIH * kQbIW + 255) / 256;  // issued together (256-thread blocks)
    int v[kLoads];
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + 256 * k;
        const int ty = i / kQbIW, tx = i - ty * kQbIW;
        if (i < kQbIH * kQbIW)
            v[k] = *px<const uint16_t>(in, clampi(x0 - kQbHalo + tx, 0, in.w - 1), clampi(y0 - kQbHalo + ty, 0, in.h - 1));
    }
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + 256 * k;
        if (i < kQbIH * kQbIW) s[i] = v[k];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kQbCH * kQbCW; i += blockDim.x) {
        const int cy = i / kQbCW, cx = i - cy * kQbCW;
        const int sx = clampi(x0 - 2 + cx, 0, in.w - 1), sy = clampi(y0 - 2 + cy, 0, in.h - 1);
        // tile coordinates of the source and of its clamped neighbours (all inside the halo-3 tile)
        const int lx = sx - (x0 - kQbHalo), ly = sy - (y0 - kQbHalo);
        const int lxm = clampi(sx - 1, 0, in.w - 1) - (x0 - kQbHalo), lxp = clampi(sx + 1, 0, in.w - 1) - (x0 - kQbHalo);
        const int lym = clampi(sy - 1, 0, in.h - 1) - (y0 - kQbHalo), lyp = clampi(sy + 1, 0, in.h - 1) - (y0 - kQbHalo);
        const int g = abs(s[ly * kQbIW + lxm] - s[ly * kQbIW + lxp]) + abs(s[lym * kQbIW + lx] - s[lyp * kQbIW + lx]);
        s_vc[i] = (uint32_t)s[ly * kQbIW + lx] | ((uint32_t)qbc_color(sx, sy) << 16);
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            const int cw = div65536(64 + g + 16 * d);
            s_cw[d][i] = (uint16_t)(cw < 1 ? 1 : cw);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kQbTH * kQbTW; i += blockDim.x) {
        const int ty = i / kQbTW, tx = i - ty * kQbTW;
        const int x = x0 + tx, y = y0 + ty;
        if (x >= out.w || y >= out.h) continue;
        const uint32_t target = ((y & 1) == 0 && (x & 1) == 0) ? 0U : (((y & 1) != 0 && (x & 1) != 0) ? 2U : 1U);
        const int c0 = (ty + 2) * kQbCW + (tx + 2);
        uint32_t ws = 0, wsum = 0;
#pragma unroll
        for (int dy = -2; dy <= 2; ++dy) {
#pragma unroll
            for (int dx = -2; dx <= 2; ++dx) {
                const int c = c0 + dy * kQbCW + dx;
                const uint32_t vc = s_vc[c];
                const uint32_t wt = (vc >> 16) == target ? (uint32_t)s_cw[abs(dx) + abs(dy)][c] : 0U;
                ws += wt * (vc & 0xFFFFU);
                wsum += wt;
            }
        }
        *px<uint16_t>(out, x, y) = wsum == 0 ? 0 : (uint16_t)((ws + (wsum / 2U)) / wsum);
    }
}

// ------------------------------------------------------------ RGBA point ops
// RGBA point ops: each thread handles 32 bytes of one row (4 RGBA16F or 2
// RGBA32F pixels) with 16-byte loads and stores when the segment is whole,
// 4-channel interleaved and aligned; other segments go pixel by pixel.
template <class T, class Op>
__global__ void __launch_bounds__(kPtThreads) rgba_point_kernel(Img in, Img out, Op op) {
    constexpr int N = 32 / (4 * (int)sizeof(T));
    const int y = blockIdx.y;
    const int x0 = (blockIdx.x * kPtThreads + threadIdx.x) * N;
    if (x0 >= in.w) return;
    const T* s = px<const T>(in, x0, y);
    T* d = px<T>(out, x0, y);
    if (x0 + N <= in.w && in.pix_stride == 4 && out.pix_stride == 4 && al16(s) && al16(d)) {
        alignas(16) T v[4 * N];
        alignas(16) T o[4 * N];
#pragma unroll
        for (int i = 0; i < 2; ++i) reinterpret_cast<uint4*>(v)[i] = __ldcs(reinterpret_cast<const uint4*>(s) + i);
#pragma unroll
        for (int i = 0; i < N; ++i) op(v + 4 * i, o + 4 * i);
#pragma unroll
        for (int i = 0; i < 2; ++i) __stcs(reinterpret_cast<uint4*>(d) + i, reinterpret_cast<const uint4*>(o)[i]);
        return;
    }
    for (int i = 0; i < N && x0 + i < in.w; ++i) op(px<const T>(in, x0 + i, y), px<T>(out, x0 + i, y));
}
inline dim3 rgba_grid(int w, int h, bool f16) { return row_grid(w, h, f16 ? 4 : 2); }

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
// wb.greyworld_auto apply: v / neutral per RGB channel, alpha bits copied
// (greyworld_auto.cpp:66-77).
template <class T>
struct GreyOp {
    float n[3];
    __device__ void operator()(const T* s, T* d) const {
        const Rgba v = load_rgba(s);
        store_rgb_keep_alpha(d, Rgba{v.r / n[0], v.g / n[1], v.b / n[2], v.a}, s);
    }
};
// tone.aces_filmic (aces_filmic_generator.cpp:22-52): the Narkowicz 2016 fit
// per RGB channel, alpha passes; enabled == 0 passes every channel.
template <class T>
struct AcesOp {
    int enabled;
    __device__ void operator()(const T* s, T* d) const {
        const Rgba v = load_rgba(s);
        const Rgba o = enabled ? Rgba{aces_fit(v.r), aces_fit(v.g), aces_fit(v.b), v.a} : v;
        store_rgb_keep_alpha(d, o, s);
    }
};
// tone.reinhard (reinhard_generator.cpp:20-48): reinhard_px per RGB channel; alpha passes.
template <class T>
struct ReinhardOp {
    float wp2;
    __device__ void operator()(const T* s, T* d) const {
        const Rgba v = load_rgba(s);
        store_rgb_keep_alpha(d, Rgba{reinhard_px(v.r, wp2), reinhard_px(v.g, wp2), reinhard_px(v.b, wp2), v.a}, s);
    }
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
// guided_filter_generator.cpp:45-85, box 3x3 (R = 1, radius <= 1) or 5x5
// (R = 2).  Tile kGfTW x kGfTH; s_v holds the clamped input at coordinates
// [x0-2R, x0+TW+2R), s_a / s_b the a, b planes at the unclamped coordinates
// [x0-R, x0+TW+R) (their windows read the clamped input), then
// out = max(mean(a) v + mean(b), 0).  Box sums keep the generator's row-major
// left-associated order: a thread loads one (kGfG + 2R) x D window into
// registers and produces kGfG vertically adjacent sums from it, so each
// value (and its square) is read and formed once per thread, not per sum.
constexpr int kGfTW = 64, kGfTH = 16, kGfG = 4;
template <int R>
struct GuidedGeom {
    static constexpr int H = 2 * R, D = 2 * R + 1;
    static constexpr int IW = kGfTW + 2 * H, IH = kGfTH + 2 * H, IP = IW + 1;
    static constexpr int AW = kGfTW + 2 * R, AH = kGfTH + 2 * R, AP = AW + 1;
    static constexpr size_t bytes() { return sizeof(float) * (size_t)(3 * IP * IH + 2 * 3 * AP * AH); }
};
template <class T, bool F16, int R>
__global__ void __launch_bounds__(256, 3) guided_kernel(Img in, Img out, float eps) {
    using G = GuidedGeom<R>;
    constexpr int H = G::H, D = G::D, IW = G::IW, IH = G::IH, IP = G::IP, AW = G::AW, AH = G::AH, AP = G::AP;
    extern __shared__ __align__(16) float smem_f[];
    float* s_v = smem_f;               // [3][IH][IP]
    float* s_a = s_v + 3 * IP * IH;    // [3][AH][AP]
    float* s_b = s_a + 3 * AP * AH;
    const int x0 = blockIdx.x * kGfTW, y0 = blockIdx.y * kGfTH;
    // all of a thread's tile loads are issued before the first store (256-thread blocks)
    constexpr int kLoads = (IH * IW + 255) / 256;
    Rgba v[kLoads];
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + 256 * k;
        const int ty = i / IW, tx = i - ty * IW;
        if (i < IH * IW) v[k] = load_clamped<T>(in, x0 - H + tx, y0 - H + ty);
    }
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + 256 * k;
        const int ty = i / IW, tx = i - ty * IW;
        if (i < IH * IW) {
            s_v[ty * IP + tx] = v[k].r;
            s_v[IP * IH + ty * IP + tx] = v[k].g;
            s_v[2 * IP * IH + ty * IP + tx] = v[k].b;
        }
    }
    __syncthreads();
    constexpr float N = (float)(D * D);
    const ConstDiv cN{N, (float)(1.0 / (double)(D * D))};  // IEEE x / N (const_div)
    constexpr int AG = (AH + kGfG - 1) / kGfG;
    for (int item = threadIdx.x; item < 3 * AW * AG; item += blockDim.x) {
        const int c = item / (AW * AG);
        const int rem = item - c * AW * AG;
        const int g = rem / AW, tx = rem - g * AW;
        const int ty0 = g * kGfG;
        const float* V = s_v + c * IP * IH + ty0 * IP + tx;  // window origin of a/b sample (ty0, tx)
        float2 win[kGfG + 2 * R][D];  // (value, value^2)
#pragma unroll
        for (int r = 0; r < kGfG + 2 * R; ++r)
#pragma unroll
            for (int dx = 0; dx < D; ++dx) {
                const float t = (ty0 + r < IH) ? V[r * IP + dx] : 0.0F;
                win[r][dx] = make_float2(t, t * t);
            }
#pragma unroll
        for (int k = 0; k < kGfG; ++k) {
            if (ty0 + k >= AH) break;
            const float2 sums = box_chain2<D>(win, k);
            const float m = const_div(sums.x, cN), corr = const_div(sums.y, cN);
            const float var = max0(corr - (m * m));
            const float a = var / (var + eps);
            const int j = c * AP * AH + (ty0 + k) * AP + tx;
            s_a[j] = a;
            s_b[j] = m - (a * m);
        }
    }
    __syncthreads();
    constexpr int TG = kGfTH / kGfG;
    for (int item = threadIdx.x; item < kGfTW * TG; item += blockDim.x) {
        const int g = item / kGfTW, tx = item - g * kGfTW;
        const int ty0 = g * kGfG;
        float o[3][kGfG];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 win[kGfG + 2 * R][D];  // (a, b)
            const float* A = s_a + c * AP * AH + ty0 * AP + tx;
            const float* B = s_b + c * AP * AH + ty0 * AP + tx;
#pragma unroll
            for (int r = 0; r < kGfG + 2 * R; ++r)
#pragma unroll
                for (int dx = 0; dx < D; ++dx) win[r][dx] = make_float2(A[r * AP + dx], B[r * AP + dx]);
#pragma unroll
            for (int k = 0; k < kGfG; ++k) {
                const float2 sab = box_chain2<D>(win, k);
                const float v = s_v[c * IP * IH + (ty0 + k + H) * IP + (tx + H)];
                o[c][k] = max0((const_div(sab.x, cN) * v) + const_div(sab.y, cN));
            }
        }
        const int x = x0 + tx;
#pragma unroll
        for (int k = 0; k < kGfG; ++k) {
            const int y = y0 + ty0 + k;
            if (x >= out.w || y >= out.h) continue;
            const Rgba src = load_rgba(px<const T>(in, x, y));
            store_rgba(px<T>(out, x, y), Rgba{o[0][k], o[1][k], o[2][k], src.a});
        }
    }
}

// -------------------------------------------- color.scene_linear_to_display
// The reference node runs the OCIO processor of its config
// (share/cpipe/ocio/v0.2/config.ocio:57-79) on the host.  Restated from
// OpenColorIO's published transform definitions:
//  sRGB  : MatrixTransform (Rec.2020 -> Rec.709 primaries) on RGB, then the
//          inverse ExponentWithLinearTransform (gamma 2.4, offset 0.055:
//          e = L <= Lb ? L / slope : 1.055 L^(1/2.4) - 0.055), then
//          RangeTransform [0, 1] (a clamp); alpha untouched.
//  PQ    : RangeTransform [0, 1], then FixedFunction LIN_TO_PQ (SMPTE ST 2084,
//          linear 1.0 = 100 cd/m^2); alpha untouched.
// Quantisation as HostContext.cpp:91-99: round-half-away(clamp(v, 0, 1) * 255)
// for R8G8B8A8_UNORM, and round(clamp(v, 0, 1) * 1023) << 6 for the 10-bit
// R16G16B16A16_UNORM output.  Each thread converts 4 pixels of a row.
struct DisplayDev {
    float m[9];
    float lin_break, inv_slope;  // moncurve: linear breakpoint, 1 / slope
};
// x^e for x > 0 as exp2(e log2 x) with the PTX approximate base-2 log and exp
// (lg2.approx / ex2.approx, documented errors of order 2^-22): relative error
// below 1e-5 even after PQ's exponent of 78.8, far under the half code value
// (2e-3 of the range at 8 bits, 5e-4 at 10) that decides the output code.
__device__ __forceinline__ float pow_pos(float x, float e) {
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e * l));
    return r;
}
__device__ __forceinline__ float srgb_encode(float l, const DisplayDev& d) {
    return l <= d.lin_break ? l * d.inv_slope : (1.055F * pow_pos(l, 1.0F / 2.4F)) - 0.055F;
}
__device__ __forceinline__ float pq_encode(float v) {
    constexpr float m1 = 2610.0F / 16384.0F, m2 = 2523.0F / 4096.0F * 128.0F;
    constexpr float c2 = 2413.0F / 4096.0F * 32.0F, c3 = 2392.0F / 4096.0F * 32.0F, c1 = c3 - c2 + 1.0F;
    const float l = clampf(v, 0.0F, 1.0F) * 0.01F;
    const float y = l > 0.0F ? pow_pos(l, m1) : 0.0F;
    return pow_pos(__fdividef(c1 + (c2 * y), 1.0F + (c3 * y)), m2);
}
__device__ __forceinline__ float unorm_round(float v, float scale) { return roundf(clampf(v, 0.0F, 1.0F) * scale); }
template <unsigned TARGET>
__device__ __forceinline__ void display_px(Rgba v, const DisplayDev& d, float o[4]) {
    if (TARGET == CPIPE_DISPLAY_SRGB) {
        const float r = ((d.m[0] * v.r) + (d.m[1] * v.g)) + (d.m[2] * v.b);
        const float g = ((d.m[3] * v.r) + (d.m[4] * v.g)) + (d.m[5] * v.b);
        const float b = ((d.m[6] * v.r) + (d.m[7] * v.g)) + (d.m[8] * v.b);
        o[0] = unorm_round(srgb_encode(r, d), 255.0F);
        o[1] = unorm_round(srgb_encode(g, d), 255.0F);
        o[2] = unorm_round(srgb_encode(b, d), 255.0F);
        o[3] = unorm_round(v.a, 255.0F);
    } else {
        o[0] = unorm_round(pq_encode(v.r), 1023.0F);
        o[1] = unorm_round(pq_encode(v.g), 1023.0F);
        o[2] = unorm_round(pq_encode(v.b), 1023.0F);
        o[3] = unorm_round(v.a, 1023.0F);
    }
}
template <unsigned TARGET>
__device__ __forceinline__ void display_store(const Img& out, int x, int y, const float o[4]) {
    if (TARGET == CPIPE_DISPLAY_SRGB)
        *reinterpret_cast<uchar4*>(px<uint8_t>(out, x, y)) =
            make_uchar4((unsigned char)o[0], (unsigned char)o[1], (unsigned char)o[2], (unsigned char)o[3]);
    else
        *reinterpret_cast<ushort4*>(px<uint16_t>(out, x, y)) =
            make_ushort4((unsigned short)((unsigned)o[0] << 6), (unsigned short)((unsigned)o[1] << 6),
                          (unsigned short)((unsigned)o[2] << 6), (unsigned short)((unsigned)o[3] << 6));
}
// ------------------------------------------------------ tone.mertens_local
// mertens_local_generator.cpp:22-115: per pixel, a weight per exposure from
// its contrast (|luma - 0.5|), saturation (RGB spread around the luma) and
// well-exposedness (Gaussian around 0.5 per channel, sigma 0.2), each raised
// to its parameter (1 / the plain factor at the defaults), then the weighted
// mean of the three exposures, clamped to [0, 1]; alpha from the normal frame.
struct MertensDev {
    float wc, ws, we;
};
__device__ __forceinline__ float mertens_cew(float v) {
    constexpr float k = 2.0F * 0.20F * 0.20F;
    const float d = v - 0.5F;
    return expf(-(d * d) / k);
}
__device__ __forceinline__ float mertens_weight(const Rgba& f, const MertensDev& p) {
    const float red = max0(f.r), green = max0(f.g), blue = max0(f.b);
    const float mean = ((f.r + f.g) + f.b) / 3.0F;
    const float sat = sqrtf(((((red - mean) * (red - mean)) + ((green - mean) * (green - mean))) +
                             ((blue - mean) * (blue - mean))) / 3.0F +
                            0.0001F);
    const float well = (mertens_cew(red) * mertens_cew(green)) * mertens_cew(blue);
    const float contrast = fabsf(mean - 0.5F);
    const float cf = p.wc == 0.0F ? 1.0F : powf(contrast + 0.01F, p.wc);
    const float sf = p.ws == 1.0F ? sat + 0.01F : powf(sat + 0.01F, p.ws);
    const float ef = p.we == 1.0F ? well : powf(well + 0.0001F, p.we);
    return (cf * sf) * ef;
}
__global__ void __launch_bounds__(kPtThreads) mertens_kernel(Img under, Img normal, Img over, Img out, MertensDev p) {
    const int y = blockIdx.y, x = blockIdx.x * kPtThreads + threadIdx.x;
    if (x >= out.w) return;
    const Rgba u = load_rgba(px<const __half>(under, x, y)), n = load_rgba(px<const __half>(normal, x, y));
    const Rgba o = load_rgba(px<const __half>(over, x, y));
    const float wu = mertens_weight(u, p), wn = mertens_weight(n, p), wo = mertens_weight(o, p);
    const float total = maxf((wu + wn) + wo, 0.000001F);
    const float r = clampf((((wu * u.r) + (wn * n.r)) + (wo * o.r)) / total, 0.0F, 1.0F);
    const float g = clampf((((wu * u.g) + (wn * n.g)) + (wo * o.g)) / total, 0.0F, 1.0F);
    const float b = clampf((((wu * u.b) + (wn * n.b)) + (wo * o.b)) / total, 0.0F, 1.0F);
    const __half* ns = px<const __half>(normal, x, y);
    store_rgb_keep_alpha(px<__half>(out, x, y), Rgba{r, g, b, n.a}, ns);
}

// ------------------------------------------------------ wb.greyworld_auto
// Estimate: per-channel sums of the RGB values of an RGBA16F frame.  Every
// binary16 value is an integer multiple of 2^-24, below 2^41 of those units
// in magnitude, so a block adds its pixels as int64 integers (exact, in any
// order) over a fixed range of rows and the host adds the block totals in
// 128-bit integers: the sum is exact and rounded to double once, whatever the
// order the blocks ran in.  partial[b] = {sum R, sum G, sum B, non-finite seen}.
__device__ __forceinline__ long long h16_units(unsigned h, int* nonfinite) {
    const int e = (int)((h >> 10) & 31U), m = (int)(h & 1023U);
    if (e == 31) {
        *nonfinite = 1;
        return 0;
    }
    const long long mag = e == 0 ? (long long)m : ((long long)(1024 + m) << (e - 1));
    return (h & 0x8000U) ? -mag : mag;
}
__global__ void __launch_bounds__(256) greyworld_sum_kernel(Img in, long long* partial) {
    const int rows = (in.h + (int)gridDim.x - 1) / (int)gridDim.x;
    const int y0 = (int)blockIdx.x * rows, y1 = min(in.h, y0 + rows);
    long long s0 = 0, s1 = 0, s2 = 0;
    int bad = 0;
    for (int y = y0; y < y1; ++y) {
        // pixel pairs as 16-byte loads (cached: the apply pass reads the frame again)
        const __half* row = px<const __half>(in, 0, y);
        const int pairs = in.pix_stride == 4 && al16(row) ? in.w / 2 : 0;
#pragma unroll 4
        for (int j = threadIdx.x; j < pairs; j += blockDim.x) {
            const uint4 u = __ldg(reinterpret_cast<const uint4*>(row) + j);
            s0 += h16_units(u.x & 0xFFFFU, &bad) + h16_units(u.z & 0xFFFFU, &bad);
            s1 += h16_units(u.x >> 16, &bad) + h16_units(u.z >> 16, &bad);
            s2 += h16_units(u.y & 0xFFFFU, &bad) + h16_units(u.w & 0xFFFFU, &bad);
        }
        for (int x = 2 * pairs + threadIdx.x; x < in.w; x += blockDim.x) {
            const uint2 u = *reinterpret_cast<const uint2*>(px<const __half>(in, x, y));
            s0 += h16_units(u.x & 0xFFFFU, &bad);
            s1 += h16_units(u.x >> 16, &bad);
            s2 += h16_units(u.y & 0xFFFFU, &bad);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s0 += __shfl_down_sync(0xFFFFFFFFU, s0, off);
        s1 += __shfl_down_sync(0xFFFFFFFFU, s1, off);
        s2 += __shfl_down_sync(0xFFFFFFFFU, s2, off);
        bad |= __shfl_down_sync(0xFFFFFFFFU, bad, off);
    }
    __shared__ long long sh[8][4];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[wid][0] = s0;
        sh[wid][1] = s1;
        sh[wid][2] = s2;
        sh[wid][3] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t[4] = {0, 0, 0, 0};
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            for (int k = 0; k < 4; ++k) t[k] = k < 3 ? t[k] + sh[w][k] : (t[k] | sh[w][k]);
        for (int k = 0; k < 4; ++k) partial[4 * blockIdx.x + k] = t[k];
    }
}

// ------------------------------------------------- sharpen.edge_aware_usm
// edge_aware_usm_generator.cpp:11-75: blur = mean3x3 (R = 1: the explicit
// 9-term left-associated sum, :11-17) or mean5x5 (R = 2: 0 + the 25 terms in
// row-major order, :19-27) of the clamped input; mask = v - blur;
// RGB = max(0, |mask| >= threshold ? v + strength * mask : v); alpha = v.
// Tile 64 x TH with halo R in shared memory (three planes); a thread loads one
// (G + 2R) x D window per channel into registers and produces the G
// vertically adjacent outputs of one column (64x16 tiles, G = 4; a 64x32 tile
// with G = 8 measured no faster: the kernel is issue-bound by the exact-order
// sums and the IEEE division per channel).
constexpr int kUsmTW = 64, kUsmTH = 16, kUsmG = 4;
template <int D, int ROWS>
__device__ __forceinline__ float usm_box(const float (&win)[ROWS][D], int k) {
    float s = D == 3 ? win[k][0] : 0.0F + win[k][0];
#pragma unroll
    for (int dy = 0; dy < D; ++dy)
#pragma unroll
        for (int dx = 0; dx < D; ++dx)
            if (dy != 0 || dx != 0) s = s + win[k + dy][dx];
    return s;
}
// DISP 0: RGBA output of the input's type; 1 / 2: the f16-rounded result is
// display-encoded (sRGB / BT2020-PQ) into an RGBA8 / RGBA16 unorm output.
template <class T, int R, int TH, int G, int DISP>
__global__ void __launch_bounds__(256) usm_kernel(Img in, Img out, float strength, float threshold, DisplayDev dd) {
    static_assert(kUsmTW * TH == 256 * G, "one column of G rows per thread");
    constexpr int D = 2 * R + 1, IW = kUsmTW + 2 * R, IH = TH + 2 * R, IP = IW + 1;
    __shared__ float s_v[3][IH * IP];
    const int x0 = blockIdx.x * kUsmTW, y0 = blockIdx.y * TH;
    constexpr int kLoads = (IH * IW + 255) / 256;  // issued together (256-thread blocks)
    Rgba v[kLoads];
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + 256 * k;
        const int ty = i / IW, tx = i - ty * IW;
        if (i < IH * IW) v[k] = load_clamped<T>(in, x0 - R + tx, y0 - R + ty);
    }
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + 256 * k;
        const int ty = i / IW, tx = i - ty * IW;
        if (i < IH * IW) {
            s_v[0][ty * IP + tx] = v[k].r;
            s_v[1][ty * IP + tx] = v[k].g;
            s_v[2][ty * IP + tx] = v[k].b;
        }
    }
    __syncthreads();
    const int tx = threadIdx.x & (kUsmTW - 1), ty0 = (threadIdx.x / kUsmTW) * G;
    constexpr float N = (float)(D * D);
    const ConstDiv cN{N, (float)(1.0 / (double)(D * D))};  // IEEE x / N (const_div)
    float o[3][G];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float win[G + 2 * R][D];
        const float* V = s_v[c] + ty0 * IP + tx;
#pragma unroll
        for (int r = 0; r < G + 2 * R; ++r)
#pragma unroll
            for (int dx = 0; dx < D; ++dx) win[r][dx] = V[r * IP + dx];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            const float blur = const_div(usm_box<D>(win, k), cN);
            const float val = win[k + R][R];
            const float mask = val - blur;
            const float sh = fabsf(mask) >= threshold ? val + (strength * mask) : val;
            o[c][k] = max0(sh);
        }
    }
    const int x = x0 + tx;
#pragma unroll
    for (int k = 0; k < G; ++k) {
        const int y = y0 + ty0 + k;
        if (x >= out.w || y >= out.h) continue;
        const Rgba src = load_rgba(px<const T>(in, x, y));
        if constexpr (DISP == 0) {
            store_rgba(px<T>(out, x, y), Rgba{o[0][k], o[1][k], o[2][k], src.a});
        } else {
            constexpr unsigned kTarget = (unsigned)(DISP - 1);
            float q[4];
            display_px<kTarget>(Rgba{h16(o[0][k]), h16(o[1][k]), h16(o[2][k]), src.a}, dd, q);
            display_store<kTarget>(out, x, y, q);
        }
    }
}

template <unsigned TARGET>
__global__ void __launch_bounds__(kPtThreads) display_kernel(Img in, Img out, DisplayDev d) {
    const int y = blockIdx.y;
    const int x0 = (blockIdx.x * kPtThreads + threadIdx.x) * 4;
    if (x0 >= in.w) return;
    const __half* s = px<const __half>(in, x0, y);
    const bool whole = x0 + 4 <= in.w && in.pix_stride == 4 && out.pix_stride == 4 && al16(s) &&
                       (TARGET == CPIPE_DISPLAY_SRGB ? al16(px<uint8_t>(out, x0, y)) : al16(px<uint16_t>(out, x0, y)));
    if (!whole) {
        for (int i = 0; i < 4 && x0 + i < in.w; ++i) {
            float o[4];
            display_px<TARGET>(load_rgba(px<const __half>(in, x0 + i, y)), d, o);
            display_store<TARGET>(out, x0 + i, y, o);
        }
        return;
    }
    alignas(16) __half v[16];
#pragma unroll
    for (int i = 0; i < 2; ++i) reinterpret_cast<uint4*>(v)[i] = __ldcs(reinterpret_cast<const uint4*>(s) + i);
    float o[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) display_px<TARGET>(load_rgba(v + 4 * i), d, o[i]);
    if (TARGET == CPIPE_DISPLAY_SRGB) {
        uint4 q;
        uint32_t* w = reinterpret_cast<uint32_t*>(&q);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            w[i] = (uint32_t)o[i][0] | ((uint32_t)o[i][1] << 8) | ((uint32_t)o[i][2] << 16) | ((uint32_t)o[i][3] << 24);
        __stcs(reinterpret_cast<uint4*>(px<uint8_t>(out, x0, y)), q);
    } else {
        uint4 q[2];
        uint32_t* w = reinterpret_cast<uint32_t*>(q);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            w[2 * i] = ((uint32_t)o[i][0] << 6) | ((uint32_t)o[i][1] << 22);
            w[2 * i + 1] = ((uint32_t)o[i][2] << 6) | ((uint32_t)o[i][3] << 22);
        }
        uint4* dq = reinterpret_cast<uint4*>(px<uint16_t>(out, x0, y));
        __stcs(dq, q[0]);
        __stcs(dq + 1, q[1]);
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
    raw_vec_kernel<uint16_t><<<row_grid(in.w, in.h, 16), kPtThreads, 0, st>>>(in, out, R16ToF32{});
    return cudaGetLastError();
}
cudaError_t launch_linearize(const Img& in, const Img& out, const uint16_t* d_table, int n, cudaStream_t st) {
    if (n > 0 && n <= kLinSmemMax)
        linearize_smem_kernel<<<dim3(row_grid(in.w, in.h, 16).x, (unsigned)(in.h < kLinRowBlocks ? in.h : kLinRowBlocks)),
                                kPtThreads, (size_t)n * sizeof(uint16_t), st>>>(in, out, d_table, n);
    else
        raw_vec_kernel<uint16_t><<<row_grid(in.w, in.h, 16), kPtThreads, 0, st>>>(in, out, Linearize{d_table, n - 1});
    return cudaGetLastError();
}
cudaError_t launch_blacklevel(const Img& in, const Img& out, const BlackDev& p, cudaStream_t st) {
    raw_vec_kernel<float><<<row_grid(in.w, in.h, 8), kPtThreads, 0, st>>>(in, out, Blacklevel{p});
    return cudaGetLastError();
}
size_t gainmap_hrows_bytes(const GainMapDev& g, int w) {
    size_t n = 0;
    for (int m = 0; m < g.map_count; ++m) n += (((size_t)g.points_v[m] * w * sizeof(float)) + 15) & ~size_t(15);
    return n;
}
cudaError_t launch_gainmap_hrows(GainMapDev* g, void* d_hrows, int w, cudaStream_t st) {
    char* p = static_cast<char*>(d_hrows);
    int pv = 1;
    for (int m = 0; m < g->map_count; ++m) {
        g->hrow[m] = reinterpret_cast<const float*>(p);
        p += (((size_t)g->points_v[m] * w * sizeof(float)) + 15) & ~size_t(15);
        pv = g->points_v[m] > pv ? g->points_v[m] : pv;
    }
    g->hw = w;
    const dim3 grid((unsigned)((w + kPtThreads - 1) / kPtThreads), (unsigned)pv, (unsigned)g->map_count);
    gainmap_hrows_kernel<<<grid, kPtThreads, 0, st>>>(*g);
    return cudaGetLastError();
}
cudaError_t launch_gainmap(const Img& in, const Img& out, const GainMapDev& g, cudaStream_t st) {
    if (g.map_count == 1) {
        gainmap_one_map_kernel<<<row_grid(in.w, in.h, kGmPx), kPtThreads, 0, st>>>(in, out, g);
        return cudaGetLastError();
    }
    gainmap_kernel<<<row_grid(in.w, in.h, kGmPx), kPtThreads, 0, st>>>(in, out, g);
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
    const dim3 g = rgba_grid(in.w, in.h, f16);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, WbOp<__half>{{n[0], n[1], n[2]}})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, WbOp<float>{{n[0], n[1], n[2]}})));
    return cudaGetLastError();
}
cudaError_t launch_colormatrix(const Img& in, const Img& out, bool f16, const float t[9], cudaStream_t st) {
    const dim3 g = rgba_grid(in.w, in.h, f16);
    CmOp<__half> oh;
    CmOp<float> of;
    for (int i = 0; i < 9; ++i) oh.t[i] = of.t[i] = t[i];
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, oh)),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, of)));
    return cudaGetLastError();
}
cudaError_t launch_filmic(const Img& in, const Img& out, bool f16, const FilmicDev& p, cudaStream_t st) {
    const dim3 g = rgba_grid(in.w, in.h, f16);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, FilmicOp<__half>{p})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, FilmicOp<float>{p})));
    return cudaGetLastError();
}
cudaError_t launch_lut3d(const Img& in, const Img& out, bool f16, const float4* d_lut, int S, int interp, cudaStream_t st) {
    const dim3 g = rgba_grid(in.w, in.h, f16);
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
template <class T, bool F16, int R>
cudaError_t guided_launch(const Img& in, const Img& out, float eps, cudaStream_t st) {
    // the whole carveout as shared memory, so that 3 blocks fit per SM
    static const cudaError_t attr = [] {
        cudaError_t e = cudaFuncSetAttribute(guided_kernel<T, F16, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)GuidedGeom<R>::bytes());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(guided_kernel<T, F16, R>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        return e;
    }();
    if (attr != cudaSuccess) return attr;
    const dim3 g((unsigned)((in.w + kGfTW - 1) / kGfTW), (unsigned)((in.h + kGfTH - 1) / kGfTH));
    guided_kernel<T, F16, R><<<g, 256, GuidedGeom<R>::bytes(), st>>>(in, out, eps);
    return cudaGetLastError();
}
cudaError_t launch_guided(const Img& in, const Img& out, bool f16, int radius, float eps, cudaStream_t st) {
    if (radius <= 1) return f16 ? guided_launch<__half, true, 1>(in, out, eps, st) : guided_launch<float, false, 1>(in, out, eps, st);
    return f16 ? guided_launch<__half, true, 2>(in, out, eps, st) : guided_launch<float, false, 2>(in, out, eps, st);
}
static DisplayDev display_dev() {
    // Rec.2020 -> Rec.709 matrix of the config's output_srgb colour space
    static const float kM[9] = {1.6604910F, -0.5876411F, -0.0728499F, -0.1245505F, 1.1328999F,
                                -0.0083494F, -0.0181508F, -0.1005789F, 1.1187297F};
    DisplayDev d;
    for (int i = 0; i < 9; ++i) d.m[i] = kM[i];
    // moncurve with gamma g, offset o: encoded breakpoint eb = o / (g - 1), linear
    // breakpoint Lb = (o g / ((g - 1)(1 + o)))^g, slope = Lb / eb (continuous)
    const double gm = 2.4, off = 0.055;
    const double eb = off / (gm - 1.0), lb = std::pow(off * gm / ((gm - 1.0) * (1.0 + off)), gm);
    d.lin_break = (float)lb;
    d.inv_slope = (float)(eb / lb);
    return d;
}
cudaError_t launch_mertens(const Img& under, const Img& normal, const Img& over, const Img& out, float wc, float ws,
                           float we, cudaStream_t st) {
    mertens_kernel<<<row_grid(out.w, out.h, 1), kPtThreads, 0, st>>>(under, normal, over, out, MertensDev{wc, ws, we});
    return cudaGetLastError();
}
cudaError_t launch_greyworld_sums(const Img& in, long long* d_partial, int blocks, cudaStream_t st) {
    greyworld_sum_kernel<<<(unsigned)blocks, 256, 0, st>>>(in, d_partial);
    return cudaGetLastError();
}
cudaError_t launch_greyworld_apply(const Img& in, const Img& out, const float n[3], cudaStream_t st) {
    const dim3 g = rgba_grid(in.w, in.h, true);
    rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, GreyOp<__half>{{n[0], n[1], n[2]}});
    return cudaGetLastError();
}
cudaError_t launch_aces(const Img& in, const Img& out, bool f16, int enabled, cudaStream_t st) {
    const dim3 g = rgba_grid(in.w, in.h, f16);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, AcesOp<__half>{enabled})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, AcesOp<float>{enabled})));
    return cudaGetLastError();
}
cudaError_t launch_reinhard(const Img& in, const Img& out, bool f16, float white_point, cudaStream_t st) {
    const float wp2 = white_point * white_point;
    const dim3 g = rgba_grid(in.w, in.h, f16);
    RGBA_DISPATCH(f16, (rgba_point_kernel<__half><<<g, kPtThreads, 0, st>>>(in, out, ReinhardOp<__half>{wp2})),
                  (rgba_point_kernel<float><<<g, kPtThreads, 0, st>>>(in, out, ReinhardOp<float>{wp2})));
    return cudaGetLastError();
}
cudaError_t launch_usm(const Img& in, const Img& out, bool f16, float strength, int radius, float threshold,
                       cudaStream_t st) {
    const dim3 g((unsigned)((in.w + kUsmTW - 1) / kUsmTW), (unsigned)((in.h + kUsmTH - 1) / kUsmTH));
    if (radius <= 1) {
        RGBA_DISPATCH(f16, (usm_kernel<__half, 1, kUsmTH, kUsmG, 0><<<g, 256, 0, st>>>(in, out, strength, threshold, DisplayDev{})),
                      (usm_kernel<float, 1, kUsmTH, kUsmG, 0><<<g, 256, 0, st>>>(in, out, strength, threshold, DisplayDev{})));
    } else {
        RGBA_DISPATCH(f16, (usm_kernel<__half, 2, kUsmTH, kUsmG, 0><<<g, 256, 0, st>>>(in, out, strength, threshold, DisplayDev{})),
                      (usm_kernel<float, 2, kUsmTH, kUsmG, 0><<<g, 256, 0, st>>>(in, out, strength, threshold, DisplayDev{})));
    }
    return cudaGetLastError();
}
cudaError_t launch_usm_display(const Img& in, const Img& out, float strength, int radius, float threshold,
                               unsigned target, cudaStream_t st) {
    const dim3 g((unsigned)((in.w + kUsmTW - 1) / kUsmTW), (unsigned)((in.h + kUsmTH - 1) / kUsmTH));
    const DisplayDev dd = display_dev();
#define USMD(R, D) usm_kernel<__half, R, kUsmTH, kUsmG, D><<<g, 256, 0, st>>>(in, out, strength, threshold, dd)
    if (target == CPIPE_DISPLAY_SRGB) {
        if (radius <= 1) USMD(1, 1); else USMD(2, 1);
    } else {
        if (radius <= 1) USMD(1, 2); else USMD(2, 2);
    }
#undef USMD
    return cudaGetLastError();
}
cudaError_t launch_display(const Img& in, const Img& out, unsigned target, cudaStream_t st) {
    const DisplayDev d = display_dev();
    const dim3 g = row_grid(in.w, in.h, 4);
    if (target == CPIPE_DISPLAY_SRGB) display_kernel<CPIPE_DISPLAY_SRGB><<<g, kPtThreads, 0, st>>>(in, out, d);
    else display_kernel<CPIPE_DISPLAY_BT2020_PQ><<<g, kPtThreads, 0, st>>>(in, out, d);
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
