// The fused raw->linear chain: the reference node sequence
//   precision_convert(r16u->f32) -> blacklevel -> GainMap -> demosaic ->
//   OpcodeList3 -> WB -> colormatrix -> BM3D -> guided -> wavelet -> filmic -> 3D LUT
// in three kernels instead of twelve launches and eleven intermediate frames:
//
//   K1 raw_to_rgba   u16 Bayer tile (+3 halo) -> convert/black/gain in shared
//                    memory -> demosaic -> RGBA            (2 B/px in, 8 B/px out)
//   K2 warp_wb_cm    OpcodeList3 warp (bicubic gather from K1's frame) -> WB ->
//                    colormatrix, per pixel               (8 B/px in, 8 B/px out)
//   K3 denoise_tone  BM3D (parity form) -> guided -> wavelet -> filmic -> LUT on a
//                    shared-memory tile with the halo the guided box-of-boxes
//                    and the 2x2 blocks need             (8 B/px in, 8 B/px out)
//
// Every node boundary keeps the reference storage rounding (binary16 for the
// RGBA nodes; none in the FP32 plain form), so the fused result equals running
// the nodes one by one.  OpcodeList3 lists other than a single WarpRectilinear
// run through the per-node OpcodeList3 path between K1 and a WB+colormatrix K2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "filters_impl.h"
#include "kernels.h"
#include "bm3d_spec.h"
#include "spec_denoise.h"
#include "surrogate.h"
#include "demosaic.cuh"
#include "nodes.cuh"

namespace cpb {
namespace {

// ------------------------------------------------------------------ K1
struct RawParams {
    BlackDev black;
    GainMapDev gain;
    int has_gain;
    Cfa cfa;
};

// precision_convert -> blacklevel -> GainMap at a clamped coordinate
struct RawLoader {
    Img raw;
    const RawParams* p;
    __device__ __forceinline__ float operator()(int gx, int gy) const {
        float v = (float)*px<const uint16_t>(raw, gx, gy);
        v = blacklevel_px(v, gx, gy, p->black);
        if (p->has_gain) v = v * gain_px(gain_map_index(gx, gy, p->gain), gx, gy, p->gain);
        return v;
    }
};

template <int ALGO, class TOut>
__global__ void __launch_bounds__(256) raw_to_rgba_kernel(Img raw, Img out, RawParams p) {
    demosaic_tile<ALGO, TOut>(RawLoader{raw, &p}, raw.w, raw.h, out, p.cfa);
}

// ------------------------------------------------------------------ K2
struct ColorParams {
    float neutral[3];
    float cm[9];
};

// A single warp's bicubic taps for every output pixel, computed once when the
// chain is made (warp_taps_kernel; the same warp_tap as the inline path):
// ixy = ix | iy << 16, tx, ty; n = w * h entries each.
struct WarpTaps {
    const uint32_t* ixy;
    const float* tx;
    const float* ty;
};
__global__ void __launch_bounds__(256) warp_taps_kernel(int w, int h, WarpDev wd, uint32_t* ixy, float* tx, float* ty) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const WarpTap t = warp_tap_px(wd, x, y);
    const size_t i = (size_t)y * w + x;
    ixy[i] = (uint32_t)t.ix | ((uint32_t)t.iy << 16);
    tx[i] = t.tx;
    ty[i] = t.ty;
}

// WARP 0: no warp; 1: the warp evaluated per pixel; 2: read from the tap table.
template <class T, bool F16, int WARP>
__device__ __forceinline__ void warp_wb_cm_px(const Img& in, const Img& out, const WarpDev& w, const ColorParams& cp,
                                              int x, int y, const WarpTaps& taps = WarpTaps{}) {
    Rgba v;
    if (WARP != 0) {
        Rgba wv;
        if (WARP == 2) {
            const size_t i = (size_t)y * out.w + x;
            const uint32_t p = __ldg(taps.ixy + i);
            wv = bicubic_at<T>(in, WarpTap{(int)(p & 0xFFFFU), (int)(p >> 16), __ldg(taps.tx + i), __ldg(taps.ty + i)});
        } else {
            wv = warp_px<T>(in, w, x, y);
        }
        v = Rgba{rnd<F16>(wv.r), rnd<F16>(wv.g), rnd<F16>(wv.b), rnd<F16>(wv.a)};
    } else {
        v = load_rgba(px<const T>(in, x, y));
    }
    Rgba b = wb_px(v, cp.neutral);
    b = Rgba{rnd<F16>(b.r), rnd<F16>(b.g), rnd<F16>(b.b), v.a};
    const Rgba c = cm_px(b, cp.cm);
    store_rgba(px<T>(out, x, y), Rgba{c.r, c.g, c.b, v.a});
}

template <class T, bool F16, int WARP>
__global__ void __launch_bounds__(128) warp_wb_cm_kernel(Img in, Img out, WarpDev w, ColorParams cp, WarpTaps taps) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= out.w) return;
    warp_wb_cm_px<T, F16, WARP>(in, out, w, cp, x, y, taps);
}

// ------------------------------------------------------------------ K3
// Tile TW x TH; R = guided box radius (0: no guided node, 1: 3x3, 2: 5x5).
// Shared-memory planes (3 colour channels each, float: every value stored is
// either an f16 node output or an f32 intermediate, so no precision is lost),
// indexed by unclamped coordinate relative to the tile origin:
//   s_bm : BM3D output at clamp(coord), coords [x0-2R, x0+TW+2R)
//   s_a/s_b : guided a, b at coords [x0-R, x0+TW+R)
//   s_gf : guided output for the tile (needed whole for the wavelet 2x2 blocks)
// BM3D is evaluated per 2x2 block of the extent (x0 and 2R are even, so the
// extent is made of whole blocks): an interior block reads its four input
// pixels with two 16-byte loads and yields four outputs; a block that overlaps
// the frame border evaluates each cell at its clamped coordinate.
// Box sums keep the generator's row-major left-to-right order; a thread loads
// one (G+2R) x (2R+1) window into registers and produces G outputs from it.
constexpr int kCTW = 64, kCTH = 16, kCG = 4;

struct ToneParams {
    int has_wavelet;
    float bm3d_strength;
    float eps;
    float wavelet_th;
    FilmicDev filmic;
    int tone_op;        // 0 tone.filmic_rgb, 1 tone.aces_filmic, 2 tone.reinhard
    float reinhard_wp2; // white point squared (tone_op 2)
    const float4* lut;
    int lut_size, lut_interp;
    int has_lut;
};

template <int R>
struct ToneGeom {
    static constexpr int H = 2 * R;
    static constexpr int CW = kCTW + 2 * H, CH = kCTH + 2 * H;  // bm3d extent
    static constexpr int CP = CW + 1;                           // padded row pitch
    static constexpr int AW = kCTW + 2 * R, AH = kCTH + 2 * R;  // a / b extent
    static constexpr int AP = AW + 1;
    static constexpr int AB = R > 0 ? AP * AH : 0;
    static constexpr int D = 2 * R + 1;
    static constexpr size_t bytes() { return sizeof(float) * (size_t)(3 * CP * CH + 2 * 3 * AB + 3 * kCTW * kCTH); }
};

template <class T>
__device__ __forceinline__ void load_pair(const Img& in, int x, int y, Rgba* a, Rgba* b);
// Two adjacent RGBA16F pixels; one 16-byte load when the pair is 16-byte
// aligned (always for even x when the row pitch is a multiple of 16 bytes),
// else two 8-byte loads.
template <>
__device__ __forceinline__ void load_pair<__half>(const Img& in, int x, int y, Rgba* a, Rgba* b) {
    const __half* p0 = px<const __half>(in, x, y);
    if ((reinterpret_cast<uintptr_t>(p0) & 15) != 0) {
        *a = load_rgba(p0);
        *b = load_rgba(p0 + in.pix_stride);
        return;
    }
    const uint4 u = *reinterpret_cast<const uint4*>(p0);
    const __half2 h0 = *reinterpret_cast<const __half2*>(&u.x), h1 = *reinterpret_cast<const __half2*>(&u.y);
    const __half2 h2 = *reinterpret_cast<const __half2*>(&u.z), h3 = *reinterpret_cast<const __half2*>(&u.w);
    *a = Rgba{__low2float(h0), __high2float(h0), __low2float(h1), __high2float(h1)};
    *b = Rgba{__low2float(h2), __high2float(h2), __low2float(h3), __high2float(h3)};
}
template <>
__device__ __forceinline__ void load_pair<float>(const Img& in, int x, int y, Rgba* a, Rgba* b) {
    *a = load_rgba(px<const float>(in, x, y));
    *b = load_rgba(px<const float>(in, x + 1, y));
}

// One kCTW x kCTH output tile at (x0, y0); smem_f: denoise_tone_smem bytes.
template <class T, bool F16, int R>
__device__ __forceinline__ void denoise_tone_tile(const Img& in, const Img& out, const ToneParams& p, int x0, int y0,
                                                  float* smem_f) {
    using Gm = ToneGeom<R>;
    constexpr int H = Gm::H, CW = Gm::CW, CH = Gm::CH, CP = Gm::CP, AW = Gm::AW, AH = Gm::AH, AP = Gm::AP;
    constexpr int AB = Gm::AB, D = Gm::D;
    float* s_bm = smem_f;
    float* s_a = s_bm + 3 * CP * CH;
    float* s_b = s_a + 3 * AB;
    float* s_gf = s_b + 3 * AB;
    const int cx0 = x0 - H, cy0 = y0 - H;
    const float s = p.bm3d_strength;
    // 1) BM3D parity form (bm3d_step1_generator.cpp:42-56) per 2x2 block of the extent
    for (int item = threadIdx.x; item < (CW / 2) * (CH / 2); item += blockDim.x) {
        const int by2 = item / (CW / 2), bx2 = item - by2 * (CW / 2);
        const int u = cx0 + 2 * bx2, v = cy0 + 2 * by2;  // unclamped block origin
        const int l = (2 * by2) * CP + 2 * bx2;
        if (u >= 0 && u + 1 < in.w && v >= 0 && v + 1 < in.h) {
            Rgba q[4];
            load_pair<T>(in, u, v, &q[0], &q[1]);
            load_pair<T>(in, u, v + 1, &q[2], &q[3]);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int o = l + (k >> 1) * CP + (k & 1);
                s_bm[o] = rnd<F16>(bm3d_blend(q[k].r, q[0].r, q[1].r, q[2].r, q[3].r, s));
                s_bm[CP * CH + o] = rnd<F16>(bm3d_blend(q[k].g, q[0].g, q[1].g, q[2].g, q[3].g, s));
                s_bm[2 * CP * CH + o] = rnd<F16>(bm3d_blend(q[k].b, q[0].b, q[1].b, q[2].b, q[3].b, s));
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int xc = clampi(u + (k & 1), 0, in.w - 1), yc = clampi(v + (k >> 1), 0, in.h - 1);
                const int bx = xc & ~1, by = yc & ~1;
                const int bx1 = min(bx + 1, in.w - 1), by1 = min(by + 1, in.h - 1);
                const Rgba q0 = load_rgba(px<const T>(in, bx, by)), q1 = load_rgba(px<const T>(in, bx1, by));
                const Rgba q2 = load_rgba(px<const T>(in, bx, by1)), q3 = load_rgba(px<const T>(in, bx1, by1));
                const Rgba c = load_rgba(px<const T>(in, xc, yc));
                const int o = l + (k >> 1) * CP + (k & 1);
                s_bm[o] = rnd<F16>(bm3d_blend(c.r, q0.r, q1.r, q2.r, q3.r, s));
                s_bm[CP * CH + o] = rnd<F16>(bm3d_blend(c.g, q0.g, q1.g, q2.g, q3.g, s));
                s_bm[2 * CP * CH + o] = rnd<F16>(bm3d_blend(c.b, q0.b, q1.b, q2.b, q3.b, s));
            }
        }
    }
    __syncthreads();
    constexpr float N = (float)(D * D);
    const ConstDiv cN{N, (float)(1.0 / (double)(D * D))};  // IEEE x / N (const_div)
    if (R == 0) {  // no guided node: the wavelet reads the BM3D output
        for (int i = threadIdx.x; i < 3 * kCTW * kCTH; i += blockDim.x) {
            const int c = i / (kCTW * kCTH);
            const int j = i - c * kCTW * kCTH;
            const int ty = j / kCTW, tx = j - ty * kCTW;
            s_gf[i] = s_bm[c * CP * CH + ty * CP + tx];
        }
    } else {
        // 2) guided a, b (guided_filter_generator.cpp:60-76) at unclamped
        //    coordinates [x0-R, x0+TW+R), kCG rows per thread
        constexpr int AG = (AH + kCG - 1) / kCG;
        for (int item = threadIdx.x; item < 3 * AW * AG; item += blockDim.x) {
            const int c = item / (AW * AG);
            const int rem = item - c * AW * AG;
            const int g = rem / AW, tx = rem - g * AW;
            const int ty0 = g * kCG;
            const float* V = s_bm + c * CP * CH + ty0 * CP + tx;  // window origin of output (ty0, tx)
            float2 win[kCG + 2 * R][D];  // (value, value^2)
#pragma unroll
            for (int r = 0; r < kCG + 2 * R; ++r)
#pragma unroll
                for (int dx = 0; dx < D; ++dx) {
                    const float t = (ty0 + r < CH) ? V[r * CP + dx] : 0.0F;
                    win[r][dx] = make_float2(t, t * t);
                }
#pragma unroll
            for (int k = 0; k < kCG; ++k) {
                if (ty0 + k >= AH) break;
                const float2 sums = box_chain2<D>(win, k);
                const float m = const_div(sums.x, cN), corr = const_div(sums.y, cN);
                const float var = max0(corr - (m * m));
                const float a = var / (var + p.eps);
                const int j = c * AB + (ty0 + k) * AP + tx;
                s_a[j] = a;
                s_b[j] = m - (a * m);
            }
        }
        __syncthreads();
        // 3) guided output for the tile: mean(a) * v + mean(b)
        constexpr int TG = kCTH / kCG;
        for (int item = threadIdx.x; item < 3 * kCTW * TG; item += blockDim.x) {
            const int c = item / (kCTW * TG);
            const int rem = item - c * kCTW * TG;
            const int g = rem / kCTW, tx = rem - g * kCTW;
            const int ty0 = g * kCG;
            float2 win[kCG + 2 * R][D];  // (a, b)
            const float* A = s_a + c * AB + ty0 * AP + tx;
            const float* B = s_b + c * AB + ty0 * AP + tx;
#pragma unroll
            for (int r = 0; r < kCG + 2 * R; ++r)
#pragma unroll
                for (int dx = 0; dx < D; ++dx) win[r][dx] = make_float2(A[r * AP + dx], B[r * AP + dx]);
#pragma unroll
            for (int k = 0; k < kCG; ++k) {
                const int ty = ty0 + k;
                const float2 sab = box_chain2<D>(win, k);
                const float v = s_bm[c * CP * CH + (ty + H) * CP + (tx + H)];
                s_gf[c * kCTW * kCTH + ty * kCTW + tx] = rnd<F16>(max0((const_div(sab.x, cN) * v) + const_div(sab.y, cN)));
            }
        }
    }
    __syncthreads();
    // 4) wavelet on the aligned 2x2 block, filmic, LUT; one thread per pixel
    for (int j = threadIdx.x; j < kCTW * kCTH; j += blockDim.x) {
        const int ty = j / kCTW, tx = j - ty * kCTW;
        const int x = x0 + tx, y = y0 + ty;
        if (x >= out.w || y >= out.h) continue;
        const int bx = x & ~1, by = y & ~1;
        const int xs0 = bx - x0, xs1 = min(bx + 1, out.w - 1) - x0;
        const int ys0 = by - y0, ys1 = min(by + 1, out.h - 1) - y0;
        Rgba q[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int l = ((k >> 1) ? ys1 : ys0) * kCTW + ((k & 1) ? xs1 : xs0);
            q[k] = Rgba{s_gf[l], s_gf[kCTW * kCTH + l], s_gf[2 * kCTW * kCTH + l], 0.0F};
        }
        // alpha runs through unchanged except the wavelet's max(0, .)
        const int ox = x & 1, oy = y & 1;
        const Rgba own = oy ? (ox ? q[3] : q[2]) : (ox ? q[1] : q[0]);
        Rgba v{own.r, own.g, own.b, load_rgba(px<const T>(in, x, y)).a};
        if (p.has_wavelet) {
            v = wavelet_px(q, v, ox, oy, p.wavelet_th);
            v = Rgba{rnd<F16>(v.r), rnd<F16>(v.g), rnd<F16>(v.b), rnd<F16>(v.a)};
        }
        if (p.tone_op == 0) v = filmic_px(v, p.filmic);
        else if (p.tone_op == 1) v = Rgba{aces_fit(v.r), aces_fit(v.g), aces_fit(v.b), v.a};
        else v = Rgba{reinhard_px(v.r, p.reinhard_wp2), reinhard_px(v.g, p.reinhard_wp2), reinhard_px(v.b, p.reinhard_wp2), v.a};
        if (p.has_lut) {
            v = Rgba{rnd<F16>(v.r), rnd<F16>(v.g), rnd<F16>(v.b), v.a};
            v = lut_px(v, p.lut, p.lut_size, p.lut_interp);
        }
        store_rgba(px<T>(out, x, y), v);
    }
}

template <class T, bool F16, int R>
__global__ void __launch_bounds__(256, 3) denoise_tone_kernel(Img in, Img out, ToneParams p) {
    extern __shared__ __align__(16) float smem_f[];
    denoise_tone_tile<T, F16, R>(in, out, p, (int)blockIdx.x * kCTW, (int)blockIdx.y * kCTH, smem_f);
}

template <class T, bool F16, int R>
size_t denoise_tone_smem() {
    return ToneGeom<R>::bytes();
}

}  // namespace
}  // namespace cpb

using namespace cpb;

namespace cpb {
struct SpotOrigins {
    int x[16], y[16];
};
struct SpotStats {
    unsigned frames, fallbacks;
    float worst_mse;
};
namespace spot {
// tiles of src at the origins -> dense [n][edge][edge][4]
template <class T>
__global__ void gather_kernel(Img src, T* __restrict__ dst, int edge, SpotOrigins o) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, t = blockIdx.z;
    if (x >= edge) return;
    const T* s = px<const T>(src, o.x[t] + x, o.y[t] + y);
    T* d = dst + (((size_t)t * edge + y) * edge + x) * 4;
    store_rgba(d, load_rgba(s));
}
// Mean squared RGB difference between the frame (at the origins) and the
// reference tiles, in two steps: mse_kernel sums kMseRows rows of one tile per
// CTA into part[tile][chunk]; decide_kernel adds a tile's chunks in a fixed
// order (so the decision does not depend on scheduling) and tests the worst tile.
constexpr int kMseRows = 8;
constexpr int kMseChunks = 256 / kMseRows;  // chunks per tile at the largest edge (256)
template <class T>
__global__ void mse_kernel(Img den, const T* __restrict__ ref, int edge, SpotOrigins o, float* __restrict__ part) {
    const int t = blockIdx.y, chunk = blockIdx.x;
    __shared__ float warps[8];
    float acc = 0.0F;
    const int y1 = min(edge, (chunk + 1) * kMseRows);
    for (int y = chunk * kMseRows + (int)(threadIdx.x >> 5); y < y1; y += (int)(blockDim.x >> 5))
        for (int x = (int)(threadIdx.x & 31); x < edge; x += 32) {
            const Rgba a = load_rgba(px<const T>(den, o.x[t] + x, o.y[t] + y));
            const Rgba b = load_rgba(ref + (((size_t)t * edge + y) * edge + x) * 4);
            const float dr = a.r - b.r, dg = a.g - b.g, db = a.b - b.b;
            acc += (dr * dr + dg * dg) + db * db;
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFU, acc, off);
    if ((threadIdx.x & 31) == 0) warps[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0F;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += warps[k];
        part[t * kMseChunks + chunk] = s;
    }
}
__global__ void decide_kernel(const float* __restrict__ part, int n, int edge, float mse_max, int* gate,
                              SpotStats* stats) {
    const int chunks = (edge + kMseRows - 1) / kMseRows;
    float worst = 0.0F;
    for (int t = 0; t < n; ++t) {
        float s = 0.0F;
        for (int k = 0; k < chunks; ++k) s += part[t * kMseChunks + k];
        worst = fmaxf(worst, s / (3.0F * (float)(edge * edge)));
    }
    const int fall = !(worst <= mse_max);  // a non-finite tile error also falls back
    *gate = fall;
    stats->frames += 1U;
    stats->fallbacks += (unsigned)fall;
    stats->worst_mse = fmaxf(stats->worst_mse, worst);
}
}  // namespace spot
}  // namespace cpb

struct cpipe_cuda_chain {
    cpipe_cuda_chain_config cfg{};
    bool f16 = true;
    int algo = 1;
    RawParams raw{};
    ColorParams color{};
    ToneParams tone{};
    WarpDev warp{};
    int warp_mode = 0;  // 0 none, 1 fused single warp, 2 general OpcodeList3 list
    // single warp with one coefficient set: its per-pixel bicubic taps (WarpTaps)
    uint32_t* d_taps_ixy = nullptr;
    float* d_taps_tx = nullptr;
    float* d_taps_ty = nullptr;
    std::vector<unsigned char> opcode3_blob;
    Opcode3View opcode3{};
    int radius = 2;
    void* d_tables = nullptr;   // gain tables + LUT cells
    void* d_mid[2] = {nullptr, nullptr};  // K1 output, K2 output (scratch frames)
    int denoise_mode = 0;
    int stop_after = 0;
    void* d_bayer = nullptr;              // remosaiced Bayer frame (Quad-Bayer input)
    Bm3dPlan bm3d{};
    void* d_denoise = nullptr;            // scratch of the mode-1 denoiser
    SurrogateNet* sg = nullptr;           // mode-2 network
    bool owns_sg = true, owns_denoise = true;  // false: a batch's shared network / BM3D scratch
    float* d_ab = nullptr;                // its noise model (a, b) on the device
    // mode-2 spot check
    int spot_tiles = 0, spot_edge = 0;
    float spot_mse_max = 0.0F;
    SpotOrigins spot{};
    Bm3dPlan tile_plan{};
    void* d_tile_in = nullptr;            // [tiles][edge][edge] RGBA, the denoiser's input
    void* d_tile_ref = nullptr;           // BM3D of the tiles
    void* d_tile_scratch = nullptr;
    float* d_tile_mse = nullptr;          // per-tile partial sums of squared differences
    int* d_gate = nullptr;                // 1: fall back to BM3D for this frame
    // finishing stages after denoise_tone: sharpen.edge_aware_usm, display encode
    bool sharpen = false;
    unsigned display = 0;  // 0 none, 1 sRGB, 2 BT2020-PQ
    // spec-mode stages between the denoiser and denoise_tone (0: none)
    bool spec_stages = false;
    bool guided_spec = false;
    AtrousPlan atrous{};
    void* d_atrous = nullptr;
    void* d_gspec = nullptr;  // spec guided filter's planes
    SpotStats* d_stats = nullptr;
    // The tiles' BM3D runs on a second stream beside the network (both read
    // only the denoiser's input), forked after K2 and joined before the MSE.
    cudaStream_t spot_stream = nullptr;
    cudaEvent_t spot_fork = nullptr, spot_join = nullptr;
    void* d_io[2] = {nullptr, nullptr};   // device staging for run_host
    size_t frame_bytes = 0;
    // profiling: 5 events per frame (start, after K1, after K2, after the denoiser, after K3)
    bool profiling = false;
    std::vector<cudaEvent_t> events;
    size_t profiled = 0;
    // captured graphs, one per (input, output, stream) triple seen, least recently used replaced
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        const void* in = nullptr;
        void* out = nullptr;
        cudaStream_t stream = nullptr;
        unsigned long long used = 0;
    };
    static constexpr int kGraphSlots = 8;
    GraphSlot graphs[kGraphSlots];
    unsigned long long graph_clock = 0;
    // run_host_frames: two device frames each way, copy streams and their events
    void* d_pipe_in[2] = {nullptr, nullptr};
    void* d_pipe_out[2] = {nullptr, nullptr};
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
};

namespace {

constexpr int kProfileEvents = 5;

cudaEvent_t* profile_slot(cpipe_cuda_chain* c) {
    if (!c->profiling) return nullptr;
    const size_t need = (c->profiled + 1) * kProfileEvents;
    while (c->events.size() < need) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->events.push_back(e);
    }
    return &c->events[c->profiled++ * kProfileEvents];
}

// The denoiser between K2 and K3 (denoise_mode 1: two-stage BM3D; 2: the
// network with its spot check: the tiles' BM3D forked onto the side stream,
// joined before the MSE, and the full-frame BM3D gated on the device).
int denoise_stage(cpipe_cuda_chain* c, const Img& k2_out, const Img& dn_out, cudaStream_t st) {
    const int w = c->cfg.width, h = c->cfg.height;
    const bool spot = c->denoise_mode == 2 && c->spot_tiles > 0;
    cudaError_t e = cudaSuccess;
    if (spot) {  // fork: gather + the tiles' BM3D on the side stream
        const int E = c->spot_edge, n = c->spot_tiles;
        const Img tin{c->d_tile_in, E, E * n, (long long)E * 4, 4};
        const Img tref{c->d_tile_ref, E, E * n, (long long)E * 4, 4};
        const dim3 gg((unsigned)((E + 127) / 128), (unsigned)E, (unsigned)n);
        cudaStream_t ss = c->spot_stream;
        e = cudaEventRecord(c->spot_fork, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ss, c->spot_fork, 0);
        if (e != cudaSuccess) return cuda_status(e, "chain spot fork");
        if (c->f16) spot::gather_kernel<__half><<<gg, 128, 0, ss>>>(k2_out, static_cast<__half*>(c->d_tile_in), E, c->spot);
        else spot::gather_kernel<float><<<gg, 128, 0, ss>>>(k2_out, static_cast<float*>(c->d_tile_in), E, c->spot);
        e = bm3d_run(c->tile_plan, tin, tref, c->f16, c->d_tile_scratch, ss, false);
        // the join is recorded even after a launch error, so the side stream never stays forked
        const cudaError_t ej = cudaEventRecord(c->spot_join, ss);
        if (e == cudaSuccess) e = ej;
    }
    if (e == cudaSuccess)
        e = c->denoise_mode == 1 ? bm3d_run(c->bm3d, k2_out, dn_out, c->f16, c->d_denoise, st, false)
                                 : surrogate_infer(c->sg, k2_out.data, dn_out.data, 1, h, w, c->f16, c->d_ab, st);
    if (spot) {
        const cudaError_t ew = cudaStreamWaitEvent(st, c->spot_join, 0);
        if (e == cudaSuccess) e = ew;
    }
    if (e == cudaSuccess && spot) {
        const int E = c->spot_edge, n = c->spot_tiles;
        const dim3 gm((unsigned)((E + spot::kMseRows - 1) / spot::kMseRows), (unsigned)n);
        if (c->f16) spot::mse_kernel<__half><<<gm, 256, 0, st>>>(dn_out, static_cast<const __half*>(c->d_tile_ref), E, c->spot, c->d_tile_mse);
        else spot::mse_kernel<float><<<gm, 256, 0, st>>>(dn_out, static_cast<const float*>(c->d_tile_ref), E, c->spot, c->d_tile_mse);
        spot::decide_kernel<<<1, 1, 0, st>>>(c->d_tile_mse, n, E, c->spot_mse_max, c->d_gate, c->d_stats);
        e = bm3d_run(c->bm3d, k2_out, dn_out, c->f16, c->d_denoise, st, false, c->d_gate);
    }
    return e == cudaSuccess ? CPIPE_OK : cuda_status(e, "chain denoise");
}

int launch_chain(cpipe_cuda_chain* c, const void* d_raw, size_t raw_pitch, void* d_out, size_t out_pitch,
                 cudaStream_t st) {
    cudaEvent_t* ev = profile_slot(c);
    if (ev) cudaEventRecord(ev[0], st);
    const int w = c->cfg.width, h = c->cfg.height;
    const int elem = c->f16 ? 2 : 4;
    Img raw{const_cast<void*>(d_raw), w, h, (long long)(raw_pitch ? raw_pitch / 2 : (size_t)w), 1};
    if (c->d_bayer) {  // demosaic.quad_bayer_remosaic (u16 -> u16) ahead of the Bayer chain
        const Img bayer{c->d_bayer, w, h, (long long)w, 1};
        const cudaError_t e = launch_qbc_remosaic(raw, bayer, st);
        if (e != cudaSuccess) return cuda_status(e, "chain remosaic");
        raw = bayer;
    }
    const Img mid0{c->d_mid[0], w, h, (long long)w * 4, 4};
    const Img mid1{c->d_mid[1], w, h, (long long)w * 4, 4};
    const int out_elem = c->display == 1 ? 1 : (c->display == 2 ? 2 : elem);
    const Img out{d_out, w, h, (long long)(out_pitch ? out_pitch / out_elem : (size_t)w * 4), 4};
    const dim3 ga((unsigned)((w + kDmTW - 1) / kDmTW), (unsigned)((h + kDmTH - 1) / kDmTH));
#define K1(A)                                                                                        \
    if (c->f16) raw_to_rgba_kernel<A, __half><<<ga, 256, 0, st>>>(raw, mid0, c->raw);                \
    else raw_to_rgba_kernel<A, float><<<ga, 256, 0, st>>>(raw, mid0, c->raw);
    if (c->algo == 0) { K1(0) } else if (c->algo == 1) { K1(1) } else { K1(2) }
#undef K1
    if (ev) cudaEventRecord(ev[1], st);
    Img k2_in = mid0;
    if (c->warp_mode == 2) {
        // General OpcodeList3 list through the per-node path (its scratch is stream-ordered).
        Call call;
        call.stream = st;
        int s = cpb_opcode3_run(call, c->opcode3, mid0, mid1, elem);
        if (s != CPIPE_OK) return s;
        s = call.finish(CPIPE_OK);
        if (s != CPIPE_OK) return s;
        k2_in = mid1;
    }
    const dim3 gb((unsigned)((w + 127) / 128), (unsigned)h);
    Img k2_out = c->stop_after == 1 ? out : (c->warp_mode == 2) ? mid0 : mid1;
    const WarpTaps taps{c->d_taps_ixy, c->d_taps_tx, c->d_taps_ty};
    if (c->warp_mode == 1 && c->d_taps_ixy) {
        if (c->f16) warp_wb_cm_kernel<__half, true, 2><<<gb, 128, 0, st>>>(k2_in, k2_out, c->warp, c->color, taps);
        else warp_wb_cm_kernel<float, false, 2><<<gb, 128, 0, st>>>(k2_in, k2_out, c->warp, c->color, taps);
    } else if (c->warp_mode == 1) {
        if (c->f16) warp_wb_cm_kernel<__half, true, 1><<<gb, 128, 0, st>>>(k2_in, k2_out, c->warp, c->color, taps);
        else warp_wb_cm_kernel<float, false, 1><<<gb, 128, 0, st>>>(k2_in, k2_out, c->warp, c->color, taps);
    } else {
        if (c->f16) warp_wb_cm_kernel<__half, true, 0><<<gb, 128, 0, st>>>(k2_in, k2_out, c->warp, c->color, taps);
        else warp_wb_cm_kernel<float, false, 0><<<gb, 128, 0, st>>>(k2_in, k2_out, c->warp, c->color, taps);
    }
    if (ev) cudaEventRecord(ev[2], st);
    if (c->stop_after == 1) {
        if (ev) cudaEventRecord(ev[3], st);
        if (ev) cudaEventRecord(ev[4], st);
        return cuda_status(cudaGetLastError(), "chain launch");
    }
    if (c->denoise_mode != 0) {
        const Img dn_out = c->stop_after == 2 ? out : (k2_out.data == mid1.data) ? mid0 : mid1;
        const int ds = denoise_stage(c, k2_out, dn_out, st);
        if (ds != CPIPE_OK) return ds;
        k2_out = dn_out;
    }
    if (c->stop_after == 2) {
        if (ev) cudaEventRecord(ev[3], st);
        if (ev) cudaEventRecord(ev[4], st);
        return cuda_status(cudaGetLastError(), "chain launch");
    }
    if (c->spec_stages) {
        // bm3d (mode 0: the reference's 2x2 blend, here as its own kernel) ->
        // guided -> wavelet, ping-ponging between the two scratch frames; the
        // tone kernel then runs filmic and the LUT (its blend at strength 0 is
        // the identity on these non-negative values)
        auto other = [&](const Img& cur) { return cur.data == mid0.data ? mid1 : mid0; };
        Img x = k2_out;
        cudaError_t e = cudaSuccess;
        if (c->denoise_mode == 0) {
            const Img y = other(x);
            e = launch_bm3d_parity(x, y, c->f16, c->cfg.bm3d_sigma, st);
            x = y;
        }
        if (e == cudaSuccess && c->cfg.guided_radius > 0) {
            const Img y = other(x);
            e = c->guided_spec ? guided_spec_run(x, y, c->f16, c->cfg.guided_radius, c->cfg.guided_eps, c->d_gspec, st)
                               : launch_guided(x, y, c->f16, c->cfg.guided_radius, c->cfg.guided_eps, st);
            x = y;
        }
        if (e == cudaSuccess && c->atrous.levels > 0) {
            const Img y = other(x);
            e = atrous_run(c->atrous, x, y, c->f16, c->d_atrous, st);
            x = y;
        }
        if (e != cudaSuccess) return cuda_status(e, "chain spec stages");
        k2_out = x;
    }
    if (ev) cudaEventRecord(ev[3], st);
    // with finishing stages the tone kernel writes a scratch frame they read
    const bool finish = c->sharpen || c->display != 0;
    const Img k3_out = !finish ? out : (k2_out.data == mid0.data ? mid1 : mid0);
    const dim3 gc((unsigned)((w + kCTW - 1) / kCTW), (unsigned)((h + kCTH - 1) / kCTH));
#define K3(TT, F, R)                                                                                       \
    denoise_tone_kernel<TT, F, R><<<gc, 256, denoise_tone_smem<TT, F, R>(), st>>>(k2_out, k3_out, c->tone);
    if (c->f16) {
        if (c->radius == 0) { K3(__half, true, 0) } else if (c->radius == 1) { K3(__half, true, 1) } else { K3(__half, true, 2) }
    } else {
        if (c->radius == 0) { K3(float, false, 0) } else if (c->radius == 1) { K3(float, false, 1) } else { K3(float, false, 2) }
    }
#undef K3
    if (finish) {
        const cpipe_cuda_chain_config& f = c->cfg;
        cudaError_t e;
        if (c->sharpen && c->display)
            e = launch_usm_display(k3_out, out, f.sharpen_strength, f.sharpen_radius, f.sharpen_threshold,
                                   c->display - 1, st);
        else if (c->sharpen)
            e = launch_usm(k3_out, out, true, f.sharpen_strength, f.sharpen_radius, f.sharpen_threshold, st);
        else
            e = launch_display(k3_out, out, c->display - 1, st);
        if (e != cudaSuccess) return cuda_status(e, "chain finishing stages");
    }
    if (ev) cudaEventRecord(ev[4], st);
    return cuda_status(cudaGetLastError(), "chain launch");
}

template <class T, bool F, int R>
cudaError_t allow_smem() {
    cudaError_t e = cudaFuncSetAttribute(denoise_tone_kernel<T, F, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)denoise_tone_smem<T, F, R>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(denoise_tone_kernel<T, F, R>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    return e;
}

}  // namespace

extern "C" {

// A batch's denoiser resources shared by its frames' chains (frames are
// denoised one after another on one stream): the network, reserved for the
// largest frame, and the full-frame BM3D scratch of the largest plan.
struct ChainShared {
    SurrogateNet* sg = nullptr;
    void* d_denoise = nullptr;
};
static cpipe_cuda_chain* chain_create(const cpipe_cuda_chain_config* cfg, int* status, const ChainShared* shared);

cpipe_cuda_chain* cpipe_cuda_chain_create(const cpipe_cuda_chain_config* cfg, int* status) {
    return chain_create(cfg, status, nullptr);
}

static cpipe_cuda_chain* chain_create(const cpipe_cuda_chain_config* cfg, int* status, const ChainShared* shared) {
    auto fail = [&](int st, cpipe_cuda_chain* c) -> cpipe_cuda_chain* {
        if (status) *status = st;
        if (c) cpipe_cuda_chain_destroy(c);
        return nullptr;
    };
    if (!cfg || cfg->width <= 0 || cfg->height <= 0) return fail(CPIPE_BAD_INDEX, nullptr);
    if (!device_ready()) return fail(CPIPE_INTERNAL_ERROR, nullptr);
    auto* c = new (std::nothrow) cpipe_cuda_chain();
    if (!c) return fail(CPIPE_OOM, nullptr);
    c->cfg = *cfg;
    c->f16 = cfg->plain_f32 == 0;
    c->algo = cfg->demosaic < 0 || cfg->demosaic > 2 ? 1 : cfg->demosaic;
    const int w = cfg->width, h = cfg->height;
    // raw stage
    int st = cpb_blacklevel_dev(&cfg->black, w, h, &c->raw.black);
    if (st != CPIPE_OK) return fail(st, c);
    for (int i = 0; i < 4; ++i) c->raw.cfa.p[i] = cfg->black.cfa_pattern[i];
    std::vector<char> table;
    size_t offsets[3][4] = {};
    if (cfg->gainmap_blob && cfg->gainmap_blob_size) {
        st = cpb_gainmap_prepare(cfg->gainmap_blob, cfg->gainmap_blob_size, w, h, &table, &c->raw.gain, offsets);
        if (st != CPIPE_OK) return fail(st, c);
        c->raw.has_gain = 1;
    }
    // LUT cells after the gain tables
    std::vector<float4> cells;
    size_t lut_off = (table.size() + 15) & ~size_t(15);
    if (cfg->lut_blob && cfg->lut_blob_size) {
        st = cpb_lut_prepare(cfg->lut_blob, cfg->lut_blob_size, &cells, &c->tone.lut_size, &c->tone.lut_interp);
        if (st != CPIPE_OK) return fail(st, c);
        c->tone.has_lut = 1;
    }
    // per-grid-row gain table after the LUT, filled on the device below
    const size_t hrows_off = (lut_off + cells.size() * sizeof(float4) + 15) & ~size_t(15);
    const size_t total = hrows_off + (c->raw.has_gain ? gainmap_hrows_bytes(c->raw.gain, w) : 0);
    if (total) {
        if (cudaMalloc(&c->d_tables, total) != cudaSuccess) return fail(CPIPE_OOM, c);
        std::vector<char> host(total, 0);
        if (!table.empty()) std::memcpy(host.data(), table.data(), table.size());
        if (!cells.empty()) std::memcpy(host.data() + lut_off, cells.data(), cells.size() * sizeof(float4));
        if (cudaMemcpy(c->d_tables, host.data(), total, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(CPIPE_INTERNAL_ERROR, c);
        if (c->raw.has_gain) {
            cpb_gainmap_bind(&c->raw.gain, static_cast<const char*>(c->d_tables), offsets);
            if (launch_gainmap_hrows(&c->raw.gain, static_cast<char*>(c->d_tables) + hrows_off, w, nullptr) !=
                    cudaSuccess ||
                cudaStreamSynchronize(nullptr) != cudaSuccess)
                return fail(CPIPE_INTERNAL_ERROR, c);
        }
        if (c->tone.has_lut) c->tone.lut = reinterpret_cast<const float4*>(static_cast<char*>(c->d_tables) + lut_off);
    }
    // OpcodeList3
    if (cfg->opcode3_blob && cfg->opcode3_blob_size) {
        c->opcode3_blob.assign(static_cast<const unsigned char*>(cfg->opcode3_blob),
                               static_cast<const unsigned char*>(cfg->opcode3_blob) + cfg->opcode3_blob_size);
        st = cpb_opcode3_parse(c->opcode3_blob.data(), c->opcode3_blob.size(), &c->opcode3);
        if (st != CPIPE_OK) return fail(st, c);
        int applied = 0, warps = 0;
        const cpipe_Opcode3DispatchRecord* warp_rec = nullptr;
        for (uint32_t i = 0; i < c->opcode3.count; ++i) {
            const auto& r = c->opcode3.records[i];
            if (r.id == CPIPE_OPCODE3_UNKNOWN) {
                if (!r.optional) return fail(CPIPE_UNSUPPORTED, c);
                continue;
            }
            ++applied;
            if (r.id == CPIPE_OPCODE3_WARP_RECTILINEAR) {
                ++warps;
                warp_rec = &r;
            }
        }
        if (applied == 1 && warps == 1) c->warp_mode = cpb_warp_dev(warp_rec, w, h, &c->warp) == CPIPE_OK ? 1 : 0;
        else if (applied > 0) c->warp_mode = 2;
        // the frame geometry is fixed per chain: a single warp's taps are
        // computed once here and read by K2 (12 bytes per pixel)
        if (c->warp_mode == 1 && c->warp.count == 1 && w <= 65535 && h <= 65535) {
            const size_t n = (size_t)w * h;
            if (cudaMalloc(&c->d_taps_ixy, n * sizeof(uint32_t)) != cudaSuccess ||
                cudaMalloc(&c->d_taps_tx, n * sizeof(float)) != cudaSuccess ||
                cudaMalloc(&c->d_taps_ty, n * sizeof(float)) != cudaSuccess)
                return fail(CPIPE_OOM, c);
            const dim3 g((unsigned)((w + 255) / 256), (unsigned)h);
            warp_taps_kernel<<<g, 256>>>(w, h, c->warp, c->d_taps_ixy, c->d_taps_tx, c->d_taps_ty);
            if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(nullptr) != cudaSuccess)
                return fail(CPIPE_INTERNAL_ERROR, c);
        }
    }
    // colour, denoise, tone
    std::memcpy(c->color.neutral, cfg->as_shot_neutral, sizeof(c->color.neutral));
    std::memcpy(c->color.cm, cfg->colormatrix, sizeof(c->color.cm));
    c->denoise_mode = cfg->denoise_mode;
    c->stop_after = cfg->stop_after;
    if (cfg->quad_bayer && cudaMalloc(&c->d_bayer, (size_t)w * h * sizeof(uint16_t)) != cudaSuccess)
        return fail(CPIPE_OOM, c);
    if (c->denoise_mode < 0 || c->denoise_mode > 2) return fail(CPIPE_UNSUPPORTED, c);
    if (c->stop_after < 0 || c->stop_after > 2 || (c->stop_after == 2 && c->denoise_mode == 0))
        return fail(CPIPE_UNSUPPORTED, c);
    if (c->denoise_mode == 2) {
        if (shared) {
            c->sg = shared->sg;
            c->owns_sg = false;
        } else {
            c->sg = surrogate_new(cfg->surrogate_blob, cfg->surrogate_blob_size, &st);
        }
        if (!c->sg) return fail(st, c);
        const float ab[2] = {cfg->noise_a, cfg->noise_b};
        if (cudaMalloc(&c->d_ab, sizeof(ab)) != cudaSuccess) return fail(CPIPE_OOM, c);
        if (cudaMemcpy(c->d_ab, ab, sizeof(ab), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(CPIPE_INTERNAL_ERROR, c);
        if (!shared && surrogate_reserve(c->sg, (long long)w * h) != cudaSuccess) return fail(CPIPE_OOM, c);
        c->spot_tiles = cfg->spot_tiles < 0 ? 0 : (cfg->spot_tiles > 16 ? 16 : cfg->spot_tiles);
        if (c->spot_tiles > 0) {
            // stratified tiles: the centres of a 4x4 grid of cells, clamped inside the frame
            const int E = std::min(256, std::min(w, h));
            c->spot_edge = E;
            c->spot_mse_max = (float)std::pow(10.0, -(double)cfg->spot_min_psnr_db / 10.0);
            for (int t = 0; t < c->spot_tiles; ++t) {
                const int i = t % 4, j = t / 4;
                c->spot.x[t] = std::min(std::max((2 * i + 1) * w / 8 - E / 2, 0), w - E);
                c->spot.y[t] = std::min(std::max((2 * j + 1) * h / 8 - E / 2, 0), h - E);
            }
            cpipe_Bm3dSpecParams sp = cfg->bm3d_spec;
            if (!(sp.sigma > 0.0F)) sp.sigma = cfg->bm3d_sigma;
            if ((st = bm3d_plan(&sp, w, h, &c->bm3d)) != CPIPE_OK) return fail(st, c);
            // the check screens the network's output against BM3D with single FP16
            // transform products (2^-11 relative each, far below the decision
            // margin); the fallback keeps the configured form
            cpipe_Bm3dSpecParams spot_sp = sp;
            if (spot_sp.transform == 0) spot_sp.transform = 2;
            if ((st = bm3d_plan(&spot_sp, E, E, &c->tile_plan, c->spot_tiles)) != CPIPE_OK) return fail(st, c);
            const size_t tile_bytes = (size_t)E * E * c->spot_tiles * 4 * (c->f16 ? 2 : 4);
            if (cudaMalloc(&c->d_tile_in, tile_bytes) != cudaSuccess || cudaMalloc(&c->d_tile_ref, tile_bytes) != cudaSuccess ||
                (!c->tile_plan.copy && cudaMalloc(&c->d_tile_scratch, c->tile_plan.bytes) != cudaSuccess) ||
                (!c->bm3d.copy && !shared && cudaMalloc(&c->d_denoise, c->bm3d.bytes) != cudaSuccess) ||
                cudaMalloc(&c->d_tile_mse, sizeof(float) * 16 * spot::kMseChunks) != cudaSuccess ||
                cudaMalloc(&c->d_gate, sizeof(int)) != cudaSuccess || cudaMalloc(&c->d_stats, sizeof(SpotStats)) != cudaSuccess)
                return fail(CPIPE_OOM, c);
            if (cudaMemset(c->d_stats, 0, sizeof(SpotStats)) != cudaSuccess || cudaMemset(c->d_gate, 0, sizeof(int)) != cudaSuccess)
                return fail(CPIPE_INTERNAL_ERROR, c);
            // the check runs at the device's highest stream priority, so its small
            // launches take free SM slots ahead of the network's next layer
            int prio_low = 0, prio_high = 0;
            if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess ||
                cudaStreamCreateWithPriority(&c->spot_stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->spot_fork, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->spot_join, cudaEventDisableTiming) != cudaSuccess)
                return fail(CPIPE_INTERNAL_ERROR, c);
            if (cudaError_t e = bm3d_setup(c->bm3d); e != cudaSuccess) return fail(cuda_status(e, "bm3d setup"), c);
            if (cudaError_t e = bm3d_setup(c->tile_plan); e != cudaSuccess) return fail(cuda_status(e, "bm3d setup"), c);
        }
    }
    c->tone.bm3d_strength = c->denoise_mode == 0 ? fminf(1.0F, fmaxf(0.0F, cfg->bm3d_sigma / 0.03F)) : 0.0F;
    if (c->denoise_mode == 1) {
        cpipe_Bm3dSpecParams sp = cfg->bm3d_spec;
        if (!(sp.sigma > 0.0F)) sp.sigma = cfg->bm3d_sigma;
        if ((st = bm3d_plan(&sp, w, h, &c->bm3d)) != CPIPE_OK) return fail(st, c);
        if (!c->bm3d.copy && !shared && cudaMalloc(&c->d_denoise, c->bm3d.bytes) != cudaSuccess) return fail(CPIPE_OOM, c);
        if (cudaError_t e = bm3d_setup(c->bm3d); e != cudaSuccess) return fail(cuda_status(e, "bm3d setup"), c);
    }
    if (shared) {
        c->d_denoise = shared->d_denoise;
        c->owns_denoise = false;
    }
    // guided_radius 0 leaves the guided node out; otherwise the reference box
    // is 3x3 for radius <= 1 and 5x5 above (guided_filter_generator.cpp:66-70).
    c->radius = cfg->guided_radius <= 0 ? 0 : (cfg->guided_radius == 1 ? 1 : 2);
    c->tone.has_wavelet = cfg->wavelet_strength >= 0.0F;
    // spec-mode guided / a-trous: run as their own stages ahead of the tone kernel
    if (cfg->guided_spec && (cfg->guided_radius < 1 || cfg->guided_radius > kGuidedSpecMaxRadius))
        return fail(CPIPE_BAD_INDEX, c);
    if (cfg->atrous_levels < 0 || cfg->atrous_levels > kAtrousMaxLevels) return fail(CPIPE_BAD_INDEX, c);
    c->guided_spec = cfg->guided_spec != 0;
    c->spec_stages = c->guided_spec || cfg->atrous_levels > 0;
    if (c->spec_stages) {
        if (c->guided_spec && guided_spec_setup() != cudaSuccess) return fail(CPIPE_INTERNAL_ERROR, c);
        if (c->guided_spec &&
            cudaMalloc(&c->d_gspec, guided_spec_scratch_bytes(w, h, cfg->guided_radius)) != cudaSuccess)
            return fail(CPIPE_OOM, c);
        if (cfg->atrous_levels > 0) {
            const cpipe_AtrousWaveletParams ap{cfg->atrous_levels, cfg->bm3d_sigma, cfg->atrous_luma_strength,
                                               cfg->wavelet_strength >= 0.0F ? cfg->wavelet_strength : 1.0F};
            if ((st = atrous_plan(&ap, w, h, &c->atrous)) != CPIPE_OK) return fail(st, c);
            if (cudaMalloc(&c->d_atrous, c->atrous.bytes) != cudaSuccess) return fail(CPIPE_OOM, c);
            if (atrous_setup() != cudaSuccess) return fail(CPIPE_INTERNAL_ERROR, c);
            c->tone.has_wavelet = 0;
        }
        if (c->denoise_mode == 0) c->tone.bm3d_strength = 0.0F;
        c->radius = 0;
    }
    c->tone.eps = cfg->guided_eps;
    c->tone.wavelet_th = 0.035F * cfg->wavelet_strength;
    c->tone.filmic = cpb_filmic_dev(&cfg->filmic);
    // tone stage: filmic (default), or tone.aces_filmic / tone.reinhard with the
    // reference nodes' parameter handling (Reinhard: unset -> 1e6, else 0.1..10)
    if (cfg->tone < 0 || cfg->tone > 2) return fail(CPIPE_BAD_INDEX, c);
    c->tone.tone_op = cfg->tone;
    {
        const float wp = cfg->reinhard_white_point < 0.0F ? 1000000.0F
                                                           : std::clamp(cfg->reinhard_white_point, 0.1F, 10.0F);
        c->tone.reinhard_wp2 = wp * wp;
    }
    // scratch frames
    c->frame_bytes = (size_t)w * h * 4 * (c->f16 ? 2 : 4);
    // finishing stages (sharpen.edge_aware_usm, display encode): f16 form, whole chain
    if (cfg->sharpen || cfg->display) {
        if (cfg->display < 0 || cfg->display > 2 || cfg->stop_after != 0) return fail(CPIPE_BAD_INDEX, c);
        if (!c->f16) return fail(CPIPE_BAD_PRECISION, c);
        c->sharpen = cfg->sharpen != 0;
        c->display = (unsigned)cfg->display;
        // the node's parameter clamps (edge_aware_usm.cpp:38-41)
        c->cfg.sharpen_strength = std::clamp(cfg->sharpen_strength, 0.0F, 2.0F);
        c->cfg.sharpen_radius = std::clamp(cfg->sharpen_radius, 1, 32);
        c->cfg.sharpen_threshold = std::clamp(cfg->sharpen_threshold, 0.0F, 0.1F);
        if (c->display) c->frame_bytes = (size_t)w * h * 4 * (c->display == 1 ? 1 : 2);
    }
    const size_t mid_bytes = (size_t)w * h * 4 * (c->f16 ? 2 : 4);  // RGBA working frames
    for (void*& p : c->d_mid)
        if (cudaMalloc(&p, mid_bytes) != cudaSuccess) return fail(CPIPE_OOM, c);
    cudaError_t e = cudaSuccess;
    if (c->f16) e = c->radius == 0 ? allow_smem<__half, true, 0>() : c->radius == 1 ? allow_smem<__half, true, 1>() : allow_smem<__half, true, 2>();
    else e = c->radius == 0 ? allow_smem<float, false, 0>() : c->radius == 1 ? allow_smem<float, false, 1>() : allow_smem<float, false, 2>();
    if (e != cudaSuccess) return fail(cuda_status(e, "chain smem"), c);
    if (status) *status = CPIPE_OK;
    return c;
}

void cpipe_cuda_chain_destroy(cpipe_cuda_chain* c) {
    if (!c) return;
    for (cudaEvent_t e : c->events) cudaEventDestroy(e);
    for (auto& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (void* p : c->d_pipe_in) cudaFree(p);
    for (void* p : c->d_pipe_out) cudaFree(p);
    for (int k = 0; k < 2; ++k)
        for (cudaEvent_t e : {c->ev_in[k], c->ev_done[k], c->ev_out[k]})
            if (e) cudaEventDestroy(e);
    if (c->s_h2d) cudaStreamDestroy(c->s_h2d);
    if (c->s_d2h) cudaStreamDestroy(c->s_d2h);
    cudaFree(c->d_tables);
    cudaFree(c->d_gspec);
    cudaFree(c->d_taps_ixy);
    cudaFree(c->d_taps_tx);
    cudaFree(c->d_taps_ty);
    if (c->owns_denoise) cudaFree(c->d_denoise);
    cudaFree(c->d_bayer);
    cudaFree(c->d_ab);
    cudaFree(c->d_tile_in);
    cudaFree(c->d_tile_ref);
    cudaFree(c->d_tile_scratch);
    cudaFree(c->d_tile_mse);
    cudaFree(c->d_gate);
    cudaFree(c->d_stats);
    cudaFree(c->d_atrous);
    if (c->spot_fork) cudaEventDestroy(c->spot_fork);
    if (c->spot_join) cudaEventDestroy(c->spot_join);
    if (c->spot_stream) cudaStreamDestroy(c->spot_stream);
    if (c->owns_sg) surrogate_free(c->sg);
    for (void* p : c->d_mid) cudaFree(p);
    for (void* p : c->d_io) cudaFree(p);
    delete c;
}

size_t cpipe_cuda_chain_output_bytes(const cpipe_cuda_chain* c) { return c ? c->frame_bytes : 0; }

int cpipe_cuda_chain_run(cpipe_cuda_chain* c, const void* d_raw, void* d_out, void* stream) {
    if (!c || !d_raw || !d_out) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (c->cfg.use_graph && c->warp_mode != 2 && !c->profiling) {
        using Slot = cpipe_cuda_chain::GraphSlot;
        Slot* hit = nullptr;
        Slot* lru = &c->graphs[0];
        for (Slot& g : c->graphs) {
            if (g.exec && g.in == d_raw && g.out == d_out && g.stream == st) hit = &g;
            if (!g.exec || (lru->exec && g.used < lru->used)) lru = &g;
        }
        if (!hit) {
            hit = lru;
            if (hit->exec) cudaGraphExecDestroy(hit->exec);
            hit->exec = nullptr;
            cudaGraph_t g;
            cudaStream_t cap = st;
            cudaStream_t own = nullptr;
            if (cap == nullptr) {  // the legacy stream cannot be captured
                if (cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
                cap = own;
            }
            int s = cuda_status(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
            if (s == CPIPE_OK) {
                const int ls = launch_chain(c, d_raw, 0, d_out, 0, cap);
                s = cuda_status(cudaStreamEndCapture(cap, &g), "end capture");
                if (ls != CPIPE_OK) s = ls;
            }
            if (s == CPIPE_OK) {
                s = cuda_status(cudaGraphInstantiate(&hit->exec, g, cudaGraphInstantiateFlagUseNodePriority), "instantiate");
                cudaGraphDestroy(g);
            }
            if (own) cudaStreamDestroy(own);
            if (s != CPIPE_OK) return s;
            hit->in = d_raw;
            hit->out = d_out;
            hit->stream = st;
        }
        hit->used = ++c->graph_clock;
        return cuda_status(cudaGraphLaunch(hit->exec, st), "graph launch");
    }
    return launch_chain(c, d_raw, 0, d_out, 0, st);
}

int cpipe_cuda_chain_run_host(cpipe_cuda_chain* c, const uint16_t* h_raw, void* h_out, void* stream) {
    if (!c || !h_raw || !h_out) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t raw_bytes = (size_t)c->cfg.width * c->cfg.height * sizeof(uint16_t);
    if (!c->d_io[0] && cudaMalloc(&c->d_io[0], raw_bytes) != cudaSuccess) return CPIPE_OOM;
    if (!c->d_io[1] && cudaMalloc(&c->d_io[1], c->frame_bytes) != cudaSuccess) return CPIPE_OOM;
    int s = cuda_status(cudaMemcpyAsync(c->d_io[0], h_raw, raw_bytes, cudaMemcpyHostToDevice, st), "chain H2D");
    if (s == CPIPE_OK) s = cpipe_cuda_chain_run(c, c->d_io[0], c->d_io[1], stream);
    if (s == CPIPE_OK)
        s = cuda_status(cudaMemcpyAsync(h_out, c->d_io[1], c->frame_bytes, cudaMemcpyDeviceToHost, st), "chain D2H");
    const int ss = cuda_status(cudaStreamSynchronize(st), "chain sync");
    return s != CPIPE_OK ? s : ss;
}

int cpipe_cuda_chain_run_host_frames(cpipe_cuda_chain* c, const uint16_t* const* h_raws, void* const* h_outs, int n,
                                     void* stream) {
    if (!c || !h_raws || !h_outs || n < 0) return CPIPE_BAD_INDEX;
    for (int i = 0; i < n; ++i)
        if (!h_raws[i] || !h_outs[i]) return CPIPE_BAD_INDEX;
    if (n == 0) return CPIPE_OK;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t raw_bytes = (size_t)c->cfg.width * c->cfg.height * sizeof(uint16_t);
    for (int k = 0; k < 2; ++k) {
        if (!c->d_pipe_in[k] && cudaMalloc(&c->d_pipe_in[k], raw_bytes) != cudaSuccess) return CPIPE_OOM;
        if (!c->d_pipe_out[k] && cudaMalloc(&c->d_pipe_out[k], c->frame_bytes) != cudaSuccess) return CPIPE_OOM;
        for (cudaEvent_t* e : {&c->ev_in[k], &c->ev_done[k], &c->ev_out[k]})
            if (!*e && cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    }
    if (!c->s_h2d && cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    if (!c->s_d2h && cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    // Frame i uses device frames k = i & 1: its upload waits until frame i - 2's
    // chain has read input k, its chain until the upload is in and frame i - 2's
    // download has emptied output k; the download follows the chain.
    int s = CPIPE_OK;
    for (int i = 0; i < n && s == CPIPE_OK; ++i) {
        const int k = i & 1;
        if (i >= 2) s = cuda_status(cudaStreamWaitEvent(c->s_h2d, c->ev_done[k], 0), "pipe wait");
        if (s == CPIPE_OK)
            s = cuda_status(cudaMemcpyAsync(c->d_pipe_in[k], h_raws[i], raw_bytes, cudaMemcpyHostToDevice, c->s_h2d),
                            "pipe H2D");
        if (s == CPIPE_OK) s = cuda_status(cudaEventRecord(c->ev_in[k], c->s_h2d), "pipe record");
        if (s == CPIPE_OK) s = cuda_status(cudaStreamWaitEvent(st, c->ev_in[k], 0), "pipe wait");
        if (s == CPIPE_OK && i >= 2) s = cuda_status(cudaStreamWaitEvent(st, c->ev_out[k], 0), "pipe wait");
        if (s == CPIPE_OK) s = cpipe_cuda_chain_run(c, c->d_pipe_in[k], c->d_pipe_out[k], stream);
        if (s == CPIPE_OK) s = cuda_status(cudaEventRecord(c->ev_done[k], st), "pipe record");
        if (s == CPIPE_OK) s = cuda_status(cudaStreamWaitEvent(c->s_d2h, c->ev_done[k], 0), "pipe wait");
        if (s == CPIPE_OK)
            s = cuda_status(cudaMemcpyAsync(h_outs[i], c->d_pipe_out[k], c->frame_bytes, cudaMemcpyDeviceToHost, c->s_d2h),
                            "pipe D2H");
        if (s == CPIPE_OK) s = cuda_status(cudaEventRecord(c->ev_out[k], c->s_d2h), "pipe record");
    }
    // every queued copy and chain finishes before the call returns, also after an error
    const int s1 = cuda_status(cudaStreamSynchronize(c->s_h2d), "pipe sync");
    const int s2 = cuda_status(cudaStreamSynchronize(st), "pipe sync");
    const int s3 = cuda_status(cudaStreamSynchronize(c->s_d2h), "pipe sync");
    return s != CPIPE_OK ? s : s1 != CPIPE_OK ? s1 : s2 != CPIPE_OK ? s2 : s3;
}

int cpipe_cuda_chain_set_profiling(cpipe_cuda_chain* c, int enable) {
    if (!c) return CPIPE_BAD_INDEX;
    c->profiling = enable != 0;
    c->profiled = 0;
    return CPIPE_OK;
}

int cpipe_cuda_chain_profile(cpipe_cuda_chain* c, double ms_per_stage[4], int* frames) {
    if (!c || !ms_per_stage || !frames) return CPIPE_BAD_INDEX;
    for (int k = 0; k < kProfileEvents - 1; ++k) ms_per_stage[k] = 0.0;
    for (size_t f = 0; f < c->profiled; ++f) {
        cudaEvent_t* ev = &c->events[f * kProfileEvents];
        const int st = cuda_status(cudaEventSynchronize(ev[kProfileEvents - 1]), "profile sync");
        if (st != CPIPE_OK) return st;
        for (int k = 0; k < kProfileEvents - 1; ++k) {
            float ms = 0.0F;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            ms_per_stage[k] += ms;
        }
    }
    *frames = (int)c->profiled;
    c->profiled = 0;
    return CPIPE_OK;
}

int cpipe_cuda_chain_denoise_stats(cpipe_cuda_chain* c, uint32_t* frames, uint32_t* fallbacks, float* worst_tile_psnr_db) {
    if (!c || !frames || !fallbacks || !worst_tile_psnr_db) return CPIPE_BAD_INDEX;
    SpotStats h{};
    if (c->d_stats) {
        const int st = cuda_status(cudaDeviceSynchronize(), "stats sync");
        if (st != CPIPE_OK) return st;
        if (cudaMemcpy(&h, c->d_stats, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    }
    *frames = h.frames;
    *fallbacks = h.fallbacks;
    *worst_tile_psnr_db = h.frames == 0 ? 0.0F : (h.worst_mse > 0.0F ? (float)(-10.0 * std::log10((double)h.worst_mse)) : INFINITY);
    return CPIPE_OK;
}

int cpipe_cuda_stream_create(void** out) {
    if (!out) return CPIPE_BAD_INDEX;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    *out = s;
    return CPIPE_OK;
}
void cpipe_cuda_stream_destroy(void* s) { cudaStreamDestroy(static_cast<cudaStream_t>(s)); }
int cpipe_cuda_stream_synchronize(void* s) {
    return cuda_status(cudaStreamSynchronize(static_cast<cudaStream_t>(s)), "stream sync");
}
int cpipe_cuda_event_create(void** out) {
    if (!out) return CPIPE_BAD_INDEX;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    *out = e;
    return CPIPE_OK;
}
void cpipe_cuda_event_destroy(void* e) { cudaEventDestroy(static_cast<cudaEvent_t>(e)); }
int cpipe_cuda_event_record(void* e, void* stream) {
    return cuda_status(cudaEventRecord(static_cast<cudaEvent_t>(e), static_cast<cudaStream_t>(stream)), "event record");
}
int cpipe_cuda_event_elapsed_ms(void* start, void* stop, float* ms) {
    if (!ms) return CPIPE_BAD_INDEX;
    int st = cuda_status(cudaEventSynchronize(static_cast<cudaEvent_t>(stop)), "event sync");
    if (st == CPIPE_OK)
        st = cuda_status(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(stop)), "elapsed");
    return st;
}
int cpipe_cuda_device_alloc(size_t bytes, void** out) {
    if (!out) return CPIPE_BAD_INDEX;
    if (cudaMalloc(out, bytes) != cudaSuccess) {
        cudaGetLastError();
        return CPIPE_OOM;
    }
    return CPIPE_OK;
}
void cpipe_cuda_device_free(void* p) { cudaFree(p); }
int cpipe_cuda_memcpy_h2d(void* dst, const void* src, size_t bytes) {
    return cuda_status(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "h2d");
}
int cpipe_cuda_memcpy_d2h(void* dst, const void* src, size_t bytes) {
    return cuda_status(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "d2h");
}
}  // extern "C"

namespace cpb {
namespace util {
__global__ void count_nonfinite_kernel(const void* d, size_t n, int f16, unsigned long long* out) {
    unsigned long long c = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = f16 ? __half2float(static_cast<const __half*>(d)[i]) : static_cast<const float*>(d)[i];
        c += isfinite(v) ? 0ULL : 1ULL;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xFFFFFFFFU, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}
}  // namespace util
}  // namespace cpb

extern "C" {

int cpipe_cuda_count_nonfinite(const void* d, size_t count, int f16, uint64_t* out, void* stream) {
    if (!d || !out) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long* dc = nullptr;
    int s = cuda_status(cudaMallocAsync(&dc, sizeof(*dc), st), "count alloc");
    if (s != CPIPE_OK) return s;
    unsigned long long h = 0;
    cudaMemsetAsync(dc, 0, sizeof(*dc), st);
    cpb::util::count_nonfinite_kernel<<<kSmCount * 4, 256, 0, st>>>(d, count, f16, dc);
    s = cuda_status(cudaMemcpyAsync(&h, dc, sizeof(h), cudaMemcpyDeviceToHost, st), "count copy");
    cudaFreeAsync(dc, st);
    const int ss = cuda_status(cudaStreamSynchronize(st), "count sync");
    *out = h;
    return s != CPIPE_OK ? s : ss;
}

int cpipe_cuda_memcpy_d2d_async(void* dst, const void* src, size_t bytes, void* stream) {
    return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)),
                       "d2d");
}
int cpipe_cuda_set_device(int device) { return cuda_status(cudaSetDevice(device), "set device"); }

int cpipe_cuda_pinned_alloc(size_t bytes, void** out) {
    if (!out) return CPIPE_BAD_INDEX;
    return cudaHostAlloc(out, bytes, cudaHostAllocDefault) == cudaSuccess ? CPIPE_OK : CPIPE_OOM;
}
void cpipe_cuda_pinned_free(void* p) { cudaFreeHost(p); }

}  // extern "C"

// ------------------------------------------------------------- batched form
// Frames of any size, CFA and bit depth through the same chain in one launch
// per stage: persistent kernels walk a queue of (frame, tile) work items.
// Tile t belongs to the frame f with prefix[f] <= t < prefix[f + 1] (binary
// search over the per-frame tile counts); the frame's descriptor (buffers and
// node parameters) is copied to shared memory when a CTA moves to a new frame.
// Per frame, the host-side preparation is that of a single-frame chain
// (cpipe_cuda_chain_create), whose intermediate frames the batch uses.
namespace cpb {
namespace batch {

constexpr int kMaxFrames = 64;
constexpr int kK2Rows = 8;  // stage-2 work item: 128 pixels x 8 rows

struct Frame {
    Img bayer, mid0, mid1, out;  // bayer: the raw input, or its remosaic for Quad-Bayer frames
    Img tone_in;                 // mid1, or the denoiser's output (mid0) when a denoiser runs between
    RawParams raw;
    WarpDev warp;
    WarpTaps taps;      // the frame chain's per-pixel warp taps (null when it evaluates the warp per pixel)
    ColorParams color;
    ToneParams tone;
    int t1x, t2x, t3x;  // work items per row, per stage
    int rows2;          // rows per stage-2 work item (autotuned)
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// First node of a batch run: the start time and each frame's count of
// stage-3 items still to finish.
__global__ void batch_clock_kernel(const int* __restrict__ prefix3, int n, int* __restrict__ left,
                                   unsigned long long* __restrict__ t0) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) left[i] = prefix3[i + 1] - prefix3[i];
    if (threadIdx.x == 0) *t0 = global_ns();
}

__device__ __forceinline__ int find_frame(const int* prefix, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Work item t of this stage: returns its frame's local index, having loaded
// the frame descriptor into s_f when the frame changed (uniform per CTA).
__device__ __forceinline__ int next_item(const Frame* __restrict__ frames, const int* s_prefix, int n, int t,
                                         Frame* s_f, int* cur) {
    const int f = find_frame(s_prefix, n, t);
    if (f != *cur) {
        __syncthreads();
        const int* src = reinterpret_cast<const int*>(frames + f);
        int* dst = reinterpret_cast<int*>(s_f);
        for (int i = threadIdx.x; i < (int)(sizeof(Frame) / 4); i += blockDim.x) dst[i] = src[i];
        *cur = f;
        __syncthreads();
    }
    return t - s_prefix[f];
}

template <int ALGO>
__global__ void __launch_bounds__(256) batch_raw_kernel(const Frame* __restrict__ frames,
                                                        const int* __restrict__ prefix, int n) {
    __shared__ int s_prefix[kMaxFrames + 1];
    __shared__ Frame s_f;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) s_prefix[i] = prefix[i];
    __syncthreads();
    int cur = -1;
    for (int t = blockIdx.x; t < s_prefix[n]; t += gridDim.x) {
        const int local = next_item(frames, s_prefix, n, t, &s_f, &cur);
        demosaic_tile_at<ALGO, __half>(RawLoader{s_f.bayer, &s_f.raw}, s_f.bayer.w, s_f.bayer.h, s_f.mid0, s_f.raw.cfa,
                                       (local % s_f.t1x) * kDmTW, (local / s_f.t1x) * kDmTH);
        __syncthreads();
    }
}

template <bool WARP>
__global__ void __launch_bounds__(128) batch_color_kernel(const Frame* __restrict__ frames,
                                                          const int* __restrict__ prefix, int n) {
    __shared__ int s_prefix[kMaxFrames + 1];
    __shared__ Frame s_f;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) s_prefix[i] = prefix[i];
    __syncthreads();
    int cur = -1;
    for (int t = blockIdx.x; t < s_prefix[n]; t += gridDim.x) {
        const int local = next_item(frames, s_prefix, n, t, &s_f, &cur);
        const int rows = s_f.rows2;
        const int x = (local % s_f.t2x) * 128 + (int)threadIdx.x, y0 = (local / s_f.t2x) * rows;
        if (x < s_f.mid1.w) {
            if (WARP && s_f.taps.ixy != nullptr) {  // the tap table, as the frame's own chain reads it
                for (int r = 0; r < rows && y0 + r < s_f.mid1.h; ++r)
                    warp_wb_cm_px<__half, true, 2>(s_f.mid0, s_f.mid1, s_f.warp, s_f.color, x, y0 + r, s_f.taps);
            } else {
                for (int r = 0; r < rows && y0 + r < s_f.mid1.h; ++r)
                    warp_wb_cm_px<__half, true, WARP>(s_f.mid0, s_f.mid1, s_f.warp, s_f.color, x, y0 + r);
            }
        }
    }
}

template <int R>
__global__ void __launch_bounds__(256, 3) batch_tone_kernel(const Frame* __restrict__ frames,
                                                            const int* __restrict__ prefix, int n,
                                                            int* __restrict__ left,
                                                            unsigned long long* __restrict__ done) {
    extern __shared__ __align__(16) float smem_f[];
    __shared__ int s_prefix[kMaxFrames + 1];
    __shared__ Frame s_f;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) s_prefix[i] = prefix[i];
    __syncthreads();
    int cur = -1;
    for (int t = blockIdx.x; t < s_prefix[n]; t += gridDim.x) {
        const int local = next_item(frames, s_prefix, n, t, &s_f, &cur);
        denoise_tone_tile<__half, true, R>(s_f.tone_in, s_f.out, s_f.tone, (local % s_f.t3x) * kCTW,
                                           (local / s_f.t3x) * kCTH, smem_f);
        __syncthreads();
        // the frame's completion time: stamped by the CTA that finishes its last item
        if (threadIdx.x == 0 && left != nullptr) {
            __threadfence();
            if (atomicSub(left + cur, 1) == 1) done[cur] = global_ns();
        }
    }
}

}  // namespace batch
}  // namespace cpb

struct cpipe_cuda_batch {
    std::vector<cpipe_cuda_chain*> chains;
    std::vector<cpb::batch::Frame> frames;
    cpb::batch::Frame* d_frames = nullptr;
    int* d_prefix = nullptr;  // three arrays of n + 1
    int n = 0, algo = 1, radius = 2;
    bool warp = false;
    int per_sm[3] = {2, 8, 3};  // persistent CTAs per SM for the three stages (autotuned)
    int rows2 = cpb::batch::kK2Rows;  // rows per stage-2 work item (autotuned)
    int denoise_mode = 0;             // 0: the reference's 2x2 blend in K3; 1 / 2: BM3D / the network between K2 and K3
    std::vector<int> prefix;          // three arrays of n + 1 (host copy)
    SurrogateNet* shared_sg = nullptr;  // denoiser resources shared by the frames' chains
    void* shared_denoise = nullptr;
    int* d_left = nullptr;            // per frame: stage-3 items not finished yet
    unsigned long long* d_times = nullptr;  // [0]: start; [1 + i]: frame i's completion (globaltimer ns)
    cudaGraphExec_t graph = nullptr;
    std::vector<const void*> graph_in;
    std::vector<void*> graph_out;
    cudaStream_t graph_stream = nullptr;
};

namespace {

using cpb::batch::Frame;

int batch_launch_stage(cpipe_cuda_batch* b, int stage, cudaStream_t st, bool timed = false) {
    // per_sm 0: one work item per CTA (the queue's limit case: a grid of all items)
    const int items = b->prefix[(size_t)stage * (b->n + 1) + b->n];
    const int grid = b->per_sm[stage] > 0 ? kSmCount * b->per_sm[stage] : (items > 0 ? items : 1);
    const int* pf = b->d_prefix + stage * (b->n + 1);
    if (stage == 0) {
        if (b->algo == 0) cpb::batch::batch_raw_kernel<0><<<grid, 256, 0, st>>>(b->d_frames, pf, b->n);
        else if (b->algo == 1) cpb::batch::batch_raw_kernel<1><<<grid, 256, 0, st>>>(b->d_frames, pf, b->n);
        else cpb::batch::batch_raw_kernel<2><<<grid, 256, 0, st>>>(b->d_frames, pf, b->n);
    } else if (stage == 1) {
        if (b->warp) cpb::batch::batch_color_kernel<true><<<grid, 128, 0, st>>>(b->d_frames, pf, b->n);
        else cpb::batch::batch_color_kernel<false><<<grid, 128, 0, st>>>(b->d_frames, pf, b->n);
    } else {
        // completion stamps only in a full run (the autotuner times stages alone)
        int* left = timed ? b->d_left : nullptr;
        unsigned long long* done = b->d_times + 1;
        if (b->radius == 0)
            cpb::batch::batch_tone_kernel<0><<<grid, 256, denoise_tone_smem<__half, true, 0>(), st>>>(b->d_frames, pf, b->n, left, done);
        else if (b->radius == 1)
            cpb::batch::batch_tone_kernel<1><<<grid, 256, denoise_tone_smem<__half, true, 1>(), st>>>(b->d_frames, pf, b->n, left, done);
        else
            cpb::batch::batch_tone_kernel<2><<<grid, 256, denoise_tone_smem<__half, true, 2>(), st>>>(b->d_frames, pf, b->n, left, done);
    }
    return cuda_status(cudaGetLastError(), "batch stage");
}

int batch_launch(cpipe_cuda_batch* b, cudaStream_t st) {
    for (int i = 0; i < b->n; ++i) {  // demosaic.quad_bayer_remosaic for Quad-Bayer frames
        cpipe_cuda_chain* c = b->chains[i];
        if (c->d_bayer) {
            const cudaError_t e = launch_qbc_remosaic(Img{const_cast<void*>(b->graph_in[i]), c->cfg.width, c->cfg.height,
                                                          (long long)c->cfg.width, 1},
                                                      b->frames[i].bayer, st);
            if (e != cudaSuccess) return cuda_status(e, "batch remosaic");
        }
    }
    cpb::batch::batch_clock_kernel<<<1, 64, 0, st>>>(b->d_prefix + 2 * (b->n + 1), b->n, b->d_left, b->d_times);
    for (int stage = 0; stage < 3; ++stage) {
        const int s = batch_launch_stage(b, stage, st, true);
        if (s != CPIPE_OK) return s;
        if (stage == 1 && b->denoise_mode != 0) {
            // the denoiser of every frame between its K2 and K3 (its chain's
            // network, spot check and gated BM3D, or its BM3D)
            for (int i = 0; i < b->n; ++i) {
                const int ds = denoise_stage(b->chains[i], b->frames[i].mid1, b->frames[i].mid0, st);
                if (ds != CPIPE_OK) return ds;
            }
        }
    }
    return CPIPE_OK;
}

// Stage prefixes for the current stage-2 rows per item; copied to the device.
int batch_prefix(cpipe_cuda_batch* b) {
    const int n = b->n;
    b->prefix.assign(3 * (n + 1), 0);
    for (int i = 0; i < n; ++i) {
        cpb::batch::Frame& f = b->frames[i];
        const int h = f.mid0.h;
        f.rows2 = b->rows2;
        b->prefix[0 * (n + 1) + i + 1] = b->prefix[0 * (n + 1) + i] + f.t1x * ((h + kDmTH - 1) / kDmTH);
        b->prefix[1 * (n + 1) + i + 1] = b->prefix[1 * (n + 1) + i] + f.t2x * ((h + b->rows2 - 1) / b->rows2);
        b->prefix[2 * (n + 1) + i + 1] = b->prefix[2 * (n + 1) + i] + f.t3x * ((h + kCTH - 1) / kCTH);
    }
    return cuda_status(cudaMemcpy(b->d_prefix, b->prefix.data(), sizeof(int) * b->prefix.size(), cudaMemcpyHostToDevice),
                       "batch prefix");
}

template <int R>
cudaError_t allow_batch_smem() {
    cudaError_t e = cudaFuncSetAttribute(cpb::batch::batch_tone_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)denoise_tone_smem<__half, true, R>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(cpb::batch::batch_tone_kernel<R>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    return e;
}

}  // namespace

extern "C" {

void cpipe_cuda_batch_destroy(cpipe_cuda_batch* b) {
    if (!b) return;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (cpipe_cuda_chain* c : b->chains) cpipe_cuda_chain_destroy(c);
    surrogate_free(b->shared_sg);
    cudaFree(b->shared_denoise);
    cudaFree(b->d_frames);
    cudaFree(b->d_prefix);
    cudaFree(b->d_left);
    cudaFree(b->d_times);
    delete b;
}

cpipe_cuda_batch* cpipe_cuda_batch_create(const cpipe_cuda_chain_config* cfgs, size_t n, int* status) {
    auto fail = [&](int st, cpipe_cuda_batch* b) -> cpipe_cuda_batch* {
        if (status) *status = st;
        cpipe_cuda_batch_destroy(b);
        return nullptr;
    };
    if (!cfgs || n == 0 || n > (size_t)cpb::batch::kMaxFrames) return fail(CPIPE_BAD_INDEX, nullptr);
    auto* b = new (std::nothrow) cpipe_cuda_batch();
    if (!b) return fail(CPIPE_OOM, nullptr);
    b->n = (int)n;
    b->denoise_mode = cfgs[0].denoise_mode;
    ChainShared shared{};
    if (b->denoise_mode == 1 || b->denoise_mode == 2) {
        // one network reserved for the largest frame and one BM3D scratch of
        // the largest plan serve every frame (they are denoised in turn)
        long long max_px = 0;
        size_t max_bytes = 0;
        for (size_t i = 0; i < n; ++i) {
            const cpipe_cuda_chain_config& c = cfgs[i];
            if (c.denoise_mode == 2 && (c.surrogate_blob_size != cfgs[0].surrogate_blob_size ||
                                        (c.surrogate_blob != cfgs[0].surrogate_blob &&
                                         std::memcmp(c.surrogate_blob, cfgs[0].surrogate_blob, c.surrogate_blob_size)))) {
                set_error("batch: %s", "every frame needs the same network weights");
                return fail(CPIPE_UNSUPPORTED, b);
            }
            max_px = std::max(max_px, (long long)c.width * c.height);
            cpipe_Bm3dSpecParams sp = c.bm3d_spec;
            if (!(sp.sigma > 0.0F)) sp.sigma = c.bm3d_sigma;
            Bm3dPlan q;
            if (bm3d_plan(&sp, c.width, c.height, &q) == CPIPE_OK && !q.copy) max_bytes = std::max(max_bytes, q.bytes);
        }
        if (b->denoise_mode == 2) {
            int st = CPIPE_OK;
            b->shared_sg = surrogate_new(cfgs[0].surrogate_blob, cfgs[0].surrogate_blob_size, &st);
            if (!b->shared_sg) return fail(st, b);
            if (surrogate_reserve(b->shared_sg, max_px) != cudaSuccess) return fail(CPIPE_OOM, b);
        }
        if (max_bytes && cudaMalloc(&b->shared_denoise, max_bytes) != cudaSuccess) return fail(CPIPE_OOM, b);
        shared.sg = b->shared_sg;
        shared.d_denoise = b->shared_denoise;
    }
    for (size_t i = 0; i < n; ++i) {
        cpipe_cuda_chain_config c = cfgs[i];
        if (c.plain_f32 || c.denoise_mode != b->denoise_mode || c.stop_after != 0 || c.guided_spec || c.atrous_levels ||
            c.sharpen || c.display) {
            set_error("batch: %s", "frames run the binary16 chain with one denoiser for all (the reference's "
                                   "denoise.bm3d, two-stage BM3D or the network)");
            return fail(CPIPE_UNSUPPORTED, b);
        }
        c.use_graph = 0;
        int st = CPIPE_OK;
        cpipe_cuda_chain* ch = chain_create(&c, &st, b->denoise_mode != 0 ? &shared : nullptr);
        if (!ch) return fail(st, b);
        b->chains.push_back(ch);
        if (i == 0) {
            b->algo = ch->algo;
            b->radius = ch->radius;
            b->warp = ch->warp_mode == 1;
        }
        if (ch->algo != b->algo || ch->radius != b->radius || (ch->warp_mode == 1) != b->warp || ch->warp_mode == 2) {
            set_error("batch: %s", "all frames need the same demosaic, guided radius class and warp form");
            return fail(CPIPE_UNSUPPORTED, b);
        }
        const int w = c.width, h = c.height;
        Frame f{};
        f.mid0 = Img{ch->d_mid[0], w, h, (long long)w * 4, 4};
        f.mid1 = Img{ch->d_mid[1], w, h, (long long)w * 4, 4};
        f.tone_in = b->denoise_mode != 0 ? f.mid0 : f.mid1;
        f.raw = ch->raw;
        f.warp = ch->warp;
        f.taps = WarpTaps{ch->d_taps_ixy, ch->d_taps_tx, ch->d_taps_ty};
        f.color = ch->color;
        f.tone = ch->tone;
        f.t1x = (w + kDmTW - 1) / kDmTW;
        f.t2x = (w + 127) / 128;
        f.t3x = (w + kCTW - 1) / kCTW;
        b->frames.push_back(f);
    }
    if (cudaMalloc(&b->d_frames, sizeof(Frame) * n) != cudaSuccess ||
        cudaMalloc(&b->d_prefix, sizeof(int) * 3 * (n + 1)) != cudaSuccess ||
        cudaMalloc(&b->d_left, sizeof(int) * n) != cudaSuccess ||
        cudaMalloc(&b->d_times, sizeof(unsigned long long) * (n + 1)) != cudaSuccess)
        return fail(CPIPE_OOM, b);
    if (batch_prefix(b) != CPIPE_OK) return fail(CPIPE_INTERNAL_ERROR, b);
    cudaError_t e = b->radius == 0 ? allow_batch_smem<0>() : b->radius == 1 ? allow_batch_smem<1>() : allow_batch_smem<2>();
    if (e != cudaSuccess) return fail(cuda_status(e, "batch smem"), b);
    if (status) *status = CPIPE_OK;
    return b;
}

static int batch_bind(cpipe_cuda_batch* b, const void* const* d_raw, void* const* d_out) {
    for (int i = 0; i < b->n; ++i) {
        if (!d_raw[i] || !d_out[i]) return CPIPE_BAD_INDEX;
        cpipe_cuda_chain* c = b->chains[i];
        const int w = c->cfg.width, h = c->cfg.height;
        b->frames[i].bayer = c->d_bayer ? Img{c->d_bayer, w, h, (long long)w, 1}
                                        : Img{const_cast<void*>(d_raw[i]), w, h, (long long)w, 1};
        b->frames[i].out = Img{d_out[i], w, h, (long long)w * 4, 4};
    }
    b->graph_in.assign(d_raw, d_raw + b->n);
    b->graph_out.assign(d_out, d_out + b->n);
    return cuda_status(cudaMemcpy(b->d_frames, b->frames.data(), sizeof(Frame) * b->n, cudaMemcpyHostToDevice),
                       "batch descriptors");
}

int cpipe_cuda_batch_run(cpipe_cuda_batch* b, const void* const* d_raw, void* const* d_out, void* stream) {
    if (!b || !d_raw || !d_out) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    bool same = b->graph && b->graph_stream == st;
    for (int i = 0; same && i < b->n; ++i) same = b->graph_in[i] == d_raw[i] && b->graph_out[i] == d_out[i];
    if (!same) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        int s = batch_bind(b, d_raw, d_out);
        if (s != CPIPE_OK) return s;
        cudaStream_t cap = st, own = nullptr;
        if (cap == nullptr) {
            if (cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
            cap = own;
        }
        cudaGraph_t g;
        s = cuda_status(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "batch capture");
        if (s == CPIPE_OK) {
            const int ls = batch_launch(b, cap);
            s = cuda_status(cudaStreamEndCapture(cap, &g), "batch end capture");
            if (ls != CPIPE_OK) s = ls;
        }
        if (s == CPIPE_OK) {
            s = cuda_status(cudaGraphInstantiate(&b->graph, g, 0), "batch instantiate");
            cudaGraphDestroy(g);
        }
        if (own) cudaStreamDestroy(own);
        if (s != CPIPE_OK) return s;
        b->graph_stream = st;
    }
    return cuda_status(cudaGraphLaunch(b->graph, st), "batch graph launch");
}

int cpipe_cuda_batch_autotune(cpipe_cuda_batch* b, const void* const* d_raw, void* const* d_out, void* stream,
                              int per_sm_out[3]) {
    if (!b || !d_raw || !d_out) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int s = batch_bind(b, d_raw, d_out);
    if (s != CPIPE_OK) return s;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    static const int cand[3][7] = {{1, 2, 3, 4, 6, 8, 0}, {2, 4, 8, 12, 16, 24, 0}, {1, 2, 3, 4, 6, 8, 0}};
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    s = batch_launch(b, st);  // fills every stage's input once
    // stage 2 also picks its work-item shape: 128 pixels x rows2 rows
    static const int rows_cand[4] = {4, 8, 16, 32};
    for (int stage = 0; stage < 3 && s == CPIPE_OK; ++stage) {
        float best = 1e30F;
        int best_k = b->per_sm[stage], best_rows = b->rows2;
        for (int ri = 0; ri < (stage == 1 ? 4 : 1) && s == CPIPE_OK; ++ri) {
            if (stage == 1) {
                b->rows2 = rows_cand[ri];
                s = batch_prefix(b);
                if (s == CPIPE_OK)
                    s = cuda_status(cudaMemcpy(b->d_frames, b->frames.data(), sizeof(Frame) * b->n, cudaMemcpyHostToDevice),
                                    "batch descriptors");
            }
            for (int k : cand[stage]) {
                if (s != CPIPE_OK) break;
                b->per_sm[stage] = k;
                float total = 0.0F;
                for (int r = 0; r < 3 && s == CPIPE_OK; ++r) {
                    cudaEventRecord(e0, st);
                    s = batch_launch_stage(b, stage, st);
                    cudaEventRecord(e1, st);
                    if (cudaEventSynchronize(e1) != cudaSuccess) s = CPIPE_INTERNAL_ERROR;
                    float ms = 0.0F;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (r > 0) total += ms;  // the first run warms up
                }
                if (total < best) {
                    best = total;
                    best_k = k;
                    best_rows = b->rows2;
                }
            }
        }
        b->per_sm[stage] = best_k;
        if (stage == 1 && s == CPIPE_OK) {
            b->rows2 = best_rows;
            s = batch_prefix(b);
            if (s == CPIPE_OK)
                s = cuda_status(cudaMemcpy(b->d_frames, b->frames.data(), sizeof(Frame) * b->n, cudaMemcpyHostToDevice),
                                "batch descriptors");
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (per_sm_out)
        for (int i = 0; i < 3; ++i) per_sm_out[i] = b->per_sm[i];
    return s;
}

cpipe_cuda_chain* cpipe_cuda_batch_frame_chain(cpipe_cuda_batch* b, size_t i) {
    return (b && i < b->chains.size()) ? b->chains[i] : nullptr;
}

int cpipe_cuda_batch_schedule(cpipe_cuda_batch* b, int per_sm[3], int* rows_per_item) {
    if (!b) return CPIPE_BAD_INDEX;
    if (per_sm)
        for (int i = 0; i < 3; ++i) per_sm[i] = b->per_sm[i];
    if (rows_per_item) *rows_per_item = b->rows2;
    return CPIPE_OK;
}

int cpipe_cuda_batch_frame_times(cpipe_cuda_batch* b, void* stream, float* ms, size_t n) {
    if (!b || !ms || n < (size_t)b->n) return CPIPE_BAD_INDEX;
    std::vector<unsigned long long> t((size_t)b->n + 1);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int s = cuda_status(cudaMemcpyAsync(t.data(), b->d_times, sizeof(unsigned long long) * t.size(),
                                        cudaMemcpyDeviceToHost, st), "batch times");
    if (s == CPIPE_OK) s = cuda_status(cudaStreamSynchronize(st), "batch times");
    if (s != CPIPE_OK) return s;
    for (int i = 0; i < b->n; ++i) ms[i] = t[i + 1] >= t[0] ? (float)((double)(t[i + 1] - t[0]) * 1e-6) : -1.0F;
    return CPIPE_OK;
}

}  // extern "C"
