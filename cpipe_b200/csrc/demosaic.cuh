// Shared-memory tile demosaic (bilinear / RCD / AMaZE), shared by the per-node
// demosaic filters and the fused chain's first kernel.  The `Loader` functor
// fills a tile cell from the clamped input coordinate: a plain R32F read for
// the node, or unpack + black level + GainMap for the chain.
#pragma once

#include "nodes.cuh"

namespace cpb {

constexpr int kDmTW = 64, kDmTH = 16, kDmHalo = 3, kDmThreads = 256;
constexpr int kDmIW = kDmTW + 2 * kDmHalo, kDmIH = kDmTH + 2 * kDmHalo;
constexpr int kDmGW = kDmTW + 2, kDmGH = kDmTH + 2;

struct DmTap {
    const float* base;
    int pitch;
    __device__ __forceinline__ float operator()(int dx, int dy) const { return base[dy * pitch + dx]; }
};

// Staged halo: RCD / AMaZE read green / chroma at +-1 whose stencils reach
// +-2 (halo 3); bilinear reads +-1 only (halo 1, a smaller tile to load).
template <int ALGO>
struct DmGeom {
    static constexpr int kHalo = ALGO == 0 ? 1 : kDmHalo;
    static constexpr int kIW = kDmTW + 2 * kHalo, kIH = kDmTH + 2 * kHalo;
};

// Tile of kDmTW x kDmTH outputs; shared memory holds the loaded input with a
// halo of 3 (RCD/AMaZE read green/chroma at +-1 whose stencils reach +-2), and
// for the tile plus a halo of 1 the green plane and the per-cell quantity the
// neighbours read: the RCD ratio c / max(g, 1e-6) (demosaic_rcd_generator.cpp:37-40)
// or the AMaZE chroma c - g (demosaic_amaze_generator.cpp:48-49), computed once
// per cell instead of once per reading pixel (same values).
template <int ALGO, class TOut, class Loader>
__device__ __forceinline__ void demosaic_tile_at(const Loader& load, int w, int h, const Img& out, const Cfa& cfa, int x0,
                                                 int y0) {
    constexpr int HL = DmGeom<ALGO>::kHalo, IW = DmGeom<ALGO>::kIW, IH = DmGeom<ALGO>::kIH;
    __shared__ float s_in[IH * IW];
    __shared__ float s_g[ALGO != 0 ? kDmGH * kDmGW : 1];
    __shared__ float s_q[ALGO != 0 ? kDmGH * kDmGW : 1];
    // Every caller launches kDmThreads threads per block; a thread's tile loads
    // are all issued before its first shared-memory store.
    constexpr int kLoads = (IH * IW + kDmThreads - 1) / kDmThreads;
    float v[kLoads];
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + kDmThreads * k;
        const int ty = i / IW, tx = i - ty * IW;
        if (i < IH * IW) v[k] = load(clampi(x0 - HL + tx, 0, w - 1), clampi(y0 - HL + ty, 0, h - 1));
    }
#pragma unroll
    for (int k = 0; k < kLoads; ++k) {
        const int i = threadIdx.x + kDmThreads * k;
        if (i < IH * IW) s_in[i] = v[k];
    }
    __syncthreads();
    if (ALGO != 0) {
        for (int i = threadIdx.x; i < kDmGH * kDmGW; i += blockDim.x) {
            const int ty = i / kDmGW, tx = i - ty * kDmGW;
            const DmTap T{s_in + (ty + HL - 1) * IW + (tx + HL - 1), IW};
            const float g = ALGO == 1 ? rcd_green(T, x0 - 1 + tx, y0 - 1 + ty, cfa)
                                      : amaze_green(T, x0 - 1 + tx, y0 - 1 + ty, cfa);
            s_g[i] = g;
            s_q[i] = ALGO == 1 ? T(0, 0) / maxf(g, 0.000001F) : T(0, 0) - g;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kDmTH * kDmTW; i += blockDim.x) {
        const int ty = i / kDmTW, tx = i - ty * kDmTW;
        const int x = x0 + tx, y = y0 + ty;
        if (x >= out.w || y >= out.h) continue;
        const float* c = s_in + (ty + HL) * IW + (tx + HL);
        const DmTap T{c, IW};
        const float ctr = c[0];
        const int site = cfa.at(x, y);
        const bool red = site == 0, blue = site == 2;
        const bool hred = cfa.at(x - 1, y) == 0, hblue = cfa.at(x - 1, y) == 2;
        float r, g, b;
        if (ALGO == 0) {  // demosaic_bilinear_generator.cpp:23-41
            const float hz = 0.5F * (T(-1, 0) + T(1, 0));
            const float vt = 0.5F * (T(0, -1) + T(0, 1));
            const float cross = 0.25F * (T(-1, 0) + T(1, 0) + T(0, -1) + T(0, 1));
            const float diag = 0.25F * (T(-1, -1) + T(1, -1) + T(-1, 1) + T(1, 1));
            r = red ? ctr : blue ? diag : hred ? hz : vt;
            g = (red || blue) ? cross : ctr;
            b = blue ? ctr : red ? diag : hred ? vt : hz;
        } else {
            const float gc = s_g[(ty + 1) * kDmGW + (tx + 1)];
            const float* Q = s_q + (ty + 1) * kDmGW + (tx + 1);
#define QQ(dx, dy) Q[(dy) * kDmGW + (dx)]
            if (ALGO == 1) {  // demosaic_rcd_generator.cpp:41-63
                const float rh = gc * 0.5F * (QQ(-1, 0) + QQ(1, 0));
                const float rv = gc * 0.5F * (QQ(0, -1) + QQ(0, 1));
                const float rd = gc * 0.25F * (QQ(-1, -1) + QQ(1, -1) + QQ(-1, 1) + QQ(1, 1));
                r = max0(red ? ctr : blue ? rd : hred ? rh : rv);
                g = max0(gc);
                b = max0(blue ? ctr : red ? rd : hblue ? rh : rv);
            } else {  // demosaic_amaze_generator.cpp:50-66
                const float chh = 0.5F * (QQ(-1, 0) + QQ(1, 0));
                const float chv = 0.5F * (QQ(0, -1) + QQ(0, 1));
                const float chd = 0.25F * (QQ(-1, -1) + QQ(1, -1) + QQ(-1, 1) + QQ(1, 1));
                const float rh = gc + chh, rv = gc + chv, rd = gc + chd;
                r = max0(red ? ctr : (blue ? rd : hred ? rh : rv));
                g = max0(gc);
                b = max0(blue ? ctr : (red ? rd : hblue ? rh : rv));
            }
#undef QQ
        }
        store_rgba(px<TOut>(out, x, y), Rgba{r, g, b, 1.0F});
    }
}

// One kDmTW x kDmTH tile at the block's grid position.
template <int ALGO, class TOut, class Loader>
__device__ __forceinline__ void demosaic_tile(const Loader& load, int w, int h, const Img& out, const Cfa& cfa) {
    demosaic_tile_at<ALGO, TOut>(load, w, h, out, cfa, (int)blockIdx.x * kDmTW, (int)blockIdx.y * kDmTH);
}

}  // namespace cpb
