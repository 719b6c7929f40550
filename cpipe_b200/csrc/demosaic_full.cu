// Full-form RCD and AMaZE demosaics (node parameter algorithm = "full";
// aot_ids "demosaic_rcd_full" and "demosaic_amaze_full").
//
// The reference's demosaic.rcd / demosaic.amaze nodes compute reduced 5x5
// stencils (demosaic_rcd_generator.cpp:8-77, demosaic_amaze_generator.cpp:8-79);
// these kernels compute the published algorithms the nodes are named after --
// RCD (L. Sanz Rodriguez, v2.3) and AMaZE (E. Martinec) -- in the stage
// definitions this project fixes for them (listed stage by stage in the
// oracle's header, oracle/oracle_demosaic_full.c).  Every expression below is
// evaluated in binary32 in the oracle's operation order (the library is built
// without contraction), so the results equal the oracle's binary32
// instantiation bit for bit; the FP64 instantiation gives the error figure.
//
// Boundary: the mosaic is read through reflect-101 extension (period 2(n-1),
// the CFA phase is kept), and every intermediate quantity outside the frame is
// evaluated at its own position from that extension, as in the oracle.
//
// RCD: one kernel.  A 32x32 output tile stages the mosaic with a halo of 10 in
// shared memory, then evaluates each stage over the region the next stage
// reads: the squared high-passes (two buffers), the vertical/horizontal and
// diagonal discriminations, the low-pass, green at red/blue sites, the other
// colour at red/blue sites, and the outputs (50 KB of shared memory).
//
// AMaZE: three kernels over an extended domain (the frame plus a margin of 16)
// in scratch planes: (1) colour differences, their vertical weight and the
// Nyquist flag; (2) the Nyquist vote, area weights, green, curvature refinement;
// (3) the other colour at red/blue sites and red/blue at green sites.  Each
// stages its inputs with their halo in shared memory.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>

#include "filters_impl.h"
#include "nodes.cuh"

namespace cpb {
namespace dmf {

__device__ __forceinline__ int refl(int i, int n) {
    if (n <= 1) return 0;
    const int p = 2 * (n - 1);
    i %= p;
    if (i < 0) i += p;
    return i >= n ? p - i : i;
}
__device__ __forceinline__ float absr(float a) { return fabsf(a); }
__device__ __forceinline__ float maxr(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minr(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float intp(float a, float b, float c) { return __fadd_rn(__fmul_rn(a, b), __fmul_rn(__fsub_rn(1.0F, a), c)); }

// A square plane region [o, o + n) x [o, o + n) relative to the tile origin.
struct Plane {
    float* p;
    int o, n;
    __device__ __forceinline__ float& at(int x, int y) const { return p[(y - o) * n + (x - o)]; }
};

// ------------------------------------------------------------------ RCD
constexpr int kRT = 32, kRH = 10, kRI = kRT + 2 * kRH;  // tile, halo, staged edge
constexpr int kRThreads = 256;
constexpr int kRSmemFloats = kRI * kRI + 44 * 44 + 46 * 46 + 40 * 40 + 46 * 46 + 46 * 46;

__device__ __forceinline__ float rcd_hpf(const Plane& c, int x, int y, int dx, int dy) {
    const float t1 = ((c.at(x - 3 * dx, y - 3 * dy) - c.at(x - dx, y - dy)) - c.at(x + dx, y + dy)) +
                     c.at(x + 3 * dx, y + 3 * dy);
    const float t2 = 3.0F * (c.at(x - 2 * dx, y - 2 * dy) + c.at(x + 2 * dx, y + 2 * dy));
    const float t = (t1 - t2) + 6.0F * c.at(x, y);
    return t * t;
}

__device__ __forceinline__ float disc(const Plane& d, int x, int y) {
    const float ctr = d.at(x, y);
    const float nb = 0.25F * (((d.at(x - 1, y - 1) + d.at(x + 1, y - 1)) + d.at(x - 1, y + 1)) + d.at(x + 1, y + 1));
    return absr(0.5F - ctr) < absr(0.5F - nb) ? nb : ctr;
}

template <class TOut>
__global__ void __launch_bounds__(kRThreads) rcd_full_kernel(Img in, Img out, Cfa cfa) {
    extern __shared__ float smem[];
    const int x0 = blockIdx.x * kRT, y0 = blockIdx.y * kRT;
    const float eps = 0.00001F, eps2 = 1e-10F;
    const Plane C{smem, -kRH, kRI};
    const Plane VH{C.p + kRI * kRI, -6, 44};
    const Plane LP{VH.p + 44 * 44, -7, 46};
    const Plane PQ{LP.p + 46 * 46, -4, 40};
    float* bufA = PQ.p + 40 * 40;
    float* bufB = bufA + 46 * 46;
    const float* src = static_cast<const float*>(in.data);
    for (int i = threadIdx.x; i < kRI * kRI; i += kRThreads) {
        const int ty = i / kRI, tx = i - ty * kRI;
        const int sx = refl(x0 - kRH + tx, in.w), sy = refl(y0 - kRH + ty, in.h);
        C.p[i] = src[(long long)sy * in.row_stride + sx];
    }
    __syncthreads();
    // squared high-passes: vertical over rows [-7, T+7) x cols [-6, T+6),
    // horizontal over rows [-6, T+6) x cols [-7, T+7) (both stored 46 x 46)
    const Plane HV{bufA, -7, 46}, HH{bufB, -7, 46};
    for (int i = threadIdx.x; i < 46 * 46; i += kRThreads) {
        const int y = i / 46 - 7, x = i % 46 - 7;
        if (x >= -6 && x < kRT + 6) HV.at(x, y) = rcd_hpf(C, x, y, 0, 1);
        if (y >= -6 && y < kRT + 6) HH.at(x, y) = rcd_hpf(C, x, y, 1, 0);
    }
    // low-pass over [-7, T+7)
    for (int i = threadIdx.x; i < 46 * 46; i += kRThreads) {
        const int y = i / 46 - 7, x = i % 46 - 7;
        LP.at(x, y) = ((0.25F * C.at(x, y)) +
                       (0.125F * (((C.at(x, y - 1) + C.at(x, y + 1)) + C.at(x - 1, y)) + C.at(x + 1, y)))) +
                      (0.0625F * (((C.at(x - 1, y - 1) + C.at(x + 1, y - 1)) + C.at(x - 1, y + 1)) + C.at(x + 1, y + 1)));
    }
    __syncthreads();
    // vertical / horizontal discrimination over [-6, T+6)
    for (int i = threadIdx.x; i < 44 * 44; i += kRThreads) {
        const int y = i / 44 - 6, x = i % 44 - 6;
        const float sv = maxr(eps2, (HV.at(x, y - 1) + HV.at(x, y)) + HV.at(x, y + 1));
        const float sh = maxr(eps2, (HH.at(x - 1, y) + HH.at(x, y)) + HH.at(x + 1, y));
        VH.at(x, y) = sv / (sv + sh);
    }
    __syncthreads();
    // diagonal squared high-passes over [-5, T+5)
    const Plane HP{bufA, -5, 42}, HQ{bufB, -5, 42};
    for (int i = threadIdx.x; i < 42 * 42; i += kRThreads) {
        const int y = i / 42 - 5, x = i % 42 - 5;
        HP.at(x, y) = rcd_hpf(C, x, y, 1, 1);
        HQ.at(x, y) = rcd_hpf(C, x, y, -1, 1);
    }
    __syncthreads();
    // diagonal discrimination over [-4, T+4)
    for (int i = threadIdx.x; i < 40 * 40; i += kRThreads) {
        const int y = i / 40 - 4, x = i % 40 - 4;
        const float sp = maxr(eps2, (HP.at(x - 1, y - 1) + HP.at(x, y)) + HP.at(x + 1, y + 1));
        const float sq = maxr(eps2, (HQ.at(x + 1, y - 1) + HQ.at(x, y)) + HQ.at(x - 1, y + 1));
        PQ.at(x, y) = sp / (sp + sq);
    }
    __syncthreads();
    // green over [-5, T+5)
    const Plane G{bufA, -5, 42};
    for (int i = threadIdx.x; i < 42 * 42; i += kRThreads) {
        const int y = i / 42 - 5, x = i % 42 - 5;
        if (cfa.at(x0 + x, y0 + y) == 1) {
            G.at(x, y) = C.at(x, y);
            continue;
        }
        const float l0 = LP.at(x, y);
        const float gn = (((eps + absr(C.at(x, y - 1) - C.at(x, y + 1))) + absr(C.at(x, y) - C.at(x, y - 2))) +
                          absr(C.at(x, y - 1) - C.at(x, y - 3))) + absr(C.at(x, y - 2) - C.at(x, y - 4));
        const float gs = (((eps + absr(C.at(x, y - 1) - C.at(x, y + 1))) + absr(C.at(x, y) - C.at(x, y + 2))) +
                          absr(C.at(x, y + 1) - C.at(x, y + 3))) + absr(C.at(x, y + 2) - C.at(x, y + 4));
        const float gw = (((eps + absr(C.at(x - 1, y) - C.at(x + 1, y))) + absr(C.at(x, y) - C.at(x - 2, y))) +
                          absr(C.at(x - 1, y) - C.at(x - 3, y))) + absr(C.at(x - 2, y) - C.at(x - 4, y));
        const float ge = (((eps + absr(C.at(x - 1, y) - C.at(x + 1, y))) + absr(C.at(x, y) - C.at(x + 2, y))) +
                          absr(C.at(x + 1, y) - C.at(x + 3, y))) + absr(C.at(x + 2, y) - C.at(x + 4, y));
        const float en = (C.at(x, y - 1) * (l0 + l0)) / ((eps + l0) + LP.at(x, y - 2));
        const float es = (C.at(x, y + 1) * (l0 + l0)) / ((eps + l0) + LP.at(x, y + 2));
        const float ew = (C.at(x - 1, y) * (l0 + l0)) / ((eps + l0) + LP.at(x - 2, y));
        const float ee = (C.at(x + 1, y) * (l0 + l0)) / ((eps + l0) + LP.at(x + 2, y));
        const float ve = ((gs * en) + (gn * es)) / (gn + gs);
        const float he = ((ge * ew) + (gw * ee)) / (gw + ge);
        G.at(x, y) = intp(disc(VH, x, y), he, ve);
    }
    __syncthreads();
    // the other colour at red/blue sites over [-3, T+3)
    const Plane RB{bufB, -3, 38};
    for (int i = threadIdx.x; i < 38 * 38; i += kRThreads) {
        const int y = i / 38 - 3, x = i % 38 - 3;
        if (cfa.at(x0 + x, y0 + y) == 1) continue;
        const float g0 = G.at(x, y);
        const float gnw = ((eps + absr(C.at(x - 1, y - 1) - C.at(x + 1, y + 1))) + absr(C.at(x - 1, y - 1) - C.at(x - 3, y - 3))) +
                          absr(g0 - G.at(x - 2, y - 2));
        const float gne = ((eps + absr(C.at(x + 1, y - 1) - C.at(x - 1, y + 1))) + absr(C.at(x + 1, y - 1) - C.at(x + 3, y - 3))) +
                          absr(g0 - G.at(x + 2, y - 2));
        const float gsw = ((eps + absr(C.at(x + 1, y - 1) - C.at(x - 1, y + 1))) + absr(C.at(x - 1, y + 1) - C.at(x - 3, y + 3))) +
                          absr(g0 - G.at(x - 2, y + 2));
        const float gse = ((eps + absr(C.at(x - 1, y - 1) - C.at(x + 1, y + 1))) + absr(C.at(x + 1, y + 1) - C.at(x + 3, y + 3))) +
                          absr(g0 - G.at(x + 2, y + 2));
        const float enw = C.at(x - 1, y - 1) - G.at(x - 1, y - 1);
        const float ene = C.at(x + 1, y - 1) - G.at(x + 1, y - 1);
        const float esw = C.at(x - 1, y + 1) - G.at(x - 1, y + 1);
        const float ese = C.at(x + 1, y + 1) - G.at(x + 1, y + 1);
        const float pe = ((gse * enw) + (gnw * ese)) / (gnw + gse);
        const float qe = ((gsw * ene) + (gne * esw)) / (gne + gsw);
        RB.at(x, y) = g0 + intp(disc(PQ, x, y), qe, pe);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRT * kRT; i += kRThreads) {
        const int y = i / kRT, x = i - (i / kRT) * kRT;
        if (x0 + x >= out.w || y0 + y >= out.h) continue;
        const int site = cfa.at(x0 + x, y0 + y);
        const float g0 = G.at(x, y);
        float o[3];
        o[1] = g0;
        if (site != 1) {
            o[site] = C.at(x, y);
            o[2 - site] = RB.at(x, y);
        } else {
            const float d = disc(VH, x, y);
#pragma unroll
            for (int k = 0; k <= 2; k += 2) {
#define XK(dx, dy) (cfa.at(x0 + x + (dx), y0 + y + (dy)) == k ? C.at(x + (dx), y + (dy)) : RB.at(x + (dx), y + (dy)))
                const float gn = ((eps + absr(g0 - G.at(x, y - 2))) + absr(XK(0, -1) - XK(0, 1))) + absr(XK(0, -1) - XK(0, -3));
                const float gs = ((eps + absr(g0 - G.at(x, y + 2))) + absr(XK(0, 1) - XK(0, -1))) + absr(XK(0, 1) - XK(0, 3));
                const float gw = ((eps + absr(g0 - G.at(x - 2, y))) + absr(XK(-1, 0) - XK(1, 0))) + absr(XK(-1, 0) - XK(-3, 0));
                const float ge = ((eps + absr(g0 - G.at(x + 2, y))) + absr(XK(1, 0) - XK(-1, 0))) + absr(XK(1, 0) - XK(3, 0));
                const float en = XK(0, -1) - G.at(x, y - 1);
                const float es = XK(0, 1) - G.at(x, y + 1);
                const float ew = XK(-1, 0) - G.at(x - 1, y);
                const float ee = XK(1, 0) - G.at(x + 1, y);
#undef XK
                const float ve = ((gs * en) + (gn * es)) / (gn + gs);
                const float he = ((ge * ew) + (gw * ee)) / (gw + ge);
                o[k] = g0 + intp(d, he, ve);
            }
        }
        store_rgba(px<TOut>(out, x0 + x, y0 + y), Rgba{maxr(0.0F, o[0]), maxr(0.0F, o[1]), maxr(0.0F, o[2]), 1.0F});
    }
}

// ---------------------------------------------------------------- AMaZE
// Scratch planes over the extended domain [-kAM, w + kAM) x [-kAM, h + kAM).
constexpr int kAM = 16;
struct AmazePlanes {
    float *vcd, *hcd, *hvw, *dg, *g, *hvf;
    unsigned char* nyq;
    int pw, ph;  // extended extent
    __device__ __forceinline__ long long idx(int x, int y) const { return (long long)(y + kAM) * pw + (x + kAM); }
};
struct AmazeWeights {
    float odd[4], grad[6], quinc[4];
};

constexpr int kAT = 32;  // tile edge of the AMaZE kernels
constexpr int kAThreads = 256;

// Kernel 1 over the whole extended domain: stages A-D at each position
// (vcd, hcd, the vertical weight hvw, the Nyquist flag).  Staged: the mosaic
// with a halo of 7 and the colour differences / fluctuations with a halo of 3.
constexpr int kA1H = 7, kA1I = kAT + 2 * kA1H;      // 46: mosaic
constexpr int kA1D = kAT + 2 * 3;                   // 38: vcd, hcd, dgv, dgh, cdsq over [-3, T+3)
constexpr int kA1W = kAT + 2 * 5;                   // 42: directional weights over [-5, T+5)
constexpr int kA1SmemFloats = kA1I * kA1I + 5 * kA1D * kA1D + 2 * kA1W * kA1W;

__global__ void __launch_bounds__(kAThreads) amaze_cd_kernel(Img in, AmazePlanes P, Cfa cfa, AmazeWeights W) {
    extern __shared__ float smem[];
    const int x0 = blockIdx.x * kAT - kAM, y0 = blockIdx.y * kAT - kAM;  // tile origin in frame coordinates
    const float eps = 0.00001F, eps2 = 1e-10F, arthresh = 0.75F, clip8 = 0.8F;
    const Plane C{smem, -kA1H, kA1I};
    const Plane D0{C.p + kA1I * kA1I, -5, kA1W}, D1{D0.p + kA1W * kA1W, -5, kA1W};
    const Plane VC{D1.p + kA1W * kA1W, -3, kA1D}, HC{VC.p + kA1D * kA1D, -3, kA1D};
    const Plane DV{HC.p + kA1D * kA1D, -3, kA1D}, DH{DV.p + kA1D * kA1D, -3, kA1D};
    const Plane SQ{DH.p + kA1D * kA1D, -3, kA1D};
    const float* src = static_cast<const float*>(in.data);
    for (int i = threadIdx.x; i < kA1I * kA1I; i += kAThreads) {
        const int ty = i / kA1I, tx = i - ty * kA1I;
        C.p[i] = src[(long long)refl(y0 - kA1H + ty, in.h) * in.row_stride + refl(x0 - kA1H + tx, in.w)];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kA1W * kA1W; i += kAThreads) {
        const int y = i / kA1W - 5, x = i % kA1W - 5;
        const float dh = absr(C.at(x + 1, y) - C.at(x - 1, y));
        const float dv = absr(C.at(x, y + 1) - C.at(x, y - 1));
        D0.at(x, y) = ((eps + absr(C.at(x, y + 2) - C.at(x, y))) + absr(C.at(x, y) - C.at(x, y - 2))) + dv;
        D1.at(x, y) = ((eps + absr(C.at(x + 2, y) - C.at(x, y))) + absr(C.at(x, y) - C.at(x - 2, y))) + dh;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kA1D * kA1D; i += kAThreads) {
        const int y = i / kA1D - 3, x = i % kA1D - 3;
        const float c0 = C.at(x, y);
        const float sgn = cfa.at(x0 + x, y0 + y) == 1 ? -1.0F : 1.0F;
        const float d0 = D0.at(x, y), d1 = D1.at(x, y);
        const float cru = (C.at(x, y - 1) * (D0.at(x, y - 2) + d0)) / ((D0.at(x, y - 2) * (eps + c0)) + (d0 * (eps + C.at(x, y - 2))));
        const float crd = (C.at(x, y + 1) * (D0.at(x, y + 2) + d0)) / ((D0.at(x, y + 2) * (eps + c0)) + (d0 * (eps + C.at(x, y + 2))));
        const float crl = (C.at(x - 1, y) * (D1.at(x - 2, y) + d1)) / ((D1.at(x - 2, y) * (eps + c0)) + (d1 * (eps + C.at(x - 2, y))));
        const float crr = (C.at(x + 1, y) * (D1.at(x + 2, y) + d1)) / ((D1.at(x + 2, y) * (eps + c0)) + (d1 * (eps + C.at(x + 2, y))));
        const float guha = C.at(x, y - 1) + (0.5F * (c0 - C.at(x, y - 2)));
        const float gdha = C.at(x, y + 1) + (0.5F * (c0 - C.at(x, y + 2)));
        const float glha = C.at(x - 1, y) + (0.5F * (c0 - C.at(x - 2, y)));
        const float grha = C.at(x + 1, y) + (0.5F * (c0 - C.at(x + 2, y)));
        float guar = absr(1.0F - cru) < arthresh ? c0 * cru : guha;
        float gdar = absr(1.0F - crd) < arthresh ? c0 * crd : gdha;
        float glar = absr(1.0F - crl) < arthresh ? c0 * crl : glha;
        float grar = absr(1.0F - crr) < arthresh ? c0 * crr : grha;
        const float hwt = D1.at(x - 1, y) / (D1.at(x - 1, y) + D1.at(x + 1, y));
        const float vwt = D0.at(x, y - 1) / (D0.at(x, y + 1) + D0.at(x, y - 1));
        const float gvha = (vwt * gdha) + ((1.0F - vwt) * guha);
        const float ghha = (hwt * grha) + ((1.0F - hwt) * glha);
        float vc = sgn * (((vwt * gdar) + ((1.0F - vwt) * guar)) - c0);
        float hc = sgn * (((hwt * grar) + ((1.0F - hwt) * glar)) - c0);
        if (c0 > clip8 || gvha > clip8 || ghha > clip8) {
            guar = guha;
            gdar = gdha;
            glar = glha;
            grar = grha;
            vc = sgn * (gvha - c0);
            hc = sgn * (ghha - c0);
        }
        VC.at(x, y) = vc;
        HC.at(x, y) = hc;
        DV.at(x, y) = minr((guha - gdha) * (guha - gdha), (guar - gdar) * (guar - gdar));
        DH.at(x, y) = minr((glha - grha) * (glha - grha), (glar - grar) * (glar - grar));
        SQ.at(x, y) = (vc - hc) * (vc - hc);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kAT * kAT; i += kAThreads) {
        const int y = i / kAT, x = i - (i / kAT) * kAT;
        const int fx = x0 + x, fy = y0 + y;
        if (fx >= in.w + kAM || fy >= in.h + kAM) continue;
        const float hwt = D1.at(x - 1, y) / (D1.at(x - 1, y) + D1.at(x + 1, y));
        const float vwt = D0.at(x, y - 1) / (D0.at(x, y + 1) + D0.at(x, y - 1));
        float su = 0.0F, sd = 0.0F, sl = 0.0F, sr = 0.0F;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            su = su + VC.at(x, y - k);
            sd = sd + VC.at(x, y + k);
            sl = sl + HC.at(x - k, y);
            sr = sr + HC.at(x + k, y);
        }
        const float mu = 0.25F * su, md = 0.25F * sd, ml = 0.25F * sl, mr = 0.25F * sr;
        float vu = 0.0F, vd = 0.0F, vl = 0.0F, vr = 0.0F;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            vu = vu + (VC.at(x, y - k) - mu) * (VC.at(x, y - k) - mu);
            vd = vd + (VC.at(x, y + k) - md) * (VC.at(x, y + k) - md);
            vl = vl + (HC.at(x - k, y) - ml) * (HC.at(x - k, y) - ml);
            vr = vr + (HC.at(x + k, y) - mr) * (HC.at(x + k, y) - mr);
        }
        const float vvar = (eps2 + (vwt * vd)) + ((1.0F - vwt) * vu);
        const float hvar = (eps2 + (hwt * vr)) + ((1.0F - hwt) * vl);
        const float fu = (DV.at(x, y) + DV.at(x, y - 1)) + DV.at(x, y - 2);
        const float fd = (DV.at(x, y) + DV.at(x, y + 1)) + DV.at(x, y + 2);
        const float fl = (DH.at(x, y) + DH.at(x - 1, y)) + DH.at(x - 2, y);
        const float fr = (DH.at(x, y) + DH.at(x + 1, y)) + DH.at(x + 2, y);
        const float vvar1 = (eps2 + (vwt * fd)) + ((1.0F - vwt) * fu);
        const float hvar1 = (eps2 + (hwt * fr)) + ((1.0F - hwt) * fl);
        const float varwt = hvar / (vvar + hvar);
        const float diffwt = hvar1 / (vvar1 + hvar1);
        const long long o = P.idx(fx, fy);
        P.hvw[o] = ((0.5F - varwt) * (0.5F - diffwt) > 0.0F && absr(0.5F - diffwt) < absr(0.5F - varwt)) ? varwt : diffwt;
        P.vcd[o] = VC.at(x, y);
        P.hcd[o] = HC.at(x, y);
        unsigned char nq = 0;
        if (cfa.at(fx, fy) != 1) {
            float a = W.odd[0] * SQ.at(x, y);
            a = a + W.odd[1] * (((SQ.at(x - 1, y - 1) + SQ.at(x + 1, y - 1)) + SQ.at(x - 1, y + 1)) + SQ.at(x + 1, y + 1));
            a = a + W.odd[2] * (((SQ.at(x, y - 2) + SQ.at(x - 2, y)) + SQ.at(x + 2, y)) + SQ.at(x, y + 2));
            a = a + W.odd[3] * (((SQ.at(x - 2, y - 2) + SQ.at(x + 2, y - 2)) + SQ.at(x - 2, y + 2)) + SQ.at(x + 2, y + 2));
            // squared gradients delh^2 + delv^2 over the 5x5 window
#define DHV(dx, dy)                                                                                   \
    ((absr(C.at(x + (dx) + 1, y + (dy)) - C.at(x + (dx) - 1, y + (dy))) *                              \
      absr(C.at(x + (dx) + 1, y + (dy)) - C.at(x + (dx) - 1, y + (dy)))) +                             \
     (absr(C.at(x + (dx), y + (dy) + 1) - C.at(x + (dx), y + (dy) - 1)) *                              \
      absr(C.at(x + (dx), y + (dy) + 1) - C.at(x + (dx), y + (dy) - 1))))
            float b = W.grad[0] * DHV(0, 0);
            b = b + W.grad[1] * (((DHV(0, -1) + DHV(-1, 0)) + DHV(1, 0)) + DHV(0, 1));
            b = b + W.grad[2] * (((DHV(-1, -1) + DHV(1, -1)) + DHV(-1, 1)) + DHV(1, 1));
            b = b + W.grad[3] * (((DHV(0, -2) + DHV(-2, 0)) + DHV(2, 0)) + DHV(0, 2));
            b = b + W.grad[4] * (((((((DHV(-1, -2) + DHV(1, -2)) + DHV(-2, -1)) + DHV(2, -1)) + DHV(-2, 1)) + DHV(2, 1)) +
                                  DHV(-1, 2)) + DHV(1, 2));
            b = b + W.grad[5] * (((DHV(-2, -2) + DHV(2, -2)) + DHV(-2, 2)) + DHV(2, 2));
#undef DHV
            nq = (a - b) > 0.0F ? 1 : 0;
        }
        P.nyq[o] = nq;
    }
}

// Kernel 2 over [-4, w + 4) x [-4, h + 4): the Nyquist vote (over [-13, T+13)),
// the area weights (over [-7, T+7)), green and the refined weight (over
// [-6, T+6)), curvatures and their refinement of green in Nyquist areas.
constexpr int kA2O = 4;                       // output margin of kernel 2
constexpr int kA2NQ = kAT + 2 * 15;           // nyq staged over [-15, T+15) (62)
constexpr int kA2N2 = kAT + 2 * 13;           // nyq2 over [-13, T+13) (58)
constexpr int kA2C = kAT + 2 * 14;            // mosaic over [-14, T+14) (60)
constexpr int kA2E = kAT + 2 * 7;             // hve over [-7, T+7) (46)
constexpr int kA2F = kAT + 2 * 6;             // g, dg, cvh, cvv over [-6, T+6) (44)
constexpr int kA2SmemBytes = (kA2C * kA2C + kA2E * kA2E + 5 * kA2F * kA2F) * 4 + kA2NQ * kA2NQ + kA2N2 * kA2N2;

__global__ void __launch_bounds__(kAThreads) amaze_green_kernel(Img in, AmazePlanes P, Cfa cfa, AmazeWeights W) {
    extern __shared__ float smem[];
    // tiles cover [-kA2O, w + kA2O): origin in frame coordinates
    const int x0 = blockIdx.x * kAT - kA2O, y0 = blockIdx.y * kAT - kA2O;
    const int xe = in.w + kA2O, ye = in.h + kA2O;
    const float eps2 = 1e-10F;
    const Plane C{smem, -14, kA2C};
    const Plane E{C.p + kA2C * kA2C, -7, kA2E};
    const Plane G{E.p + kA2E * kA2E, -6, kA2F}, DG{G.p + kA2F * kA2F, -6, kA2F};
    const Plane CH{DG.p + kA2F * kA2F, -6, kA2F}, CV{CH.p + kA2F * kA2F, -6, kA2F};
    const Plane HF{CV.p + kA2F * kA2F, -6, kA2F};
    unsigned char* nq = reinterpret_cast<unsigned char*>(HF.p + kA2F * kA2F);
    unsigned char* nq2 = nq + kA2NQ * kA2NQ;
#define NQ(x, y) nq[((y) + 15) * kA2NQ + ((x) + 15)]
#define NQ2(x, y) nq2[((y) + 13) * kA2N2 + ((x) + 13)]
    const float* src = static_cast<const float*>(in.data);
    for (int i = threadIdx.x; i < kA2C * kA2C; i += kAThreads) {
        const int ty = i / kA2C, tx = i - ty * kA2C;
        C.p[i] = src[(long long)refl(y0 - 14 + ty, in.h) * in.row_stride + refl(x0 - 14 + tx, in.w)];
    }
    // the Nyquist flags are stored over [-kAM, w + kAM); the tile reads within [-19, ...], so clamp to the
    // stored margin (flags past it are never used by an output of the frame: see the ranges above)
    for (int i = threadIdx.x; i < kA2NQ * kA2NQ; i += kAThreads) {
        const int ty = i / kA2NQ, tx = i - ty * kA2NQ;
        const int fx = x0 - 15 + tx, fy = y0 - 15 + ty;
        unsigned char v = 0;
        if (fx >= -kAM && fy >= -kAM && fx < in.w + kAM && fy < in.h + kAM) v = P.nyq[P.idx(fx, fy)];
        nq[i] = v;
    }
    for (int i = threadIdx.x; i < kA2E * kA2E; i += kAThreads) {
        const int ty = i / kA2E, tx = i - ty * kA2E;
        const int fx = x0 - 7 + tx, fy = y0 - 7 + ty;
        E.p[i] = (fx >= -kAM && fy >= -kAM && fx < in.w + kAM && fy < in.h + kAM) ? P.hvw[P.idx(fx, fy)] : 0.0F;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kA2N2 * kA2N2; i += kAThreads) {
        const int y = i / kA2N2 - 13, x = i % kA2N2 - 13;
        unsigned char v = 0;
        if (cfa.at(x0 + x, y0 + y) != 1) {
            const int s = NQ(x - 1, y - 1) + NQ(x + 1, y - 1) + NQ(x - 1, y + 1) + NQ(x + 1, y + 1) + NQ(x, y - 2) +
                          NQ(x - 2, y) + NQ(x + 2, y) + NQ(x, y + 2);
            v = s > 4 ? 1 : (s < 4 ? 0 : NQ(x, y));
        }
        NQ2(x, y) = v;
    }
    __syncthreads();
    // area weights over [-7, T+7) (E holds hvw; replaced where nyq2)
    for (int i = threadIdx.x; i < kA2E * kA2E; i += kAThreads) {
        const int y = i / kA2E - 7, x = i % kA2E - 7;
        if (cfa.at(x0 + x, y0 + y) == 1 || !NQ2(x, y)) continue;
        float sh = 0.0F, sv = 0.0F, qh = 0.0F, qv = 0.0F, n = 0.0F;
        for (int a = -6; a <= 6; a += 2)
            for (int b = -6; b <= 6; b += 2) {
                const int qx = x + b, qy = y + a;
                if (!NQ2(qx, qy)) continue;
                const float q0 = C.at(qx, qy);
                sh = sh + (q0 - 0.5F * (C.at(qx - 1, qy) + C.at(qx + 1, qy)));
                sv = sv + (q0 - 0.5F * (C.at(qx, qy - 1) + C.at(qx, qy + 1)));
                qh = qh + 0.5F * ((q0 - C.at(qx - 1, qy)) * (q0 - C.at(qx - 1, qy)) + (q0 - C.at(qx + 1, qy)) * (q0 - C.at(qx + 1, qy)));
                qv = qv + 0.5F * ((q0 - C.at(qx, qy - 1)) * (q0 - C.at(qx, qy - 1)) + (q0 - C.at(qx, qy + 1)) * (q0 - C.at(qx, qy + 1)));
                n = n + 1.0F;
            }
        const float hvar = eps2 + absr((n * qh) - (sh * sh));
        const float vvar = eps2 + absr((n * qv) - (sv * sv));
        // in place: the cells of this loop read nyq2 and the mosaic, never E
        E.at(x, y) = hvar / (vvar + hvar);
    }
    __syncthreads();
    // refined weight, green, curvatures over [-6, T+6)
    for (int i = threadIdx.x; i < kA2F * kA2F; i += kAThreads) {
        const int y = i / kA2F - 6, x = i % kA2F - 6;
        const int fx = x0 + x, fy = y0 + y;
        float gv = C.at(x, y), dgv = 0.0F, hv = 0.0F, ch = 0.0F, cv = 0.0F;
        if (cfa.at(fx, fy) != 1) {
            const float hv0 = E.at(x, y);
            const float alt = 0.25F * (((E.at(x - 1, y - 1) + E.at(x + 1, y - 1)) + E.at(x - 1, y + 1)) + E.at(x + 1, y + 1));
            hv = absr(0.5F - hv0) < absr(0.5F - alt) ? alt : hv0;
            const bool in_ext = fx >= -kAM && fy >= -kAM && fx < in.w + kAM && fy < in.h + kAM;
            const long long o = in_ext ? P.idx(fx, fy) : 0;
            const float hc = in_ext ? P.hcd[o] : 0.0F, vc = in_ext ? P.vcd[o] : 0.0F;
            dgv = (hc * (1.0F - hv)) + (vc * hv);
            gv = C.at(x, y) + dgv;
            if (NQ2(x, y)) {
                const float th = gv - 0.5F * (C.at(x - 1, y) + C.at(x + 1, y));
                const float tv = gv - 0.5F * (C.at(x, y - 1) + C.at(x, y + 1));
                ch = th * th;
                cv = tv * tv;
            }
        }
        G.at(x, y) = gv;
        DG.at(x, y) = dgv;
        CH.at(x, y) = ch;
        CV.at(x, y) = cv;
        HF.at(x, y) = hv;
    }
    __syncthreads();
    // curvature refinement and write-out over the tile
    for (int i = threadIdx.x; i < kAT * kAT; i += kAThreads) {
        const int y = i / kAT, x = i - (i / kAT) * kAT;
        const int fx = x0 + x, fy = y0 + y;
        if (fx >= xe || fy >= ye) continue;
        float gv = G.at(x, y), dgv = DG.at(x, y);
        if (cfa.at(fx, fy) != 1 && NQ2(x, y)) {
            float gh = W.quinc[0] * CH.at(x, y), gvv = W.quinc[0] * CV.at(x, y);
            gh = gh + W.quinc[1] * (((CH.at(x - 1, y - 1) + CH.at(x + 1, y - 1)) + CH.at(x - 1, y + 1)) + CH.at(x + 1, y + 1));
            gvv = gvv + W.quinc[1] * (((CV.at(x - 1, y - 1) + CV.at(x + 1, y - 1)) + CV.at(x - 1, y + 1)) + CV.at(x + 1, y + 1));
            gh = gh + W.quinc[2] * (((CH.at(x, y - 2) + CH.at(x - 2, y)) + CH.at(x + 2, y)) + CH.at(x, y + 2));
            gvv = gvv + W.quinc[2] * (((CV.at(x, y - 2) + CV.at(x - 2, y)) + CV.at(x + 2, y)) + CV.at(x, y + 2));
            gh = gh + W.quinc[3] * (((CH.at(x - 2, y - 2) + CH.at(x + 2, y - 2)) + CH.at(x - 2, y + 2)) + CH.at(x + 2, y + 2));
            gvv = gvv + W.quinc[3] * (((CV.at(x - 2, y - 2) + CV.at(x + 2, y - 2)) + CV.at(x - 2, y + 2)) + CV.at(x + 2, y + 2));
            gh = eps2 + gh;
            gvv = eps2 + gvv;
            const long long o = P.idx(fx, fy);
            dgv = ((P.hcd[o] * gvv) + (P.vcd[o] * gh)) / (gvv + gh);
            gv = C.at(x, y) + dgv;
        }
        const long long o = P.idx(fx, fy);
        P.g[o] = gv;
        P.dg[o] = dgv;
        P.hvf[o] = HF.at(x, y);
    }
#undef NQ
#undef NQ2
}

// Kernel 3 over the frame: the other colour's difference at red/blue sites
// (over [-1, T+1), from dg over [-4, T+4)) and the outputs.
constexpr int kA3D = kAT + 2 * 4;  // dg staged over [-4, T+4) (40)
constexpr int kA3O = kAT + 2;      // cdo, hvf over [-1, T+1) (34)
template <class TOut>
__global__ void __launch_bounds__(kAThreads) amaze_out_kernel(Img in, Img out, AmazePlanes P, Cfa cfa) {
    __shared__ float s_dg[kA3D * kA3D];
    __shared__ float s_cdo[kA3O * kA3O];
    __shared__ float s_hvf[kA3O * kA3O];
    const int x0 = blockIdx.x * kAT, y0 = blockIdx.y * kAT;
    const float eps = 0.00001F;
    const Plane DG{s_dg, -4, kA3D}, CO{s_cdo, -1, kA3O}, HF{s_hvf, -1, kA3O};
    for (int i = threadIdx.x; i < kA3D * kA3D; i += kAThreads) {
        const int y = i / kA3D - 4, x = i % kA3D - 4;
        const int fx = min(x0 + x, in.w + 3), fy = min(y0 + y, in.h + 3);  // within the stored [-4, w + 4)
        s_dg[i] = P.dg[P.idx(fx, fy)];
    }
    for (int i = threadIdx.x; i < kA3O * kA3O; i += kAThreads) {
        const int y = i / kA3O - 1, x = i % kA3O - 1;
        const int fx = min(x0 + x, in.w), fy = min(y0 + y, in.h);
        s_hvf[i] = P.hvf[P.idx(fx, fy)];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kA3O * kA3O; i += kAThreads) {
        const int y = i / kA3O - 1, x = i % kA3O - 1;
        if (cfa.at(x0 + x, y0 + y) == 1) continue;
        float num = 0.0F, den = 0.0F;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int dx = (k & 1) ? 1 : -1, dy = (k & 2) ? 1 : -1;
            const float d1 = DG.at(x + dx, y + dy), dm = DG.at(x - dx, y - dy), d3 = DG.at(x + 3 * dx, y + 3 * dy);
            const float wt = 1.0F / (((eps + absr(d1 - dm)) + absr(d1 - d3)) + absr(dm - d3));
            const float est = (((1.325F * d1) - (0.175F * d3)) - (0.075F * DG.at(x + 3 * dx, y + dy))) -
                              (0.075F * DG.at(x + dx, y + 3 * dy));
            num = num + wt * est;
            den = den + wt;
        }
        CO.at(x, y) = num / den;
    }
    __syncthreads();
    const float* src = static_cast<const float*>(in.data);
    for (int i = threadIdx.x; i < kAT * kAT; i += kAThreads) {
        const int y = i / kAT, x = i - (i / kAT) * kAT;
        const int fx = x0 + x, fy = y0 + y;
        if (fx >= out.w || fy >= out.h) continue;
        const int site = cfa.at(fx, fy);
        const float g0 = P.g[P.idx(fx, fy)];
        float o[3];
        o[1] = g0;
        if (site != 1) {
            o[site] = src[(long long)fy * in.row_stride + fx];
            o[2 - site] = g0 - CO.at(x, y);
        } else {
            const float wn = HF.at(x, y - 1), ws = HF.at(x, y + 1);
            const float ww = 1.0F - HF.at(x - 1, y), we = 1.0F - HF.at(x + 1, y);
            const float t = 1.0F / (((wn + we) + ww) + ws);
#pragma unroll
            for (int k = 0; k <= 2; k += 2) {
#define CDK(dx, dy) (cfa.at(fx + (dx), fy + (dy)) == k ? DG.at(x + (dx), y + (dy)) : CO.at(x + (dx), y + (dy)))
                const float s = (((wn * CDK(0, -1)) + (we * CDK(1, 0))) + (ww * CDK(-1, 0))) + (ws * CDK(0, 1));
#undef CDK
                o[k] = g0 - (s * t);
            }
        }
        store_rgba(px<TOut>(out, fx, fy), Rgba{maxr(0.0F, o[0]), maxr(0.0F, o[1]), maxr(0.0F, o[2]), 1.0F});
    }
}

AmazeWeights amaze_weights() {
    // Gaussian weights from their definitions (see the oracle's header):
    // quincunx d^2 = 0, 2, 4, 8 (1, 4, 4, 4 sites); 5x5 d^2 = 0, 1, 2, 4, 5, 8
    // (1, 4, 4, 4, 8, 4 sites); computed in double, rounded to binary32.
    const double qd[4] = {0.0, 2.0, 4.0, 8.0}, qn[4] = {1.0, 4.0, 4.0, 4.0};
    const double gd[6] = {0.0, 1.0, 2.0, 4.0, 5.0, 8.0}, gn[6] = {1.0, 4.0, 4.0, 4.0, 8.0, 4.0};
    AmazeWeights W;
    double s = 0.0;
    for (int i = 0; i < 4; ++i) s += qn[i] * std::exp(-qd[i] / (2.0 * 2.88));
    for (int i = 0; i < 4; ++i) W.odd[i] = (float)(std::exp(-qd[i] / (2.0 * 2.88)) / s);
    s = 0.0;
    for (int i = 0; i < 6; ++i) s += gn[i] * std::exp(-gd[i] / (2.0 * 2.88));
    for (int i = 0; i < 6; ++i) W.grad[i] = (float)(0.5 * std::exp(-gd[i] / (2.0 * 2.88)) / s);
    s = 0.0;
    for (int i = 0; i < 4; ++i) s += qn[i] * std::exp(-qd[i] / (2.0 * 2.25));
    for (int i = 0; i < 4; ++i) W.quinc[i] = (float)(std::exp(-qd[i] / (2.0 * 2.25)) / s);
    return W;
}

}  // namespace dmf

size_t demosaic_full_scratch_bytes(int algo, int w, int h) {
    if (algo != 2) return 0;
    const size_t n = (size_t)(w + 2 * dmf::kAM) * (size_t)(h + 2 * dmf::kAM);
    return n * (6 * sizeof(float)) + ((n + 255) / 256) * 256;
}

cudaError_t launch_demosaic_full(int algo, const Img& in, const Img& out, bool out_f16, const int cfa4[4], void* scratch,
                                 cudaStream_t st) {
    const Cfa cfa{{cfa4[0], cfa4[1], cfa4[2], cfa4[3]}};
    if (algo == 1) {
        const size_t smem = dmf::kRSmemFloats * sizeof(float);
        const dim3 grid((in.w + dmf::kRT - 1) / dmf::kRT, (in.h + dmf::kRT - 1) / dmf::kRT);
        cudaError_t e;
        if (out_f16) {
            e = cudaFuncSetAttribute(dmf::rcd_full_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            dmf::rcd_full_kernel<__half><<<grid, dmf::kRThreads, smem, st>>>(in, out, cfa);
        } else {
            e = cudaFuncSetAttribute(dmf::rcd_full_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            dmf::rcd_full_kernel<float><<<grid, dmf::kRThreads, smem, st>>>(in, out, cfa);
        }
        return cudaGetLastError();
    }
    dmf::AmazePlanes P;
    P.pw = in.w + 2 * dmf::kAM;
    P.ph = in.h + 2 * dmf::kAM;
    const size_t n = (size_t)P.pw * P.ph;
    float* f = static_cast<float*>(scratch);
    P.vcd = f;
    P.hcd = f + n;
    P.hvw = f + 2 * n;
    P.dg = f + 3 * n;
    P.g = f + 4 * n;
    P.hvf = f + 5 * n;
    P.nyq = reinterpret_cast<unsigned char*>(f + 6 * n);
    const dmf::AmazeWeights W = dmf::amaze_weights();
    const size_t s1 = dmf::kA1SmemFloats * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(dmf::amaze_cd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1);
    if (e != cudaSuccess) return e;
    const dim3 g1((P.pw + dmf::kAT - 1) / dmf::kAT, (P.ph + dmf::kAT - 1) / dmf::kAT);
    dmf::amaze_cd_kernel<<<g1, dmf::kAThreads, s1, st>>>(in, P, cfa, W);
    const size_t s2 = dmf::kA2SmemBytes;
    e = cudaFuncSetAttribute(dmf::amaze_green_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);
    if (e != cudaSuccess) return e;
    const dim3 g2((in.w + 2 * dmf::kA2O + dmf::kAT - 1) / dmf::kAT, (in.h + 2 * dmf::kA2O + dmf::kAT - 1) / dmf::kAT);
    dmf::amaze_green_kernel<<<g2, dmf::kAThreads, s2, st>>>(in, P, cfa, W);
    const dim3 g3((in.w + dmf::kAT - 1) / dmf::kAT, (in.h + dmf::kAT - 1) / dmf::kAT);
    if (out_f16) dmf::amaze_out_kernel<__half><<<g3, dmf::kAThreads, 0, st>>>(in, out, P, cfa);
    else dmf::amaze_out_kernel<float><<<g3, dmf::kAThreads, 0, st>>>(in, out, P, cfa);
    return cudaGetLastError();
}

}  // namespace cpb
