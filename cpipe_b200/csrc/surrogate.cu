// Learned surrogate denoiser on sm_100a: an 8-layer, 32-channel residual
// network of 3x3 convolutions with BF16 weights and activations and FP32
// accumulation, trained on the GPU by the kernels in this file.
//
// There is no reference counterpart: the reference's AI denoise node is
// planned but not implemented (docs/research/08-ai-isp-algorithms.md:37) and
// its inference suite returns UNSUPPORTED (src/cpipe/runtime/HostContext.cpp:997-1000).
//
// Layout.  Activations are NHWC bf16: the input a0 has 8 channels (R, G, B,
// sigma/0.03, four zeros), hidden activations a1..a7 32 channels (post-ReLU).
// The tcgen05 inference path keeps its hidden activations in 8-channel planes,
// [n][4][h][w][8] (surrogate_tc.cu); a0 is the same in both layouts.
// Layer l is an implicit GEMM  out[p][co] = sum_k A[p][k] * W[co][k]  with
// k = tap * CIN + ci (tap = 3*(dy+1) + (dx+1)), K padded to a multiple of 16;
// the weights are stored [COUT][K] (the col-major B operand of mma).
//
// Kernels.
//   sg_prep_kernel   RGBA frame(s) -> a0 (noise map from the per-image model)
//   sg_conv_kernel   one 8x16-pixel output tile per CTA iteration (4 warps, a
//                    row pair each), persistent over tiles; the input tile with
//                    its 1-pixel halo and all weights are staged in shared
//                    memory (rows padded to 80 B / 592 B so ldmatrix is
//                    conflict free); A and B fragments by ldmatrix,
//                    mma.sync.m16n8k16 bf16 -> f32.  Epilogues: bias + ReLU ->
//                    bf16; ReLU-mask of the backward pass -> bf16; residual
//                    add -> RGBA frame; residual + MSE loss gradient (training).
//                    The backward-data pass of a layer is the same kernel with
//                    the weights transposed and spatially flipped.
//   sg_wgrad_kernel  dW[co][k] = sum_p dY[p][co] * A[p][k]: the same tiles,
//                    A^T and the im2col operand by transposing ldmatrix,
//                    per-CTA register accumulation over its tiles, then one
//                    atomic add per weight; bias gradients alongside.
//   sg_adam_kernel   Adam on the FP32 master parameters (blob order), after a
//                    global gradient-norm clip (sg_gradnorm_kernel); a step
//                    with a non-finite gradient is skipped.
//   sg_pack_kernel   master parameters -> bf16 forward and backward layouts.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "common.cuh"
#include "filters_impl.h"
#include "surrogate.h"
#include "surrogate_tc.h"

namespace cpb {
namespace sg {

using bf16 = __nv_bfloat16;

constexpr int kLayers = 8;
constexpr int kCh = 32;
constexpr int kTileH = 8, kTileW = 16, kHaloW = kTileW + 2, kHaloPix = (kTileH + 2) * kHaloW;
constexpr float kSigmaScale = 1.0F / 0.03F;
constexpr float kGradClip = 1e-2F;  // global gradient L2 norm bound (the loss is a per-pixel mean)

__host__ __device__ constexpr int kpad(int cin) { return (9 * cin + 15) / 16 * 16; }
__host__ __device__ constexpr int cin_pad(int l) { return l == 0 ? 8 : kCh; }
__host__ __device__ constexpr int cout_pad(int l) { return l == kLayers - 1 ? 8 : kCh; }
__host__ __device__ constexpr int cin_real(int l) { return l == 0 ? 4 : kCh; }
__host__ __device__ constexpr int cout_real(int l) { return l == kLayers - 1 ? 3 : kCh; }

// --------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t& r0, uint32_t& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t& r0, uint32_t& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r0), "=r"(r1)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------------ prep
// a0[p] = (R, G, B, sigma/0.03, 0, 0, 0, 0); dense RGBA frames [n][h][w][4].
template <class T>
__global__ void sg_prep_kernel(const T* __restrict__ in, bf16* __restrict__ a0, const float* __restrict__ ab,
                               long long npx_img, int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npx_img * n) return;
    const int img = (int)(i / npx_img);
    const Rgba p = load_rgba(in + 4 * i);
    const float L = ((p.r + p.g) + p.b) * (1.0F / 3.0F);
    const float var = fmaxf(0.0F, ab[2 * img + 1] + ab[2 * img] * fmaxf(L, 0.0F));
    const float s = sqrtf(var) * kSigmaScale;
    __nv_bfloat162 v[4];
    v[0] = __floats2bfloat162_rn(p.r, p.g);
    v[1] = __floats2bfloat162_rn(p.b, s);
    v[2] = __floats2bfloat162_rn(0.0F, 0.0F);
    v[3] = v[2];
    *reinterpret_cast<uint4*>(a0 + 8 * i) = *reinterpret_cast<const uint4*>(v);
}

// ------------------------------------------------------------------ conv
enum Epi { kEpiRelu = 0, kEpiMask = 1, kEpiResidual = 2, kEpiLoss = 3 };

struct ConvArgs {
    const bf16* x;     // [n][h][w][CIN]
    const bf16* w;     // [COUT][KP]
    const float* bias; // [cout_real] or null
    int cout_real;
    int n, h, w_px;
    bf16* y;           // kEpiRelu / kEpiMask / kEpiLoss: [n][h][w][COUT]
    const bf16* mask;  // kEpiMask: activation whose > 0 gates the gradient
    const void* rgba;  // kEpiResidual / kEpiLoss: the network input frame (RGBA, T)
    void* out;         // kEpiResidual: RGBA output frame (T)
    const __half* target;  // kEpiLoss: RGBA16F target
    float grad_scale;  // kEpiLoss: 2 / (3 * pixels)
    float* loss;       // kEpiLoss: sum of squared errors (atomic)
};

template <int CIN, int COUT>
struct ConvShape {
    static constexpr int KP = kpad(CIN);
    static constexpr int KSTEPS = KP / 16;
    static constexpr int XS = CIN == 32 ? 40 : 8;  // smem pixel stride (elements)
    static constexpr int WS = KP + 8;              // smem weight row stride (elements)
    static constexpr int NT = COUT / 8;
};

template <int CIN, int COUT, int EPI, class T>
__global__ void __launch_bounds__(128) sg_conv_kernel(ConvArgs a) {
    using S = ConvShape<CIN, COUT>;
    __shared__ __align__(16) bf16 s_x[kHaloPix * S::XS];
    __shared__ __align__(16) bf16 s_w[COUT * S::WS];
    __shared__ float s_bias[COUT];
    for (int i = threadIdx.x; i < COUT * (S::KP / 8); i += blockDim.x) {
        const int nn = i / (S::KP / 8), kk = (i % (S::KP / 8)) * 8;
        *reinterpret_cast<uint4*>(&s_w[nn * S::WS + kk]) = *reinterpret_cast<const uint4*>(&a.w[nn * S::KP + kk]);
    }
    if (threadIdx.x < COUT) s_bias[threadIdx.x] = (a.bias && (int)threadIdx.x < a.cout_real) ? a.bias[threadIdx.x] : 0.0F;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (a.w_px + kTileW - 1) / kTileW, tiles_y = (a.h + kTileH - 1) / kTileH;
    const int per_img = tiles_x * tiles_y, tiles = per_img * a.n;
    const long long npx_img = (long long)a.h * a.w_px;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int img = tile / per_img, r = tile - img * per_img;
        const int y0 = (r / tiles_x) * kTileH, x0 = (r % tiles_x) * kTileW;
        __syncthreads();
        const bf16* xin = a.x + (size_t)img * npx_img * CIN;
        for (int i = threadIdx.x; i < kHaloPix * (CIN / 8); i += blockDim.x) {
            const int pix = i / (CIN / 8), q = i - pix * (CIN / 8);
            const int gy = y0 + pix / kHaloW - 1, gx = x0 + pix % kHaloW - 1;
            uint4 v = make_uint4(0U, 0U, 0U, 0U);
            if (gy >= 0 && gy < a.h && gx >= 0 && gx < a.w_px)
                v = *reinterpret_cast<const uint4*>(xin + ((size_t)gy * a.w_px + gx) * CIN + q * 8);
            *reinterpret_cast<uint4*>(&s_x[pix * S::XS + q * 8]) = v;
        }
        __syncthreads();
        float acc[2][S::NT][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int j = 0; j < S::NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[mt][j][e] = 0.0F;
        const int mi = lane >> 3, rr = lane & 7;
#pragma unroll
        for (int ks = 0; ks < S::KSTEPS; ++ks) {
            uint32_t af[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int row = warp * 2 + mt;
                const int m = rr + 8 * (mi & 1);
                int tap, ch;
                if (CIN == 32) {
                    tap = ks >> 1;
                    ch = (ks & 1) * 16 + 8 * (mi >> 1);
                } else {
                    tap = min(2 * ks + (mi >> 1), 8);
                    ch = 0;
                }
                ldsm_x4(af[mt], &s_x[((row + tap / 3) * kHaloW + m + tap % 3) * S::XS + ch]);
            }
            if constexpr (S::NT == 1) {
                uint32_t b0, b1;
                ldsm_x2(b0, b1, &s_w[rr * S::WS + ks * 16 + 8 * (mi & 1)]);
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) mma_bf16(acc[mt][0], af[mt], b0, b1);
            } else {
#pragma unroll
                for (int j = 0; j < S::NT; j += 2) {
                    uint32_t b[4];
                    ldsm_x4(b, &s_w[((j + (mi >> 1)) * 8 + rr) * S::WS + ks * 16 + 8 * (mi & 1)]);
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        mma_bf16(acc[mt][j], af[mt], b[0], b[1]);
                        mma_bf16(acc[mt][j + 1], af[mt], b[2], b[3]);
                    }
                }
            }
        }
        // epilogue: acc[mt][j][0..1] at pixel (row, g), channels 8j+2q+{0,1}; [2..3] at pixel g+8
        const int g = lane >> 2, q = lane & 3;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int gy = y0 + warp * 2 + mt;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int gx = x0 + g + 8 * half;
                const bool inside = gy < a.h && gx < a.w_px;
                const long long p = (long long)img * npx_img + (long long)gy * a.w_px + gx;
                if constexpr (EPI == kEpiRelu || EPI == kEpiMask) {
                    if (inside) {
#pragma unroll
                        for (int j = 0; j < S::NT; ++j) {
                            const int c = 8 * j + 2 * q;
                            float v0 = acc[mt][j][2 * half], v1 = acc[mt][j][2 * half + 1];
                            if constexpr (EPI == kEpiRelu) {
                                v0 = fmaxf(v0 + s_bias[c], 0.0F);
                                v1 = fmaxf(v1 + s_bias[c + 1], 0.0F);
                            } else {
                                const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(a.mask + p * COUT + c);
                                v0 = __low2float(mk) > 0.0F ? v0 : 0.0F;
                                v1 = __high2float(mk) > 0.0F ? v1 : 0.0F;
                            }
                            *reinterpret_cast<__nv_bfloat162*>(a.y + p * COUT + c) = __floats2bfloat162_rn(v0, v1);
                        }
                    }
                } else {
                    // COUT == 8: lanes q = 0 and 1 hold channels 0,1 and 2,3 of the pixel
                    const float c0 = acc[mt][0][2 * half] + s_bias[2 * q];
                    const float c1 = acc[mt][0][2 * half + 1] + s_bias[2 * q + 1];
                    const float c2 = __shfl_down_sync(0xFFFFFFFFU, c0, 1);
                    if (EPI == kEpiResidual) {
                        if (inside && q == 0) {
                            const T* src = static_cast<const T*>(a.rgba) + 4 * p;
                            const Rgba x = load_rgba(src);
                            store_rgb_keep_alpha(static_cast<T*>(a.out) + 4 * p, Rgba{x.r + c0, x.g + c1, x.b + c2, 0.0F},
                                                 src);
                        }
                    } else {
                        float sq = 0.0F;
                        if (inside && q == 0) {
                            const Rgba x = load_rgba(static_cast<const __half*>(a.rgba) + 4 * p);
                            const Rgba t = load_rgba(a.target + 4 * p);
                            const float d0 = (x.r + c0) - t.r, d1 = (x.g + c1) - t.g, d2 = (x.b + c2) - t.b;
                            sq = d0 * d0 + d1 * d1 + d2 * d2;
                            __nv_bfloat162 v[4];
                            v[0] = __floats2bfloat162_rn(d0 * a.grad_scale, d1 * a.grad_scale);
                            v[1] = __floats2bfloat162_rn(d2 * a.grad_scale, 0.0F);
                            v[2] = __floats2bfloat162_rn(0.0F, 0.0F);
                            v[3] = v[2];
                            *reinterpret_cast<uint4*>(a.y + p * 8) = *reinterpret_cast<const uint4*>(v);
                        }
#pragma unroll
                        for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(0xFFFFFFFFU, sq, off);
                        if (lane == 0 && sq != 0.0F) atomicAdd(a.loss, sq);
                    }
                }
            }
        }
    }
}

// ----------------------------------------------------------------- wgrad
struct WgradArgs {
    const bf16* x;   // layer input [n][h][w][CIN]
    const bf16* dy;  // gradient of the layer output (pre-activation) [n][h][w][COUT]
    int n, h, w_px;
    float* dw;       // [COUT][KP] (atomic)
    float* db;       // [COUT] (atomic)
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) sg_wgrad_kernel(WgradArgs a) {
    using S = ConvShape<CIN, COUT>;
    constexpr int DS = COUT == 32 ? 40 : 16;  // dY smem pixel stride; COUT 8 is zero padded to 16 rows of A
    constexpr int MT = COUT == 32 ? 2 : 1;
    constexpr int NTOT = 9 * CIN / 8;         // n8 tiles over the real K
    constexpr int NPW = (NTOT + 3) / 4;       // per warp
    __shared__ __align__(16) bf16 s_x[kHaloPix * S::XS];
    __shared__ __align__(16) bf16 s_d[kTileH * kTileW * DS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (a.w_px + kTileW - 1) / kTileW, tiles_y = (a.h + kTileH - 1) / kTileH;
    const int per_img = tiles_x * tiles_y, tiles = per_img * a.n;
    const long long npx_img = (long long)a.h * a.w_px;
    float acc[MT][NPW][4];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int j = 0; j < NPW; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mt][j][e] = 0.0F;
    float bsum = 0.0F;
    const int mi = lane >> 3, rr = lane & 7;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int img = tile / per_img, r = tile - img * per_img;
        const int y0 = (r / tiles_x) * kTileH, x0 = (r % tiles_x) * kTileW;
        __syncthreads();
        const bf16* xin = a.x + (size_t)img * npx_img * CIN;
        for (int i = threadIdx.x; i < kHaloPix * (CIN / 8); i += blockDim.x) {
            const int pix = i / (CIN / 8), qq = i - pix * (CIN / 8);
            const int gy = y0 + pix / kHaloW - 1, gx = x0 + pix % kHaloW - 1;
            uint4 v = make_uint4(0U, 0U, 0U, 0U);
            if (gy >= 0 && gy < a.h && gx >= 0 && gx < a.w_px)
                v = *reinterpret_cast<const uint4*>(xin + ((size_t)gy * a.w_px + gx) * CIN + qq * 8);
            *reinterpret_cast<uint4*>(&s_x[pix * S::XS + qq * 8]) = v;
        }
        const bf16* din = a.dy + (size_t)img * npx_img * COUT;
        for (int i = threadIdx.x; i < kTileH * kTileW * (DS / 8); i += blockDim.x) {
            const int pix = i / (DS / 8), qq = i - pix * (DS / 8);
            const int gy = y0 + pix / kTileW, gx = x0 + pix % kTileW;
            uint4 v = make_uint4(0U, 0U, 0U, 0U);
            if (qq < COUT / 8 && gy < a.h && gx < a.w_px)
                v = *reinterpret_cast<const uint4*>(din + ((size_t)gy * a.w_px + gx) * COUT + qq * 8);
            *reinterpret_cast<uint4*>(&s_d[pix * DS + qq * 8]) = v;
        }
        __syncthreads();
        if (threadIdx.x < COUT)
            for (int p = 0; p < kTileH * kTileW; ++p) bsum += __bfloat162float(s_d[p * DS + threadIdx.x]);
#pragma unroll
        for (int ks = 0; ks < kTileH; ++ks) {  // k-step = one tile row of 16 pixels
            uint32_t af[MT][4];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
                ldsm_x4_t(af[mt], &s_d[(ks * kTileW + rr + 8 * (mi >> 1)) * DS + 16 * mt + 8 * (mi & 1)]);
#pragma unroll
            for (int j = 0; j < NPW; ++j) {
                const int nt = warp * NPW + j;
                if (nt < NTOT) {
                    const int tap = nt / (CIN / 8), c8 = (nt % (CIN / 8)) * 8;
                    const int px = rr + 8 * (mi & 1);
                    uint32_t b0, b1;
                    ldsm_x2_t(b0, b1, &s_x[((ks + tap / 3) * kHaloW + px + tap % 3) * S::XS + c8]);
#pragma unroll
                    for (int mt = 0; mt < MT; ++mt) mma_bf16(acc[mt][j], af[mt], b0, b1);
                }
            }
        }
    }
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int j = 0; j < NPW; ++j) {
            const int nt = warp * NPW + j;
            if (nt >= NTOT) continue;
            const int k = nt * 8 + 2 * q;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int co = 16 * mt + g + 8 * half;
                if (co < COUT) {
                    atomicAdd(&a.dw[co * S::KP + k], acc[mt][j][2 * half]);
                    atomicAdd(&a.dw[co * S::KP + k + 1], acc[mt][j][2 * half + 1]);
                }
            }
        }
    if (threadIdx.x < COUT) atomicAdd(&a.db[threadIdx.x], bsum);
}

// ------------------------------------------------------------ adam / pack
struct LayerTable {
    int woff[kLayers], boff[kLayers];  // master parameter offsets (blob order)
    int goff[kLayers], gboff[kLayers];  // gradient offsets (padded [COUT][KP], then [COUT])
    int fwoff[kLayers], bwoff[kLayers];  // packed bf16 forward / backward weight offsets
};

// Squared L2 norm of the gradient buffer (one CTA; deterministic order).
__global__ void __launch_bounds__(1024) sg_gradnorm_kernel(const float* __restrict__ g, int n, float* __restrict__ out) {
    __shared__ float part[32];
    float s = 0.0F;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = __fmaf_rn(g[i], g[i], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xFFFFFFFFU, s, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0.0F;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xFFFFFFFFU, s, off);
        if (threadIdx.x == 0) *out = s;
    }
}

// Adam on the master parameters.  The gradient is scaled to a global L2 norm
// of at most `clip`; a step whose gradient norm is not finite is skipped.
__global__ void sg_adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                               const float* __restrict__ grad, const float* __restrict__ gnorm2, LayerTable t,
                               int total, float lr, float b1, float b2, float eps, float c1, float c2, float clip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const float n2 = *gnorm2;
    if (!isfinite(n2)) return;
    const float scale = n2 > clip * clip ? clip * rsqrtf(n2) : 1.0F;
    int l = 0;
    while (l + 1 < kLayers && i >= t.woff[l + 1]) ++l;
    const int ci_r = cin_real(l), co_r = cout_real(l);
    float gr;
    if (i < t.boff[l]) {
        const int r = i - t.woff[l], co = r / (ci_r * 9), rem = r - co * ci_r * 9, ci = rem / 9, tap = rem % 9;
        gr = grad[t.goff[l] + co * kpad(cin_pad(l)) + tap * cin_pad(l) + ci];
    } else {
        gr = grad[t.gboff[l] + (i - t.boff[l])];
    }
    (void)co_r;
    gr *= scale;
    const float mm = b1 * m[i] + (1.0F - b1) * gr;
    const float vv = b2 * v[i] + (1.0F - b2) * gr * gr;
    m[i] = mm;
    v[i] = vv;
    p[i] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
}

// One thread per packed element of layer l's forward [COUT][KP] and backward
// [CIN][KPB] matrices.
__global__ void sg_pack_kernel(const float* __restrict__ p, bf16* __restrict__ packed, LayerTable t) {
    const int l = blockIdx.y;
    const int cinp = cin_pad(l), coutp = cout_pad(l), ci_r = cin_real(l), co_r = cout_real(l);
    const int kp = kpad(cinp), kpb = kpad(coutp);
    const int nf = coutp * kp, nb = l > 0 ? cinp * kpb : 0;
    const float* w = p + t.woff[l];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf + nb; i += gridDim.x * blockDim.x) {
        float v = 0.0F;
        if (i < nf) {
            const int co = i / kp, k = i - co * kp, tap = k / cinp, ci = k - tap * cinp;
            if (co < co_r && ci < ci_r && tap < 9) v = w[(co * ci_r + ci) * 9 + tap];
            packed[t.fwoff[l] + i] = __float2bfloat16_rn(v);
        } else {
            const int j = i - nf, ci = j / kpb, k = j - ci * kpb, tap = k / coutp, co = k - tap * coutp;
            if (co < co_r && ci < ci_r && tap < 9) v = w[(co * ci_r + ci) * 9 + (8 - tap)];
            packed[t.bwoff[l] + j] = __float2bfloat16_rn(v);
        }
    }
}

int grid_for(long long tiles, int per_sm) {
    const long long g = (long long)kSmCount * per_sm;
    return (int)(tiles < g ? tiles : g);
}

}  // namespace sg

using namespace sg;

struct SurrogateNet {
    LayerTable t{};
    int nparams = 0, ngrad = 0, npacked = 0;
    float* d_params = nullptr;  // master FP32 (blob order)
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_grad = nullptr;
    bf16* d_packed = nullptr;
    float* d_loss = nullptr;
    float* d_gnorm = nullptr;    // squared gradient norm of the last step
    float* d_ab = nullptr;       // per-image noise model (a, b)
    int ab_cap = 0;
    int* d_err = nullptr;        // nonzero: a tcgen05 pipeline wait ran out
    bool use_tc = true;          // inference on tcgen05 (else the mma.sync kernels)
    int step = 0;
    // activations for a batch of n x h x w
    long long act_px = 0;
    bf16* d_act = nullptr;       // a0 (8 ch) then a1..a7 (32 ch)
    bf16* d_g[2] = {nullptr, nullptr};  // gradient ping-pong (32 ch)
    bf16* d_gout = nullptr;             // dLoss/dOut (8 ch)
};

static void layout(SurrogateNet* s) {
    int o = 0, go = 0, po = 0;
    for (int l = 0; l < kLayers; ++l) {
        s->t.woff[l] = o;
        o += cout_real(l) * cin_real(l) * 9;
        s->t.boff[l] = o;
        o += cout_real(l);
        s->t.goff[l] = go;
        go += cout_pad(l) * kpad(cin_pad(l));
        s->t.gboff[l] = go;
        go += cout_pad(l);
        s->t.fwoff[l] = po;
        po += cout_pad(l) * kpad(cin_pad(l));
        s->t.bwoff[l] = po;
        if (l > 0) po += cin_pad(l) * kpad(cout_pad(l));
    }
    s->nparams = o;
    s->ngrad = go;
    s->npacked = po;
}

static size_t blob_bytes() {
    SurrogateNet tmp;
    layout(&tmp);
    return sizeof(cpipe_SurrogateHeader) + sizeof(float) * (size_t)tmp.nparams;
}

static cudaError_t pack(SurrogateNet* s, cudaStream_t st) {
    sg_pack_kernel<<<dim3(16, kLayers), 256, 0, st>>>(s->d_params, s->d_packed, s->t);
    return cudaGetLastError();
}

static void free_acts(SurrogateNet* s) {
    cudaFree(s->d_act);
    cudaFree(s->d_g[0]);
    cudaFree(s->d_g[1]);
    cudaFree(s->d_gout);
    s->d_act = s->d_g[0] = s->d_g[1] = s->d_gout = nullptr;
    s->act_px = 0;
}

static cudaError_t ensure_acts(SurrogateNet* s, long long px, bool training) {
    const long long need = training ? px : -px;  // training needs every activation and the gradients
    if (s->act_px == need) return cudaSuccess;
    // inference keeps a larger allocation: the layer buffers are laid out by
    // the call's pixel count inside it (frames of a batch share one network)
    if (!training && s->act_px < 0 && -s->act_px >= px) return cudaSuccess;
    free_acts(s);
    const size_t a0 = (size_t)px * 8, hid = (size_t)px * kCh;
    const size_t acts = training ? a0 + 7 * hid : a0 + 2 * hid;
    cudaError_t e = cudaMalloc(&s->d_act, acts * sizeof(bf16));
    if (e == cudaSuccess && training) e = cudaMalloc(&s->d_g[0], hid * sizeof(bf16));
    if (e == cudaSuccess && training) e = cudaMalloc(&s->d_g[1], hid * sizeof(bf16));
    if (e == cudaSuccess && training) e = cudaMalloc(&s->d_gout, (size_t)px * 8 * sizeof(bf16));
    if (e != cudaSuccess) {
        free_acts(s);
        return e;
    }
    s->act_px = need;
    return cudaSuccess;
}

template <int CIN, int COUT, int EPI, class T>
static void conv(const ConvArgs& a, long long tiles, cudaStream_t st) {
    sg_conv_kernel<CIN, COUT, EPI, T><<<grid_for(tiles, 4), 128, 0, st>>>(a);
}
template <int CIN, int COUT>
static void wgrad(const WgradArgs& a, long long tiles, cudaStream_t st) {
    sg_wgrad_kernel<CIN, COUT><<<grid_for(tiles, 4), 128, 0, st>>>(a);
}

static ConvArgs conv_args(const SurrogateNet* s, int l, const bf16* x, bf16* y, int n, int h, int w) {
    ConvArgs a{};
    a.x = x;
    a.w = s->d_packed + s->t.fwoff[l];
    a.bias = s->d_params + s->t.boff[l];
    a.cout_real = cout_real(l);
    a.n = n;
    a.h = h;
    a.w_px = w;
    a.y = y;
    return a;
}

// Forward through layers 0..6 (ReLU); a0 must hold the prepared input.
// training: activations a1..a7 kept; else ping-pong in two buffers.
static const bf16* forward_hidden(SurrogateNet* s, int n, int h, int w, bool training, cudaStream_t st,
                                  cudaEvent_t* ev = nullptr) {
    const long long px = (long long)n * h * w;
    const long long tiles = (long long)n * ((h + kTileH - 1) / kTileH) * ((w + kTileW - 1) / kTileW);
    const bf16* cur = s->d_act;
    bf16* hid = s->d_act + (size_t)px * 8;
    for (int l = 0; l < kLayers - 1; ++l) {
        bf16* nxt = training ? hid + (size_t)l * px * kCh : hid + (size_t)(l & 1) * px * kCh;
        const ConvArgs a = conv_args(s, l, cur, nxt, n, h, w);
        if (l == 0) conv<8, kCh, kEpiRelu, __half>(a, tiles, st);
        else conv<kCh, kCh, kEpiRelu, __half>(a, tiles, st);
        if (ev) cudaEventRecord(ev[l + 2], st);
        cur = nxt;
    }
    return cur;
}

static cudaError_t upload_ab(SurrogateNet* s, const float* ab, int n, cudaStream_t st) {
    if (n > s->ab_cap) {
        cudaFree(s->d_ab);
        s->d_ab = nullptr;
        s->ab_cap = 0;
        cudaError_t e = cudaMalloc(&s->d_ab, sizeof(float) * 2 * (size_t)n);
        if (e != cudaSuccess) return e;
        s->ab_cap = n;
    }
    return cudaMemcpyAsync(s->d_ab, ab, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice, st);
}

cudaError_t surrogate_reserve(SurrogateNet* s, long long pixels) { return ensure_acts(s, pixels, false); }

// ev (optional): kLayers + 2 events recorded before the input preparation,
// after it, and after each layer.
static cudaError_t infer(SurrogateNet* s, const void* in, void* out, int n, int h, int w, bool f16,
                         const float* d_ab, cudaStream_t st, cudaEvent_t* ev) {
    const long long px = (long long)n * h * w;
    cudaError_t e = ensure_acts(s, px, false);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[0], st);
    if (f16) sg_prep_kernel<__half><<<(unsigned)((px + 255) / 256), 256, 0, st>>>(static_cast<const __half*>(in), s->d_act, d_ab, (long long)h * w, n);
    else sg_prep_kernel<float><<<(unsigned)((px + 255) / 256), 256, 0, st>>>(static_cast<const float*>(in), s->d_act, d_ab, (long long)h * w, n);
    if (ev) cudaEventRecord(ev[1], st);
    if (s->use_tc) {
        const bf16* cur = s->d_act;
        bf16* hid = s->d_act + (size_t)px * 8;
        for (int l = 0; l < kLayers; ++l) {
            TcConvArgs t{};
            t.n = n;
            t.h = h;
            t.w = w;
            t.w_rows = cout_pad(l);
            t.bias = s->d_params + s->t.boff[l];
            t.cout_real = cout_real(l);
            t.err = s->d_err;
            cudaError_t e2;
            if (l < kLayers - 1) {
                bf16* nxt = hid + (size_t)(l & 1) * px * kCh;
                t.y = nxt;
                e2 = tc_conv(cin_pad(l), kCh, 0, f16, cur, s->d_packed + s->t.fwoff[l], t, st);
                cur = nxt;
            } else {
                t.rgba = in;
                t.out = out;
                e2 = tc_conv(kCh, 16, 1, f16, cur, s->d_packed + s->t.fwoff[l], t, st);
            }
            if (e2 != cudaSuccess) return e2;
            if (ev) cudaEventRecord(ev[l + 2], st);
        }
        return cudaGetLastError();
    }
    const bf16* a7 = forward_hidden(s, n, h, w, false, st, ev);
    ConvArgs a = conv_args(s, kLayers - 1, a7, nullptr, n, h, w);
    a.rgba = in;
    a.out = out;
    const long long tiles = (long long)n * ((h + kTileH - 1) / kTileH) * ((w + kTileW - 1) / kTileW);
    if (f16) conv<kCh, 8, kEpiResidual, __half>(a, tiles, st);
    else conv<kCh, 8, kEpiResidual, float>(a, tiles, st);
    if (ev) cudaEventRecord(ev[kLayers + 1], st);
    return cudaGetLastError();
}

cudaError_t surrogate_infer(SurrogateNet* s, const void* in, void* out, int n, int h, int w, bool f16,
                            const float* d_ab, cudaStream_t st) {
    return infer(s, in, out, n, h, w, f16, d_ab, st, nullptr);
}

SurrogateNet* surrogate_new(const void* blob, size_t size, int* status) {
    auto fail = [&](int st, SurrogateNet* s) -> SurrogateNet* {
        if (status) *status = st;
        if (s) surrogate_free(s);
        return nullptr;
    };
    if (!blob || size != blob_bytes()) return fail(CPIPE_BAD_INDEX, nullptr);
    cpipe_SurrogateHeader hd;
    std::memcpy(&hd, blob, sizeof(hd));
    if (std::memcmp(hd.magic, "CPSN", 4) != 0 || hd.version != 1 || hd.layers != kLayers || hd.channels != kCh ||
        hd.in_channels != 4 || hd.out_channels != 3)
        return fail(CPIPE_BAD_INDEX, nullptr);
    auto* s = new (std::nothrow) SurrogateNet();
    if (!s) return fail(CPIPE_OOM, nullptr);
    layout(s);
    const float* params = reinterpret_cast<const float*>(static_cast<const char*>(blob) + sizeof(hd));
    for (int i = 0; i < s->nparams; ++i)
        if (!std::isfinite(params[i])) return fail(CPIPE_BAD_INDEX, s);
    if (cudaMalloc(&s->d_params, sizeof(float) * s->nparams) != cudaSuccess ||
        cudaMalloc(&s->d_packed, sizeof(bf16) * s->npacked) != cudaSuccess ||
        cudaMalloc(&s->d_loss, sizeof(float)) != cudaSuccess || cudaMalloc(&s->d_gnorm, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->d_err, sizeof(int)) != cudaSuccess || cudaMemset(s->d_err, 0, sizeof(int)) != cudaSuccess)
        return fail(CPIPE_OOM, s);
    if (cudaMemcpy(s->d_params, params, sizeof(float) * s->nparams, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(CPIPE_INTERNAL_ERROR, s);
    if (pack(s, nullptr) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return fail(CPIPE_INTERNAL_ERROR, s);
    s->use_tc = tc_conv_available();
    if (status) *status = CPIPE_OK;
    return s;
}

void surrogate_free(SurrogateNet* s) {
    if (!s) return;
    free_acts(s);
    cudaFree(s->d_params);
    cudaFree(s->d_m);
    cudaFree(s->d_v);
    cudaFree(s->d_grad);
    cudaFree(s->d_packed);
    cudaFree(s->d_loss);
    cudaFree(s->d_gnorm);
    cudaFree(s->d_err);
    cudaFree(s->d_ab);
    delete s;
}

}  // namespace cpb

using namespace cpb;

struct cpipe_surrogate {
    SurrogateNet* net;
};

extern "C" {

size_t cpipe_surrogate_blob_size(void) { return blob_bytes(); }

cpipe_surrogate* cpipe_surrogate_create(const void* blob, size_t blob_size, int* status) {
    if (!device_ready()) {
        if (status) *status = CPIPE_INTERNAL_ERROR;
        return nullptr;
    }
    SurrogateNet* n = surrogate_new(blob, blob_size, status);
    if (!n) {
        set_error("surrogate: %s", "bad weight blob or out of device memory");
        return nullptr;
    }
    return new cpipe_surrogate{n};
}

void cpipe_surrogate_destroy(cpipe_surrogate* s) {
    if (!s) return;
    surrogate_free(s->net);
    delete s;
}

int cpipe_surrogate_export(const cpipe_surrogate* s, void* blob, size_t blob_size) {
    if (!s || !blob || blob_size != blob_bytes()) return CPIPE_BAD_INDEX;
    cpipe_SurrogateHeader hd{};
    std::memcpy(hd.magic, "CPSN", 4);
    hd.version = 1;
    hd.layers = kLayers;
    hd.channels = kCh;
    hd.in_channels = 4;
    hd.out_channels = 3;
    std::memcpy(blob, &hd, sizeof(hd));
    return cuda_status(cudaMemcpy(static_cast<char*>(blob) + sizeof(hd), s->net->d_params,
                                  sizeof(float) * s->net->nparams, cudaMemcpyDeviceToHost),
                       "surrogate export");
}

int cpipe_surrogate_denoise(cpipe_surrogate* s, const void* d_in, void* d_out, int n, int width, int height, int f16,
                            const float* noise_ab, void* stream) {
    if (!s || !d_in || !d_out || !noise_ab || n <= 0 || width <= 0 || height <= 0) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = upload_ab(s->net, noise_ab, n, st);
    if (e == cudaSuccess) e = surrogate_infer(s->net, d_in, d_out, n, height, width, f16 != 0, s->net->d_ab, st);
    return cuda_status(e, "surrogate denoise");
}

int cpipe_surrogate_set_engine(cpipe_surrogate* s, int engine) {
    if (!s || (engine != 0 && engine != 1)) return CPIPE_BAD_INDEX;
    if (engine == 1 && !tc_conv_available()) {
        set_error("surrogate: %s", "tensor-map encoder unavailable for the tcgen05 engine");
        return CPIPE_UNSUPPORTED;
    }
    s->net->use_tc = engine == 1;
    return CPIPE_OK;
}

int cpipe_surrogate_check(cpipe_surrogate* s) {
    if (!s) return CPIPE_BAD_INDEX;
    int err = 0;
    const int st = cuda_status(cudaDeviceSynchronize(), "surrogate check");
    if (st != CPIPE_OK) return st;
    if (cudaMemcpy(&err, s->net->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return CPIPE_INTERNAL_ERROR;
    if (err) {
        set_error("surrogate: tcgen05 pipeline wait ran out (%s)", err == 1 ? "input stage" : err == 2 ? "tile load"
                                                                    : err == 3 ? "accumulator" : "MMA completion");
        return CPIPE_INTERNAL_ERROR;
    }
    return CPIPE_OK;
}

int cpipe_surrogate_profile(cpipe_surrogate* s, const void* d_in, void* d_out, int n, int width, int height, int f16,
                            const float* noise_ab, float ms[9], void* stream) {
    if (!s || !d_in || !d_out || !noise_ab || !ms || n <= 0 || width <= 0 || height <= 0) return CPIPE_BAD_INDEX;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[kLayers + 2] = {};
    int status = CPIPE_OK;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) status = CPIPE_INTERNAL_ERROR;
    cudaError_t e = status == CPIPE_OK ? upload_ab(s->net, noise_ab, n, st) : cudaSuccess;
    if (status == CPIPE_OK && e == cudaSuccess)
        e = infer(s->net, d_in, d_out, n, height, width, f16 != 0, s->net->d_ab, st, ev);
    if (status == CPIPE_OK && e == cudaSuccess) e = cudaEventSynchronize(ev[kLayers + 1]);
    if (status == CPIPE_OK && e == cudaSuccess)
        for (int k = 0; k <= kLayers; ++k) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    return status != CPIPE_OK ? status : cuda_status(e, "surrogate profile");
}

int cpipe_surrogate_train_step(cpipe_surrogate* s, const void* d_noisy, const void* d_target, const float* noise_ab,
                               int n, int width, int height, float lr, int update, float* loss, void* stream) {
    if (!s || !d_noisy || !d_target || !noise_ab || n <= 0 || width <= 0 || height <= 0) return CPIPE_BAD_INDEX;
    SurrogateNet* net = s->net;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long px = (long long)n * height * width;
    const long long tiles = (long long)n * ((height + kTileH - 1) / kTileH) * ((width + kTileW - 1) / kTileW);
    cudaError_t e = ensure_acts(net, px, true);
    if (e == cudaSuccess && !net->d_grad) {
        e = cudaMalloc(&net->d_grad, sizeof(float) * net->ngrad);
        if (e == cudaSuccess) e = cudaMalloc(&net->d_m, sizeof(float) * net->nparams);
        if (e == cudaSuccess) e = cudaMalloc(&net->d_v, sizeof(float) * net->nparams);
        if (e == cudaSuccess) e = cudaMemsetAsync(net->d_m, 0, sizeof(float) * net->nparams, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(net->d_v, 0, sizeof(float) * net->nparams, st);
    }
    if (e == cudaSuccess) e = upload_ab(net, noise_ab, n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(net->d_loss, 0, sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(net->d_grad, 0, sizeof(float) * net->ngrad, st);
    if (e != cudaSuccess) return cuda_status(e, "surrogate train setup");
    sg_prep_kernel<__half><<<(unsigned)((px + 255) / 256), 256, 0, st>>>(static_cast<const __half*>(d_noisy), net->d_act,
                                                                        net->d_ab, (long long)height * width, n);
    const bf16* a7 = forward_hidden(net, n, height, width, true, st);
    {
        ConvArgs a = conv_args(net, kLayers - 1, a7, net->d_gout, n, height, width);
        a.rgba = d_noisy;
        a.target = static_cast<const __half*>(d_target);
        a.grad_scale = 2.0F / (3.0F * (float)px);
        a.loss = net->d_loss;
        conv<kCh, 8, kEpiLoss, __half>(a, tiles, st);
    }
    // backward: g = dLoss/d(pre-activation of layer l's output)
    const bf16* act0 = net->d_act;
    auto act = [&](int l) -> const bf16* {  // input of layer l
        return l == 0 ? act0 : net->d_act + (size_t)px * 8 + (size_t)(l - 1) * px * kCh;
    };
    const bf16* g = net->d_gout;
    for (int l = kLayers - 1; l >= 0; --l) {
        WgradArgs wa{act(l), g, n, height, width, net->d_grad + net->t.goff[l], net->d_grad + net->t.gboff[l]};
        if (l == kLayers - 1) wgrad<kCh, 8>(wa, tiles, st);
        else if (l == 0) wgrad<8, kCh>(wa, tiles, st);
        else wgrad<kCh, kCh>(wa, tiles, st);
        if (l == 0) break;
        bf16* gn = net->d_g[l & 1];
        ConvArgs a{};
        a.x = g;
        a.w = net->d_packed + net->t.bwoff[l];
        a.cout_real = kCh;
        a.n = n;
        a.h = height;
        a.w_px = width;
        a.y = gn;
        a.mask = act(l);
        if (l == kLayers - 1) conv<8, kCh, kEpiMask, __half>(a, tiles, st);
        else conv<kCh, kCh, kEpiMask, __half>(a, tiles, st);
        g = gn;
    }
    if (update) {
        net->step += 1;
        const float b1 = 0.9F, b2 = 0.999F, eps = 1e-8F;
        const float c1 = 1.0F / (1.0F - std::pow(b1, (float)net->step));
        const float c2 = 1.0F / (1.0F - std::pow(b2, (float)net->step));
        sg_gradnorm_kernel<<<1, 1024, 0, st>>>(net->d_grad, net->ngrad, net->d_gnorm);
        sg_adam_kernel<<<(net->nparams + 255) / 256, 256, 0, st>>>(net->d_params, net->d_m, net->d_v, net->d_grad,
                                                                   net->d_gnorm, net->t, net->nparams, lr, b1, b2, eps,
                                                                   c1, c2, kGradClip);
        e = pack(net, st);
        if (e != cudaSuccess) return cuda_status(e, "surrogate pack");
    }
    e = cudaGetLastError();
    if (e == cudaSuccess && loss) {
        float sum = 0.0F;
        e = cudaMemcpyAsync(&sum, net->d_loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        *loss = sum / (3.0F * (float)px);
    }
    return cuda_status(e, "surrogate train step");
}

int cpipe_surrogate_gradients(const cpipe_surrogate* s, float* grad, size_t count) {
    if (!s || !grad || !s->net->d_grad || count != (size_t)s->net->nparams) return CPIPE_BAD_INDEX;
    const SurrogateNet* net = s->net;
    std::vector<float> padded(net->ngrad);
    const int st = cuda_status(cudaMemcpy(padded.data(), net->d_grad, sizeof(float) * net->ngrad, cudaMemcpyDeviceToHost),
                               "surrogate gradients");
    if (st != CPIPE_OK) return st;
    for (int l = 0; l < kLayers; ++l) {
        const int ci_r = cin_real(l), co_r = cout_real(l), kp = kpad(cin_pad(l));
        for (int co = 0; co < co_r; ++co) {
            for (int ci = 0; ci < ci_r; ++ci)
                for (int tap = 0; tap < 9; ++tap)
                    grad[net->t.woff[l] + (co * ci_r + ci) * 9 + tap] = padded[net->t.goff[l] + co * kp + tap * cin_pad(l) + ci];
            grad[net->t.boff[l] + co] = padded[net->t.gboff[l] + co];
        }
    }
    return CPIPE_OK;
}

}  // extern "C"
