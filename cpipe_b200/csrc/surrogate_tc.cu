// Surrogate-denoiser convolutions on the 5th-generation tensor cores
// (tcgen05, sm_100a): the inference path of cpipe_b200/csrc/surrogate.cu.
//
// One CTA iteration computes an 8 x 16-pixel output tile (M = 128 pixels) for
// all output channels (N = 32, or 16 for the 3-channel last layer padded with
// zero weights) as an implicit GEMM over K = 9 taps x CIN channels:
//
//  * Activations between the layers are bf16 in 8-channel planes,
//    [n][C/8][h][w][8], so one plane row is a contiguous run of 16-byte pixels
//    (whole sectors for the copy engine and for the epilogue's stores).  TMA
//    (cp.async.bulk.tensor.4d, no multicast) loads the 10 x 18-pixel halo tile
//    as CIN/8 planes ([row][col][8 ch]); out-of-image pixels are zero-filled by
//    the copy, which is the convolution's zero padding.
//  * In that layout the im2col operand of one tap is a K-major, unswizzled
//    shared-memory matrix: 8 consecutive output pixels of a row are one core
//    matrix (16 B apart), the next output row is one halo row further (SBO =
//    160 B) and the second 8-channel chunk of the 16-wide K slice is the next
//    plane (LBO).  So every MMA reads the halo tile in place: no im2col copy.
//  * Weights are staged once per CTA in core-matrix order; one elected thread
//    issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) into TMEM, four
//    accumulator buffers so the epilogues of earlier tiles overlap the MMAs of
//    the next; tcgen05.commit signals the mbarriers that free an input stage
//    and publish an accumulator.
//  * Two epilogue warpgroups take alternate tiles; each warp reads its 32 TMEM
//    lanes (tcgen05.ld 32x32b), adds the bias and applies ReLU (hidden layers:
//    bf16 planes out) or adds the residual to the RGBA input (last layer).
//
// Warp roles: 0-7 epilogue, 8 TMA producer, 9 MMA issuer and TMEM owner.  A
// 3-stage input ring and every mbarrier wait is bounded: a wait that runs out
// records an error code in *err and ends that role, and the CTA still reaches
// its teardown (TMEM released) so the context stays usable.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "../../include/cpipe_node_abi.h"
#include "common.cuh"
#include "surrogate_tc.h"

namespace cpb {
namespace sgtc {

using bf16 = __nv_bfloat16;

constexpr int kTW = 8, kTH = 16;               // output tile: 8 columns x 16 rows = 128 pixels
constexpr int kHW = kTW + 2, kHH = kTH + 2;    // halo tile
constexpr int kPlaneBytes = kHW * kHH * 16;    // one 8-channel plane as TMA writes it (2880 B)
constexpr int kPlaneStride = 2944;             // planes 128-byte aligned
constexpr int kStages = 3;
constexpr int kAcc = 4;                         // TMEM accumulators of up to 32 columns
constexpr int kTmemCols = kAcc * 32;
constexpr int kEpiWarps = 8;                    // two epilogue warpgroups, alternate tiles
constexpr int kThreads = 32 * (kEpiWarps + 2);  // + TMA producer warp + MMA warp
constexpr int kBarBytes = 256;  // mbarriers (2 per stage + 2 per accumulator) and the TMEM address slot
static_assert((2 * kStages + 2 * kAcc) * 8 + 4 <= kBarBytes, "barrier area");
constexpr uint32_t kSpinLimit = 1U << 20;  // try_wait suspends between polls: about a second in all

__host__ __device__ constexpr int kpad(int cin) { return (9 * cin + 15) / 16 * 16; }

// ----------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
// Bounded wait for the completion of phase `parity`; false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = saddr(bar);
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle (SM100 version field 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFU) | ((uint64_t)((lbo >> 4) & 0x3FFFU) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFU) << 32) | (1ULL << 46);
}
// Instruction descriptor: D = F32, A = B = BF16, both K-major, M = 128, N.
template <int N>
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1U << 4) | (1U << 7) | (1U << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(saddr(bar))
                 : "memory");
}

template <int N>
__device__ __forceinline__ void tmem_load(uint32_t taddr, float (&v)[N]);
template <>
__device__ __forceinline__ void tmem_load<32>(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
        "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
template <>
__device__ __forceinline__ void tmem_load<16>(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ int tap_offset(int t) { return ((t / 3) * kHW + (t % 3)) * 16; }

template <int CIN, int N>
struct TcShape {
    static constexpr int PLANES = CIN / 8;
    static constexpr int STAGE = PLANES * kPlaneStride;
    static constexpr int STAGE_TX = PLANES * kPlaneBytes;
    static constexpr int KP = kpad(CIN);
    static constexpr int KG = KP / 8;
    static constexpr int KSLICES = KP / 16;
    static constexpr int WBYTES = N * KP * 2;
    static constexpr int BAR_OFF = kStages * STAGE + WBYTES;
    static constexpr int SMEM = BAR_OFF + kBarBytes + N * 4 + 1024;  // + barriers/TMEM slot, bias, alignment slack
};

enum { kTcRelu = 0, kTcResidual = 1 };

template <int CIN, int N, int EPI, class T>
__global__ void __launch_bounds__(kThreads, 1)
    sg_tc_conv_kernel(const __grid_constant__ CUtensorMap tmap, const bf16* __restrict__ wpk, TcConvArgs a) {
    using S = TcShape<CIN, N>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t* s_in = smem;
    uint8_t* s_w = smem + kStages * S::STAGE;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::BAR_OFF);
    uint64_t* empty = full + kStages;
    uint64_t* accf = empty + kStages;
    uint64_t* acce = accf + kAcc;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(acce + kAcc);
    float* s_bias = reinterpret_cast<float*>(smem + S::BAR_OFF + kBarBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // weights -> core-matrix order: (n-group, k-group) at (kg * N/8 + ng) * 128 B
    for (int i = threadIdx.x; i < N * S::KG; i += blockDim.x) {
        const int n = i / S::KG, kg = i - n * S::KG;
        uint4 v = make_uint4(0U, 0U, 0U, 0U);
        if (n < a.w_rows) v = *reinterpret_cast<const uint4*>(wpk + (size_t)n * S::KP + kg * 8);
        *reinterpret_cast<uint4*>(s_w + (kg * (N / 8) + n / 8) * 128 + (n % 8) * 16) = v;
    }
    if (threadIdx.x < N) s_bias[threadIdx.x] = (a.bias && (int)threadIdx.x < a.cout_real) ? a.bias[threadIdx.x] : 0.0F;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < kAcc; ++s) {
            mbar_init(&accf[s], 1);
            mbar_init(&acce[s], 4);  // the four warps of the warpgroup that drains it
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // generic-proxy writes of the weights must be visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    if (warp == kEpiWarps + 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;

    const int tiles_x = (a.w + kTW - 1) / kTW, tiles_y = (a.h + kTH - 1) / kTH;
    const int per_img = tiles_x * tiles_y, tiles = per_img * a.n;

    if (warp == kEpiWarps) {
        if (lane == 0) {  // TMA producer
            int i = 0;
            for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++i) {
                const int s = i % kStages, u = i / kStages;
                if (u > 0 && !mbar_wait(&empty[s], (uint32_t)(u - 1) & 1U)) {
                    atomicExch(a.err, 1);
                    break;
                }
                const int img = tile / per_img, r = tile - img * per_img;
                const int x0 = (r % tiles_x) * kTW - 1, y0 = (r / tiles_x) * kTH - 1;
                mbar_expect_tx(&full[s], S::STAGE_TX);
#pragma unroll
                for (int p = 0; p < S::PLANES; ++p)
                    tma_load_4d(s_in + s * S::STAGE + p * kPlaneStride, &tmap, &full[s], x0 * 8, y0,
                                img * S::PLANES + p, 0);
            }
        }
    } else if (warp == kEpiWarps + 1) {
        if (lane == 0) {  // MMA issuer
            constexpr uint32_t idesc = instr_desc<N>();
            const uint32_t wbase = saddr(s_w);
            int i = 0;
            for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++i) {
                const int s = i % kStages, u = i / kStages, acc = i % kAcc, v = i / kAcc;
                if (!mbar_wait(&full[s], (uint32_t)u & 1U)) {
                    atomicExch(a.err, 2);
                    break;
                }
                if (v > 0 && !mbar_wait(&acce[acc], (uint32_t)(v - 1) & 1U)) {
                    atomicExch(a.err, 3);
                    break;
                }
                tc_fence_after();
                const uint32_t abase = saddr(s_in + s * S::STAGE);
                const uint32_t d = tmem + (uint32_t)(acc * 32);
#pragma unroll
                for (int ks = 0; ks < S::KSLICES; ++ks) {
                    uint64_t ad;
                    if (CIN == 32) {
                        const int tap = ks >> 1, pair = ks & 1;
                        ad = smem_desc(abase + 2 * pair * kPlaneStride + tap_offset(tap), kPlaneStride, kHW * 16);
                    } else {
                        const int t0 = 2 * ks, t1 = 2 * ks + 1 > 8 ? 8 : 2 * ks + 1;
                        ad = smem_desc(abase + tap_offset(t0), tap_offset(t1) - tap_offset(t0), kHW * 16);
                    }
                    const uint64_t bd = smem_desc(wbase + 2 * ks * (N / 8) * 128, (N / 8) * 128, 128);
                    mma_f16(d, ad, bd, idesc, ks > 0 ? 1U : 0U);
                }
                mma_commit(&empty[s]);
                mma_commit(&accf[acc]);
            }
        }
    } else {  // epilogue warps: TMEM lanes 32*(warp%4) .. +31 = tile pixels; warpgroup warp/4 takes every other tile
        const int m = (warp & 3) * 32 + lane, wg = warp >> 2;
        float bias_r[N];
#pragma unroll
        for (int k = 0; k < N; ++k) bias_r[k] = s_bias[k];
        int i = 0;
        for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++i) {
            if ((i & 1) != wg) continue;
            const int acc = i % kAcc, v = i / kAcc;
            if (!mbar_wait(&accf[acc], (uint32_t)v & 1U)) {
                atomicExch(a.err, 4);
                break;
            }
            tc_fence_after();
            float c[N];
            tmem_load<N>(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(acc * 32), c);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[acc]);
            const int img = tile / per_img, r = tile - img * per_img;
            const int gx = (r % tiles_x) * kTW + (m & 7), gy = (r / tiles_x) * kTH + (m >> 3);
            if (gx >= a.w || gy >= a.h) continue;
            const long long p = ((long long)img * a.h + gy) * a.w + gx;
            if constexpr (EPI == kTcRelu) {
                __nv_bfloat162 o[N / 2];
#pragma unroll
                for (int k = 0; k < N / 2; ++k)
                    o[k] = __floats2bfloat162_rn(fmaxf(c[2 * k] + bias_r[2 * k], 0.0F),
                                                 fmaxf(c[2 * k + 1] + bias_r[2 * k + 1], 0.0F));
                // planar output [img][N / 8][h][w][8]: each store of a warp is four 128-byte rows
                const long long plane = (long long)a.h * a.w;
                uint4* dst = reinterpret_cast<uint4*>(a.y) + (long long)img * (N / 8) * plane + (long long)gy * a.w + gx;
#pragma unroll
                for (int k = 0; k < N / 8; ++k) dst[k * plane] = reinterpret_cast<const uint4*>(o)[k];
            } else {
                const T* src = static_cast<const T*>(a.rgba) + 4 * p;
                const Rgba x = load_rgba(src);
                store_rgb_keep_alpha(static_cast<T*>(a.out) + 4 * p,
                                     Rgba{x.r + (c[0] + bias_r[0]), x.g + (c[1] + bias_r[1]), x.b + (c[2] + bias_r[2]),
                                          0.0F},
                                     src);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == kEpiWarps + 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
    }
}

// ------------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool make_map(CUtensorMap* map, const bf16* act, int cin, int n, int h, int w) {
    auto fn = encode_fn();
    if (!fn) return false;
    // [n][cin / 8][h][w][8] seen as rows of w * 8 elements: a box row is one
    // contiguous 160-byte run (the copy engine fetches whole sectors), and the
    // x coordinate 8 * px is a multiple of 16 bytes for every pixel px
    const cuuint64_t dims[4] = {(cuuint64_t)w * 8, (cuuint64_t)h, (cuuint64_t)n * (cuuint64_t)(cin / 8), 1};
    const cuuint64_t strides[3] = {(cuuint64_t)w * 16, (cuuint64_t)h * w * 16, (cuuint64_t)n * (cin / 8) * h * w * 16};
    const cuuint32_t box[4] = {(cuuint32_t)kHW * 8, (cuuint32_t)kHH, 1, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(act), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CIN, int N, int EPI, class T>
cudaError_t launch(const bf16* x, const bf16* wpk, const TcConvArgs& a, cudaStream_t st) {
    using S = TcShape<CIN, N>;
    static std::once_flag attr;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr, [] {
        attr_err = cudaFuncSetAttribute(sg_tc_conv_kernel<CIN, N, EPI, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        S::SMEM);
    });
    if (attr_err != cudaSuccess) return attr_err;
    CUtensorMap map;
    if (!make_map(&map, x, CIN, a.n, a.h, a.w)) return cudaErrorNotSupported;
    const long long tiles = (long long)a.n * ((a.h + kTH - 1) / kTH) * ((a.w + kTW - 1) / kTW);
    const long long cap = (long long)kSmCount * 2;
    const int grid = (int)(tiles < cap ? tiles : cap);
    sg_tc_conv_kernel<CIN, N, EPI, T><<<grid, kThreads, S::SMEM, st>>>(map, wpk, a);
    return cudaGetLastError();
}

}  // namespace sgtc

bool tc_conv_available() { return sgtc::encode_fn() != nullptr; }

cudaError_t tc_conv(int cin, int n_out, int epi, bool f16, const __nv_bfloat16* x, const __nv_bfloat16* wpk,
                    const TcConvArgs& a, cudaStream_t st) {
    using namespace sgtc;
    if (cin == 8 && n_out == 32 && epi == 0) return launch<8, 32, kTcRelu, __half>(x, wpk, a, st);
    if (cin == 32 && n_out == 32 && epi == 0) return launch<32, 32, kTcRelu, __half>(x, wpk, a, st);
    if (cin == 32 && n_out == 16 && epi == 1)
        return f16 ? launch<32, 16, kTcResidual, __half>(x, wpk, a, st) : launch<32, 16, kTcResidual, float>(x, wpk, a, st);
    return cudaErrorInvalidValue;
}

}  // namespace cpb
