// Two-stage colour BM3D on sm_100a (aot_id denoise_bm3d_spec).
//
// The algorithm is the published one (Dabov et al., IEEE TIP 2007; colour
// grouping on luminance; parameters of Lebrun, IPOL 2012).  The reference's
// denoise.bm3d node computes a 2x2 box blend instead
// (src/cpipe/nodes/denoise/bm3d_step1_generator.cpp:33-61); that form lives in
// kernels_nodes.cu and the fused chain.  The exact definition shared with the
// FP64 CPU oracle:
//   colour    orthonormal opponent Y=(R+G+B)/sqrt3, U=(R-B)/sqrt2, V=(R-2G+B)/sqrt6
//   refs      8x8 blocks at min(i*nstep, W-8), same in y
//   matching  integer sum of squared differences of q = rint(clamp(L,0,1)*255)
//             (L = ((R+G)+B)*(1/3) for step 1, Y_basic*(1/sqrt3) for step 2)
//             over all positions within +-(ns-1)/2, d <= floor(64*tau);
//             group = reference + best (d, raster) candidates, at most n2,
//             truncated to a power of two
//   transform orthonormal 8x8 DCT-II, then orthonormal Haar along the group
//   step 1    hard threshold |c| > lambda3d*sigma, weight 1/(sigma^2*kept)
//   step 2    Wiener W = B^2/(B^2+sigma^2) from the basic estimate's group,
//             weight 1/(sigma^2*max(sum W^2, 1e-20)) (1 when the sum is 0);
//             the kernels use the weights times sigma^2, which cancels in
//             num / den and keeps FP32 from overflowing
//   aggregate weight x Kaiser(beta) 8x8 window; estimate = num / den
//
// Kernels (all FP32 on the CUDA cores; the transforms use explicit fused
// multiply-adds, the library being built without contraction):
//   bm3d_prep_kernel    RGBA -> Y,U,V planes + 8-bit matching luminance
//   bm3d_match_kernel   one thread per reference block; the search region of a
//                       16x16 tile of references is staged in shared memory as
//                       four byte-shifted word copies so every 4-pixel chunk is
//                       one aligned 32-bit load; distances with byte-SIMD
//                       |a-b| and dp4a (exact integers); a sorted register list
//                       keeps the 15 best (d << 11 | window index) keys
//   bm3d_filter_kernel  one warp per group and channel: lane = (block, row
//                       half); row DCT in registers, column DCT through a warp
//                       shared buffer, Haar along the group with warp shuffles;
//                       aggregation into a shared-memory footprint of the 8x8
//                       reference tile, then added to the frame accumulators.
//                       Tiles are launched in P x P phases so that tiles of one
//                       launch have disjoint footprints: the flush is a plain
//                       read-modify-write, no global atomics.
//   bm3d_basic_kernel   step-1 num/den -> basic estimate + step-2 luminance
//   bm3d_final_kernel   num/den -> RGB, alpha copied
#include "bm3d_spec.h"

#include <math.h>

#include <algorithm>

#include "../../include/cpipe_node_abi.h"
#include "kernels.h"

namespace cpb {
namespace {

constexpr float kInvS3 = 0.57735026918962576451F;
constexpr float kInvS2 = 0.70710678118654752440F;
constexpr float kInvS6 = 0.40824829046386301637F;
constexpr float kMinWienerEnergy = 1e-20F;  // floor of sum W^2 in the step-2 weight

// cos(m * pi / 16) for any integer m.
__host__ __device__ constexpr float cos16(int m) {
    m = ((m % 32) + 32) % 32;
    if (m > 16) m = 32 - m;
    float sgn = 1.0F;
    if (m > 8) {
        m = 16 - m;
        sgn = -1.0F;
    }
    return sgn * (m == 0   ? 1.0F
                  : m == 1 ? 0.98078528040323044913F
                  : m == 2 ? 0.92387953251128675613F
                  : m == 3 ? 0.83146961230254523708F
                  : m == 4 ? 0.70710678118654752440F
                  : m == 5 ? 0.55557023301960222474F
                  : m == 6 ? 0.38268343236508977173F
                  : m == 7 ? 0.19509032201612826785F
                           : 0.0F);
}
// Orthonormal DCT-II basis: dctc(k, n) = a(k) cos((2n+1) k pi / 16).
__host__ __device__ constexpr float dctc(int k, int n) {
    return (k == 0 ? 0.35355339059327376220F : 0.5F) * cos16((2 * n + 1) * k);
}

__device__ __forceinline__ int refpos(int i, int n, int nstep) { return min(i * nstep, n - 8); }

__device__ __forceinline__ uint8_t quantise(float l) {
    l = l > 0.0F ? l : 0.0F;
    l = fminf(l, 1.0F);
    return (uint8_t)__float2int_rn(l * 255.0F);
}

// ------------------------------------------------------------------- prep
// gate (optional): the kernels of a gated run return at once unless *gate != 0.
__device__ __forceinline__ bool gated_off(const int* gate) { return gate != nullptr && *gate == 0; }

template <class T>
__global__ void bm3d_prep_kernel(Img in, float* __restrict__ yuv, uint8_t* __restrict__ q, long long npx,
                                 const int* gate) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= in.w || gated_off(gate)) return;
    const Rgba p = load_rgba(px<const T>(in, x, y));
    const float s = (p.r + p.g) + p.b;
    const long long o = (long long)y * in.w + x;
    yuv[o] = s * kInvS3;
    yuv[npx + o] = (p.r - p.b) * kInvS2;
    yuv[2 * npx + o] = ((p.r + p.b) - 2.0F * p.g) * kInvS6;
    q[o] = quantise(s * (1.0F / 3.0F));
}

// ------------------------------------------------------------------ match
struct MatchArgs {
    int w, h, nrx, nry, nstep, R, ns, n2, wpr, rows;  // h: one image's height (blockIdx.z = image)
    uint32_t dthr;
    const uint8_t* q;
    uint32_t* list;
    uint8_t* cnt;
    const int* gate;
};

constexpr int kMatchTile = 16;  // reference blocks per CTA edge (one thread each)
constexpr int kMatchWprStd = 24;  // words per staged row for the 39x39 window at step 3

// WPR > 0: words per staged row fixed at compile time (the standard 39x39
// window), 0: taken from the arguments.
template <int WPR>
__global__ void __launch_bounds__(256) bm3d_match_kernel(MatchArgs a) {
    extern __shared__ uint32_t s_w[];
    const int wpr = WPR > 0 ? WPR : a.wpr;
    if (gated_off(a.gate)) return;
    const int img = blockIdx.z, row0 = img * a.h;  // images are stacked in rows
    const int i0 = blockIdx.x * kMatchTile, j0 = blockIdx.y * kMatchTile;
    const int iL = min(i0 + kMatchTile - 1, a.nrx - 1), jL = min(j0 + kMatchTile - 1, a.nry - 1);
    const int rx0 = max(0, refpos(i0, a.w, a.nstep) - a.R);
    const int rx1 = min(a.w, refpos(iL, a.w, a.nstep) + a.R + 8);
    const int ry0 = row0 + max(0, refpos(j0, a.h, a.nstep) - a.R);
    const int ry1 = row0 + min(a.h, refpos(jL, a.h, a.nstep) + a.R + 8);
    const int RW = rx1 - rx0, RH = ry1 - ry0;
    const int plane = a.rows * wpr;  // words per shifted copy
    // Copy s, row r, word k holds region bytes 4k+s .. 4k+s+3 (little endian).
    for (int idx = threadIdx.x; idx < 4 * RH * wpr; idx += blockDim.x) {
        const int s = idx / (RH * wpr), rem = idx - s * RH * wpr;
        const int r = rem / wpr, k = rem - r * wpr;
        const uint8_t* row = a.q + (size_t)(ry0 + r) * a.w + rx0;
        const int c0 = 4 * k + s;
        uint32_t word = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int cc = c0 + b;
            word |= (cc < RW ? (uint32_t)row[cc] : 0U) << (8 * b);
        }
        s_w[s * plane + r * wpr + k] = word;
    }
    __syncthreads();
    const int i = i0 + (int)(threadIdx.x % kMatchTile), j = j0 + (int)(threadIdx.x / kMatchTile);
    if (i >= a.nrx || j >= a.nry) return;
    const int x = refpos(i, a.w, a.nstep), y = row0 + refpos(j, a.h, a.nstep);
    uint32_t rw[16];
    {
        const int c = x - rx0;
        const uint32_t* p = s_w + (c & 3) * plane + (y - ry0) * wpr + (c >> 2);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            rw[2 * r] = p[r * wpr];
            rw[2 * r + 1] = p[r * wpr + 1];
        }
    }
    uint32_t keys[15];
#pragma unroll
    for (int m = 0; m < 15; ++m) keys[m] = 0xFFFFFFFFU;
    const int ylo = max(row0, y - a.R), yhi = min(row0 + a.h - 8, y + a.R);
    const int xlo = max(0, x - a.R), xhi = min(a.w - 8, x + a.R);
    if (a.n2 > 1) {
        // Columns of the search window outer, rows inner: the candidate's eight
        // rows sit in a register ring (slot = row & 7, rows counted from ylo), so
        // each candidate loads one new row.  Keys are unique (distance, window
        // index), so the sorted list does not depend on the visiting order.
        const int ny = yhi - ylo + 1;
        for (int xx = xlo; xx <= xhi; ++xx) {
            const int c = xx - rx0;
            const uint32_t* colp = s_w + (c & 3) * plane + (ylo - ry0) * wpr + (c >> 2);
            const uint32_t wcol = (uint32_t)((ylo - y + a.R) * a.ns + a.R - x + xx);
            uint32_t cw[8][2];
#pragma unroll
            for (int r = 0; r < 7; ++r) {
                cw[r][0] = colp[r * wpr];
                cw[r][1] = colp[r * wpr + 1];
            }
            cw[7][0] = cw[7][1] = 0U;
            for (int y0 = 0; y0 < ny; y0 += 8) {
                const uint32_t* rp = colp + (y0 + 7) * wpr;
#pragma unroll
                for (int st = 0; st < 8; ++st) {
                    if (y0 + st < ny) {
                        cw[(st + 7) & 7][0] = rp[st * wpr];
                        cw[(st + 7) & 7][1] = rp[st * wpr + 1];
                        uint32_t d = 0;
#pragma unroll
                        for (int r = 0; r < 8; ++r) {
                            const uint32_t a0 = __vabsdiffu4(rw[2 * r], cw[(st + r) & 7][0]);
                            d = __dp4a(a0, a0, d);
                            const uint32_t a1 = __vabsdiffu4(rw[2 * r + 1], cw[(st + r) & 7][1]);
                            d = __dp4a(a1, a1, d);
                        }
                        const int yy = ylo + y0 + st;
                        if (d <= a.dthr && (xx != x || yy != y)) {
                            uint32_t key = (d << 11) | (wcol + (uint32_t)((y0 + st) * a.ns));
                            if (key < keys[14]) {
#pragma unroll
                                for (int m = 0; m < 15; ++m) {
                                    const uint32_t lo = min(keys[m], key);
                                    key = max(keys[m], key);
                                    keys[m] = lo;
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    const long long ref = ((long long)img * a.nry + j) * a.nrx + i;
    uint32_t* out = a.list + ref * 16;
    out[0] = ((uint32_t)y << 16) | (uint32_t)x;
    int n = 1;
#pragma unroll
    for (int m = 0; m < 15; ++m) {
        if (m < a.n2 - 1 && keys[m] != 0xFFFFFFFFU) {
            const int widx = (int)(keys[m] & 2047U);
            const int dy = widx / a.ns - a.R, dx = widx % a.ns - a.R;
            out[1 + m] = ((uint32_t)(y + dy) << 16) | (uint32_t)(x + dx);
            ++n;
        }
    }
    a.cnt[ref] = (uint8_t)n;
}

// ----------------------------------------------------------------- filter
struct FilterArgs {
    int w, h, nrx, nry, nstep, R, ntx, nty, phases, fw;
    float sigma2, thr;
    long long npx;
    const uint32_t* list;
    const uint8_t* cnt;
    const float* noisy;
    const float* basic;
    float* acc;  // num of channel c at c*npx, den at (3+c)*npx
    const int* gate;
    float kaiser[64];
    float kaiser1[8];
    int np;  // tensor-core form: row pitch of the footprint planes (= 4 mod 32)
};

constexpr int kBufStride = 65;                 // floats per block in a warp buffer
constexpr int kWarpBuf = 16 * kBufStride;      // one group of 16 blocks
constexpr int kFilterWarps = 8;
constexpr int kRefTile = 8;                    // reference blocks per tile edge

__device__ __forceinline__ void haar_forward(float (&Z)[32], int N, int b, bool act) {
    for (int s = 1; s < N; s <<= 1) {
        const bool part = act && (b & (s - 1)) == 0;
        const bool odd = (b & s) != 0;
#pragma unroll
        for (int e = 0; e < 32; ++e) {
            const float p = __shfl_xor_sync(0xFFFFFFFFU, Z[e], 2 * s);
            if (part) Z[e] = odd ? (p - Z[e]) * kInvS2 : (Z[e] + p) * kInvS2;
        }
    }
}
__device__ __forceinline__ void haar_inverse(float (&Z)[32], int N, int b, bool act) {
    for (int s = N >> 1; s >= 1; s >>= 1) {
        const bool part = act && (b & (s - 1)) == 0;
        const bool odd = (b & s) != 0;
#pragma unroll
        for (int e = 0; e < 32; ++e) {
            const float p = __shfl_xor_sync(0xFFFFFFFFU, Z[e], 2 * s);
            if (part) Z[e] = odd ? (p - Z[e]) * kInvS2 : (Z[e] + p) * kInvS2;
        }
    }
}

// 3D transform of the group held by one warp.  Lane (b, hh) loads rows
// 4hh..4hh+3 of block b; on return it holds frequency rows 0..7 of frequency
// columns 4hh..4hh+3 (Z[kr*4 + jj]) after the Haar transform along the group.
__device__ __forceinline__ void forward3d(const float* img, int fw, int bx, int by, int hh, int b, bool act, int N,
                                          float* buf, float (&Z)[32]) {
    if (act) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float* row = img + (by + 4 * hh + r) * fw + bx;
            float v[8];
#pragma unroll
            for (int n = 0; n < 8; ++n) v[n] = row[n];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float s = dctc(k, 0) * v[0];
#pragma unroll
                for (int n = 1; n < 8; ++n) s = __fmaf_rn(dctc(k, n), v[n], s);
                buf[b * kBufStride + (4 * hh + r) * 8 + k] = s;
            }
        }
    }
    __syncwarp();
    float z[8][4];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) z[r][jj] = act ? buf[b * kBufStride + r * 8 + 4 * hh + jj] : 0.0F;
    __syncwarp();
#pragma unroll
    for (int kr = 0; kr < 8; ++kr)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            float s = dctc(kr, 0) * z[0][jj];
#pragma unroll
            for (int r = 1; r < 8; ++r) s = __fmaf_rn(dctc(kr, r), z[r][jj], s);
            Z[kr * 4 + jj] = s;
        }
    haar_forward(Z, N, b, act);
}

template <int STAGE>
__global__ void __launch_bounds__(256, 2) bm3d_filter_kernel(FilterArgs a, int phx, int phy) {
    extern __shared__ float sm[];
    const int c = blockIdx.z % 3, img = blockIdx.z / 3, row0 = img * a.h;  // h: one image's height
    const int tx = blockIdx.x * a.phases + phx, ty = blockIdx.y * a.phases + phy;
    if (tx >= a.ntx || ty >= a.nty || gated_off(a.gate)) return;
    const int i0 = tx * kRefTile, j0 = ty * kRefTile;
    const int i1 = min(i0 + kRefTile, a.nrx), j1 = min(j0 + kRefTile, a.nry);
    const int fx0 = max(0, refpos(i0, a.w, a.nstep) - a.R);
    const int fx1 = min(a.w, refpos(i1 - 1, a.w, a.nstep) + a.R + 8);
    const int fy0 = row0 + max(0, refpos(j0, a.h, a.nstep) - a.R);
    const int fy1 = row0 + min(a.h, refpos(j1 - 1, a.h, a.nstep) + a.R + 8);
    const int fw = fx1 - fx0, fn = fw * (fy1 - fy0);
    const int FN = a.fw * a.fw;
    float* s_num = sm;
    float* s_den = sm + FN;
    float* s_img = sm + 2 * FN;
    float* s_bas = sm + 3 * FN;
    float* s_buf = sm + (STAGE == 2 ? 4 : 3) * FN;
    float* s_k = s_buf + kFilterWarps * kWarpBuf;
    const float* gz = a.noisy + (long long)c * a.npx;
    const float* gb = STAGE == 2 ? a.basic + (long long)c * a.npx : nullptr;
    for (int idx = threadIdx.x; idx < fn; idx += blockDim.x) {
        const int yy = idx / fw, xx = idx - yy * fw;
        const long long o = (long long)(fy0 + yy) * a.w + fx0 + xx;
        s_num[idx] = 0.0F;
        s_den[idx] = 0.0F;
        s_img[idx] = gz[o];
        if (STAGE == 2) s_bas[idx] = gb[o];
    }
    if (threadIdx.x < 64) s_k[threadIdx.x] = a.kaiser[threadIdx.x];
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, b = lane >> 1, hh = lane & 1;
    float* buf = s_buf + warp * kWarpBuf;
    const int nti = i1 - i0, nref = nti * (j1 - j0);
    for (int k = warp; k < nref; k += kFilterWarps) {
        const long long ref = ((long long)img * a.nry + j0 + k / nti) * a.nrx + i0 + k % nti;
        const int cnt = a.cnt[ref];
        const int N = cnt >= 16 ? 16 : cnt >= 8 ? 8 : cnt >= 4 ? 4 : cnt >= 2 ? 2 : 1;
        const bool act = b < N;
        int bx = 0, by = 0;
        if (act) {
            const uint32_t p = a.list[ref * 16 + b];
            bx = (int)(p & 0xFFFFU) - fx0;
            by = (int)(p >> 16) - fy0;
        }
        float Z[32];
        forward3d(s_img, fw, bx, by, hh, b, act, N, buf, Z);
        float wgt;
        if (STAGE == 1) {
            unsigned kept = 0;
#pragma unroll
            for (int e = 0; e < 32; ++e) {
                const bool keep = fabsf(Z[e]) > a.thr;
                Z[e] = keep ? Z[e] : 0.0F;
                kept += keep ? 1U : 0U;
            }
            kept = __reduce_add_sync(0xFFFFFFFFU, kept);
            // weight x sigma^2 (the factor cancels in num / den): 1/kept, or sigma^2
            wgt = kept > 0U ? 1.0F / (float)kept : a.sigma2;
        } else {
            float B[32];
            forward3d(s_bas, fw, bx, by, hh, b, act, N, buf, B);
            float sw2 = 0.0F;
#pragma unroll
            for (int e = 0; e < 32; ++e) {
                const float b2 = B[e] * B[e];
                const float W = b2 / (b2 + a.sigma2);
                Z[e] = Z[e] * W;
                sw2 = __fmaf_rn(W, W, sw2);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) sw2 += __shfl_xor_sync(0xFFFFFFFFU, sw2, off);
            wgt = sw2 > 0.0F ? 1.0F / fmaxf(sw2, kMinWienerEnergy) : a.sigma2;
        }
        haar_inverse(Z, N, b, act);
        if (act) {
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    float s = dctc(0, r) * Z[jj];
#pragma unroll
                    for (int kr = 1; kr < 8; ++kr) s = __fmaf_rn(dctc(kr, r), Z[kr * 4 + jj], s);
                    buf[b * kBufStride + r * 8 + 4 * hh + jj] = s;
                }
        }
        __syncwarp();
        if (act) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = 4 * hh + r;
                float v[8];
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) v[kk] = buf[b * kBufStride + row * 8 + kk];
                float* dn = s_num + (by + row) * fw + bx;
                float* dd = s_den + (by + row) * fw + bx;
#pragma unroll
                for (int n = 0; n < 8; ++n) {
                    float s = dctc(0, n) * v[0];
#pragma unroll
                    for (int kk = 1; kk < 8; ++kk) s = __fmaf_rn(dctc(kk, n), v[kk], s);
                    const float kw = wgt * s_k[row * 8 + n];
                    atomicAdd(dn + n, kw * s);
                    atomicAdd(dd + n, kw);
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    float* gn = a.acc + (long long)c * a.npx;
    float* gd = a.acc + (long long)(3 + c) * a.npx;
    for (int idx = threadIdx.x; idx < fn; idx += blockDim.x) {
        const int yy = idx / fw, xx = idx - yy * fw;
        const long long o = (long long)(fy0 + yy) * a.w + fx0 + xx;
        gn[o] += s_num[idx];
        gd[o] += s_den[idx];
    }
}

// ------------------------------------------- filter on the tensor cores
// The 2D DCTs of a group as separable 8-point transforms on
// mma.sync.m16n8k8 (FP16 operands, FP32 accumulation).  Every operand is split
// hi/lo (x = hi + lo, both FP16): a*b ~ ahi*bhi + alo*bhi + ahi*blo, which keeps
// FP32-level accuracy for the threshold and Wiener decisions.  One m16 tile
// holds two blocks of the group (rows 0-7 block 2t, rows 8-15 block 2t+1):
//   forward  Rc = X^T C^T   rows (block, x), K = y  (columns of each block)
//            H  = Rc^T C^T  rows (block, v), K = x  (rows; Rc^T per 8x8 piece by
//                                                    movmatrix.trans in registers)
//   Haar     along the group, in FP32: a lane holds the same two coefficients
//            (v = g, u = 2q, 2q+1) of all 16 blocks, so every level is register
//            arithmetic (unnormalised butterflies; the normalisation is an exact
//            power of two applied in the shrink step)
//   shrink   hard threshold / Wiener on H (FP32)
//   inverse  Rr = H C       rows (block, v), K = u  (the accumulator is the A
//                                                    operand as it stands)
//            X' = Rr^T C    rows (block, x), K = v
// The DCT matrix enters only as B fragments: four registers per lane.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// 8x8 b16 matrix held as a fragment (row lane/4, columns 2(lane%4)..+1) -> its transpose.
__device__ __forceinline__ uint32_t movtrans(uint32_t x) {
    uint32_t y;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(y) : "r"(x));
    return y;
}
__device__ __forceinline__ void mma1688(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(b0));
}
// FP16 hi/lo halves of two floats, packed as (x0, x1) pairs.
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(x0, x1);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}
// c = A * B over one 8-wide k-step with A = (a0, a1) given as FP32 pairs and B split hi/lo.
__device__ __forceinline__ void mma_split(float (&c)[4], float a00, float a01, float a10, float a11, uint32_t bh,
                                          uint32_t bl) {
    uint32_t h0, l0, h1, l1;
    split2(a00, a01, h0, l0);
    split2(a10, a11, h1, l1);
    c[0] = c[1] = c[2] = c[3] = 0.0F;
    mma1688(c, h0, h1, bh);
    mma1688(c, l0, l1, bh);
    mma1688(c, h0, h1, bl);
}
// The same with A = each 8x8 piece of an accumulator tile transposed.
__device__ __forceinline__ void mma_split_t(float (&c)[4], const float (&r)[4], uint32_t bh, uint32_t bl) {
    uint32_t h0, l0, h1, l1;
    split2(r[0], r[1], h0, l0);
    split2(r[2], r[3], h1, l1);
    h0 = movtrans(h0);
    l0 = movtrans(l0);
    h1 = movtrans(h1);
    l1 = movtrans(l1);
    c[0] = c[1] = c[2] = c[3] = 0.0F;
    mma1688(c, h0, h1, bh);
    mma1688(c, l0, l1, bh);
    mma1688(c, h0, h1, bl);
}

// Single FP16 products (transform 2, the screening form): A rounded once to
// FP16, B = the DCT matrix's FP16 part, FP32 accumulation -- about 2^-11
// relative per product instead of the split form's FP32-level accuracy.
__device__ __forceinline__ uint32_t pack2(float x0, float x1) {
    const __half2 h = __floats2half2_rn(x0, x1);
    return *reinterpret_cast<const uint32_t*>(&h);
}
template <bool SPLIT>
__device__ __forceinline__ void mma_prod(float (&c)[4], float a00, float a01, float a10, float a11, uint32_t bh,
                                         uint32_t bl) {
    if (SPLIT) {
        mma_split(c, a00, a01, a10, a11, bh, bl);
    } else {
        c[0] = c[1] = c[2] = c[3] = 0.0F;
        mma1688(c, pack2(a00, a01), pack2(a10, a11), bh);
    }
}
template <bool SPLIT>
__device__ __forceinline__ void mma_prod_t(float (&c)[4], const float (&r)[4], uint32_t bh, uint32_t bl) {
    if (SPLIT) {
        mma_split_t(c, r, bh, bl);
    } else {
        c[0] = c[1] = c[2] = c[3] = 0.0F;
        mma1688(c, movtrans(pack2(r[0], r[1])), movtrans(pack2(r[2], r[3])), bh);
    }
}

struct DctFrags {
    uint32_t fh, fl;  // B[k][n] = C[n][k] (k = 2q, 2q+1; n = g): products with C^T
    uint32_t ih, il;  // B[k][n] = C[k][n]: products with C
};
__device__ __forceinline__ DctFrags dct_frags(int g, int q) {
    DctFrags d;
    split2(dctc(g, 2 * q), dctc(g, 2 * q + 1), d.fh, d.fl);
    split2(dctc(2 * q, g), dctc(2 * q + 1, g), d.ih, d.il);
    return d;
}

// One level of the unnormalised Haar along the group: block b = 2t + (e >= 2)
// pairs with b + S, (lo, hi) -> (lo + hi, lo - hi).  A level is its own
// transpose, so the inverse runs the same levels in reverse order.  The
// orthonormal transform's coefficient at position b is the unnormalised one
// times 2^(-k/2), k = log2 N for b = 0 and ctz(b) + 1 otherwise: the shrink
// step compares against thresholds scaled by 2^(k/2) (the Wiener step against
// sigma^2 2^k) and multiplies the kept coefficients by 2^-k, exactly, which is
// the forward and the inverse normalisation together.
template <int S>
__device__ __forceinline__ void haar_level(float (&H)[8][4]) {
    if (S == 1) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float lo = H[t][e], hi = H[t][e + 2];
                H[t][e] = lo + hi;
                H[t][e + 2] = lo - hi;
            }
    } else {
        constexpr int D = S / 2;  // distance in t
#pragma unroll
        for (int t = 0; t < 8; t += 2 * D)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float lo = H[t][e], hi = H[t + D][e];
                H[t][e] = lo + hi;
                H[t + D][e] = lo - hi;
            }
    }
}
// k of position b > 0 (compile-time after unrolling); position 0 uses log2 N.
__device__ __forceinline__ constexpr int haar_k(int b) { return (b & 1) ? 1 : (b & 2) ? 2 : (b & 4) ? 3 : 4; }
// 2^e for a small integer e (exact).
__device__ __forceinline__ float exp2i(int e) { return __int_as_float((127 + e) << 23); }

// Forward 2D DCT and Haar of one group of N blocks read from `img` (row pitch P;
// off[b]: block b's offset in the footprint plane).  H[t][e]: block 2t (e < 2) or 2t + 1 (e >= 2),
// coefficient (v = g, u = 2q + (e & 1)).
template <bool SPLIT>
__device__ __forceinline__ void tc_forward(const float* img, int P, const int* off, int N, const DctFrags& d,
                                           float (&H)[8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        H[t][0] = H[t][1] = H[t][2] = H[t][3] = 0.0F;
        if (2 * t >= N) continue;
        float v[2][2] = {{0.0F, 0.0F}, {0.0F, 0.0F}};
#pragma unroll
        for (int hh = 0; hh < 2; ++hh)
            if (2 * t + hh < N) {
                const float* src = img + off[2 * t + hh] + 2 * q * P + g;
                v[hh][0] = src[0];
                v[hh][1] = src[P];
            }
        float rc[4];
        mma_prod<SPLIT>(rc, v[0][0], v[0][1], v[1][0], v[1][1], d.fh, d.fl);  // rows (block, x = g), columns v
        mma_prod_t<SPLIT>(H[t], rc, d.fh, d.fl);                             // rows (block, v = g), columns u
    }
    if (N > 1) haar_level<1>(H);
    if (N > 2) haar_level<2>(H);
    if (N > 4) haar_level<4>(H);
    if (N > 8) haar_level<8>(H);
}

// Inverse Haar and 2D DCT: X[t][e] = block 2t (e < 2) or 2t + 1, pixel (x = g, y = 2q + (e & 1)).
template <bool SPLIT>
__device__ __forceinline__ void tc_inverse(float (&H)[8][4], int N, const DctFrags& d, float (&X)[8][4]) {
    if (N > 8) haar_level<8>(H);
    if (N > 4) haar_level<4>(H);
    if (N > 2) haar_level<2>(H);
    if (N > 1) haar_level<1>(H);
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        X[t][0] = X[t][1] = X[t][2] = X[t][3] = 0.0F;
        if (2 * t >= N) continue;
        float rr[4];
        mma_prod<SPLIT>(rr, H[t][0], H[t][1], H[t][2], H[t][3], d.ih, d.il);  // rows (block, v = g), columns x
        mma_prod_t<SPLIT>(X[t], rr, d.ih, d.il);                             // rows (block, x = g), columns y
    }
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

constexpr int kTcWarps = 8;
constexpr int kStageStride = 72;  // floats per block in a warp's staging buffer (64 + 8: conflict-free float2 stores)
// blocks staged per round: 4 in stage 2 keeps three CTAs of it within one SM's shared memory
__host__ __device__ constexpr int tc_stage_blocks(int stage) { return stage == 2 ? 4 : 8; }

// One launch per stage covers every tile: footprints of neighbouring tiles
// overlap, and the flush adds into the frame accumulators with global
// reductions.  The footprint planes use a row pitch P = 4 mod 32 (>= the
// footprint edge), which makes the column loads of the forward transform and
// the numerator atomics fall in 32 different banks.  Aggregation inside a tile:
//   numerator    the group's inverse-transformed blocks go through the warp's
//                staging buffer ([block][x][y]), so each shared-memory atomic
//                instruction covers 32 distinct pixels (8 rows x 4 columns) of
//                one block;
//   denominator  sum over placements of weight x Kaiser(pixel - origin): the
//                weights are added at the block origins (a weight map, one
//                atomic per block), and the separable Kaiser window is applied
//                to that map at the flush.
template <int STAGE, bool SPLIT>
__global__ void __launch_bounds__(32 * kTcWarps, 3) bm3d_filter_tc_kernel(FilterArgs a) {
    constexpr int SB = tc_stage_blocks(STAGE);
    extern __shared__ __align__(16) float sm[];
    const int c = blockIdx.z % 3, img = blockIdx.z / 3, row0 = img * a.h;
    const int tx = blockIdx.x, ty = blockIdx.y;
    if (tx >= a.ntx || ty >= a.nty || gated_off(a.gate)) return;
    const int i0 = tx * kRefTile, j0 = ty * kRefTile;
    const int i1 = min(i0 + kRefTile, a.nrx), j1 = min(j0 + kRefTile, a.nry);
    const int fx0 = max(0, refpos(i0, a.w, a.nstep) - a.R);
    const int fx1 = min(a.w, refpos(i1 - 1, a.w, a.nstep) + a.R + 8);
    const int fy0 = row0 + max(0, refpos(j0, a.h, a.nstep) - a.R);
    const int fy1 = row0 + min(a.h, refpos(j1 - 1, a.h, a.nstep) + a.R + 8);
    const int fw = fx1 - fx0, fh = fy1 - fy0;
    const int P = a.np, FP = a.fw * P;  // planes [a.fw rows][P]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* s_num = sm;
    float* s_img = sm + FP;                             // after the groups: the weight map, then den
    float* s_bas = s_img + FP;                          // stage 2
    float* s_aux = s_img + (STAGE == 2 ? 2 : 1) * FP;  // staging buffers (stage 1: at the flush the row-filtered map)
    float* s_k = s_aux + (STAGE == 2 ? kTcWarps * SB * kStageStride : max(FP, kTcWarps * SB * kStageStride));
    float* s_k1 = s_k + 64;
    float* s_wgt = s_k1 + 8;  // one aggregation weight per reference block of the tile
    uint32_t* s_list = reinterpret_cast<uint32_t*>((reinterpret_cast<uintptr_t>(s_wgt + kRefTile * kRefTile) + 15) &
                                                   ~(uintptr_t)15);
    uint32_t* s_cnt = s_list + kRefTile * kRefTile * 16;
    int* s_off = reinterpret_cast<int*>(s_cnt + kRefTile * kRefTile);  // [warp][16] block offsets of the group
    const float* gz = a.noisy + (long long)c * a.npx;
    const float* gb = STAGE == 2 ? a.basic + (long long)c * a.npx : nullptr;
    for (int yy = warp; yy < fh; yy += kTcWarps) {
        const long long o = (long long)(fy0 + yy) * a.w + fx0;
        for (int xx = lane; xx < fw; xx += 32) {
            cp_async4(s_img + yy * P + xx, gz + o + xx);
            if (STAGE == 2) cp_async4(s_bas + yy * P + xx, gb + o + xx);
        }
    }
    const int nti = i1 - i0, nref = nti * (j1 - j0);
    for (int i = threadIdx.x; i < nref * 4; i += blockDim.x) {
        const int k = i >> 2;
        const long long ref = ((long long)img * a.nry + j0 + k / nti) * a.nrx + i0 + k % nti;
        cp_async16(s_list + 4 * i, a.list + ref * 16 + 4 * (i & 3));
    }
    if (threadIdx.x < nref) {
        const int k = threadIdx.x;
        s_cnt[k] = a.cnt[((long long)img * a.nry + j0 + k / nti) * a.nrx + i0 + k % nti];
    }
    for (int idx = threadIdx.x; idx < FP; idx += blockDim.x) s_num[idx] = 0.0F;
    if (threadIdx.x < 64) s_k[threadIdx.x] = a.kaiser[threadIdx.x];
    if (threadIdx.x < 8) s_k1[threadIdx.x] = a.kaiser1[threadIdx.x];
    cp_async_wait_all();
    __syncthreads();

    const int g = lane >> 2, q = lane & 3;
    const DctFrags dct = dct_frags(g, q);
    // hard thresholds of the unnormalised coefficients: lambda sigma 2^(k/2)
    const float thr1 = a.thr * 1.41421356237309515F, thr2 = a.thr * 2.0F, thr3 = a.thr * 2.82842712474619030F,
                thr4 = a.thr * 4.0F;
    float* stg = s_aux + warp * (SB * kStageStride);
    const int ly = lane & 7, lx = lane >> 3;  // a lane's pixel in an 8x4 half-block (y, x) and (y, x + 4)
    const float kq0 = s_k[ly * 8 + lx], kq1 = s_k[ly * 8 + lx + 4];
    for (int k = warp; k < nref; k += kTcWarps) {
        const int cnt = (int)s_cnt[k];
        const int N = cnt >= 16 ? 16 : cnt >= 8 ? 8 : cnt >= 4 ? 4 : cnt >= 2 ? 2 : 1;
        const uint32_t* lst = s_list + k * 16;
        int* woff = s_off + warp * 16;
        __syncwarp();
        if (lane < 16) {
            const uint32_t p = lst[lane];
            woff[lane] = ((int)(p >> 16) - fy0) * P + (int)(p & 0xFFFFU) - fx0;
        }
        __syncwarp();
        float H[8][4];
        tc_forward<SPLIT>(s_img, P, woff, N, dct, H);
        const int L = 31 - __clz(N);
        float wgt;
        if (STAGE == 1) {
            const float th0 = L == 0 ? a.thr : L == 1 ? thr1 : L == 2 ? thr2 : L == 3 ? thr3 : thr4;
            const float sc0 = exp2i(-L);
            unsigned kept = 0;
#pragma unroll
            for (int t = 0; t < 8; ++t)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int b = 2 * t + (e >> 1), kb = haar_k(b);
                    const float th = b == 0 ? th0 : kb == 1 ? thr1 : kb == 2 ? thr2 : kb == 3 ? thr3 : thr4;
                    const float sc = b == 0 ? sc0 : (kb == 1 ? 0.5F : kb == 2 ? 0.25F : kb == 3 ? 0.125F : 0.0625F);
                    const bool keep = fabsf(H[t][e]) > th;
                    H[t][e] = keep ? H[t][e] * sc : 0.0F;
                    kept += keep ? 1U : 0U;
                }
            kept = __reduce_add_sync(0xFFFFFFFFU, kept);
            wgt = kept > 0U ? 1.0F / (float)kept : a.sigma2;
        } else {
            float B[8][4];
            tc_forward<SPLIT>(s_bas, P, woff, N, dct, B);
            const float s0 = a.sigma2 * exp2i(L), sc0 = exp2i(-L);
            float sw2 = 0.0F;
#pragma unroll
            for (int t = 0; t < 8; ++t)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int b = 2 * t + (e >> 1), kb = haar_k(b);
                    const float sk = b == 0 ? s0 : a.sigma2 * (float)(1 << kb);
                    const float sc = b == 0 ? sc0 : (kb == 1 ? 0.5F : kb == 2 ? 0.25F : kb == 3 ? 0.125F : 0.0625F);
                    const float b2 = B[t][e] * B[t][e];
                    const float W = __fdividef(b2, b2 + sk);
                    H[t][e] = (H[t][e] * W) * sc;
                    sw2 = __fmaf_rn(W, W, sw2);
                }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) sw2 += __shfl_xor_sync(0xFFFFFFFFU, sw2, off);
            wgt = sw2 > 0.0F ? 1.0F / fmaxf(sw2, kMinWienerEnergy) : a.sigma2;
        }
        if (lane == 0) s_wgt[k] = wgt;
        float X[8][4];
        tc_inverse<SPLIT>(H, N, dct, X);
        // numerator: X -> staging [block][x][y], SB blocks per round -> one block's
        // 8x4 half per atomic instruction
        const float kw0 = wgt * kq0, kw1 = wgt * kq1;
#pragma unroll
        for (int rb = 0; rb < 16 / SB; ++rb) {
            if (SB * rb >= N) break;
#pragma unroll
            for (int tt = 0; tt < SB / 2; ++tt) {
                const int t = rb * (SB / 2) + tt;
                *reinterpret_cast<float2*>(stg + (2 * tt) * kStageStride + g * 8 + 2 * q) = make_float2(X[t][0], X[t][1]);
                *reinterpret_cast<float2*>(stg + (2 * tt + 1) * kStageStride + g * 8 + 2 * q) =
                    make_float2(X[t][2], X[t][3]);
            }
            __syncwarp();
            const int nb = min(SB, N - SB * rb);
            for (int bb = 0; bb < nb; ++bb) {
                float* dst = s_num + woff[SB * rb + bb] + ly * P + lx;
                atomicAdd(dst, kw0 * stg[bb * kStageStride + lane]);
                atomicAdd(dst + 4, kw1 * stg[bb * kStageStride + 32 + lane]);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // weight map at the block origins (in the footprint's own plane, now free)
    float* s_w = s_img;
    for (int idx = threadIdx.x; idx < FP; idx += blockDim.x) s_w[idx] = 0.0F;
    __syncthreads();
    for (int i = threadIdx.x; i < nref * 16; i += blockDim.x) {
        const int k = i >> 4, cnt = (int)s_cnt[k];
        const int N = cnt >= 16 ? 16 : cnt >= 8 ? 8 : cnt >= 4 ? 4 : cnt >= 2 ? 2 : 1;
        if ((i & 15) < N) {
            const uint32_t p = s_list[i];
            atomicAdd(s_w + ((int)(p >> 16) - fy0) * P + (int)(p & 0xFFFFU) - fx0, s_wgt[k]);
        }
    }
    __syncthreads();
    // den = map correlated with the Kaiser window: rows into a free plane, then columns
    float* s_row = STAGE == 2 ? s_bas : s_aux;
    // (the window comes from the kernel arguments; bounds tests only in the first 7 columns / rows)
    for (int yy = warp; yy < fh; yy += kTcWarps)
        for (int xx = lane; xx < fw; xx += 32) {
            const float* wr = s_w + yy * P + xx;
            float h = 0.0F;
            if (xx >= 7) {
#pragma unroll
                for (int u = 0; u < 8; ++u) h = __fmaf_rn(a.kaiser1[u], wr[-u], h);
            } else {
                for (int u = 0; u <= xx; ++u) h = __fmaf_rn(a.kaiser1[u], wr[-u], h);
            }
            s_row[yy * P + xx] = h;
        }
    __syncthreads();
    float* gn = a.acc + (long long)c * a.npx;
    float* gd = a.acc + (long long)(3 + c) * a.npx;
    for (int yy = warp; yy < fh; yy += kTcWarps) {
        const long long o = (long long)(fy0 + yy) * a.w + fx0;
        for (int xx = lane; xx < fw; xx += 32) {
            const float* cr = s_row + yy * P + xx;
            float d = 0.0F;
            if (yy >= 7) {
#pragma unroll
                for (int v = 0; v < 8; ++v) d = __fmaf_rn(a.kaiser1[v], cr[-v * P], d);
            } else {
                for (int v = 0; v <= yy; ++v) d = __fmaf_rn(a.kaiser1[v], cr[-v * P], d);
            }
            if (d > 0.0F) {
                atomicAdd(gn + o + xx, s_num[yy * P + xx]);
                atomicAdd(gd + o + xx, d);
            }
        }
    }
}

// --------------------------------------------------------- basic / final
__global__ void bm3d_basic_kernel(const float* __restrict__ acc, float* __restrict__ basic, uint8_t* __restrict__ q,
                                  long long npx, const int* gate) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npx || gated_off(gate)) return;
    float y = 0.0F;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float v = acc[c * npx + i] / acc[(3 + c) * npx + i];
        basic[c * npx + i] = v;
        if (c == 0) y = v;
    }
    q[i] = quantise(y * kInvS3);
}

template <class T>
__global__ void bm3d_final_kernel(const float* __restrict__ acc, Img in, Img out, long long npx, const int* gate) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= in.w || gated_off(gate)) return;
    const long long i = (long long)y * in.w + x;
    const float Y = acc[i] / acc[3 * npx + i];
    const float U = acc[npx + i] / acc[4 * npx + i];
    const float V = acc[2 * npx + i] / acc[5 * npx + i];
    const float yy = Y * kInvS3, uu = U * kInvS2, vv = V * kInvS6;
    const Rgba o{(yy + uu) + vv, yy - 2.0F * vv, (yy - uu) + vv, 0.0F};
    store_rgb_keep_alpha(px<T>(out, x, y), o, px<const T>(in, x, y));
}

__global__ void bm3d_zero_kernel(float* __restrict__ p, long long n, const int* gate) {
    if (gated_off(gate)) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = 0.0F;
}

double bessel_i0(double x) {
    double sum = 1.0, term = 1.0;
    const double hx = 0.5 * x;
    for (int k = 1; k < 64; ++k) {
        term *= (hx / k) * (hx / k);
        sum += term;
        if (term < 1e-18 * sum) break;
    }
    return sum;
}

int ref_count(int n, int nstep) {
    if (n < 8) return 0;
    int m = (n - 8) / nstep + 1;
    if ((n - 8) % nstep) ++m;
    return m;
}

size_t align256(size_t v) { return (v + 255U) & ~(size_t)255U; }

size_t filter_smem(const Bm3dPlan& p, int stage) {
    return sizeof(float) * ((size_t)(stage == 2 ? 4 : 3) * p.fw * p.fw + (size_t)kFilterWarps * kWarpBuf + 64);
}
size_t match_smem(const Bm3dPlan& p) { return sizeof(uint32_t) * 4 * (size_t)p.mwin * p.mwpr; }
// Row pitch of the tensor-core form's footprint planes: at least fw and 4 mod
// 32 (column loads of eight columns x two rows, and atomics of eight rows x
// four columns, fall in 32 different banks).
int tile_pitch(int fw) { return fw + ((4 - fw) % 32 + 32) % 32; }
size_t filter_tc_smem(const Bm3dPlan& p, int stage) {
    const size_t fp = (size_t)p.fw * tile_pitch(p.fw);
    const size_t stg = (size_t)kTcWarps * tc_stage_blocks(stage) * kStageStride;
    const size_t aux = stage == 2 ? stg : std::max(fp, stg);
    const size_t floats = fp + (stage == 2 ? 2 : 1) * fp + aux + 64 + 8 + kRefTile * kRefTile;  // + Kaiser, its 1D factor, weights
    return sizeof(float) * floats + 16 + sizeof(uint32_t) * kRefTile * kRefTile * 17 + sizeof(int) * kTcWarps * 16;
}

}  // namespace

int bm3d_plan(const cpipe_Bm3dSpecParams* p, int w, int h, Bm3dPlan* out, int batch) {
    if (p == nullptr || out == nullptr) return CPIPE_BAD_INDEX;
    const int n2 = p->n2;
    if (!(n2 == 1 || n2 == 2 || n2 == 4 || n2 == 8 || n2 == 16)) return CPIPE_BAD_INDEX;
    if (p->ns < 1 || p->ns > 45 || (p->ns & 1) == 0) return CPIPE_BAD_INDEX;
    if (p->nstep < 1 || p->nstep > 8) return CPIPE_BAD_INDEX;
    if (!(p->tau_match1 >= 0.0F && p->tau_match1 <= 16000.0F)) return CPIPE_BAD_INDEX;
    if (!(p->tau_match2 >= 0.0F && p->tau_match2 <= 16000.0F)) return CPIPE_BAD_INDEX;
    if (p->stages != 1 && p->stages != 2) return CPIPE_BAD_INDEX;
    if (!(p->lambda3d >= 0.0F) || !(p->kaiser_beta >= 0.0F)) return CPIPE_BAD_INDEX;
    if (p->transform < 0 || p->transform > 2) return CPIPE_BAD_INDEX;
    if (w <= 0 || h <= 0 || batch < 1 || w > 65535 || (long long)h * batch > 65535) return CPIPE_BAD_INDEX;
    Bm3dPlan& q = *out;
    q = Bm3dPlan{};
    q.w = w;
    q.h = h;
    q.batch = batch;
    q.ns = p->ns;
    q.R = (p->ns - 1) / 2;
    q.n2 = n2;
    q.nstep = p->nstep;
    q.stages = p->stages;
    q.tensor = p->transform != 1;
    q.split = p->transform == 0;
    q.sigma = p->sigma;
    q.sigma2 = p->sigma * p->sigma;
    q.thr = p->lambda3d * p->sigma;
    q.dthr[0] = (uint32_t)floor(64.0 * (double)p->tau_match1);
    q.dthr[1] = (uint32_t)floor(64.0 * (double)p->tau_match2);
    q.copy = w < 8 || h < 8 || !(p->sigma > 0.0F) || !(q.sigma2 > 0.0F);
    if (q.copy) return CPIPE_OK;
    double k1[8];
    const double i0b = bessel_i0(p->kaiser_beta);
    for (int n = 0; n < 8; ++n) {
        const double t = (2.0 * n - 7.0) / 7.0;
        k1[n] = bessel_i0(p->kaiser_beta * sqrt(1.0 - t * t)) / i0b;
    }
    for (int v = 0; v < 8; ++v)
        for (int u = 0; u < 8; ++u) q.kaiser[v * 8 + u] = (float)(k1[v] * k1[u]);
    for (int n = 0; n < 8; ++n) q.kaiser1[n] = (float)k1[n];
    q.nrx = ref_count(w, q.nstep);
    q.nry = ref_count(h, q.nstep);
    q.fw = (kRefTile - 1) * q.nstep + 2 * q.R + 8;
    const int span = kRefTile * q.nstep;
    q.phases = (span + 2 * q.R + 8 + span - 1) / span;
    q.ntx = (q.nrx + kRefTile - 1) / kRefTile;
    q.nty = (q.nry + kRefTile - 1) / kRefTile;
    q.mwin = (kMatchTile - 1) * q.nstep + 2 * q.R + 8;
    q.mwpr = (q.mwin + 3) / 4 + 1;
    const size_t npx = (size_t)w * h * batch, nref = (size_t)q.nrx * q.nry * batch;
    size_t o = 0;
    q.off_yuv = o;
    o = align256(o + 3 * npx * sizeof(float));
    q.off_basic = o;
    if (q.stages == 2) o = align256(o + 3 * npx * sizeof(float));
    q.off_acc = o;
    o = align256(o + 6 * npx * sizeof(float));
    q.off_q = o;
    o = align256(o + npx);
    q.off_list = o;
    o = align256(o + nref * 16 * sizeof(uint32_t));
    q.off_cnt = o;
    o = align256(o + nref);
    q.bytes = o;
    return CPIPE_OK;
}

cudaError_t bm3d_setup(const Bm3dPlan& p) {
    if (p.copy) return cudaSuccess;
    static const size_t kSmemOptIn = 227 * 1024;
    const size_t ms = match_smem(p), fs1 = filter_smem(p, 1), fs2 = filter_smem(p, 2);
    if (ms > kSmemOptIn || fs2 > kSmemOptIn) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(bm3d_match_kernel<kMatchWprStd>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(bm3d_match_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(bm3d_filter_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fs1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(bm3d_filter_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fs2);
    if (p.tensor) {
        const size_t t1 = filter_tc_smem(p, 1), t2 = filter_tc_smem(p, 2);
        if (t2 > kSmemOptIn) return cudaErrorInvalidConfiguration;
        const void* k1 = p.split ? (const void*)bm3d_filter_tc_kernel<1, true> : (const void*)bm3d_filter_tc_kernel<1, false>;
        const void* k2 = p.split ? (const void*)bm3d_filter_tc_kernel<2, true> : (const void*)bm3d_filter_tc_kernel<2, false>;
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t1);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t2);
    }
    return e;
}

cudaError_t bm3d_run(const Bm3dPlan& p, const Img& in, const Img& out, bool f16, void* scratch, cudaStream_t st,
                     bool setup, const int* gate) {
    if (p.copy && gate) return cudaSuccess;  // a gated run leaves the output alone
    if (p.copy) {
        const int elem = f16 ? 2 : 4;
        return launch_copy(in.data, in.row_stride * elem, out.data, out.row_stride * elem, (long long)in.w * 4 * elem,
                           in.h, st);
    }
    char* base = static_cast<char*>(scratch);
    float* yuv = reinterpret_cast<float*>(base + p.off_yuv);
    float* basic = reinterpret_cast<float*>(base + p.off_basic);
    float* acc = reinterpret_cast<float*>(base + p.off_acc);
    uint8_t* q = reinterpret_cast<uint8_t*>(base + p.off_q);
    uint32_t* list = reinterpret_cast<uint32_t*>(base + p.off_list);
    uint8_t* cnt = reinterpret_cast<uint8_t*>(base + p.off_cnt);
    const long long npx = (long long)p.w * p.h * p.batch;
    cudaError_t e;
    if (setup && (e = bm3d_setup(p)) != cudaSuccess) return e;
    const size_t ms = match_smem(p), fs1 = filter_smem(p, 1), fs2 = filter_smem(p, 2);
    const size_t ts1 = filter_tc_smem(p, 1), ts2 = filter_tc_smem(p, 2);

    const dim3 pgrid((p.w + 255) / 256, p.h * p.batch);
    if (f16) bm3d_prep_kernel<__half><<<pgrid, 256, 0, st>>>(in, yuv, q, npx, gate);
    else bm3d_prep_kernel<float><<<pgrid, 256, 0, st>>>(in, yuv, q, npx, gate);

    MatchArgs ma{p.w, p.h, p.nrx, p.nry, p.nstep, p.R, p.ns, p.n2, p.mwpr, p.mwin, p.dthr[0], q, list, cnt, gate};
    const dim3 mgrid((p.nrx + kMatchTile - 1) / kMatchTile, (p.nry + kMatchTile - 1) / kMatchTile, p.batch);
    FilterArgs fa{};
    fa.w = p.w;
    fa.h = p.h;
    fa.nrx = p.nrx;
    fa.nry = p.nry;
    fa.nstep = p.nstep;
    fa.R = p.R;
    fa.ntx = p.ntx;
    fa.nty = p.nty;
    fa.phases = p.phases;
    fa.fw = p.fw;
    fa.sigma2 = p.sigma2;
    fa.thr = p.thr;
    fa.npx = npx;
    fa.list = list;
    fa.cnt = cnt;
    fa.noisy = yuv;
    fa.basic = basic;
    fa.acc = acc;
    fa.gate = gate;
    for (int i = 0; i < 64; ++i) fa.kaiser[i] = p.kaiser[i];
    for (int i = 0; i < 8; ++i) fa.kaiser1[i] = p.kaiser1[i];
    fa.np = tile_pitch(p.fw);
    FilterArgs ta = fa;  // tensor-core form: one launch over all tiles (global reductions at the flush)
    ta.phases = 1;
    const dim3 tgrid(p.ntx, p.nty, 3 * p.batch);
    const dim3 fgrid((p.ntx + p.phases - 1) / p.phases, (p.nty + p.phases - 1) / p.phases, 3 * p.batch);

    for (int stage = 1; stage <= p.stages; ++stage) {
        bm3d_zero_kernel<<<kSmCount * 8, 256, 0, st>>>(acc, 6 * npx, gate);
        ma.dthr = p.dthr[stage - 1];
        if (p.mwpr == kMatchWprStd) bm3d_match_kernel<kMatchWprStd><<<mgrid, kMatchTile * kMatchTile, ms, st>>>(ma);
        else bm3d_match_kernel<0><<<mgrid, kMatchTile * kMatchTile, ms, st>>>(ma);
        if (p.tensor) {
            if (p.split) {
                if (stage == 1) bm3d_filter_tc_kernel<1, true><<<tgrid, 32 * kTcWarps, ts1, st>>>(ta);
                else bm3d_filter_tc_kernel<2, true><<<tgrid, 32 * kTcWarps, ts2, st>>>(ta);
            } else {
                if (stage == 1) bm3d_filter_tc_kernel<1, false><<<tgrid, 32 * kTcWarps, ts1, st>>>(ta);
                else bm3d_filter_tc_kernel<2, false><<<tgrid, 32 * kTcWarps, ts2, st>>>(ta);
            }
        } else {
            for (int py = 0; py < p.phases; ++py)
                for (int pxh = 0; pxh < p.phases; ++pxh) {
                    if (stage == 1) bm3d_filter_kernel<1><<<fgrid, 32 * kFilterWarps, fs1, st>>>(fa, pxh, py);
                    else bm3d_filter_kernel<2><<<fgrid, 32 * kFilterWarps, fs2, st>>>(fa, pxh, py);
                }
        }
        if (stage == 1 && p.stages == 2)
            bm3d_basic_kernel<<<(unsigned)((npx + 255) / 256), 256, 0, st>>>(acc, basic, q, npx, gate);
    }
    if (f16) bm3d_final_kernel<__half><<<pgrid, 256, 0, st>>>(acc, in, out, npx, gate);
    else bm3d_final_kernel<float><<<pgrid, 256, 0, st>>>(acc, in, out, npx, gate);
    return cudaGetLastError();
}

}  // namespace cpb
