// Seeded synthetic raw frames generated on the GPU (training data for the
// learned surrogate, and large batches for the benchmark).
//
// Scene (the family of the benchmark's CPU generator): linear RGB gradients,
// `rects` axis-aligned rectangles of uniform reflectance in [0.05, 0.9]
// painted in order, and a sinusoidal zone plate in the central third; mosaicked
// with a 2x2 (Bayer) or 4x4 (Quad-Bayer) CFA; noise from the model var = a*x + b in normalised units in its
// Gaussian form x + sqrt(a*x + b) * N(0, 1); scaled above the black level,
// rounded and clamped to the white level.  Random numbers come from the
// counter-based Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011) keyed by the seed, so every
// pixel is independent of the launch shape: rectangle i uses counters
// (i, 1, 0, 0) and (i, 2, 0, 0), pixel p the counter (p mod 2^32, p >> 32, 3, 0);
// N(0,1) by Box-Muller from the first two words.
#include <stdint.h>

#include "../../include/cpipe_b200.h"
#include "common.cuh"
#include "filters_impl.h"

namespace cpb {
namespace {

struct Philox4 {
    uint32_t v[4];
};

__host__ __device__ inline void mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
    const uint64_t p = (uint64_t)a * b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

__host__ __device__ inline Philox4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                          uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53U, c0, &hi0, &lo0);
        mulhilo(0xCD9E8D57U, c2, &hi1, &lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9U;
        k1 += 0xBB67AE85U;
    }
    return Philox4{{c0, c1, c2, c3}};
}

// Uniform in (0, 1] from 32 random bits (exact in float64, then rounded).
__host__ __device__ inline float unit(uint32_t u) { return (float)(((double)u + 1.0) * (1.0 / 4294967296.0)); }

constexpr int kMaxRects = 64;

struct SceneArgs {
    uint16_t* out;
    int w, h, rects;
    uint32_t k0, k1;
    float a, b;
    int black, white;
    int rep;            // CFA repeat: 2 (Bayer) or 4 (Quad Bayer)
    uint8_t cfa[16];    // rep x rep pattern, row-major
    int rx0[kMaxRects], rx1[kMaxRects], ry0[kMaxRects], ry1[kMaxRects];
    float refl[kMaxRects][3];
};

__global__ void scene_raw_kernel(SceneArgs s) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= s.w) return;
    const float fx = s.w > 1 ? (float)x / (float)(s.w - 1) : 0.0F;
    const float fy = s.h > 1 ? (float)y / (float)(s.h - 1) : 0.0F;
    float rgb[3] = {0.15F + 0.55F * fx + 0.1F * fy, 0.2F + 0.4F * fy + 0.15F * fx,
                    0.1F + 0.3F * (1.0F - fx) + 0.25F * fy};
    for (int i = s.rects - 1; i >= 0; --i)
        if (x >= s.rx0[i] && x <= s.rx1[i] && y >= s.ry0[i] && y <= s.ry1[i]) {
            rgb[0] = s.refl[i][0];
            rgb[1] = s.refl[i][1];
            rgb[2] = s.refl[i][2];
            break;
        }
    const float cy = s.h * 0.5F, cx = s.w * 0.5F, rr = fminf((float)s.h, (float)s.w) / 6.0F;
    if (fabsf((float)y - cy) < rr && fabsf((float)x - cx) < rr) {
        const float d2 = (((float)y - cy) * ((float)y - cy) + ((float)x - cx) * ((float)x - cx)) / (rr * rr);
        const float zp = 0.5F + 0.4F * cosf(3.14159265358979F * 0.5F * rr * d2);
        rgb[0] = zp * 0.9F;
        rgb[1] = zp * 0.85F;
        rgb[2] = zp * 0.8F;
    }
    const float clean = fminf(fmaxf(rgb[s.cfa[(y % s.rep) * s.rep + (x % s.rep)]], 0.0F), 1.0F);
    const uint64_t p = (uint64_t)y * (uint64_t)s.w + (uint64_t)x;
    const Philox4 r = philox((uint32_t)p, (uint32_t)(p >> 32), 3U, 0U, s.k0, s.k1);
    const float u1 = unit(r.v[0]), u2 = unit(r.v[1]);
    const float nrm = sqrtf(-2.0F * logf(u1)) * cosf(6.28318530717959F * u2);
    const float noisy = clean + sqrtf(fmaxf(s.a * clean + s.b, 0.0F)) * nrm;
    const float v = rintf(noisy * (float)(s.white - s.black)) + (float)s.black;
    s.out[p] = (uint16_t)fminf(fmaxf(v, 0.0F), (float)s.white);
}

}  // namespace
}  // namespace cpb

using namespace cpb;

extern "C" int cpipe_cuda_scene_raw_cfa(void* d_out, int width, int height, uint64_t seed, int bits, int black,
                                        float noise_a, float noise_b, const uint8_t* cfa, int cfa_repeat, int rects,
                                        void* stream) {
    if (!d_out || width <= 0 || height <= 0 || bits < 8 || bits > 16 || black < 0 || black >= (1 << bits) - 1 ||
        rects < 0 || rects > kMaxRects || !cfa || (cfa_repeat != 2 && cfa_repeat != 4))
        return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    SceneArgs s{};
    s.out = static_cast<uint16_t*>(d_out);
    s.w = width;
    s.h = height;
    s.rects = rects;
    s.k0 = (uint32_t)seed;
    s.k1 = (uint32_t)(seed >> 32);
    s.a = noise_a;
    s.b = noise_b;
    s.black = black;
    s.white = (1 << bits) - 1;
    s.rep = cfa_repeat;
    for (int i = 0; i < cfa_repeat * cfa_repeat; ++i) s.cfa[i] = cfa[i] > 2 ? 1 : cfa[i];
    for (int i = 0; i < rects; ++i) {
        const Philox4 g = philox((uint32_t)i, 1U, 0U, 0U, s.k0, s.k1);
        const int xa = (int)(g.v[0] % (uint32_t)width), xb = (int)(g.v[1] % (uint32_t)width);
        const int ya = (int)(g.v[2] % (uint32_t)height), yb = (int)(g.v[3] % (uint32_t)height);
        s.rx0[i] = xa < xb ? xa : xb;
        s.rx1[i] = xa < xb ? xb : xa;
        s.ry0[i] = ya < yb ? ya : yb;
        s.ry1[i] = ya < yb ? yb : ya;
        const Philox4 c = philox((uint32_t)i, 2U, 0U, 0U, s.k0, s.k1);
        for (int k = 0; k < 3; ++k) s.refl[i][k] = 0.05F + 0.85F * unit(c.v[k]);
    }
    const dim3 grid((unsigned)((width + 255) / 256), (unsigned)height);
    scene_raw_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(s);
    return cuda_status(cudaGetLastError(), "scene_raw");
}

extern "C" int cpipe_cuda_scene_raw(void* d_out, int width, int height, uint64_t seed, int bits, int black,
                                    float noise_a, float noise_b, const uint8_t cfa[4], int rects, void* stream) {
    return cpipe_cuda_scene_raw_cfa(d_out, width, height, seed, bits, black, noise_a, noise_b, cfa, 2, rects, stream);
}
