// Shared device helpers for the sm_100a node kernels.
//
// Numerics contract: the library is compiled with -fmad=false so that every
// a*b+c in a kernel is a separate IEEE multiply and add, like the reference's
// Halide x86-64 target (no FMA feature; reference src/cpipe/nodes/CMakeLists.txt:33)
// and its plain-C++ filters.  Where a fused multiply-add is wanted (float-float
// products) it is written explicitly with __fmaf_rn.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cpb {

constexpr int kSmCount = 148;  // B200: 2 dies x 74 SMs

// Image view handed to every kernel.  Strides are in elements of the storage type.
struct Img {
    void* data;
    int w, h;
    long long row_stride;  // elements between rows
    int pix_stride;        // elements between pixels (channels for interleaved)
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
// std::max / Halide::max semantics: max(a, b) = (a < b) ? b : a.
__device__ __forceinline__ float maxf(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float max0(float x) { return maxf(0.0F, x); }

// Round to binary16 and back (RNE), the inter-node storage rounding.
__device__ __forceinline__ float h16(float v) { return __half2float(__float2half_rn(v)); }

template <bool F16>
__device__ __forceinline__ float rnd(float v) { return F16 ? h16(v) : v; }

// RGBA pixel load/store for the two interleaved storage types.
struct Rgba { float r, g, b, a; };

__device__ __forceinline__ Rgba load_rgba(const __half* p) {
    const uint2 u = *reinterpret_cast<const uint2*>(p);
    const __half2 lo = *reinterpret_cast<const __half2*>(&u.x);
    const __half2 hi = *reinterpret_cast<const __half2*>(&u.y);
    return Rgba{__low2float(lo), __high2float(lo), __low2float(hi), __high2float(hi)};
}
__device__ __forceinline__ Rgba load_rgba(const float* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    return Rgba{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ void store_rgba(__half* p, Rgba v) {
    __half2 lo = __floats2half2_rn(v.r, v.g);
    __half2 hi = __floats2half2_rn(v.b, v.a);
    uint2 u;
    u.x = *reinterpret_cast<uint32_t*>(&lo);
    u.y = *reinterpret_cast<uint32_t*>(&hi);
    *reinterpret_cast<uint2*>(p) = u;
}
__device__ __forceinline__ void store_rgba(float* p, Rgba v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.r, v.g, v.b, v.a);
}
// Store with bit-exact alpha pass-through: the reference copies the alpha
// half unchanged (e.g. wb_dual_illuminant_dispatch.cpp:38-41).
__device__ __forceinline__ void store_rgb_keep_alpha(__half* p, Rgba v, const __half* src) {
    __half2 lo = __floats2half2_rn(v.r, v.g);
    const __half a = src[3];
    __half2 hi = __halves2half2(__float2half_rn(v.b), a);
    uint2 u;
    u.x = *reinterpret_cast<uint32_t*>(&lo);
    u.y = *reinterpret_cast<uint32_t*>(&hi);
    *reinterpret_cast<uint2*>(p) = u;
}
__device__ __forceinline__ void store_rgb_keep_alpha(float* p, Rgba v, const float* src) {
    *reinterpret_cast<float4*>(p) = make_float4(v.r, v.g, v.b, src[3]);
}

template <class T>
__device__ __forceinline__ T* px(const Img& im, int x, int y) {
    return reinterpret_cast<T*>(im.data) + (long long)y * im.row_stride + (long long)x * im.pix_stride;
}
template <class T>
__device__ __forceinline__ Rgba load_clamped(const Img& im, int x, int y) {
    return load_rgba(px<const T>(im, clampi(x, 0, im.w - 1), clampi(y, 0, im.h - 1)));
}

// ---- float-float ("df64") arithmetic: value = hi + lo, |lo| <= ulp(hi)/2 ----
// Used for the OpcodeList3 source coordinates, which the reference evaluates in
// double (dng_opcode_list_3_dispatch.cpp:96-118).  Algorithms: Knuth two-sum and
// the FMA-based exact product (Dekker/Ogita-Rump-Oishi).
struct ff { float hi, lo; };
__device__ __forceinline__ ff ff_from(float a) { return ff{a, 0.0F}; }
__device__ __forceinline__ ff two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return ff{s, e};
}
__device__ __forceinline__ ff quick_two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    return ff{s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ ff ff_add(ff a, ff b) {
    ff s = two_sum(a.hi, b.hi);
    const ff t = two_sum(a.lo, b.lo);
    s.lo = __fadd_rn(s.lo, t.hi);
    s = quick_two_sum(s.hi, s.lo);
    s.lo = __fadd_rn(s.lo, t.lo);
    return quick_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ ff ff_neg(ff a) { return ff{-a.hi, -a.lo}; }
__device__ __forceinline__ ff ff_sub(ff a, ff b) { return ff_add(a, ff_neg(b)); }
__device__ __forceinline__ ff ff_mul(ff a, ff b) {
    const float p = __fmul_rn(a.hi, b.hi);
    float e = __fmaf_rn(a.hi, b.hi, -p);
    e = __fmaf_rn(a.hi, b.lo, e);
    e = __fmaf_rn(a.lo, b.hi, e);
    return quick_two_sum(p, e);
}
// floor of a float-float value, returned as an int; exact for |v| < 2^24.
__device__ __forceinline__ int ff_floor(ff v) {
    float f = floorf(v.hi);
    if (f == v.hi && v.lo < 0.0F) f -= 1.0F;
    return (int)f;
}
// (v - n) rounded to float, for integer n near v.
__device__ __forceinline__ float ff_frac(ff v, int n) {
    const ff d = ff_sub(v, ff_from((float)n));
    return __fadd_rn(d.hi, d.lo);
}

}  // namespace cpb
