// Spec-mode guided filter and a-trous wavelet denoiser: host plans and
// launchers shared by the filter entries and the fused chain.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/cpipe_b200_params.h"
#include "common.cuh"

namespace cpb {

constexpr int kGuidedSpecMaxRadius = 16;
constexpr int kAtrousMaxLevels = 6;

// Guided filter with a true (2r+1)^2 box, r in 1..kGuidedSpecMaxRadius; RGBA
// in and out (binary16 when f16, else float32), alpha copied.  scratch:
// guided_spec_scratch_bytes(w, h, r) of device memory, 8-byte aligned.
cudaError_t guided_spec_setup();
size_t guided_spec_scratch_bytes(int w, int h, int radius);
cudaError_t guided_spec_run(const Img& in, const Img& out, bool f16, int radius, float eps, void* scratch,
                            cudaStream_t stream);

struct AtrousPlan {
    int w = 0, h = 0, levels = 0;
    int tiles = 0;               // most partial-sum blocks of any level (one per level-kernel block)
    float noise[kAtrousMaxLevels][3] = {};  // band noise std per level and channel (Y, Co, Cg)
    float strength[3] = {};
    bool copy = false;           // levels 0: output = input
    size_t off_c = 0, off_part = 0, off_thr = 0, bytes = 0;  // off_c: c_1 .. c_L (3 FP32 planes each)
};

// Validates the parameters (CPIPE_BAD_INDEX when out of range) and sizes the
// scratch buffer for a w x h frame.
int atrous_plan(const cpipe_AtrousWaveletParams* p, int w, int h, AtrousPlan* out);
// Kernel attributes (none needed at present; kept for callers that set up once before a capture).
cudaError_t atrous_setup();
// RGBA in -> RGBA out; scratch: plan.bytes of device memory, 256-byte aligned.
cudaError_t atrous_run(const AtrousPlan& plan, const Img& in, const Img& out, bool f16, void* scratch,
                       cudaStream_t stream);

// White-noise gain of level j (1-based) of the B3-spline a-trous transform in
// 2D: the L2 norm of its detail filter (exact, from the filter taps).
double atrous_band_gain(int level);

}  // namespace cpb
