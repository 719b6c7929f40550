// Two-stage colour BM3D ("spec mode", aot_id denoise_bm3d_spec): host plan
// and launcher shared by the filter entry and the fused chain.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/cpipe_b200_params.h"
#include "common.cuh"

namespace cpb {

struct Bm3dPlan {
    int w = 0, h = 0;     // one image (a batch stacks `batch` images in rows)
    int batch = 1;
    int nrx = 0, nry = 0;  // reference blocks per axis
    int ns = 0, R = 0, n2 = 0, nstep = 0, stages = 0;
    float sigma = 0.0F, sigma2 = 0.0F, thr = 0.0F;
    uint32_t dthr[2] = {0, 0};  // integer match thresholds (64 * tau)
    float kaiser[64] = {};
    float kaiser1[8] = {};  // the 1D window: kaiser[v * 8 + u] = kaiser1[v] * kaiser1[u] (rounded from double)
    int fw = 0;            // filter footprint edge bound (pixels)
    int phases = 0;        // filter launch phases per axis
    int ntx = 0, nty = 0;  // filter tiles (8x8 reference blocks each)
    int mwin = 0, mwpr = 0;  // match tile region edge bound, words per smem row
    bool copy = false;       // image below 8x8 or sigma <= 0: output = input
    bool tensor = true;      // transforms on the tensor cores or FP32 CUDA cores
    bool split = true;       // tensor cores: FP16 hi/lo split products (else single FP16 products)
    size_t off_yuv = 0, off_basic = 0, off_acc = 0, off_q = 0, off_list = 0, off_cnt = 0, bytes = 0;
};

// Validates the parameters (CPIPE_BAD_INDEX when out of range) and sizes the
// scratch buffer for `batch` w x h images stacked in rows (batch * h <= 65535);
// each image is denoised on its own (search windows stay inside it).
int bm3d_plan(const cpipe_Bm3dSpecParams* p, int w, int h, Bm3dPlan* out, int batch = 1);

// Sets the kernels' shared-memory limits for the plan (host-side; call
// before capturing bm3d_run into a graph).
cudaError_t bm3d_setup(const Bm3dPlan& plan);

// RGBA in -> RGBA out (both binary16 when f16, else float32; alpha copied);
// for a batch, `in` and `out` span all batch * h rows.  scratch: plan.bytes of
// device memory, 256-byte aligned.  setup = true runs bm3d_setup first.  gate
// (optional device int): every kernel returns at once while *gate == 0, so
// the run can sit in a graph and happen only when a device-side test asks.
cudaError_t bm3d_run(const Bm3dPlan& plan, const Img& in, const Img& out, bool f16, void* scratch,
                     cudaStream_t stream, bool setup = true, const int* gate = nullptr);

}  // namespace cpb
