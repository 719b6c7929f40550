// Host-side launch functions of the per-node kernels (kernels_nodes.cu).  These
// are internal C++ entry points; the public C ABI is in include/cpipe_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "nodes.cuh"

namespace cpb {

struct VignetteParams {
    ff cx, cy, inv_m, k[5];
};

cudaError_t launch_r16u_to_f32(const Img& in, const Img& out, cudaStream_t st);
cudaError_t launch_linearize(const Img& in, const Img& out, const uint16_t* d_table, int n, cudaStream_t st);
cudaError_t launch_blacklevel(const Img& in, const Img& out, const BlackDev& p, cudaStream_t st);
// Device bytes of the per-grid-row table of g at image width w; fill it
// (sets g->hrow / g->hw to point into d_hrows) before launch_gainmap or any
// kernel that evaluates gain_px.
size_t gainmap_hrows_bytes(const GainMapDev& g, int w);
cudaError_t launch_gainmap_hrows(GainMapDev* g, void* d_hrows, int w, cudaStream_t st);
cudaError_t launch_gainmap(const Img& in, const Img& out, const GainMapDev& g, cudaStream_t st);
cudaError_t launch_copy(const void* src, long long src_pitch, void* dst, long long dst_pitch, long long row_bytes,
                        int rows, cudaStream_t st);
cudaError_t launch_demosaic(int algo, const Img& in, const Img& out, bool out_f16, const int cfa[4], cudaStream_t st);
cudaError_t launch_qbc_remosaic(const Img& in, const Img& out, cudaStream_t st);
// Full-form RCD (algo 1) and AMaZE (algo 2) demosaics (demosaic_full.cu); AMaZE
// needs demosaic_full_scratch_bytes(2, w, h) of device scratch (RCD none).
size_t demosaic_full_scratch_bytes(int algo, int w, int h);
cudaError_t launch_demosaic_full(int algo, const Img& in, const Img& out, bool out_f16, const int cfa[4], void* scratch,
                                 cudaStream_t st);
cudaError_t launch_f32_to_rgba16f(const Img& in, const Img& out, cudaStream_t st);
cudaError_t launch_rgba16f_to_unorm(const Img& in, const Img& out, int bits8, cudaStream_t st);
cudaError_t launch_wb(const Img& in, const Img& out, bool f16, const float n[3], cudaStream_t st);
cudaError_t launch_colormatrix(const Img& in, const Img& out, bool f16, const float t[9], cudaStream_t st);
cudaError_t launch_filmic(const Img& in, const Img& out, bool f16, const FilmicDev& p, cudaStream_t st);
// wb.greyworld_auto: per-block exact sums (d_partial: blocks x 4 int64, see
// greyworld_sum_kernel), then v / n per RGB channel of an RGBA16F frame.
constexpr int kGreyworldBlocks = 148 * 8;
cudaError_t launch_greyworld_sums(const Img& in, long long* d_partial, int blocks, cudaStream_t st);
cudaError_t launch_greyworld_apply(const Img& in, const Img& out, const float n[3], cudaStream_t st);
cudaError_t launch_mertens(const Img& under, const Img& normal, const Img& over, const Img& out, float wc, float ws,
                           float we, cudaStream_t st);
cudaError_t launch_aces(const Img& in, const Img& out, bool f16, int enabled, cudaStream_t st);
cudaError_t launch_reinhard(const Img& in, const Img& out, bool f16, float white_point, cudaStream_t st);
cudaError_t launch_usm(const Img& in, const Img& out, bool f16, float strength, int radius, float threshold,
                       cudaStream_t st);
cudaError_t launch_display(const Img& in, const Img& out, unsigned target, cudaStream_t st);
// sharpen.edge_aware_usm on an RGBA16F frame, its f16-rounded result encoded
// for display (target CPIPE_DISPLAY_SRGB / _BT2020_PQ) in the same kernel.
cudaError_t launch_usm_display(const Img& in, const Img& out, float strength, int radius, float threshold,
                               unsigned target, cudaStream_t st);
cudaError_t launch_lut3d(const Img& in, const Img& out, bool f16, const float4* d_lut, int S, int interp,
                         cudaStream_t st);
cudaError_t launch_bm3d_parity(const Img& in, const Img& out, bool f16, float sigma, cudaStream_t st);
cudaError_t launch_wavelet(const Img& in, const Img& out, bool f16, float strength, cudaStream_t st);
cudaError_t launch_guided(const Img& in, const Img& out, bool f16, int radius, float eps, cudaStream_t st);
cudaError_t launch_warp(const Img& in, const Img& out, bool f16, const WarpDev& w, cudaStream_t st);
cudaError_t launch_vignette(const Img& in, const Img& out, bool f16, const VignetteParams& p, cudaStream_t st);
cudaError_t launch_bad_constant(const Img& in, const Img& out, bool f16, float k, cudaStream_t st);
cudaError_t launch_bad_list(const Img& in, const Img& out, bool f16, const uint32_t* d_pts, int npts,
                            const uint32_t* d_rects, int nrects, cudaStream_t st);
cudaError_t launch_trim(const Img& in, const Img& out, bool f16, uint32_t top, uint32_t left, uint32_t bottom,
                        uint32_t right, cudaStream_t st);

}  // namespace cpb
