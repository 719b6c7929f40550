// tcgen05 (sm_100a) convolutions of the surrogate denoiser's inference path.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cpb {

struct TcConvArgs {
    int n, h, w;             // images and their size; activations NHWC bf16
    int w_rows;              // rows of the packed [rows][K] weight matrix (32, or 8 for the last layer)
    const float* bias;       // [cout_real] or null
    int cout_real;
    __nv_bfloat16* y;        // epi 0: output activation, planar [n][4][h][w][8]
    const void* rgba;        // epi 1: the network's RGBA input frame(s)
    void* out;               // epi 1: RGBA output frame(s)
    int* err;                // device int: nonzero when a pipeline wait ran out
};

// True when the driver exposes the tensor-map encoder the kernels need.
bool tc_conv_available();

// cin 8 or 32; n_out 32 (epi 0: bias + ReLU -> bf16) or 16 (epi 1: residual to
// RGBA, binary16 frames when f16 else float32).  wpk: packed forward weights
// [w_rows][9*cin padded to 16].  Activations are planar in 8-channel planes,
// x = [n][cin / 8][h][w][8] (for cin = 8 the same as NHWC), so a TMA box row
// and a warp's store are contiguous runs of whole sectors.
cudaError_t tc_conv(int cin, int n_out, int epi, bool f16, const __nv_bfloat16* x, const __nv_bfloat16* wpk,
                    const TcConvArgs& a, cudaStream_t stream);

}  // namespace cpb
