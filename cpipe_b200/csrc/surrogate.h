// Learned surrogate denoiser: the engine shared by the C ABI
// (cpipe_surrogate_*) and the fused chain's denoise_mode 2.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace cpb {

struct SurrogateNet;

// Parses and uploads a weight blob (cpipe_SurrogateHeader + FP32 parameters);
// null with *status set on failure.
SurrogateNet* surrogate_new(const void* blob, size_t size, int* status);
void surrogate_free(SurrogateNet* net);

// Allocates the inference activations for `pixels` (n x h x w) ahead of time.
cudaError_t surrogate_reserve(SurrogateNet* net, long long pixels);

// n dense RGBA frames (binary16 when f16, else float32) of h x w -> the same
// layout; d_ab holds n (a, b) noise-model pairs on the device.  Allocates the
// activation buffers on first use for a given size (reserve them before a
// graph capture).
cudaError_t surrogate_infer(SurrogateNet* net, const void* in, void* out, int n, int h, int w, bool f16,
                            const float* d_ab, cudaStream_t stream);

}  // namespace cpb
