// Self-tests of device arithmetic the kernels depend on, run by the test suite.
#include <cstdint>

#include "../../include/cpipe_b200.h"
#include "filters_impl.h"
#include "nodes.cuh"

namespace cpb {
namespace {

// Every binary32 bit pattern x with |x| in const_div's range: const_div(x) must
// equal the IEEE quotient x / d bit for bit.
__global__ void __launch_bounds__(256) const_div_check_kernel(ConstDiv c, unsigned long long* counts) {
    unsigned long long bad = 0, seen = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (1ULL << 32); i += stride) {
        const float x = __uint_as_float((uint32_t)i);
        if (!const_div_ok(x)) continue;
        ++seen;
        if (__float_as_uint(const_div(x, c)) != __float_as_uint(__fdiv_rn(x, c.d))) ++bad;
    }
    atomicAdd(&counts[0], bad);
    atomicAdd(&counts[1], seen);
}

}  // namespace
}  // namespace cpb

extern "C" int cpipe_cuda_selftest_const_division(float divisor, uint64_t* mismatches, uint64_t* checked) {
    using namespace cpb;
    if (mismatches == nullptr || checked == nullptr || !(divisor > 0.0F)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    unsigned long long* d_counts = nullptr;
    cudaError_t e = cudaMalloc(&d_counts, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_status(e, "selftest alloc");
    unsigned long long h[2] = {0, 0};
    e = cudaMemset(d_counts, 0, sizeof(h));
    const ConstDiv c{divisor, (float)(1.0 / (double)divisor)};
    if (e == cudaSuccess) {
        const_div_check_kernel<<<148 * 16, 256>>>(c, d_counts);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d_counts, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d_counts);
    if (e != cudaSuccess) return cuda_status(e, "selftest");
    *mismatches = h[0];
    *checked = h[1];
    return CPIPE_OK;
}
