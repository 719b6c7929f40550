// Allocation-free variant of the 3D LUT filter.
//
// cpipe_cuda_color_3d_lut copies the LUT of every call into device memory it
// allocates for that call.  Some callers cannot allocate device memory while
// they process frames: a camera or video loop with a fixed per-frame latency
// budget, where an allocator call may block on or synchronise the device, or a
// host that hands each plugin a fixed device-memory budget at start-up and
// forbids allocations afterwards.  This entry point takes the same arguments
// but keeps the LUT in a fixed scratch array that is part of the library's
// device image (`g_lut_scratch` below), so it allocates nothing.
//
// Costs and limits of that choice:
//  * every GPU that loads the library holds the array (kMaxLutFloats floats,
//    3.3 MB) until the process exits;
//  * the LUT edge length is at most kMaxLutSize (65); larger LUTs are rejected
//    with CPIPE_BAD_INDEX and a message in cpipe_cuda_last_error();
//  * every call shares the one array and it keeps the last call's LUT: two calls
//    whose work overlaps on the GPU (different streams, or different host
//    threads) race on it and may read each other's LUT.  Calls issued in order
//    on one stream are safe.  Nothing in the array has to start at zero: each
//    call overwrites the cells it reads;
//  * input and output must already be device buffers (halide_buffer_t.device);
//    host buffers would need staging memory, so they are rejected with
//    CPIPE_UNSUPPORTED;
//  * the first call on each device resolves the array's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture on that device;
//  * the LUT is copied from the caller's blob with cudaMemcpyAsync on the
//    call's stream.  From ordinary (pageable) host memory the CUDA runtime
//    waits for the work already queued on that stream before it copies, so the
//    call returns only once that earlier work has finished.  A blob in
//    page-locked memory (cudaHostAlloc / cudaHostRegister) is copied without
//    that wait; it must then stay unchanged until the stream reaches the copy;
//  * frames of any height are covered: the grid is at most 65535 rows high and
//    each block row steps through the frame's rows.
#include <cstring>
#include <mutex>

#include "../../include/cpipe_b200.h"
#include "filters_impl.h"
#include "nodes.cuh"

namespace {

constexpr int kMaxLutSize = 65;
constexpr size_t kMaxLutFloats = (size_t)kMaxLutSize * kMaxLutSize * kMaxLutSize * 3;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_lut_scratch[kMaxLutFloats];

std::mutex g_symbol_mutex;
float* g_symbol_ptr[kMaxDevices] = {nullptr};

// Device address of g_lut_scratch on the current device (resolved once per device).
int scratch_for_current_device(float** out) {
    int dev = 0;
    int st = cpb::cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != CPIPE_OK) return st;
    if (dev < 0 || dev >= kMaxDevices) {
        cpb::set_error("%s", "device index beyond the allocation-free LUT's device table");
        return CPIPE_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    if (g_symbol_ptr[dev] == nullptr) {
        void* p = nullptr;
        st = cpb::cuda_status(cudaGetSymbolAddress(&p, g_lut_scratch), "cudaGetSymbolAddress");
        if (st != CPIPE_OK) return st;
        g_symbol_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_symbol_ptr[dev];
    return CPIPE_OK;
}

// LUT cells stored as RGB float triplets, as the reference blob carries them.
struct LutRgbCells {
    const float* __restrict__ lut;
    __device__ __forceinline__ float4 operator()(int i) const {
        const float* c = lut + 3 * i;
        return make_float4(__ldg(c), __ldg(c + 1), __ldg(c + 2), 0.0F);
    }
};

template <class T>
__global__ void __launch_bounds__(256) lut_rgb_kernel(cpb::Img in, cpb::Img out, const float* lut, int S, int interp) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= in.w) return;
    for (int y = blockIdx.y; y < in.h; y += gridDim.y) {
        const T* s = cpb::px<const T>(in, x, y);
        cpb::store_rgb_keep_alpha(cpb::px<T>(out, x, y),
                                  cpb::lut_px_cells(cpb::load_rgba(s), LutRgbCells{lut}, S, interp), s);
    }
}

// A device RGBA buffer as an Img (no staging: host buffers are refused).
int device_rgba(halide_buffer_t* hb, cpb::Img* img, int* elem) {
    if (hb == nullptr) return CPIPE_BAD_INDEX;
    if (hb->type.code != halide_type_float || (hb->type.bits != 16 && hb->type.bits != 32)) return CPIPE_BAD_PRECISION;
    if (hb->dimensions != 3 || hb->dim[2].extent != 4 || hb->dim[2].stride != 1 || hb->dim[0].stride != 4)
        return CPIPE_BAD_INDEX;
    if (hb->device == 0) {
        cpb::set_error("%s", "the allocation-free LUT entry point needs device buffers (halide_buffer_t.device)");
        return CPIPE_UNSUPPORTED;
    }
    const int e = hb->type.bits / 8;
    const long long row = hb->dim[1].stride;
    if (hb->dim[0].extent <= 0 || hb->dim[1].extent <= 0 || row < 4LL * hb->dim[0].extent) return CPIPE_BAD_INDEX;
    if (hb->device % (4 * e) != 0 || (row * e) % (4 * e) != 0) {
        cpb::set_error("%s", "device buffer rows are not aligned for vector access");
        return CPIPE_UNSUPPORTED;
    }
    *img = cpb::Img{reinterpret_cast<void*>(hb->device), hb->dim[0].extent, hb->dim[1].extent, row, 4};
    *elem = e;
    return CPIPE_OK;
}

}  // namespace

extern "C" int cpipe_cuda_color_3d_lut_noalloc(halide_buffer_t* const* inputs, size_t n_inputs,
                                               halide_buffer_t* const* outputs, size_t n_outputs,
                                               const void* param_blob, size_t param_blob_size) {
    if (n_inputs != 1 || n_outputs != 1 || inputs == nullptr || outputs == nullptr) return CPIPE_BAD_INDEX;
    if (param_blob == nullptr || param_blob_size < sizeof(cpipe_Lut3dParamHeader)) return CPIPE_BAD_INDEX;
    cpipe_Lut3dParamHeader hd;
    std::memcpy(&hd, param_blob, sizeof(hd));
    if (hd.size < 2U || hd.value_count == 0U || (hd.value_count % 3U) != 0U) return CPIPE_BAD_INDEX;
    if (param_blob_size != sizeof(hd) + (size_t)hd.value_count * sizeof(float)) return CPIPE_BAD_INDEX;
    if (hd.size > (uint32_t)kMaxLutSize) {
        cpb::set_error("%s", "LUT edge length exceeds 65, the maximum of the allocation-free LUT entry point");
        return CPIPE_BAD_INDEX;
    }
    const size_t floats = (size_t)hd.size * hd.size * hd.size * 3;
    if ((size_t)hd.value_count < floats) return CPIPE_BAD_INDEX;
    if (!cpb::device_ready()) return CPIPE_INTERNAL_ERROR;
    cpb::Img in{}, out{};
    int ein = 0, eout = 0;
    int st = device_rgba(inputs[0], &in, &ein);
    if (st == CPIPE_OK) st = device_rgba(outputs[0], &out, &eout);
    if (st != CPIPE_OK) return st;
    if (in.w != out.w || in.h != out.h) return CPIPE_BAD_INDEX;
    if (ein != eout) return CPIPE_BAD_PRECISION;
    float* scratch = nullptr;
    if ((st = scratch_for_current_device(&scratch)) != CPIPE_OK) return st;
    const cudaStream_t stream = cpb::current_stream();
    const float* values = reinterpret_cast<const float*>(static_cast<const char*>(param_blob) + sizeof(hd));
    st = cpb::cuda_status(cudaMemcpyAsync(scratch, values, floats * sizeof(float), cudaMemcpyHostToDevice, stream),
                          "LUT upload");
    if (st != CPIPE_OK) return st;
    const dim3 grid((unsigned)((in.w + 255) / 256), (unsigned)(in.h < 65535 ? in.h : 65535));
    const int interp = hd.interpolation == 1U ? 1 : 0;
    if (ein == 2) lut_rgb_kernel<__half><<<grid, 256, 0, stream>>>(in, out, scratch, (int)hd.size, interp);
    else lut_rgb_kernel<float><<<grid, 256, 0, stream>>>(in, out, scratch, (int)hd.size, interp);
    st = cpb::cuda_status(cudaGetLastError(), "LUT launch");
    if (st == CPIPE_OK) outputs[0]->flags |= halide_buffer_flag_device_dirty;
    return st;
}
