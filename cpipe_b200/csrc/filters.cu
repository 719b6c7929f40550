// The filter seam: one extern "C" function per reference aot_id, with the
// reference's HalideParamFilterEntry / HalideFilterEntry signatures
// (src/cpipe/runtime/HalideFilterRegistry.hpp:18-21), so a reference runtime can
// register them in place of the Halide/C++ CPU filters
// (ComputeContext::register_halide_param_filter, ComputeContext.cpp:16-23).
//
// Buffers: a halide_buffer_t with device != 0 is CUDA device memory and is
// processed in place, asynchronously, on the calling thread's current stream
// (cpipe_cuda_set_stream).  Otherwise its host pointer is staged through device
// memory and the call returns only after the result is back in host memory,
// which is what a CPU-filter caller expects.  There is no CPU code path: if no
// CUDA device is usable, every filter returns CPIPE_INTERNAL_ERROR.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "bm3d_spec.h"
#include "spec_denoise.h"
#include "filters_impl.h"
#include "kernels.h"

namespace cpb {

// ------------------------------------------------------------ thread state
namespace {
thread_local cudaStream_t g_stream = nullptr;
thread_local char g_err[512] = {0};
}  // namespace

void set_error(const char* fmt, const char* detail) {
    std::snprintf(g_err, sizeof(g_err), fmt, detail ? detail : "");
}
cudaStream_t current_stream() { return g_stream; }

int cuda_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return CPIPE_OK;
    std::snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
    return CPIPE_INTERNAL_ERROR;
}

// ---------------------------------------------------------------- binding
int Call::bind(halide_buffer_t* hb, Kind kind, bool is_output, Bound* out) {
    if (hb == nullptr) return CPIPE_BAD_INDEX;
    const int code = hb->type.code, bits = hb->type.bits;
    int elem = bits / 8, ch = 1;
    switch (kind) {
        case Kind::BayerU16:
            if (code != halide_type_uint || bits != 16) return CPIPE_BAD_PRECISION;
            if (hb->dimensions != 2) return CPIPE_BAD_INDEX;
            break;
        case Kind::BayerF32:
            if (code != halide_type_float || bits != 32) return CPIPE_BAD_PRECISION;
            if (hb->dimensions != 2) return CPIPE_BAD_INDEX;
            break;
        case Kind::Rgba:
            if (code != halide_type_float || (bits != 16 && bits != 32)) return CPIPE_BAD_PRECISION;
            if (hb->dimensions != 3 || hb->dim[2].extent != 4 || hb->dim[2].stride != 1) return CPIPE_BAD_INDEX;
            ch = 4;
            break;
        case Kind::RgbaU8:
            if (code != halide_type_uint || bits != 8) return CPIPE_BAD_PRECISION;
            if (hb->dimensions != 3 || hb->dim[2].extent != 4 || hb->dim[2].stride != 1) return CPIPE_BAD_INDEX;
            ch = 4;
            break;
        case Kind::RgbaU16:
            if (code != halide_type_uint || bits != 16) return CPIPE_BAD_PRECISION;
            if (hb->dimensions != 3 || hb->dim[2].extent != 4 || hb->dim[2].stride != 1) return CPIPE_BAD_INDEX;
            ch = 4;
            break;
        case Kind::Any:
            if (bits % 8 != 0 || bits == 0) return CPIPE_BAD_PRECISION;
            if (hb->dimensions == 3) {
                if (hb->dim[2].stride != 1) return CPIPE_BAD_INDEX;
                ch = hb->dim[2].extent;
            } else if (hb->dimensions != 2) {
                return CPIPE_BAD_INDEX;
            }
            break;
    }
    const int w = hb->dim[0].extent, h = hb->dim[1].extent;
    if (w <= 0 || h <= 0) return CPIPE_BAD_INDEX;
    if (hb->dim[0].stride != ch) {
        set_error("%s", "interleaved pixels with pixel stride == channel count are required");
        return CPIPE_UNSUPPORTED;
    }
    const long long row_stride = hb->dim[1].stride;
    if (row_stride < (long long)w * ch) return CPIPE_BAD_INDEX;
    // Vector loads need 8-byte (RGBA f16) / 16-byte (RGBA f32) aligned pixels.
    const int align = (ch == 4 && kind != Kind::Any) ? elem * 4 : elem;
    Bound b;
    b.hb = hb;
    b.elem = elem;
    b.ch = ch;
    b.is_output = is_output;
    const bool on_device = hb->device != 0 && !(hb->flags & halide_buffer_flag_host_dirty && hb->host);
    if (on_device) {
        if ((hb->device % align) != 0 || ((row_stride * elem) % align) != 0) {
            set_error("%s", "device buffer rows are not aligned for vector access");
            return CPIPE_UNSUPPORTED;
        }
        b.img = Img{reinterpret_cast<void*>(hb->device), w, h, row_stride, ch};
        b.staged = false;
    } else {
        if (hb->host == nullptr) return CPIPE_BAD_INDEX;
        const size_t bytes = (size_t)w * h * ch * elem;
        void* d = nullptr;
        int st = alloc(bytes, &d);
        if (st != CPIPE_OK) return st;
        b.img = Img{d, w, h, (long long)w * ch, ch};
        b.staged = true;
        if (!is_output) {
            st = cuda_status(cudaMemcpy2DAsync(d, (size_t)w * ch * elem, hb->host, (size_t)row_stride * elem,
                                               (size_t)w * ch * elem, (size_t)h, cudaMemcpyHostToDevice, stream),
                             "stage in");
            if (st != CPIPE_OK) return st;
        }
        staged_any = true;
    }
    bounds.push_back(b);
    *out = b;
    return CPIPE_OK;
}

// The filters' per-call scratch comes from a device memory pool of the
// library's own that keeps what it has reserved (release threshold: never),
// so a call does not map fresh device memory after every synchronisation;
// cpipe_cuda_trim_scratch returns it.  One pool per device, made on first use.
static cudaError_t scratch_pool(cudaMemPool_t* out) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    pools[dev] = pool;
    *out = pool;
    return cudaSuccess;
}

int Call::alloc(size_t bytes, void** out) {
    void* d = nullptr;
    cudaMemPool_t pool;
    cudaError_t e = scratch_pool(&pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&d, bytes < 256 ? 256 : bytes, pool, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::snprintf(g_err, sizeof(g_err), "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return CPIPE_OOM;
    }
    scratch.push_back(d);
    *out = d;
    return CPIPE_OK;
}

int Call::upload(const void* host, size_t bytes, void** out) {
    int st = alloc(bytes, out);
    if (st != CPIPE_OK) return st;
    return cuda_status(cudaMemcpyAsync(*out, host, bytes, cudaMemcpyHostToDevice, stream), "upload params");
}

int Call::finish(int status) {
    if (status == CPIPE_OK) {
        status = cuda_status(cudaGetLastError(), "kernel launch");
    }
    for (const Bound& b : bounds) {
        if (!b.is_output) continue;
        if (b.staged) {
            if (status == CPIPE_OK) {
                const halide_buffer_t* hb = b.hb;
                status = cuda_status(cudaMemcpy2DAsync(hb->host, (size_t)hb->dim[1].stride * b.elem, b.img.data,
                                                       (size_t)b.img.w * b.ch * b.elem, (size_t)b.img.w * b.ch * b.elem,
                                                       (size_t)b.img.h, cudaMemcpyDeviceToHost, stream),
                                     "stage out");
            }
        } else if (status == CPIPE_OK) {
            b.hb->flags |= halide_buffer_flag_device_dirty;
        }
    }
    for (void* p : scratch) cudaFreeAsync(p, stream);
    scratch.clear();
    if (staged_any) {
        const int st = cuda_status(cudaStreamSynchronize(stream), "synchronize");
        if (status == CPIPE_OK) status = st;
    }
    return status;
}

Call::Call() : stream(current_stream()) {}
Call::~Call() {
    for (void* p : scratch) cudaFreeAsync(p, stream);
}

// Device copies of prepared filter tables (linearization tables, GainMap
// gain / axis / grid-row tables, 3D LUT cells), keyed by the exact parameter
// blob and the frame extent: a pipeline that calls a filter with the same
// parameters frame after frame prepares and uploads its tables once.  A small
// least-recently-used set per process (each entry records its device).  The
// caller holds the TableLock from lookup until its kernels are launched, so no
// entry is released under a launch; an evicted entry is freed after a device
// synchronisation.  cpipe_cuda_trim_scratch releases every entry.
namespace {
std::mutex g_tab_mu;
std::vector<TableEntry> g_tabs;
uint64_t g_tab_clock = 0;
constexpr size_t kTableEntries = 8;
}  // namespace

TableLock::TableLock() : lock(g_tab_mu) {}

const TableEntry* table_find(int kind, int w, int h, const void* key, size_t key_bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    for (TableEntry& e : g_tabs) {
        if (e.dev == dev && e.kind == kind && e.w == w && e.h == h && e.key.size() == key_bytes &&
            std::memcmp(e.key.data(), key, key_bytes) == 0) {
            e.used = ++g_tab_clock;
            return &e;
        }
    }
    return nullptr;
}

int table_add(int kind, int w, int h, const void* key, size_t key_bytes, const void* host, size_t host_bytes,
              size_t device_bytes, TableEntry** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "table cache");
    if (g_tabs.size() >= kTableEntries) {
        size_t lru = 0;
        for (size_t i = 1; i < g_tabs.size(); ++i)
            if (g_tabs[i].used < g_tabs[lru].used) lru = i;
        if ((e = cudaSetDevice(g_tabs[lru].dev)) == cudaSuccess && (e = cudaDeviceSynchronize()) == cudaSuccess)
            e = cudaFree(g_tabs[lru].d);
        cudaSetDevice(dev);
        if (e != cudaSuccess) return cuda_status(e, "table cache eviction");
        g_tabs.erase(g_tabs.begin() + (long)lru);
    }
    TableEntry t;
    t.dev = dev;
    t.kind = kind;
    t.w = w;
    t.h = h;
    t.key.assign(static_cast<const unsigned char*>(key), static_cast<const unsigned char*>(key) + key_bytes);
    if (cudaMalloc(&t.d, device_bytes < 256 ? 256 : device_bytes) != cudaSuccess) {
        cudaGetLastError();
        std::snprintf(g_err, sizeof(g_err), "device allocation of %zu bytes failed", device_bytes);
        return CPIPE_OOM;
    }
    if ((e = cudaMemcpy(t.d, host, host_bytes, cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(t.d);
        return cuda_status(e, "table upload");
    }
    t.used = ++g_tab_clock;
    g_tabs.push_back(std::move(t));
    *out = &g_tabs.back();
    return CPIPE_OK;
}

static cudaError_t table_release_all() {
    std::lock_guard<std::mutex> lock(g_tab_mu);
    cudaError_t first = cudaSuccess;
    int cur = 0;
    cudaGetDevice(&cur);
    for (TableEntry& t : g_tabs) {
        cudaError_t e = cudaSetDevice(t.dev);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaFree(t.d);
        if (first == cudaSuccess) first = e;
    }
    cudaSetDevice(cur);
    g_tabs.clear();
    return first;
}

bool device_ready() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("%s", "no CUDA device is available; the cpipe B200 filters have no CPU path");
        return false;
    }
    return true;
}

static bool same_extent(const Bound& a, const Bound& b) { return a.img.w == b.img.w && a.img.h == b.img.h; }

// float-float split of a double.
ff split(double v) {
    const float hi = (float)v;
    return ff{hi, (float)(v - (double)hi)};
}

}  // namespace cpb

using namespace cpb;

#define CHECK_ARITY(nin, nout)                                                                     \
    if (n_in != (nin) || n_out != (nout) || inputs == nullptr || outputs == nullptr ||             \
        inputs[0] == nullptr || outputs[0] == nullptr)                                             \
        return CPIPE_BAD_INDEX;
#define BIND(idx, arr, kind, is_out, var)                                                          \
    Bound var;                                                                                     \
    {                                                                                              \
        const int s_ = call.bind(arr[idx], kind, is_out, &var);                                    \
        if (s_ != CPIPE_OK) return call.finish(s_);                                                \
    }
#define REQUIRE_SAME_EXTENT(a, b) \
    if (!same_extent(a, b)) return call.finish(CPIPE_BAD_INDEX);

extern "C" {

// ----------------------------------------------------------------- stream API
int cpipe_cuda_set_stream(void* stream) {
    g_stream = static_cast<cudaStream_t>(stream);
    return CPIPE_OK;
}
void* cpipe_cuda_get_stream(void) { return g_stream; }
const char* cpipe_cuda_last_error(void) { return g_err; }
int cpipe_cuda_synchronize(void) { return cuda_status(cudaStreamSynchronize(g_stream), "synchronize"); }
int cpipe_cuda_trim_scratch(void) {
    cudaMemPool_t pool;
    cudaError_t e = table_release_all();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = scratch_pool(&pool);
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    return cuda_status(e, "trim scratch");
}
int cpipe_cuda_memory_stats(uint64_t* scratch_reserved, uint64_t* scratch_used, uint64_t* device_free,
                            uint64_t* prepared_tables) {
    cudaMemPool_t pool;
    cudaError_t e = scratch_pool(&pool);
    uint64_t reserved = 0, used = 0;
    size_t free_b = 0, total_b = 0;
    if (e == cudaSuccess) e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    if (e == cudaSuccess) e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return cuda_status(e, "memory stats");
    if (scratch_reserved) *scratch_reserved = reserved;
    if (scratch_used) *scratch_used = used;
    if (device_free) *device_free = free_b;
    if (prepared_tables) {
        std::lock_guard<std::mutex> lock(g_tab_mu);
        *prepared_tables = g_tabs.size();
    }
    return CPIPE_OK;
}
int cpipe_cuda_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// ------------------------------------------------------ a1 precision_convert
// precision_convert_generator.cpp:31-124; plain (input, output) filters
// registered with CPIPE_REGISTER_HALIDE_FILTER (precision_convert_dispatch.cpp).
int cpipe_cuda_precision_convert_r16u_to_f32(halide_buffer_t* input, halide_buffer_t* output) {
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    halide_buffer_t* ins[1] = {input};
    halide_buffer_t* outs[1] = {output};
    BIND(0, ins, Kind::BayerU16, false, in);
    BIND(0, outs, Kind::BayerF32, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    return call.finish(cuda_status(launch_r16u_to_f32(in.img, out.img, call.stream), "r16u_to_f32"));
}
int cpipe_cuda_precision_convert_f32_to_rgba16f(halide_buffer_t* input, halide_buffer_t* output) {
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    halide_buffer_t* ins[1] = {input};
    halide_buffer_t* outs[1] = {output};
    BIND(0, ins, Kind::BayerF32, false, in);
    BIND(0, outs, Kind::Rgba, true, out);
    if (out.elem != 2) return call.finish(CPIPE_BAD_PRECISION);
    REQUIRE_SAME_EXTENT(in, out);
    return call.finish(cuda_status(launch_f32_to_rgba16f(in.img, out.img, call.stream), "f32_to_rgba16f"));
}
static int rgba16f_to_unorm(halide_buffer_t* input, halide_buffer_t* output, int bits8) {
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    halide_buffer_t* ins[1] = {input};
    halide_buffer_t* outs[1] = {output};
    BIND(0, ins, Kind::Rgba, false, in);
    if (in.elem != 2) return call.finish(CPIPE_BAD_PRECISION);
    BIND(0, outs, bits8 ? Kind::RgbaU8 : Kind::RgbaU16, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    return call.finish(cuda_status(launch_rgba16f_to_unorm(in.img, out.img, bits8, call.stream), "to_unorm"));
}
int cpipe_cuda_precision_convert_rgba16f_to_rgba8(halide_buffer_t* input, halide_buffer_t* output) {
    return rgba16f_to_unorm(input, output, 1);
}
int cpipe_cuda_precision_convert_rgba16f_to_rgba16u(halide_buffer_t* input, halide_buffer_t* output) {
    return rgba16f_to_unorm(input, output, 0);
}

// --------------------------------------------------------------- a2 linearize
// linearize_dng_lut_dispatch.cpp:17-51
int cpipe_cuda_linearize_dng_lut(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                 size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_LinearizeParamsHeader)) return CPIPE_BAD_INDEX;
    const auto* hd = static_cast<const cpipe_LinearizeParamsHeader*>(blob);
    const size_t expected = sizeof(*hd) + (size_t)hd->table_size * sizeof(uint16_t);
    if (hd->table_size == 0 || blob_size < expected) return CPIPE_NEED_METADATA;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::BayerU16, false, in);
    BIND(0, outputs, Kind::BayerF32, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    const size_t tbytes = hd->table_size * sizeof(uint16_t);
    const char* table = static_cast<const char*>(blob) + sizeof(*hd);
    TableLock lock;
    const TableEntry* t = table_find(kTabLinearize, 0, 0, table, tbytes);
    if (t == nullptr) {
        TableEntry* added = nullptr;
        const int st = table_add(kTabLinearize, 0, 0, table, tbytes, table, tbytes, tbytes, &added);
        if (st != CPIPE_OK) return call.finish(st);
        t = added;
    }
    return call.finish(cuda_status(
        launch_linearize(in.img, out.img, static_cast<const uint16_t*>(t->d), (int)hd->table_size, call.stream),
        "linearize"));
}

// -------------------------------------------------------------- a3 blacklevel
// blacklevel_dng_levels_dispatch.cpp:16-47
int cpb_blacklevel_dev(const cpipe_BlacklevelParams* p, int w, int h, BlackDev* out) {
    for (int i = 0; i < 4; ++i) {
        const unsigned ch = p->cfa_pattern[i] < 3 ? p->cfa_pattern[i] : 3;
        out->black[i] = p->black_level[ch];
        out->denom[i] = (float)p->white_level - p->black_level[ch];
        const bool used = ((i & 1) == 0 || w > 1) && ((i >> 1) == 0 || h > 1);
        if (used && out->denom[i] <= 0.0F) return CPIPE_NEED_METADATA;
    }
    return CPIPE_OK;
}
int cpipe_cuda_blacklevel_dng_levels(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                     size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_BlacklevelParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::BayerF32, false, in);
    BIND(0, outputs, Kind::BayerF32, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    BlackDev p;
    const int st = cpb_blacklevel_dev(static_cast<const cpipe_BlacklevelParams*>(blob), in.img.w, in.img.h, &p);
    if (st != CPIPE_OK) return call.finish(st);
    return call.finish(cuda_status(launch_blacklevel(in.img, out.img, p, call.stream), "blacklevel"));
}

// ----------------------------------------------------------------- a4 gainmap
// shading_gainmap_dispatch.cpp:23-133.  The double-precision axis sampling is
// done here on the host, once per row and column.
static AxisSample host_sample_axis(double coord, uint32_t points) {
    AxisSample a{0, 0, 0.0F};
    if (points <= 1U || coord <= 0.0) return a;
    const double last = (double)(points - 1U);
    if (coord >= last) {
        a.low = a.high = points - 1U;
        return a;
    }
    a.low = (uint32_t)std::floor(coord);
    a.high = a.low + 1U;
    a.weight = (float)(coord - (double)a.low);
    return a;
}
int cpb_gainmap_prepare(const void* blob, size_t blob_size, int w, int h, std::vector<char>* table,
                        GainMapDev* g, size_t offsets[3][4]) {
    if (blob == nullptr || blob_size < sizeof(cpipe_GainMapDispatchHeader)) return CPIPE_BAD_INDEX;
    const auto* hd = static_cast<const cpipe_GainMapDispatchHeader*>(blob);
    if (hd->map_count == 0U || hd->map_count > 4U) return CPIPE_NEED_METADATA;
    const size_t map_bytes = hd->map_count * sizeof(cpipe_GainMapDispatchPlane);
    if (blob_size < sizeof(*hd) + map_bytes) return CPIPE_BAD_INDEX;
    const auto* maps = reinterpret_cast<const cpipe_GainMapDispatchPlane*>(static_cast<const char*>(blob) + sizeof(*hd));
    const char* gains = static_cast<const char*>(blob) + sizeof(*hd) + map_bytes;
    const size_t gain_bytes = blob_size - sizeof(*hd) - map_bytes;
    for (uint32_t i = 0; i < hd->map_count; ++i) {
        const uint64_t req = ((uint64_t)maps[i].gain_offset + maps[i].gain_count) * sizeof(float);
        if (maps[i].map_points_v == 0U || maps[i].map_points_h == 0U || maps[i].gain_count == 0U || req > gain_bytes)
            return CPIPE_BAD_INDEX;
        // the sampler reads up to (points_v-1)*points_h + points_h-1 from the map's offset
        if ((uint64_t)maps[i].map_points_v * maps[i].map_points_h > maps[i].gain_count) return CPIPE_BAD_INDEX;
    }
    g->map_count = (int)hd->map_count;
    g->qbc = hd->cfa_repeat[0] == 4U && hd->cfa_repeat[1] == 4U;
    for (int p = 0; p < 4; ++p) {
        g->plane_to_map[p] = -1;
        for (uint32_t i = 0; i < hd->map_count; ++i)
            if (maps[i].plane == (uint32_t)p) {
                g->plane_to_map[p] = (int)i;
                break;
            }
    }
    if (hd->map_count > 1) {
        // select_map returns nullptr -> CPIPE_NEED_METADATA for any pixel whose plane has no map
        for (int p = 0; p < 4; ++p) {
            const bool used = g->qbc ? (((p & 1) == 0 || w > 2) && ((p >> 1) == 0 || h > 2))
                                     : (((p & 1) == 0 || w > 1) && ((p >> 1) == 0 || h > 1));
            if (used && g->plane_to_map[p] < 0) return CPIPE_NEED_METADATA;
        }
    }
    // layout: gains | cols (w per map) | rows (h per map)
    size_t off = 0;
    table->clear();
    for (uint32_t i = 0; i < hd->map_count; ++i) {
        offsets[0][i] = off;
        const size_t n = (size_t)maps[i].map_points_v * maps[i].map_points_h * sizeof(float);
        table->resize(off + n);
        std::memcpy(table->data() + off, gains + (size_t)maps[i].gain_offset * sizeof(float), n);
        off += (n + 15) & ~size_t(15);
        g->points_h[i] = (int)maps[i].map_points_h;
        g->points_v[i] = (int)maps[i].map_points_v;
    }
    for (uint32_t i = 0; i < hd->map_count; ++i) {
        offsets[1][i] = off;
        table->resize(off + (size_t)w * sizeof(AxisSample));
        auto* cols = reinterpret_cast<AxisSample*>(table->data() + off);
        for (int x = 0; x < w; ++x)
            cols[x] = host_sample_axis(((double)x - maps[i].map_origin_h) / maps[i].map_spacing_h, maps[i].map_points_h);
        off += ((size_t)w * sizeof(AxisSample) + 15) & ~size_t(15);
    }
    for (uint32_t i = 0; i < hd->map_count; ++i) {
        offsets[2][i] = off;
        table->resize(off + (size_t)h * sizeof(AxisSample));
        auto* rows = reinterpret_cast<AxisSample*>(table->data() + off);
        for (int y = 0; y < h; ++y)
            rows[y] = host_sample_axis(((double)y - maps[i].map_origin_v) / maps[i].map_spacing_v, maps[i].map_points_v);
        off += ((size_t)h * sizeof(AxisSample) + 15) & ~size_t(15);
    }
    table->resize(off);
    return CPIPE_OK;
}
void cpb_gainmap_bind(GainMapDev* g, const char* d_table, size_t offsets[3][4]) {
    for (int i = 0; i < g->map_count; ++i) {
        g->gains[i] = reinterpret_cast<const float*>(d_table + offsets[0][i]);
        g->cols[i] = reinterpret_cast<const AxisSample*>(d_table + offsets[1][i]);
        g->rows[i] = reinterpret_cast<const AxisSample*>(d_table + offsets[2][i]);
    }
}
int cpipe_cuda_lens_shading_gainmap(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                    size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_GainMapDispatchHeader)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::BayerF32, false, in);
    BIND(0, outputs, Kind::BayerF32, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    TableLock lock;
    const TableEntry* t = table_find(kTabGainMap, in.img.w, in.img.h, blob, blob_size);
    if (t == nullptr) {
        std::vector<char> table;
        GainMapDev g{};
        size_t offsets[3][4] = {};
        int st = cpb_gainmap_prepare(blob, blob_size, in.img.w, in.img.h, &table, &g, offsets);
        if (st != CPIPE_OK) return call.finish(st);
        const size_t hoff = (table.size() + 15) & ~size_t(15);
        TableEntry* added = nullptr;
        st = table_add(kTabGainMap, in.img.w, in.img.h, blob, blob_size, table.data(), table.size(),
                       hoff + gainmap_hrows_bytes(g, in.img.w), &added);
        if (st != CPIPE_OK) return call.finish(st);
        cpb_gainmap_bind(&g, static_cast<const char*>(added->d), offsets);
        cudaError_t e = launch_gainmap_hrows(&g, static_cast<char*>(added->d) + hoff, in.img.w, call.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(call.stream);
        if (e != cudaSuccess) return call.finish(cuda_status(e, "gainmap rows"));
        added->meta.resize(sizeof(g));
        std::memcpy(added->meta.data(), &g, sizeof(g));
        t = added;
    }
    GainMapDev g;
    std::memcpy(&g, t->meta.data(), sizeof(g));
    return call.finish(cuda_status(launch_gainmap(in.img, out.img, g, call.stream), "gainmap"));
}

// ---------------------------------------------------------------- a5-a7 demosaic
static int demosaic_filter(int algo, halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                           size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_DemosaicParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::BayerF32, false, in);
    BIND(0, outputs, Kind::Rgba, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    const auto* p = static_cast<const cpipe_DemosaicParams*>(blob);
    const int cfa[4] = {p->cfa_pattern[0], p->cfa_pattern[1], p->cfa_pattern[2], p->cfa_pattern[3]};
    return call.finish(cuda_status(launch_demosaic(algo, in.img, out.img, out.elem == 2, cfa, call.stream), "demosaic"));
}
int cpipe_cuda_demosaic_bilinear(halide_buffer_t* const* i, size_t ni, halide_buffer_t* const* o, size_t no,
                                 const void* b, size_t bs) {
    return demosaic_filter(0, i, ni, o, no, b, bs);
}
int cpipe_cuda_demosaic_rcd(halide_buffer_t* const* i, size_t ni, halide_buffer_t* const* o, size_t no, const void* b,
                            size_t bs) {
    return demosaic_filter(1, i, ni, o, no, b, bs);
}
int cpipe_cuda_demosaic_amaze(halide_buffer_t* const* i, size_t ni, halide_buffer_t* const* o, size_t no,
                              const void* b, size_t bs) {
    return demosaic_filter(2, i, ni, o, no, b, bs);
}

// Full-form RCD / AMaZE (no reference filter: the reference's nodes compute the
// reduced stencils above).  Bayer patterns with the two greens on a diagonal.
static int demosaic_full_filter(int algo, halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_DemosaicParams)) return CPIPE_BAD_INDEX;
    const auto* p = static_cast<const cpipe_DemosaicParams*>(blob);
    const int cfa[4] = {p->cfa_pattern[0], p->cfa_pattern[1], p->cfa_pattern[2], p->cfa_pattern[3]};
    const bool bayer = ((cfa[0] == 1 && cfa[3] == 1 && cfa[1] + cfa[2] == 2 && cfa[1] != 1) ||
                        (cfa[1] == 1 && cfa[2] == 1 && cfa[0] + cfa[3] == 2 && cfa[0] != 1));
    if (!bayer) {
        set_error("%s", "full-form demosaic needs a 2x2 Bayer pattern (RGGB, BGGR, GRBG, GBRG)");
        return CPIPE_UNSUPPORTED;
    }
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::BayerF32, false, in);
    BIND(0, outputs, Kind::Rgba, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    void* scratch = nullptr;
    const size_t bytes = demosaic_full_scratch_bytes(algo, in.img.w, in.img.h);
    if (bytes) {
        const int st = call.alloc(bytes, &scratch);
        if (st != CPIPE_OK) return call.finish(st);
    }
    return call.finish(cuda_status(launch_demosaic_full(algo, in.img, out.img, out.elem == 2, cfa, scratch, call.stream),
                                   "demosaic full"));
}
int cpipe_cuda_demosaic_rcd_full(halide_buffer_t* const* i, size_t ni, halide_buffer_t* const* o, size_t no,
                                 const void* b, size_t bs) {
    return demosaic_full_filter(1, i, ni, o, no, b, bs);
}
int cpipe_cuda_demosaic_amaze_full(halide_buffer_t* const* i, size_t ni, halide_buffer_t* const* o, size_t no,
                                   const void* b, size_t bs) {
    return demosaic_full_filter(2, i, ni, o, no, b, bs);
}

// ------------------------------------------------------------ a8 QBC remosaic
int cpipe_cuda_demosaic_quad_bayer_remosaic(halide_buffer_t* input, halide_buffer_t* output) {
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    halide_buffer_t* ins[1] = {input};
    halide_buffer_t* outs[1] = {output};
    BIND(0, ins, Kind::BayerU16, false, in);
    BIND(0, outs, Kind::BayerU16, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    return call.finish(cuda_status(launch_qbc_remosaic(in.img, out.img, call.stream), "qbc_remosaic"));
}

// -------------------------------------------------------- a9/a10 WB, colormatrix
int cpipe_cuda_wb_dual_illuminant(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                  size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_WbParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::Rgba, false, in);
    BIND(0, outputs, Kind::Rgba, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    if (in.elem != out.elem) return call.finish(CPIPE_BAD_PRECISION);
    const auto* p = static_cast<const cpipe_WbParams*>(blob);
    return call.finish(cuda_status(launch_wb(in.img, out.img, in.elem == 2, p->as_shot_neutral, call.stream), "wb"));
}
int cpipe_cuda_colormatrix_dng_to_working(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                          size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_ColormatrixParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::Rgba, false, in);
    BIND(0, outputs, Kind::Rgba, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    if (in.elem != out.elem) return call.finish(CPIPE_BAD_PRECISION);
    const auto* p = static_cast<const cpipe_ColormatrixParams*>(blob);
    return call.finish(cuda_status(launch_colormatrix(in.img, out.img, in.elem == 2, p->transform, call.stream), "cm"));
}

// ---------------------------------------------------------- a11-a13 denoise
static int rgba_pair(Call& call, halide_buffer_t* const* inputs, halide_buffer_t* const* outputs, Bound* in, Bound* out) {
    int st = call.bind(inputs[0], Kind::Rgba, false, in);
    if (st != CPIPE_OK) return st;
    st = call.bind(outputs[0], Kind::Rgba, true, out);
    if (st != CPIPE_OK) return st;
    if (!same_extent(*in, *out)) return CPIPE_BAD_INDEX;
    if (in->elem != out->elem) return CPIPE_BAD_PRECISION;
    return CPIPE_OK;
}
int cpipe_cuda_denoise_bm3d_step1(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                  size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_Bm3dParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    const float sigma = static_cast<const cpipe_Bm3dParams*>(blob)->sigma;
    return call.finish(cuda_status(launch_bm3d_parity(in.img, out.img, in.elem == 2, sigma, call.stream), "bm3d"));
}
// bm3d_step2_generator.cpp:33-42: a sigma-aware identity.
int cpipe_cuda_denoise_bm3d_step2(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                  size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_Bm3dParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    return call.finish(cuda_status(launch_copy(in.img.data, in.img.row_stride * in.elem, out.img.data,
                                               out.img.row_stride * out.elem, (long long)in.img.w * 4 * in.elem,
                                               in.img.h, call.stream),
                                   "bm3d_step2"));
}
// Two-stage colour BM3D (bm3d_spec.cu); no reference counterpart.
int cpipe_cuda_denoise_bm3d_spec(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                 size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_Bm3dSpecParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    cpipe_Bm3dSpecParams prm;
    std::memcpy(&prm, blob, sizeof(prm));
    Call call;
    Bound in, out;
    int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    Bm3dPlan plan;
    if ((st = bm3d_plan(&prm, in.img.w, in.img.h, &plan)) != CPIPE_OK) {
        set_error("bm3d_spec: %s", "parameters out of range");
        return call.finish(st);
    }
    void* scratch = nullptr;
    if (!plan.copy && (st = call.alloc(plan.bytes, &scratch)) != CPIPE_OK) return call.finish(st);
    return call.finish(cuda_status(bm3d_run(plan, in.img, out.img, in.elem == 2, scratch, call.stream), "bm3d_spec"));
}
int cpipe_cuda_denoise_guided_filter_spec(halide_buffer_t* const* inputs, size_t n_in,
                                          halide_buffer_t* const* outputs, size_t n_out, const void* blob,
                                          size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_GuidedFilterParams)) return CPIPE_BAD_INDEX;
    cpipe_GuidedFilterParams prm;
    std::memcpy(&prm, blob, sizeof(prm));
    if (prm.radius < 1 || prm.radius > kGuidedSpecMaxRadius || !(prm.eps > 0.0F) || !std::isfinite(prm.eps)) {
        set_error("guided_filter_spec: %s", "radius must be 1..16 and eps positive");
        return CPIPE_BAD_INDEX;
    }
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    static const cudaError_t setup = guided_spec_setup();
    if (setup != cudaSuccess) return cuda_status(setup, "guided_filter_spec setup");
    Call call;
    Bound in, out;
    int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    void* scratch = nullptr;
    if ((st = call.alloc(guided_spec_scratch_bytes(in.img.w, in.img.h, prm.radius), &scratch)) != CPIPE_OK)
        return call.finish(st);
    return call.finish(cuda_status(
        guided_spec_run(in.img, out.img, in.elem == 2, prm.radius, prm.eps, scratch, call.stream), "guided_spec"));
}
int cpipe_cuda_denoise_wavelet_atrous_spec(halide_buffer_t* const* inputs, size_t n_in,
                                           halide_buffer_t* const* outputs, size_t n_out, const void* blob,
                                           size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_AtrousWaveletParams)) return CPIPE_BAD_INDEX;
    cpipe_AtrousWaveletParams prm;
    std::memcpy(&prm, blob, sizeof(prm));
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    static const cudaError_t setup = atrous_setup();
    if (setup != cudaSuccess) return cuda_status(setup, "wavelet_atrous_spec setup");
    Call call;
    Bound in, out;
    int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    AtrousPlan plan;
    if ((st = atrous_plan(&prm, in.img.w, in.img.h, &plan)) != CPIPE_OK) {
        set_error("wavelet_atrous_spec: %s", "parameters out of range");
        return call.finish(st);
    }
    void* scratch = nullptr;
    if (!plan.copy && (st = call.alloc(plan.bytes, &scratch)) != CPIPE_OK) return call.finish(st);
    return call.finish(cuda_status(atrous_run(plan, in.img, out.img, in.elem == 2, scratch, call.stream), "atrous"));
}
int cpipe_cuda_denoise_guided_filter(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                     size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_GuidedFilterParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    const auto* p = static_cast<const cpipe_GuidedFilterParams*>(blob);
    return call.finish(
        cuda_status(launch_guided(in.img, out.img, in.elem == 2, p->radius, p->eps, call.stream), "guided"));
}
int cpipe_cuda_denoise_wavelet_bayes_shrink(halide_buffer_t* const* inputs, size_t n_in,
                                            halide_buffer_t* const* outputs, size_t n_out, const void* blob,
                                            size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_WaveletBayesShrinkParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    const float strength = static_cast<const cpipe_WaveletBayesShrinkParams*>(blob)->chroma_strength;
    return call.finish(cuda_status(launch_wavelet(in.img, out.img, in.elem == 2, strength, call.stream), "wavelet"));
}

// -------------------------------------------------------------- a15 3D LUT
int cpb_lut_prepare(const void* blob, size_t blob_size, std::vector<float4>* cells, int* S, int* interp) {
    if (blob == nullptr || blob_size < sizeof(cpipe_Lut3dParamHeader)) return CPIPE_BAD_INDEX;
    cpipe_Lut3dParamHeader hd;
    std::memcpy(&hd, blob, sizeof(hd));
    if (hd.size < 2U || hd.value_count == 0U || (hd.value_count % 3U) != 0U) return CPIPE_BAD_INDEX;
    if (blob_size != sizeof(hd) + (size_t)hd.value_count * sizeof(float) || hd.size > 256U) return CPIPE_BAD_INDEX;
    const size_t ncell = (size_t)hd.size * hd.size * hd.size;
    if ((size_t)hd.value_count / 3U < ncell) return CPIPE_BAD_INDEX;
    const float* v = reinterpret_cast<const float*>(static_cast<const char*>(blob) + sizeof(hd));
    cells->resize(ncell);
    for (size_t i = 0; i < ncell; ++i) (*cells)[i] = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0F);
    *S = (int)hd.size;
    *interp = hd.interpolation == 1U ? 1 : 0;
    return CPIPE_OK;
}
int cpipe_cuda_color_3d_lut(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                            size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr) return CPIPE_BAD_INDEX;
    TableLock lock;
    const TableEntry* t = table_find(kTabLut, 0, 0, blob, blob_size);
    std::vector<float4> cells;
    int lut_si[2] = {0, 0};  // size, interpolation
    if (t == nullptr) {
        const int pst = cpb_lut_prepare(blob, blob_size, &cells, &lut_si[0], &lut_si[1]);
        if (pst != CPIPE_OK) return pst;
    } else {
        std::memcpy(lut_si, t->meta.data(), sizeof(lut_si));
    }
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    if (t == nullptr) {
        TableEntry* added = nullptr;
        const size_t bytes = cells.size() * sizeof(float4);
        if ((st = table_add(kTabLut, 0, 0, blob, blob_size, cells.data(), bytes, bytes, &added)) != CPIPE_OK)
            return call.finish(st);
        added->meta.resize(sizeof(lut_si));
        std::memcpy(added->meta.data(), lut_si, sizeof(lut_si));
        t = added;
    }
    return call.finish(cuda_status(launch_lut3d(in.img, out.img, in.elem == 2, static_cast<const float4*>(t->d),
                                                lut_si[0], lut_si[1], call.stream),
                                   "lut"));
}

// ----------------------------------------------------------------- a16 filmic
FilmicDev cpb_filmic_dev(const cpipe_FilmicRgbParams* p) {
    FilmicDev f;
    f.exposure = std::pow(2.0F, p->ev);
    f.inv_contrast = 1.0F / p->contrast;
    f.saturation = p->saturation;
    f.highlights = p->highlights;
    f.shadows = p->shadows;
    f.log_white = (float)std::log(109.0);  // log(1 + 6 * 18), folded by the generator
    return f;
}
int cpipe_cuda_tone_filmic_rgb(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                               size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_FilmicRgbParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    const FilmicDev f = cpb_filmic_dev(static_cast<const cpipe_FilmicRgbParams*>(blob));
    return call.finish(cuda_status(launch_filmic(in.img, out.img, in.elem == 2, f, call.stream), "filmic"));
}

// ------------------------------------------------------- wb.greyworld_auto
// greyworld_auto.cpp:44-77 on the GPU: exact channel sums (greyworld_sum_kernel
// block totals added here in 128-bit integers, then rounded to double once),
// the neutral (R/G, 1, B/G) rounded to float as the reference does, v / neutral.
int cpipe_cuda_wb_greyworld_auto(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                 size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_GreyworldParams)) return CPIPE_BAD_INDEX;
    cpipe_GreyworldParams p;
    std::memcpy(&p, blob, sizeof(p));
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    if (in.elem != 2) return call.finish(CPIPE_BAD_PRECISION);
    void* d_partial = nullptr;
    if ((st = call.alloc(sizeof(long long) * 4 * kGreyworldBlocks, &d_partial)) != CPIPE_OK) return call.finish(st);
    std::vector<long long> part(4 * kGreyworldBlocks);
    cudaError_t e = launch_greyworld_sums(in.img, static_cast<long long*>(d_partial), kGreyworldBlocks, call.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(part.data(), d_partial, part.size() * sizeof(long long), cudaMemcpyDeviceToHost,
                            call.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(call.stream);
    if (e != cudaSuccess) return call.finish(cuda_status(e, "greyworld sums"));
    __int128 t[3] = {0, 0, 0};
    long long bad = 0;
    for (int b = 0; b < kGreyworldBlocks; ++b) {
        for (int k = 0; k < 3; ++k) t[k] += part[4 * b + k];
        bad |= part[4 * b + 3];
    }
    double sums[3];
    for (int k = 0; k < 3; ++k) sums[k] = std::ldexp((double)t[k], -24);
    for (double v : sums)
        if (bad || !(v > 0.0)) {
            set_error("wb_greyworld_auto: %s", "invalid channel mean");
            return call.finish(CPIPE_NEED_METADATA);
        }
    const float n[3] = {(float)(sums[0] / sums[1]), 1.0F, (float)(sums[2] / sums[1])};
    if ((e = launch_greyworld_apply(in.img, out.img, n, call.stream)) != cudaSuccess)
        return call.finish(cuda_status(e, "greyworld apply"));
    if (p.neutral_out) std::memcpy(reinterpret_cast<void*>((uintptr_t)p.neutral_out), n, sizeof(n));
    return call.finish(CPIPE_OK);
}

// ------------------------------------------------------ tone.mertens_local
// mertens_local_dispatch.cpp:18-37: inputs under, normal, over (RGBA16F, one extent).
int cpipe_cuda_tone_mertens_local(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                  size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(3, 1);
    if (inputs[1] == nullptr || inputs[2] == nullptr) return CPIPE_BAD_INDEX;
    if (blob == nullptr || blob_size < sizeof(cpipe_MertensLocalParams)) return CPIPE_BAD_INDEX;
    cpipe_MertensLocalParams p;
    std::memcpy(&p, blob, sizeof(p));
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::Rgba, false, under);
    BIND(1, inputs, Kind::Rgba, false, normal);
    BIND(2, inputs, Kind::Rgba, false, over);
    BIND(0, outputs, Kind::Rgba, true, out);
    if (under.elem != 2 || normal.elem != 2 || over.elem != 2 || out.elem != 2) return call.finish(CPIPE_BAD_PRECISION);
    REQUIRE_SAME_EXTENT(under, out);
    REQUIRE_SAME_EXTENT(normal, out);
    REQUIRE_SAME_EXTENT(over, out);
    return call.finish(cuda_status(launch_mertens(under.img, normal.img, over.img, out.img, p.weight_contrast,
                                                  p.weight_saturation, p.weight_well_exposedness, call.stream),
                                   "mertens"));
}

// ------------------------------------------------ tone.aces_filmic / reinhard
// aces_filmic_dispatch.cpp:17-31, reinhard_dispatch.cpp:16-29 (4-byte blobs).
int cpipe_cuda_tone_aces_filmic(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_AcesFilmicParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    cpipe_AcesFilmicParams p;
    std::memcpy(&p, blob, sizeof(p));
    return call.finish(cuda_status(launch_aces(in.img, out.img, in.elem == 2, p.enabled, call.stream), "aces"));
}
int cpipe_cuda_tone_reinhard(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                             size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_ReinhardParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    cpipe_ReinhardParams p;
    std::memcpy(&p, blob, sizeof(p));
    return call.finish(
        cuda_status(launch_reinhard(in.img, out.img, in.elem == 2, p.white_point, call.stream), "reinhard"));
}

// --------------------------------------------------- sharpen.edge_aware_usm
// edge_aware_usm_dispatch.cpp:18-31 (blob EdgeAwareUsmParams, 12 bytes).
int cpipe_cuda_sharpen_edge_aware_usm(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                      size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_EdgeAwareUsmParams)) return CPIPE_BAD_INDEX;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    const int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    cpipe_EdgeAwareUsmParams p;
    std::memcpy(&p, blob, sizeof(p));
    return call.finish(cuda_status(
        launch_usm(in.img, out.img, in.elem == 2, p.strength, p.radius, p.threshold, call.stream), "usm"));
}

// -------------------------------------------- color.scene_linear_to_display
// RGBA16F in; RGBA8 unorm out (sRGB) or RGBA16 unorm (BT2020-PQ, 10-bit codes
// in the top bits), as the reference's write_ocio_output (HostContext.cpp:155-185).
int cpipe_cuda_scene_linear_to_display(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                       size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    if (blob == nullptr || blob_size < sizeof(cpipe_DisplayParams)) return CPIPE_BAD_INDEX;
    cpipe_DisplayParams p;
    std::memcpy(&p, blob, sizeof(p));
    if (p.target != CPIPE_DISPLAY_SRGB && p.target != CPIPE_DISPLAY_BT2020_PQ) {
        set_error("scene_linear_to_display: %s", "target must be 0 (sRGB) or 1 (BT2020-PQ)");
        return CPIPE_UNSUPPORTED;
    }
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::Rgba, false, in);
    if (in.elem != 2) return call.finish(CPIPE_BAD_PRECISION);
    BIND(0, outputs, p.target == CPIPE_DISPLAY_SRGB ? Kind::RgbaU8 : Kind::RgbaU16, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    return call.finish(cuda_status(launch_display(in.img, out.img, p.target, call.stream), "display"));
}

// ------------------------------------------------------------ a14 OpcodeList3
// dng_opcode_list_3_dispatch.cpp:254-398.  Records run in order, each from the
// previous result; two device scratch images ping-pong between them.
static double max_corner_distance(double cx, double cy, int w, int h) {
    const double x1 = (double)(w - 1), y1 = (double)(h - 1);
    const double d00 = (cx * cx) + (cy * cy), d10 = ((x1 - cx) * (x1 - cx)) + (cy * cy);
    const double d01 = (cx * cx) + ((y1 - cy) * (y1 - cy)), d11 = ((x1 - cx) * (x1 - cx)) + ((y1 - cy) * (y1 - cy));
    double m = d00;
    if (d10 > m) m = d10;
    if (d01 > m) m = d01;
    if (d11 > m) m = d11;
    return std::sqrt(m);
}
int cpb_warp_dev(const cpipe_Opcode3DispatchRecord* r, int w, int h, WarpDev* out) {
    // returns CPIPE_OK when a warp applies, CPIPE_REPLY_DEFAULT for the copy cases
    if (r->coefficient_count == 0U || w <= 1 || h <= 1) return CPIPE_REPLY_DEFAULT;
    const double cx = r->cx_hat * (double)(w - 1), cy = r->cy_hat * (double)(h - 1);
    const double m = max_corner_distance(cx, cy, w, h);
    if (m <= 2.220446049250313e-16) return CPIPE_REPLY_DEFAULT;
    out->count = (int)(r->coefficient_count < 4U ? r->coefficient_count : 4U);
    for (int i = 0; i < out->count; ++i) {
        const cpipe_Opcode3WarpCoefficient& k = r->coefficients[i];
        WarpCoefDev& d = out->k[i];
        d.kr0m1 = split(k.kr0 - 1.0);
        d.kr1 = split(k.kr1);
        d.kr2 = split(k.kr2);
        d.kr3 = split(k.kr3);
        d.t0 = split(k.kt0 / m);
        d.t1 = split(k.kt1 / m);
        d.has_kr3 = k.kr3 != 0.0;
        d.has_tan = k.kt0 != 0.0 || k.kt1 != 0.0;
    }
    out->cx = split(cx);
    out->cy = split(cy);
    out->inv_m2 = split(1.0 / (m * m));
    out->xmax = (float)(w - 1);
    out->ymax = (float)(h - 1);
    return CPIPE_OK;
}
int cpb_opcode3_parse(const void* blob, size_t blob_size, Opcode3View* v) {
    if (blob == nullptr || blob_size < sizeof(cpipe_Opcode3DispatchHeader)) return CPIPE_BAD_INDEX;
    const char* base = static_cast<const char*>(blob);
    const auto* hd = reinterpret_cast<const cpipe_Opcode3DispatchHeader*>(base);
    const size_t rec_bytes = (size_t)hd->opcode_count * sizeof(cpipe_Opcode3DispatchRecord);
    if (blob_size < sizeof(*hd) + rec_bytes) return CPIPE_BAD_INDEX;
    const auto* recs = reinterpret_cast<const cpipe_Opcode3DispatchRecord*>(base + sizeof(*hd));
    size_t npt = 0, nrc = 0;
    for (uint32_t i = 0; i < hd->opcode_count; ++i) {
        npt = std::max(npt, (size_t)recs[i].point_offset + recs[i].point_count);
        nrc = std::max(nrc, (size_t)recs[i].rect_offset + recs[i].rect_count);
    }
    const size_t pts_off = sizeof(*hd) + rec_bytes;
    const size_t rc_off = pts_off + npt * sizeof(cpipe_Opcode3BadPoint);
    if (blob_size < rc_off + nrc * sizeof(cpipe_Opcode3BadRect)) return CPIPE_BAD_INDEX;
    v->count = hd->opcode_count;
    v->records = recs;
    v->points = reinterpret_cast<const cpipe_Opcode3BadPoint*>(base + pts_off);
    v->rects = reinterpret_cast<const cpipe_Opcode3BadRect*>(base + rc_off);
    v->npoints = npt;
    v->nrects = nrc;
    return CPIPE_OK;
}
int cpb_opcode3_run(Call& call, const Opcode3View& v, const Img& in, const Img& out, int elem) {
    const bool f16 = elem == 2;
    const int w = in.w, h = in.h;
    for (uint32_t i = 0; i < v.count; ++i)
        if (v.records[i].id != CPIPE_OPCODE3_UNKNOWN && v.records[i].id != CPIPE_OPCODE3_WARP_RECTILINEAR &&
            v.records[i].id != CPIPE_OPCODE3_FIX_VIGNETTE_RADIAL && v.records[i].id != CPIPE_OPCODE3_FIX_BAD_PIXELS_CONSTANT &&
            v.records[i].id != CPIPE_OPCODE3_FIX_BAD_PIXELS_LIST && v.records[i].id != CPIPE_OPCODE3_TRIM_BOUNDS)
            return CPIPE_UNSUPPORTED;
        else if (v.records[i].id == CPIPE_OPCODE3_UNKNOWN && v.records[i].optional == 0U)
            return CPIPE_UNSUPPORTED;
    // Device copies of the point / rect lists.
    void* d_pts = nullptr;
    void* d_rects = nullptr;
    int st = CPIPE_OK;
    if (v.npoints) st = call.upload(v.points, v.npoints * sizeof(cpipe_Opcode3BadPoint), &d_pts);
    if (st == CPIPE_OK && v.nrects) st = call.upload(v.rects, v.nrects * sizeof(cpipe_Opcode3BadRect), &d_rects);
    if (st != CPIPE_OK) return st;
    // Ping-pong: the working image starts as `in`; every applied opcode writes a
    // scratch image (or `out` for the last applied one).
    int last = -1;
    for (uint32_t i = 0; i < v.count; ++i)
        if (v.records[i].id != CPIPE_OPCODE3_UNKNOWN) last = (int)i;
    const long long row_bytes = (long long)w * 4 * elem;
    if (last < 0) return cuda_status(launch_copy(in.data, in.row_stride * elem, out.data, out.row_stride * elem,
                                                 row_bytes, h, call.stream), "opcode3 copy");
    void* tmp[2] = {nullptr, nullptr};
    Img work = in;
    int slot = 0;
    for (uint32_t i = 0; i < v.count; ++i) {
        const cpipe_Opcode3DispatchRecord& r = v.records[i];
        if (r.id == CPIPE_OPCODE3_UNKNOWN) continue;
        Img dst = out;
        if ((int)i != last) {
            if (tmp[slot] == nullptr) {
                st = call.alloc((size_t)w * h * 4 * elem, &tmp[slot]);
                if (st != CPIPE_OK) return st;
            }
            dst = Img{tmp[slot], w, h, (long long)w * 4, 4};
            slot ^= 1;
        }
        cudaError_t e = cudaSuccess;
        switch (r.id) {
            case CPIPE_OPCODE3_WARP_RECTILINEAR: {
                WarpDev wd;
                if (cpb_warp_dev(&r, w, h, &wd) == CPIPE_OK) e = launch_warp(work, dst, f16, wd, call.stream);
                else e = launch_copy(work.data, work.row_stride * elem, dst.data, dst.row_stride * elem, row_bytes, h, call.stream);
                break;
            }
            case CPIPE_OPCODE3_FIX_VIGNETTE_RADIAL: {
                const double cx = r.vignette_cx_hat * (double)(w - 1), cy = r.vignette_cy_hat * (double)(h - 1);
                const double m = (w <= 1 || h <= 1) ? 0.0 : max_corner_distance(cx, cy, w, h);
                if (w <= 1 || h <= 1 || m <= 2.220446049250313e-16) {
                    e = launch_copy(work.data, work.row_stride * elem, dst.data, dst.row_stride * elem, row_bytes, h, call.stream);
                } else {
                    VignetteParams vp;
                    vp.cx = split(cx);
                    vp.cy = split(cy);
                    vp.inv_m = split(1.0 / m);
                    for (int k = 0; k < 5; ++k) vp.k[k] = split(r.vignette_k[k]);
                    e = launch_vignette(work, dst, f16, vp, call.stream);
                }
                break;
            }
            case CPIPE_OPCODE3_FIX_BAD_PIXELS_CONSTANT:
                e = launch_bad_constant(work, dst, f16, (float)r.constant, call.stream);
                break;
            case CPIPE_OPCODE3_FIX_BAD_PIXELS_LIST:
                e = launch_copy(work.data, work.row_stride * elem, dst.data, dst.row_stride * elem, row_bytes, h, call.stream);
                if (e == cudaSuccess && (r.point_count || r.rect_count))
                    e = launch_bad_list(work, dst, f16,
                                        static_cast<const uint32_t*>(d_pts) + 2 * (size_t)r.point_offset, (int)r.point_count,
                                        static_cast<const uint32_t*>(d_rects) + 4 * (size_t)r.rect_offset, (int)r.rect_count,
                                        call.stream);
                break;
            case CPIPE_OPCODE3_TRIM_BOUNDS:
                e = launch_trim(work, dst, f16, r.top, r.left, r.bottom, r.right, call.stream);
                break;
            default:
                return CPIPE_UNSUPPORTED;
        }
        st = cuda_status(e, "opcode3");
        if (st != CPIPE_OK) return st;
        work = dst;
    }
    return CPIPE_OK;
}
int cpipe_cuda_lens_dng_opcode_list_3(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs,
                                      size_t n_out, const void* blob, size_t blob_size) {
    CHECK_ARITY(1, 1);
    Opcode3View v;
    const int pst = cpb_opcode3_parse(blob, blob_size, &v);
    if (pst != CPIPE_OK) return pst;
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    Bound in, out;
    int st = rgba_pair(call, inputs, outputs, &in, &out);
    if (st != CPIPE_OK) return call.finish(st);
    return call.finish(cpb_opcode3_run(call, v, in.img, out.img, in.elem));
}

// ----------------------------------------------------------- pass-through
// Device copy used by the node plugins for their pass-through cases (no GainMap,
// no OpcodeList3, Bayer input to the Quad-Bayer remosaic), in place of the
// reference's lock_cpu + memcpy.  The blob is ignored.
int cpipe_cuda_copy(halide_buffer_t* const* inputs, size_t n_in, halide_buffer_t* const* outputs, size_t n_out,
                    const void* blob, size_t blob_size) {
    (void)blob;
    (void)blob_size;
    CHECK_ARITY(1, 1);
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    BIND(0, inputs, Kind::Any, false, in);
    BIND(0, outputs, Kind::Any, true, out);
    REQUIRE_SAME_EXTENT(in, out);
    if (in.elem != out.elem || in.ch != out.ch) return call.finish(CPIPE_BAD_PRECISION);
    return call.finish(cuda_status(launch_copy(in.img.data, in.img.row_stride * in.elem, out.img.data,
                                               out.img.row_stride * out.elem, (long long)in.img.w * in.ch * in.elem,
                                               in.img.h, call.stream),
                                   "copy"));
}

// -------------------------------------------------------------- filter table
static const cpipe_cuda_filter_desc kFilters[] = {
    {"precision_convert_r16u_to_f32", (void*)&cpipe_cuda_precision_convert_r16u_to_f32, 0},
    {"precision_convert_f32_to_rgba16f", (void*)&cpipe_cuda_precision_convert_f32_to_rgba16f, 0},
    {"precision_convert_rgba16f_to_rgba8", (void*)&cpipe_cuda_precision_convert_rgba16f_to_rgba8, 0},
    {"precision_convert_rgba16f_to_rgba16u", (void*)&cpipe_cuda_precision_convert_rgba16f_to_rgba16u, 0},
    {"demosaic_quad_bayer_remosaic", (void*)&cpipe_cuda_demosaic_quad_bayer_remosaic, 0},
    {"linearize_dng_lut", (void*)&cpipe_cuda_linearize_dng_lut, 1},
    {"blacklevel_dng_levels", (void*)&cpipe_cuda_blacklevel_dng_levels, 1},
    {"lens_shading_gainmap", (void*)&cpipe_cuda_lens_shading_gainmap, 1},
    {"demosaic_bilinear", (void*)&cpipe_cuda_demosaic_bilinear, 1},
    {"demosaic_rcd", (void*)&cpipe_cuda_demosaic_rcd, 1},
    {"demosaic_amaze", (void*)&cpipe_cuda_demosaic_amaze, 1},
    {"demosaic_rcd_full", (void*)&cpipe_cuda_demosaic_rcd_full, 1},
    {"demosaic_amaze_full", (void*)&cpipe_cuda_demosaic_amaze_full, 1},
    {"wb_dual_illuminant", (void*)&cpipe_cuda_wb_dual_illuminant, 1},
    {"colormatrix_dng_to_working", (void*)&cpipe_cuda_colormatrix_dng_to_working, 1},
    {"denoise_bm3d_step1", (void*)&cpipe_cuda_denoise_bm3d_step1, 1},
    {"denoise_bm3d_step2", (void*)&cpipe_cuda_denoise_bm3d_step2, 1},
    {"denoise_bm3d_spec", (void*)&cpipe_cuda_denoise_bm3d_spec, 1},
    {"denoise_guided_filter", (void*)&cpipe_cuda_denoise_guided_filter, 1},
    {"denoise_wavelet_bayes_shrink", (void*)&cpipe_cuda_denoise_wavelet_bayes_shrink, 1},
    {"denoise_guided_filter_spec", (void*)&cpipe_cuda_denoise_guided_filter_spec, 1},
    {"denoise_wavelet_atrous_spec", (void*)&cpipe_cuda_denoise_wavelet_atrous_spec, 1},
    {"lens_dng_opcode_list_3", (void*)&cpipe_cuda_lens_dng_opcode_list_3, 1},
    {"color_3d_lut", (void*)&cpipe_cuda_color_3d_lut, 1},
    {"tone_filmic_rgb", (void*)&cpipe_cuda_tone_filmic_rgb, 1},
    {"cpipe_wb_greyworld_auto", (void*)&cpipe_cuda_wb_greyworld_auto, 1},
    {"tone_mertens_local", (void*)&cpipe_cuda_tone_mertens_local, 1},
    {"tone_aces_filmic", (void*)&cpipe_cuda_tone_aces_filmic, 1},
    {"tone_reinhard", (void*)&cpipe_cuda_tone_reinhard, 1},
    {"sharpen_edge_aware_usm", (void*)&cpipe_cuda_sharpen_edge_aware_usm, 1},
    {"cpipe_scene_linear_to_display", (void*)&cpipe_cuda_scene_linear_to_display, 1},
    {"cpipe_copy", (void*)&cpipe_cuda_copy, 1},
};

const cpipe_cuda_filter_desc* cpipe_cuda_filters(size_t* count) {
    if (count) *count = sizeof(kFilters) / sizeof(kFilters[0]);
    return kFilters;
}
const cpipe_cuda_filter_desc* cpipe_cuda_find_filter(const char* aot_id) {
    if (aot_id == nullptr) return nullptr;
    for (const auto& f : kFilters)
        if (std::strcmp(f.aot_id, aot_id) == 0) return &f;
    return nullptr;
}

}  // extern "C"
