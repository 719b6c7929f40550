// Internal helpers shared by the filter seam (filters.cu), the node plugins
// (nodes_plugin.cpp) and the fused chain (chain.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "kernels.h"

namespace cpb {

enum class Kind { BayerU16, BayerF32, Rgba, RgbaU8, RgbaU16, Any };

struct Bound {
    Img img{};
    halide_buffer_t* hb = nullptr;
    int elem = 0, ch = 0;
    bool staged = false, is_output = false;
};

// One filter invocation: binds halide buffers (device in place, or host staged
// through device memory), owns per-call device scratch (stream-ordered
// allocations), and on finish() copies staged outputs back and synchronises.
struct Call {
    cudaStream_t stream;
    std::vector<Bound> bounds;
    std::vector<void*> scratch;
    bool staged_any = false;
    Call();
    ~Call();
    int bind(halide_buffer_t* hb, Kind kind, bool is_output, Bound* out);
    int alloc(size_t bytes, void** out);
    int upload(const void* host, size_t bytes, void** out);
    int finish(int status);
};

// Prepared-table cache (filters.cu): a device copy of a filter's prepared
// tables keyed by (kind, frame extent, parameter blob bytes).  Hold a
// TableLock from table_find / table_add until the kernels that read the entry
// are launched.
enum TableKind { kTabLinearize = 1, kTabGainMap = 2, kTabLut = 3 };
struct TableEntry {
    int dev = 0, kind = 0, w = 0, h = 0;
    std::vector<unsigned char> key;
    void* d = nullptr;
    std::vector<unsigned char> meta;  // kind-specific host values (GainMapDev, LUT size / interpolation)
    uint64_t used = 0;
};
struct TableLock {
    std::unique_lock<std::mutex> lock;
    TableLock();
};
const TableEntry* table_find(int kind, int w, int h, const void* key, size_t key_bytes);
// Copies host_bytes of `host` into a new device entry of device_bytes (which
// may leave room for tables filled on the device), evicting the least recently
// used entry when the set is full.
int table_add(int kind, int w, int h, const void* key, size_t key_bytes, const void* host, size_t host_bytes,
              size_t device_bytes, TableEntry** out);

struct Opcode3View {
    uint32_t count = 0;
    const cpipe_Opcode3DispatchRecord* records = nullptr;
    const cpipe_Opcode3BadPoint* points = nullptr;
    const cpipe_Opcode3BadRect* rects = nullptr;
    size_t npoints = 0, nrects = 0;
};

void set_error(const char* fmt, const char* detail);
cudaStream_t current_stream();
int cuda_status(cudaError_t e, const char* where);
bool device_ready();
ff split(double v);
// Lossless JPEG segments (lj92.cu; cpipe_cuda_lj92_decode's contract).
int lj92_decode(const uint8_t* const* streams, const size_t* bytes, uint32_t count, uint32_t across, uint32_t seg_w,
                uint32_t seg_h, uint32_t width, uint32_t height, uint16_t* d_raw);

}  // namespace cpb

// Host-side parameter preparation, shared with the chain builder (C linkage
// so the definitions inside filters.cu's extern "C" block match).
extern "C" {
int cpb_blacklevel_dev(const cpipe_BlacklevelParams* p, int w, int h, cpb::BlackDev* out);
int cpb_gainmap_prepare(const void* blob, size_t blob_size, int w, int h, std::vector<char>* table,
                        cpb::GainMapDev* g, size_t offsets[3][4]);
void cpb_gainmap_bind(cpb::GainMapDev* g, const char* d_table, size_t offsets[3][4]);
int cpb_lut_prepare(const void* blob, size_t blob_size, std::vector<float4>* cells, int* S, int* interp);
cpb::FilmicDev cpb_filmic_dev(const cpipe_FilmicRgbParams* p);
int cpb_warp_dev(const cpipe_Opcode3DispatchRecord* r, int w, int h, cpb::WarpDev* out);
int cpb_opcode3_parse(const void* blob, size_t blob_size, cpb::Opcode3View* v);
int cpb_opcode3_run(cpb::Call& call, const cpb::Opcode3View& v, const cpb::Img& in, const cpb::Img& out, int elem);
}  // extern "C"
