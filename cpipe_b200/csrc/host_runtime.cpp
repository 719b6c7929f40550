// A small host runtime for the node plugins: the reference host suites
// ("buffer", "metadata", "metadata_builder", "compute", "param", "inference";
// reference src/cpipe/runtime/HostContext.cpp:191-283) implemented over
// device-resident Image2D buffers.
//
// Differences from the reference host that matter for this path:
//  * Buffers live in device memory for their whole life; lock_cpu is a
//    synchronised device->host mirror (write access copies back on unlock).
//  * compute.submit_halide[_with_params] resolves the aot_id in this library's
//    CUDA filter table and passes halide buffers whose `device` field is the
//    device pointer, so filters run in place on the host's CUDA stream.
//  * A device-memory cap makes buffer creation fail with CPIPE_OOM
//    (reference Pipeline.cpp:587-592 checks its planner's peak against a cap).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <memory>
#include <optional>
#include <set>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "../../include/cpipe_b200_dng.h"
#include "host_internal.h"

namespace {

struct Metadata {
    bool has_cfa = false;
    uint8_t cfa_repeat[2] = {0, 0};
    uint8_t cfa_pattern[16] = {0};
    float black[4] = {0, 0, 0, 0};
    uint32_t white = 0;
    std::vector<uint16_t> lin_table;
    std::optional<std::array<float, 9>> m[4];  // color1, color2, forward1, forward2
    uint16_t illum1 = 0, illum2 = 0;
    std::vector<float> noise_beta, noise_lambda;
    float as_shot_neutral[3] = {1.0F, 1.0F, 1.0F};
    std::string cs_role;
    std::vector<std::string> steps;
    std::map<std::string, std::vector<unsigned char>> blobs;
};

uint64_t format_bytes(int fmt) {
    switch (fmt) {
        case CPIPE_FMT_R16_UINT: return 2;
        case CPIPE_FMT_R8G8B8A8_UNORM: return 4;
        case CPIPE_FMT_R16G16B16A16_SFLOAT: return 8;
        case CPIPE_FMT_R16G16B16A16_UNORM: return 8;
        case CPIPE_FMT_R32G32B32A32_SFLOAT: return 16;
        case CPIPE_FMT_R32_SFLOAT: return 4;
        default: return 0;
    }
}
int format_channels(int fmt) {
    switch (fmt) {
        case CPIPE_FMT_R8G8B8A8_UNORM:
        case CPIPE_FMT_R16G16B16A16_SFLOAT:
        case CPIPE_FMT_R16G16B16A16_UNORM:
        case CPIPE_FMT_R32G32B32A32_SFLOAT: return 4;
        default: return 1;
    }
}
halide_type_t halide_type_for(int fmt) {
    switch (fmt) {
        case CPIPE_FMT_R16G16B16A16_SFLOAT: return halide_type_t{halide_type_float, 16, 1};
        case CPIPE_FMT_R32G32B32A32_SFLOAT:
        case CPIPE_FMT_R32_SFLOAT: return halide_type_t{halide_type_float, 32, 1};
        case CPIPE_FMT_R16_UINT:
        case CPIPE_FMT_R16G16B16A16_UNORM: return halide_type_t{halide_type_uint, 16, 1};
        default: return halide_type_t{halide_type_uint, 8, 1};
    }
}

}  // namespace

struct cpipe_b200_host {
    cpipe_host_t abi;  // must stay the first member: suites recover the host from it
    cpipe_buffer_suite_v1 buffer_suite;
    cpipe_metadata_suite_v1 metadata_suite;
    cpipe_metadata_builder_suite_v1 builder_suite;
    cpipe_compute_suite_v1 compute_suite;
    cpipe_param_suite_v1 param_suite;
    cpipe_inference_suite_v1 inference_suite;
    cudaStream_t stream = nullptr;
    uint64_t cap = 0, allocated = 0;
    std::string error;
    std::set<cpipe_b200_buffer*> live;  // buffers still holding device memory
};

struct cpipe_b200_buffer {
    cpipe_b200_host* host = nullptr;
    int format = 0;
    uint32_t w = 0, h = 0;
    void* dev = nullptr;
    size_t bytes = 0;
    bool owned = true;  // false: a view over device memory someone else owns (planner slots)
    std::shared_ptr<Metadata> meta = std::make_shared<Metadata>();
    std::vector<unsigned char> mirror;
    int lock_access = -1;
};

struct cpipe_b200_params {
    std::map<std::string, double> num;
    std::map<std::string, std::string> str;
    std::map<std::string, int> boolean;
};

namespace {

struct Builder {
    Metadata m;
    std::vector<std::shared_ptr<Metadata>> inputs;
};
struct Compute {
    cpipe_b200_host* host;
};

inline cpipe_b200_buffer* B(const cpipe_buffer_t* b) {
    return reinterpret_cast<cpipe_b200_buffer*>(const_cast<cpipe_buffer_t*>(b));
}
inline const Metadata* M(const cpipe_metadata_t* m) { return reinterpret_cast<const Metadata*>(m); }
inline Builder* BL(cpipe_metadata_builder_t* b) { return reinterpret_cast<Builder*>(b); }
inline const cpipe_b200_params* P(const cpipe_props_t* p) { return reinterpret_cast<const cpipe_b200_params*>(p); }
inline cpipe_b200_host* H(cpipe_host_t* h) { return reinterpret_cast<cpipe_b200_host*>(h); }

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}

// ------------------------------------------------------------- buffer suite
int b_get_dims(const cpipe_buffer_t* b, uint8_t* ndim, uint32_t dims[8]) {
    if (!b || !ndim || !dims) return CPIPE_BAD_INDEX;
    *ndim = 2;
    dims[0] = B(b)->w;
    dims[1] = B(b)->h;
    return CPIPE_OK;
}
int b_get_format(const cpipe_buffer_t* b, int* f) {
    if (!b || !f) return CPIPE_BAD_INDEX;
    *f = B(b)->format;
    return CPIPE_OK;
}
int b_get_kind(const cpipe_buffer_t* b, int* k) {
    if (!b || !k) return CPIPE_BAD_INDEX;
    *k = 0;  // Image2D
    return CPIPE_OK;
}
int b_get_stride(const cpipe_buffer_t* b, uint64_t s[8]) {
    if (!b || !s) return CPIPE_BAD_INDEX;
    const uint64_t px = format_bytes(B(b)->format);
    s[0] = px;
    s[1] = px * B(b)->w;
    return CPIPE_OK;
}
int b_get_color_role(const cpipe_buffer_t* b, const char** r) {
    if (!b || !r) return CPIPE_BAD_INDEX;
    *r = B(b)->meta->cs_role.c_str();
    return CPIPE_OK;
}
int b_lock_cpu(cpipe_buffer_t* b, int access, void** ptr) {
    return guarded([&]() -> int {
        if (!b || !ptr) return CPIPE_BAD_INDEX;
        cpipe_b200_buffer* buf = B(b);
        buf->mirror.resize(buf->bytes);
        if (access != CPIPE_CPU_ACCESS_WRITE) {
            if (cudaStreamSynchronize(buf->host->stream) != cudaSuccess ||
                cudaMemcpy(buf->mirror.data(), buf->dev, buf->bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
                return CPIPE_INTERNAL_ERROR;
        }
        buf->lock_access = access;
        *ptr = buf->mirror.data();
        return CPIPE_OK;
    });
}
int b_flush(cpipe_buffer_t* b) {
    if (!b) return CPIPE_BAD_INDEX;
    cpipe_b200_buffer* buf = B(b);
    if (buf->mirror.size() != buf->bytes) return CPIPE_OK;
    return cudaMemcpy(buf->dev, buf->mirror.data(), buf->bytes, cudaMemcpyHostToDevice) == cudaSuccess
               ? CPIPE_OK : CPIPE_INTERNAL_ERROR;
}
int b_unlock_cpu(cpipe_buffer_t* b) {
    if (!b) return CPIPE_BAD_INDEX;
    cpipe_b200_buffer* buf = B(b);
    const int access = buf->lock_access;
    buf->lock_access = -1;
    if (access == CPIPE_CPU_ACCESS_WRITE || access == CPIPE_CPU_ACCESS_READ_WRITE) return b_flush(b);
    return CPIPE_OK;
}
int b_get_metadata(const cpipe_buffer_t* b, const cpipe_metadata_t** out) {
    if (!b || !out) return CPIPE_BAD_INDEX;
    *out = reinterpret_cast<const cpipe_metadata_t*>(B(b)->meta.get());
    return CPIPE_OK;
}

// ----------------------------------------------------------- metadata suite
int m_lin_table(const cpipe_metadata_t* m, size_t max, size_t* n, uint16_t* out) {
    if (!m || !n) return CPIPE_BAD_INDEX;
    const auto& t = M(m)->lin_table;
    *n = t.size();
    if (out) std::copy_n(t.begin(), std::min(max, t.size()), out);
    return CPIPE_OK;
}
int m_noise(const cpipe_metadata_t* m, size_t max, size_t* n, float* a, float* b) {
    if (!m || !n) return CPIPE_BAD_INDEX;
    const Metadata* md = M(m);
    *n = md->noise_beta.size();
    const size_t k = std::min(max, md->noise_beta.size());
    if (a) std::copy_n(md->noise_beta.begin(), k, a);
    if (b) std::copy_n(md->noise_lambda.begin(), k, b);
    return CPIPE_OK;
}
int m_get_calibration(const cpipe_metadata_t* m, cpipe_calibration_view* out) {
    if (!m || !out) return CPIPE_BAD_INDEX;
    const Metadata* md = M(m);
    *out = cpipe_calibration_view{};
    out->has_cfa = md->has_cfa;
    std::memcpy(out->cfa_repeat, md->cfa_repeat, 2);
    std::memcpy(out->cfa_pattern, md->cfa_pattern, 16);
    std::memcpy(out->black_level, md->black, sizeof(md->black));
    out->white_level = md->white;
    out->has_linearization_table = !md->lin_table.empty();
    out->get_linearization_table = &m_lin_table;
    float* dst[4] = {out->color_matrix1, out->color_matrix2, out->forward_matrix1, out->forward_matrix2};
    int* has[4] = {&out->has_color_matrix1, &out->has_color_matrix2, &out->has_forward_matrix1, &out->has_forward_matrix2};
    for (int i = 0; i < 4; ++i) {
        *has[i] = md->m[i].has_value();
        if (md->m[i]) std::memcpy(dst[i], md->m[i]->data(), 9 * sizeof(float));
    }
    out->calibration_illuminant1 = md->illum1;
    out->calibration_illuminant2 = md->illum2;
    out->get_noise_profile = &m_noise;
    return CPIPE_OK;
}
int m_get_capture(const cpipe_metadata_t* m, cpipe_capture_view* out) {
    if (!m || !out) return CPIPE_BAD_INDEX;
    *out = cpipe_capture_view{};
    std::memcpy(out->as_shot_neutral, M(m)->as_shot_neutral, sizeof(float) * 3);
    return CPIPE_OK;
}
int m_get_tq(const cpipe_metadata_t* m, cpipe_tensor_quant_view* out) {
    if (!m || !out) return CPIPE_BAD_INDEX;
    *out = cpipe_tensor_quant_view{};
    return CPIPE_OK;
}
int m_get_cs_role(const cpipe_metadata_t* m, const char** out) {
    if (!m || !out) return CPIPE_BAD_INDEX;
    *out = M(m)->cs_role.c_str();
    return CPIPE_OK;
}
int m_get_active_area(const cpipe_metadata_t*, uint32_t*, uint32_t*, uint32_t*, uint32_t*) { return CPIPE_UNSUPPORTED; }
int m_has_step(const cpipe_metadata_t* m, const char* step, int* out) {
    if (!m || !step || !out) return CPIPE_BAD_INDEX;
    const auto& s = M(m)->steps;
    *out = std::find(s.begin(), s.end(), step) != s.end();
    return CPIPE_OK;
}
int m_list_steps(const cpipe_metadata_t* m, size_t max, size_t* n, const char** out) {
    if (!m || !n) return CPIPE_BAD_INDEX;
    const auto& s = M(m)->steps;
    *n = s.size();
    if (out)
        for (size_t i = 0; i < std::min(max, s.size()); ++i) out[i] = s[i].c_str();
    return CPIPE_OK;
}
int m_get_blob(const cpipe_metadata_t* m, const char* key, const void** ptr, size_t* size) {
    if (!m || !key || !ptr || !size) return CPIPE_BAD_INDEX;
    const auto it = M(m)->blobs.find(key);
    if (it == M(m)->blobs.end()) return CPIPE_NEED_METADATA;
    *ptr = it->second.data();
    *size = it->second.size();
    return CPIPE_OK;
}
int m_list_blobs(const cpipe_metadata_t* m, size_t max, size_t* total, const char** keys) {
    if (!m || !total) return CPIPE_BAD_INDEX;
    *total = M(m)->blobs.size();
    size_t i = 0;
    if (keys)
        for (const auto& kv : M(m)->blobs) {
            if (i >= max) break;
            keys[i++] = kv.first.c_str();
        }
    return CPIPE_OK;
}

// ---------------------------------------------------- metadata builder suite
int mb_share_cal(cpipe_metadata_builder_t* b, size_t idx) {
    if (!b || idx >= BL(b)->inputs.size()) return CPIPE_BAD_INDEX;
    const Metadata& s = *BL(b)->inputs[idx];
    Metadata& d = BL(b)->m;
    d.has_cfa = s.has_cfa;
    std::memcpy(d.cfa_repeat, s.cfa_repeat, 2);
    std::memcpy(d.cfa_pattern, s.cfa_pattern, 16);
    std::memcpy(d.black, s.black, sizeof(d.black));
    d.white = s.white;
    d.lin_table = s.lin_table;
    for (int i = 0; i < 4; ++i) d.m[i] = s.m[i];
    d.illum1 = s.illum1;
    d.illum2 = s.illum2;
    d.noise_beta = s.noise_beta;
    d.noise_lambda = s.noise_lambda;
    return CPIPE_OK;
}
int mb_clear_cal(cpipe_metadata_builder_t* b) {
    if (!b) return CPIPE_BAD_INDEX;
    Metadata& d = BL(b)->m;
    Metadata fresh;
    fresh.as_shot_neutral[0] = d.as_shot_neutral[0];
    fresh.as_shot_neutral[1] = d.as_shot_neutral[1];
    fresh.as_shot_neutral[2] = d.as_shot_neutral[2];
    fresh.cs_role = d.cs_role;
    fresh.steps = d.steps;
    fresh.blobs = d.blobs;
    d = fresh;
    return CPIPE_OK;
}
int mb_clear_cfa(cpipe_metadata_builder_t* b) {
    if (!b) return CPIPE_BAD_INDEX;
    BL(b)->m.has_cfa = false;
    std::memset(BL(b)->m.cfa_repeat, 0, 2);
    std::memset(BL(b)->m.cfa_pattern, 0, 16);
    return CPIPE_OK;
}
int mb_set_asn(cpipe_metadata_builder_t* b, const float rgb[3]) {
    if (!b || !rgb) return CPIPE_BAD_INDEX;
    std::memcpy(BL(b)->m.as_shot_neutral, rgb, sizeof(float) * 3);
    return CPIPE_OK;
}
int mb_set_orient(cpipe_metadata_builder_t* b, uint8_t) { return b ? CPIPE_OK : CPIPE_BAD_INDEX; }
int mb_set_cs_role(cpipe_metadata_builder_t* b, const char* r) {
    if (!b || !r) return CPIPE_BAD_INDEX;
    BL(b)->m.cs_role = r;
    return CPIPE_OK;
}
int mb_add_step(cpipe_metadata_builder_t* b, const char* s) {
    if (!b || !s) return CPIPE_BAD_INDEX;
    auto& v = BL(b)->m.steps;
    if (std::find(v.begin(), v.end(), s) == v.end()) v.emplace_back(s);
    return CPIPE_OK;
}
int mb_remove_step(cpipe_metadata_builder_t* b, const char* s) {
    if (!b || !s) return CPIPE_BAD_INDEX;
    auto& v = BL(b)->m.steps;
    v.erase(std::remove(v.begin(), v.end(), std::string(s)), v.end());
    return CPIPE_OK;
}
int mb_set_active_area(cpipe_metadata_builder_t* b, uint32_t, uint32_t, uint32_t, uint32_t) {
    return b ? CPIPE_UNSUPPORTED : CPIPE_BAD_INDEX;
}
int mb_set_tq(cpipe_metadata_builder_t* b, int, int, int8_t, const float*, size_t, const int32_t*, size_t) {
    return b ? CPIPE_UNSUPPORTED : CPIPE_BAD_INDEX;
}
int mb_set_blob(cpipe_metadata_builder_t* b, const char* key, const void* p, size_t n) {
    if (!b || !key || (!p && n)) return CPIPE_BAD_INDEX;
    const auto* c = static_cast<const unsigned char*>(p);
    BL(b)->m.blobs[key] = std::vector<unsigned char>(c, c + n);
    return CPIPE_OK;
}
int mb_merge_from(cpipe_metadata_builder_t* b, size_t idx, int) {
    if (!b || idx >= BL(b)->inputs.size()) return CPIPE_BAD_INDEX;
    for (const auto& kv : BL(b)->inputs[idx]->blobs) BL(b)->m.blobs.insert(kv);
    for (const auto& s : BL(b)->inputs[idx]->steps) mb_add_step(b, s.c_str());
    return CPIPE_OK;
}
int mb_set_cfa(cpipe_metadata_builder_t* b, const uint8_t repeat[2], const uint8_t pattern[16]) {
    if (!b || !repeat || !pattern) return CPIPE_BAD_INDEX;
    BL(b)->m.has_cfa = true;
    std::memcpy(BL(b)->m.cfa_repeat, repeat, 2);
    std::memcpy(BL(b)->m.cfa_pattern, pattern, 16);
    return CPIPE_OK;
}

// ------------------------------------------------------------ compute suite
void make_halide(cpipe_b200_buffer* b, halide_buffer_t* hb, halide_dimension_t dims[3]) {
    const int ch = format_channels(b->format);
    *hb = halide_buffer_t{};
    hb->device = reinterpret_cast<uint64_t>(b->dev);
    hb->type = halide_type_for(b->format);
    hb->dim = dims;
    if (ch > 1) {
        hb->dimensions = 3;
        dims[0] = halide_dimension_t{0, (int32_t)b->w, ch, 0};
        dims[1] = halide_dimension_t{0, (int32_t)b->h, (int32_t)(b->w * ch), 0};
        dims[2] = halide_dimension_t{0, ch, 1, 0};
    } else {
        hb->dimensions = 2;
        dims[0] = halide_dimension_t{0, (int32_t)b->w, 1, 0};
        dims[1] = halide_dimension_t{0, (int32_t)b->h, (int32_t)b->w, 0};
    }
}
int submit(cpipe_compute_t* c, const char* aot_id, const cpipe_buffer_t* const* ins, size_t n_in,
           cpipe_buffer_t* const* outs, size_t n_out, const void* blob, size_t blob_size, bool with_params) {
    return guarded([&]() -> int {
        if (!c || !aot_id) return CPIPE_BAD_INDEX;
        const cpipe_cuda_filter_desc* f = cpipe_cuda_find_filter(aot_id);
        if (!f) return CPIPE_UNSUPPORTED;
        if ((f->takes_params != 0) != with_params) return CPIPE_UNSUPPORTED;
        std::vector<halide_buffer_t> hb(n_in + n_out);
        std::vector<std::array<halide_dimension_t, 3>> dims(n_in + n_out);
        std::vector<halide_buffer_t*> pin, pout;
        for (size_t i = 0; i < n_in; ++i) {
            if (!ins[i]) return CPIPE_BAD_INDEX;
            make_halide(B(ins[i]), &hb[i], dims[i].data());
            pin.push_back(&hb[i]);
        }
        for (size_t i = 0; i < n_out; ++i) {
            if (!outs[i]) return CPIPE_BAD_INDEX;
            make_halide(B(outs[i]), &hb[n_in + i], dims[n_in + i].data());
            pout.push_back(&hb[n_in + i]);
        }
        cpipe_b200_host* host = reinterpret_cast<Compute*>(c)->host;
        void* prev = cpipe_cuda_get_stream();
        cpipe_cuda_set_stream(host->stream);
        int st;
        if (with_params) {
            using Entry = int (*)(halide_buffer_t* const*, size_t, halide_buffer_t* const*, size_t, const void*, size_t);
            st = reinterpret_cast<Entry>(f->entry)(pin.data(), pin.size(), pout.data(), pout.size(), blob, blob_size);
        } else {
            if (n_in != 1 || n_out != 1) st = CPIPE_BAD_INDEX;
            else {
                using Entry = int (*)(halide_buffer_t*, halide_buffer_t*);
                st = reinterpret_cast<Entry>(f->entry)(pin[0], pout[0]);
            }
        }
        cpipe_cuda_set_stream(prev);
        if (st != CPIPE_OK) host->error = cpipe_cuda_last_error();
        return st;
    });
}
int c_submit_halide(cpipe_compute_t* c, const char* id, const cpipe_buffer_t* const* i, size_t ni,
                    cpipe_buffer_t* const* o, size_t no) {
    return submit(c, id, i, ni, o, no, nullptr, 0, false);
}
int c_submit_halide_params(cpipe_compute_t* c, const char* id, const cpipe_buffer_t* const* i, size_t ni,
                           cpipe_buffer_t* const* o, size_t no, const void* blob, size_t bs) {
    return submit(c, id, i, ni, o, no, blob, bs, true);
}
int c_submit_slang(cpipe_compute_t*, const char*, const char*, const cpipe_buffer_t* const*, size_t,
                   cpipe_buffer_t* const*, size_t, const void*, size_t) {
    return CPIPE_UNSUPPORTED;
}
int c_request_scratch(cpipe_compute_t*, uint64_t, int, cpipe_buffer_t**) { return CPIPE_UNSUPPORTED; }
void c_record_marker(cpipe_compute_t*, const char*) {}
int c_submit_ocio(cpipe_compute_t*, cpipe_ocio_processor_t*, const cpipe_buffer_t*, cpipe_buffer_t*) {
    return CPIPE_UNSUPPORTED;
}
int i_submit_inference(cpipe_inference_t*, const char*, const cpipe_buffer_t* const*, size_t, cpipe_buffer_t* const*,
                       size_t) {
    return CPIPE_UNSUPPORTED;
}

// -------------------------------------------------------------- param suite
int p_get_double(const cpipe_props_t* p, const char* key, double* out) {
    if (!p || !key || !out) return CPIPE_NEED_PARAM;
    const auto it = P(p)->num.find(key);
    if (it == P(p)->num.end()) return CPIPE_NEED_PARAM;
    *out = it->second;
    return CPIPE_OK;
}
int p_get_int(const cpipe_props_t* p, const char* key, int64_t* out) {
    double d;
    const int st = p_get_double(p, key, &d);
    if (st == CPIPE_OK) *out = (int64_t)d;
    return st;
}
int p_get_bool(const cpipe_props_t* p, const char* key, int* out) {
    if (!p || !key || !out) return CPIPE_NEED_PARAM;
    const auto it = P(p)->boolean.find(key);
    if (it == P(p)->boolean.end()) return CPIPE_NEED_PARAM;
    *out = it->second;
    return CPIPE_OK;
}
int p_get_enum(const cpipe_props_t* p, const char* key, const char** out) {
    if (!p || !key || !out) return CPIPE_NEED_PARAM;
    const auto it = P(p)->str.find(key);
    if (it == P(p)->str.end()) return CPIPE_NEED_PARAM;
    *out = it->second.c_str();
    return CPIPE_OK;
}
int p_get_curve(const cpipe_props_t*, const char*, const float**, const float**, size_t*) { return CPIPE_UNSUPPORTED; }
int p_get_color(const cpipe_props_t*, const char*, float[4]) { return CPIPE_UNSUPPORTED; }

// --------------------------------------------------------------------- host
const void* h_get_suite(cpipe_host_t* self, const char* name, int version) {
    if (!self || !name || version != 1) return nullptr;
    cpipe_b200_host* h = H(self);
    if (!std::strcmp(name, "buffer")) return &h->buffer_suite;
    if (!std::strcmp(name, "compute")) return &h->compute_suite;
    if (!std::strcmp(name, "param")) return &h->param_suite;
    if (!std::strcmp(name, "inference")) return &h->inference_suite;
    if (!std::strcmp(name, "metadata")) return &h->metadata_suite;
    if (!std::strcmp(name, "metadata_builder")) return &h->builder_suite;
    return nullptr;
}
void h_log(cpipe_host_t* self, int, const char* msg) {
    if (self && msg) H(self)->error = msg;
}
void* h_alloc(cpipe_host_t*, size_t n) { return std::malloc(n); }
void h_free(cpipe_host_t*, void* p) { std::free(p); }
cpipe_ocio_processor_t* h_ocio(cpipe_host_t*, const char*, const char*, const char*) { return nullptr; }

}  // namespace

extern "C" {

cpipe_b200_host* cpipe_b200_host_create(void) {
    auto* h = new (std::nothrow) cpipe_b200_host();
    if (!h) return nullptr;
    h->abi = cpipe_host_t{CPIPE_ABI_MAJOR, CPIPE_ABI_MINOR, &h_get_suite, &h_log, &h_alloc, &h_free, &h_ocio};
    h->buffer_suite = cpipe_buffer_suite_v1{&b_get_dims, &b_get_format, &b_get_kind, &b_get_stride, &b_get_color_role,
                                            &b_lock_cpu, &b_unlock_cpu, &b_flush, &b_get_metadata};
    h->metadata_suite = cpipe_metadata_suite_v1{&m_get_calibration, &m_get_capture, &m_get_tq, &m_get_cs_role,
                                                &m_get_active_area, &m_has_step, &m_list_steps, &m_get_blob,
                                                &m_list_blobs};
    h->builder_suite = cpipe_metadata_builder_suite_v1{&mb_share_cal, &mb_clear_cal, &mb_clear_cfa, &mb_set_asn,
                                                       &mb_set_orient, &mb_set_cs_role, &mb_add_step, &mb_remove_step,
                                                       &mb_set_active_area, &mb_set_tq, &mb_set_blob, &mb_merge_from,
                                                       &mb_set_cfa};
    h->compute_suite = cpipe_compute_suite_v1{&c_submit_halide, &c_submit_slang, &c_request_scratch, &c_record_marker,
                                              &c_submit_halide_params, &c_submit_ocio};
    h->param_suite = cpipe_param_suite_v1{&p_get_double, &p_get_int, &p_get_bool, &p_get_enum, &p_get_curve, &p_get_color};
    h->inference_suite = cpipe_inference_suite_v1{&i_submit_inference};
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return nullptr;
    }
    return h;
}
// Destroying the host releases the device memory of every buffer still alive;
// those buffer handles stay valid for cpipe_b200_buffer_destroy (which then only
// frees the handle), whatever order the caller releases things in.
void cpipe_b200_host_destroy(cpipe_b200_host* h) {
    if (!h) return;
    cudaStreamSynchronize(h->stream);
    for (cpipe_b200_buffer* b : h->live) {
        cudaFree(b->dev);
        b->dev = nullptr;
        b->host = nullptr;
    }
    cudaStreamDestroy(h->stream);
    delete h;
}
cpipe_host_t* cpipe_b200_host_abi(cpipe_b200_host* h) { return h ? &h->abi : nullptr; }
int cpipe_b200_host_set_memory_cap(cpipe_b200_host* h, uint64_t bytes) {
    if (!h) return CPIPE_BAD_INDEX;
    h->cap = bytes;
    return CPIPE_OK;
}
const char* cpipe_b200_host_last_error(cpipe_b200_host* h) { return h ? h->error.c_str() : ""; }

cpipe_b200_buffer* cpipe_b200_buffer_create(cpipe_b200_host* h, int format, uint32_t w, uint32_t hgt) {
    if (!h || w == 0 || hgt == 0 || format_bytes(format) == 0) return nullptr;
    const size_t bytes = (size_t)w * hgt * format_bytes(format);
    if (h->cap && h->allocated + bytes > h->cap) {
        h->error = "device memory cap exceeded (CPIPE_OOM)";
        return nullptr;
    }
    auto* b = new (std::nothrow) cpipe_b200_buffer();
    if (!b) return nullptr;
    if (cudaMalloc(&b->dev, bytes) != cudaSuccess) {
        cudaGetLastError();
        h->error = "cudaMalloc failed (CPIPE_OOM)";
        delete b;
        return nullptr;
    }
    b->host = h;
    h->live.insert(b);
    b->format = format;
    b->w = w;
    b->h = hgt;
    b->bytes = bytes;
    h->allocated += bytes;
    return b;
}
void cpipe_b200_buffer_destroy(cpipe_b200_buffer* b) {
    if (!b) return;
    if (b->host && b->owned) {
        cudaStreamSynchronize(b->host->stream);
        cudaFree(b->dev);
        b->host->allocated -= b->bytes;
        b->host->live.erase(b);
    }
    delete b;
}
int cpipe_b200_buffer_upload(cpipe_b200_buffer* b, const void* data, size_t bytes) {
    if (!b || !b->host || !data || bytes != b->bytes) return CPIPE_BAD_INDEX;
    if (cudaMemcpyAsync(b->dev, data, bytes, cudaMemcpyHostToDevice, b->host->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->host->stream) != cudaSuccess)
        return CPIPE_INTERNAL_ERROR;
    return CPIPE_OK;
}
int cpipe_b200_buffer_download(cpipe_b200_buffer* b, void* data, size_t bytes) {
    if (!b || !b->host || !data || bytes != b->bytes) return CPIPE_BAD_INDEX;
    if (cudaMemcpyAsync(data, b->dev, bytes, cudaMemcpyDeviceToHost, b->host->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->host->stream) != cudaSuccess)
        return CPIPE_INTERNAL_ERROR;
    return CPIPE_OK;
}
void* cpipe_b200_buffer_device_ptr(cpipe_b200_buffer* b) { return b ? b->dev : nullptr; }
int cpipe_b200_buffer_format(const cpipe_b200_buffer* b) { return b ? b->format : 0; }
const cpipe_buffer_t* cpipe_b200_buffer_abi(cpipe_b200_buffer* b) { return reinterpret_cast<const cpipe_buffer_t*>(b); }

int cpipe_b200_buffer_set_cfa(cpipe_b200_buffer* b, const uint8_t repeat[2], const uint8_t pattern[16]) {
    if (!b || !repeat || !pattern) return CPIPE_BAD_INDEX;
    b->meta->has_cfa = true;
    std::memcpy(b->meta->cfa_repeat, repeat, 2);
    std::memcpy(b->meta->cfa_pattern, pattern, 16);
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_levels(cpipe_b200_buffer* b, const float black[4], uint32_t white) {
    if (!b || !black) return CPIPE_BAD_INDEX;
    std::memcpy(b->meta->black, black, sizeof(float) * 4);
    b->meta->white = white;
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_matrix(cpipe_b200_buffer* b, int which, const float m[9]) {
    if (!b || which < 1 || which > 4) return CPIPE_BAD_INDEX;
    if (!m) {
        b->meta->m[which - 1].reset();
        return CPIPE_OK;
    }
    std::array<float, 9> a;
    std::memcpy(a.data(), m, sizeof(float) * 9);
    b->meta->m[which - 1] = a;
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_illuminants(cpipe_b200_buffer* b, uint16_t i1, uint16_t i2) {
    if (!b) return CPIPE_BAD_INDEX;
    b->meta->illum1 = i1;
    b->meta->illum2 = i2;
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_linearization_table(cpipe_b200_buffer* b, const uint16_t* v, size_t n) {
    if (!b || (!v && n)) return CPIPE_BAD_INDEX;
    b->meta->lin_table.assign(v, v + n);
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_noise_profile(cpipe_b200_buffer* b, const float* beta, const float* lambda, size_t n) {
    if (!b || ((!beta || !lambda) && n)) return CPIPE_BAD_INDEX;
    b->meta->noise_beta.assign(beta, beta + n);
    b->meta->noise_lambda.assign(lambda, lambda + n);
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_as_shot_neutral(cpipe_b200_buffer* b, const float rgb[3]) {
    if (!b || !rgb) return CPIPE_BAD_INDEX;
    std::memcpy(b->meta->as_shot_neutral, rgb, sizeof(float) * 3);
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_cs_role(cpipe_b200_buffer* b, const char* role) {
    if (!b || !role) return CPIPE_BAD_INDEX;
    b->meta->cs_role = role;
    return CPIPE_OK;
}
int cpipe_b200_buffer_add_applied_step(cpipe_b200_buffer* b, const char* step) {
    if (!b || !step) return CPIPE_BAD_INDEX;
    auto& v = b->meta->steps;
    if (std::find(v.begin(), v.end(), step) == v.end()) v.emplace_back(step);
    return CPIPE_OK;
}
int cpipe_b200_buffer_set_blob(cpipe_b200_buffer* b, const char* key, const void* data, size_t size) {
    if (!b || !key || (!data && size)) return CPIPE_BAD_INDEX;
    const auto* c = static_cast<const unsigned char*>(data);
    b->meta->blobs[key] = std::vector<unsigned char>(c, c + size);
    return CPIPE_OK;
}
int cpipe_b200_buffer_has_applied_step(cpipe_b200_buffer* b, const char* step) {
    if (!b || !step) return 0;
    const auto& v = b->meta->steps;
    return std::find(v.begin(), v.end(), step) != v.end();
}
const char* cpipe_b200_buffer_cs_role(cpipe_b200_buffer* b) { return b ? b->meta->cs_role.c_str() : ""; }
int cpipe_b200_buffer_get_blob(cpipe_b200_buffer* b, const char* key, const void** data, size_t* size) {
    if (!b || !key || !data || !size) return CPIPE_BAD_INDEX;
    const auto it = b->meta->blobs.find(key);
    if (it == b->meta->blobs.end()) return CPIPE_NEED_METADATA;
    *data = it->second.data();
    *size = it->second.size();
    return CPIPE_OK;
}
int cpipe_b200_buffer_get_cfa(cpipe_b200_buffer* b, int* has_cfa, uint8_t repeat[2], uint8_t pattern[16]) {
    if (!b || !has_cfa || !repeat || !pattern) return CPIPE_BAD_INDEX;
    *has_cfa = b->meta->has_cfa;
    std::memcpy(repeat, b->meta->cfa_repeat, 2);
    std::memcpy(pattern, b->meta->cfa_pattern, 16);
    return CPIPE_OK;
}

cpipe_b200_params* cpipe_b200_params_create(void) { return new (std::nothrow) cpipe_b200_params(); }
void cpipe_b200_params_destroy(cpipe_b200_params* p) { delete p; }
int cpipe_b200_params_set_double(cpipe_b200_params* p, const char* k, double v) {
    if (!p || !k) return CPIPE_BAD_INDEX;
    p->num[k] = v;
    return CPIPE_OK;
}
int cpipe_b200_params_set_string(cpipe_b200_params* p, const char* k, const char* v) {
    if (!p || !k || !v) return CPIPE_BAD_INDEX;
    p->str[k] = v;
    return CPIPE_OK;
}
int cpipe_b200_params_set_bool(cpipe_b200_params* p, const char* k, int v) {
    if (!p || !k) return CPIPE_BAD_INDEX;
    p->boolean[k] = v != 0;
    return CPIPE_OK;
}

int cpipe_b200_run_node(cpipe_b200_host* h, const char* node_id, const cpipe_b200_params* params,
                        cpipe_b200_buffer* const* inputs, size_t n_in, cpipe_b200_buffer* const* outputs,
                        size_t n_out) {
    if (!h || !node_id) return CPIPE_BAD_INDEX;
    const cpipe_plugin_desc_t* desc = cpipe_b200_find_node(node_id);
    if (!desc) {
        h->error = std::string("unknown node id ") + node_id;
        return CPIPE_BAD_INDEX;
    }
    return cpb_run_node(h, desc, params, inputs, n_in, outputs, n_out, true);
}

}  // extern "C"

// ------------------------------------------------------- pipeline runner hooks
cpipe_b200_buffer* cpb_buffer_view(cpipe_b200_host* h, int format, uint32_t w, uint32_t hgt, void* dev) {
    if (!h || !dev || w == 0 || hgt == 0 || format_bytes(format) == 0) return nullptr;
    auto* b = new (std::nothrow) cpipe_b200_buffer();
    if (!b) return nullptr;
    b->host = h;
    b->format = format;
    b->w = w;
    b->h = hgt;
    b->dev = dev;
    b->bytes = (size_t)w * hgt * format_bytes(format);
    b->owned = false;
    return b;
}
size_t cpb_format_bytes(int format) { return (size_t)format_bytes(format); }
int cpb_buffer_format(const cpipe_b200_buffer* b) { return b ? b->format : 0; }
void cpb_buffer_extent(const cpipe_b200_buffer* b, uint32_t* w, uint32_t* h) {
    *w = b ? b->w : 0;
    *h = b ? b->h : 0;
}
void cpb_buffer_share_metadata(cpipe_b200_buffer* dst, const cpipe_b200_buffer* src) {
    if (dst && src) dst->meta = src->meta;
}
cudaStream_t cpb_host_stream(cpipe_b200_host* h) { return h ? h->stream : nullptr; }
bool cpb_is_own_host(const cpipe_host_t* h) { return h && h->get_suite == &h_get_suite; }
cudaStream_t cpb_abi_host_stream(cpipe_host_t* h) { return cpb_is_own_host(h) ? H(h)->stream : nullptr; }
void* cpb_buffer_device(const cpipe_buffer_t* b) { return b ? B(b)->dev : nullptr; }
// The DNG's calibration, capture and blobs as DngReader attaches them
// (DngReader.cpp:214-230), written into one of this host's builders.
int cpb_builder_set_dng(cpipe_metadata_builder_t* builder, const cpipe_DngInfo* info, const uint8_t* file,
                        size_t file_bytes) {
    if (!builder || !info || !file) return CPIPE_BAD_INDEX;
    Metadata& m = BL(builder)->m;
    m = Metadata{};
    m.has_cfa = true;
    m.cfa_repeat[0] = (uint8_t)info->cfa_repeat[0];
    m.cfa_repeat[1] = (uint8_t)info->cfa_repeat[1];
    std::memcpy(m.cfa_pattern, info->cfa_pattern, 16);
    std::memcpy(m.black, info->black_level, sizeof(m.black));
    m.white = info->white_level;
    for (int k = 0; k < 4; ++k) {
        if (!info->has_matrix[k]) continue;
        std::array<float, 9> a;
        std::memcpy(a.data(), info->matrix[k], sizeof(float) * 9);
        m.m[k] = a;
    }
    m.illum1 = (uint16_t)info->calibration_illuminant[0];
    m.illum2 = (uint16_t)info->calibration_illuminant[1];
    std::memcpy(m.as_shot_neutral, info->as_shot_neutral, sizeof(m.as_shot_neutral));
    m.cs_role = "raw_camera";
    auto range = [&](uint32_t off, uint32_t n) -> const uint8_t* {
        return (n && (uint64_t)off + n <= file_bytes) ? file + off : nullptr;
    };
    if (const uint8_t* p = range(info->linearization_offset, 2 * info->linearization_count)) {
        m.lin_table.resize(info->linearization_count);
        for (uint32_t i = 0; i < info->linearization_count; ++i) m.lin_table[i] = (uint16_t)(p[2 * i] | (p[2 * i + 1] << 8));
    }
    static const char* kOpcodeKeys[3] = {"com.cpipe.dng.opcode_list_1_bytes", "com.cpipe.dng.opcode_list_2_bytes",
                                         "com.cpipe.dng.opcode_list_3_bytes"};
    for (int k = 0; k < 3; ++k)
        if (const uint8_t* p = range(info->opcode_list_offset[k], info->opcode_list_bytes[k]))
            m.blobs[kOpcodeKeys[k]] = std::vector<unsigned char>(p, p + info->opcode_list_bytes[k]);
    return CPIPE_OK;
}
uint64_t cpb_host_memory_cap(cpipe_b200_host* h) { return h ? h->cap : 0; }
void cpb_host_set_error(cpipe_b200_host* h, const std::string& e) {
    if (h) h->error = e;
}
const std::string& cpb_host_error(cpipe_b200_host* h) { return h->error; }

// One node through its main_entry (create, process, destroy) on the host's
// stream; with sync == false its kernels stay queued (the pipeline runner
// synchronises once per run).
int cpb_run_node(cpipe_b200_host* h, const cpipe_plugin_desc_t* desc, const cpipe_b200_params* params,
                 cpipe_b200_buffer* const* inputs, size_t n_in, cpipe_b200_buffer* const* outputs, size_t n_out,
                 bool sync) {
    cpipe_b200_params empty;
    cpipe_props_t* props = reinterpret_cast<cpipe_props_t*>(const_cast<cpipe_b200_params*>(params ? params : &empty));
    void* instance = nullptr;
    int st = desc->main_entry(CPIPE_ACTION_CREATE, &h->abi, nullptr, props, nullptr, &instance);
    if (st != CPIPE_OK) return st;
    std::vector<const cpipe_buffer_t*> ins(n_in);
    std::vector<cpipe_buffer_t*> outs(n_out);
    std::vector<Builder> builders(n_out);
    std::vector<cpipe_metadata_builder_t*> bptrs(n_out);
    for (size_t i = 0; i < n_in; ++i) ins[i] = reinterpret_cast<const cpipe_buffer_t*>(inputs[i]);
    for (size_t i = 0; i < n_out; ++i) {
        outs[i] = reinterpret_cast<cpipe_buffer_t*>(outputs[i]);
        // inherits_from: the first input's metadata (reference Pipeline.cpp:744-760)
        if (n_in > 0 && inputs[0]) builders[i].m = *inputs[0]->meta;
        for (size_t k = 0; k < n_in; ++k)
            if (inputs[k]) builders[i].inputs.push_back(inputs[k]->meta);
        bptrs[i] = reinterpret_cast<cpipe_metadata_builder_t*>(&builders[i]);
    }
    Compute compute{h};
    cpipe_process_ctx ctx{reinterpret_cast<cpipe_compute_t*>(&compute), nullptr, ins.data(), n_in, outs.data(), n_out,
                          bptrs.data()};
    h->error.clear();
    st = desc->main_entry(CPIPE_ACTION_PROCESS, &h->abi, reinterpret_cast<cpipe_node_t*>(instance), props, &ctx, nullptr);
    const int dst = desc->main_entry(CPIPE_ACTION_DESTROY, &h->abi, nullptr, props, instance, nullptr);
    const cudaError_t e = sync ? cudaStreamSynchronize(h->stream) : cudaGetLastError();
    if (st == CPIPE_OK && e != cudaSuccess) {
        h->error = cudaGetErrorString(e);
        st = CPIPE_INTERNAL_ERROR;
    }
    if (st == CPIPE_OK) {
        for (size_t i = 0; i < n_out; ++i)
            if (outputs[i]) outputs[i]->meta = std::make_shared<Metadata>(builders[i].m);
    }
    return st != CPIPE_OK ? st : dst;
}
