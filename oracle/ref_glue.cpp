/* Glue for the oracle's reference build: the reference's own plain-C++ filters
 * (compiled unmodified from the reference tree, see oracle/Makefile) register
 * themselves through the stand-in HalideFilterRegistry.hpp; this file keeps the
 * table and exposes C entry points so the tests can call a reference filter by
 * its aot_id, and the reference white-balance helpers (WbMetadata.hpp).
 * Test infrastructure only: never linked into the product library. */
#include <HalideRuntime.h>
#include <cpipe/runtime/HalideFilterRegistry.hpp>

#include <cstring>
#include <map>
#include <string>

#include "wb/WbMetadata.hpp"

namespace {
std::map<std::string, RefParamFilterEntry>& param_table() {
    static std::map<std::string, RefParamFilterEntry> t;
    return t;
}
std::map<std::string, RefFilterEntry>& plain_table() {
    static std::map<std::string, RefFilterEntry> t;
    return t;
}
}  // namespace

void cpipe_ref_register_filter(const char* aot_id, RefFilterEntry entry) { plain_table()[aot_id] = entry; }
void cpipe_ref_register_param_filter(const char* aot_id, RefParamFilterEntry entry) {
    param_table()[aot_id] = entry;
}

extern "C" int cpipe_ref_call(const char* aot_id, halide_buffer_t* const* in, size_t n_in,
                              halide_buffer_t* const* out, size_t n_out, const void* blob,
                              size_t blob_size) {
    auto it = param_table().find(aot_id);
    if (it == param_table().end()) return -1;
    return it->second(in, n_in, out, n_out, blob, blob_size);
}

extern "C" int cpipe_ref_has(const char* aot_id) { return param_table().count(aot_id) ? 1 : 0; }

/* Reference dual-illuminant interpolation (WbMetadata.hpp interpolate_calibration).
 * fm1/fm2 may be NULL.  Returns the cpipe status; fills camera_to_xyz[9], cct, weight. */
extern "C" int cpipe_ref_wb_interpolate(const float neutral[3], const float cm1[9], const float cm2[9],
                                        const float* fm1, const float* fm2, unsigned illum1,
                                        unsigned illum2, float camera_to_xyz[9], double* cct,
                                        float* weight) {
    using namespace cpipe::nodes::wb_detail;
    cpipe::sdk::CalibrationView cal;
    Matrix3 a{}, b{};
    std::memcpy(a.data(), cm1, sizeof(float) * 9);
    std::memcpy(b.data(), cm2, sizeof(float) * 9);
    cal.color_matrix1 = a;
    cal.color_matrix2 = b;
    if (fm1 && fm2) {
        Matrix3 f1{}, f2{};
        std::memcpy(f1.data(), fm1, sizeof(float) * 9);
        std::memcpy(f2.data(), fm2, sizeof(float) * 9);
        cal.forward_matrix1 = f1;
        cal.forward_matrix2 = f2;
    }
    cal.calibration_illuminant1 = static_cast<std::uint16_t>(illum1);
    cal.calibration_illuminant2 = static_cast<std::uint16_t>(illum2);
    const Vec3 n{neutral[0], neutral[1], neutral[2]};
    const auto r = interpolate_calibration(cal, n);
    if (!r) return r.error().code;
    std::memcpy(camera_to_xyz, r->camera_to_xyz_d50.data(), sizeof(float) * 9);
    *cct = r->scene_cct;
    *weight = r->blend_weight;
    return 0;
}
