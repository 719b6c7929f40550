// Node plugins: one cpipe_plugin_desc_t per reference node id, placed in the
// `cpipe_registry` ELF section so a reference host's Registry::load_builtin_nodes
// (reference src/cpipe/runtime/Registry.cpp:13-26) discovers them, and listed by
// cpipe_b200_node_descs().  Each main_entry follows the reference node's
// process() (cited per node): buffer/format/metadata checks with the same
// status codes, host-side parameter preparation, then the kernel is submitted
// through the host's compute suite by aot_id (which this library's host
// resolves to the CUDA filters), and finally the metadata builder edits.
//
// Actions (reference include/cpipe/sdk/sdk.hpp:632-703): "describe" ->
// CPIPE_REPLY_DEFAULT, "create" -> a per-instance object, "prepare" -> OK,
// "process" -> run, "destroy" -> free.  No C++ exception crosses main_entry.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "../../include/cpipe_b200_dng.h"
#include "host_internal.h"
#include "host_prep.h"

namespace {

using cpb::prep::Mat3;
using cpb::prep::Vec3;

// ------------------------------------------------------------ suite access
struct Ctx {
    cpipe_host_t* host;
    const cpipe_buffer_suite_v1* buf;
    const cpipe_metadata_suite_v1* meta;
    const cpipe_metadata_builder_suite_v1* mb;
    const cpipe_compute_suite_v1* compute;
    const cpipe_param_suite_v1* param;
    const cpipe_props_t* props;
    cpipe_process_ctx* pc;
    std::string msg;

    bool init() {
        buf = static_cast<const cpipe_buffer_suite_v1*>(host->get_suite(host, "buffer", 1));
        meta = static_cast<const cpipe_metadata_suite_v1*>(host->get_suite(host, "metadata", 1));
        mb = static_cast<const cpipe_metadata_builder_suite_v1*>(host->get_suite(host, "metadata_builder", 1));
        compute = static_cast<const cpipe_compute_suite_v1*>(host->get_suite(host, "compute", 1));
        param = static_cast<const cpipe_param_suite_v1*>(host->get_suite(host, "param", 1));
        return buf && meta && mb && compute;
    }
    const cpipe_buffer_t* in(size_t i) const { return pc->inputs[i]; }
    cpipe_buffer_t* out(size_t i) const { return pc->outputs[i]; }
    cpipe_metadata_builder_t* builder() const { return pc->out_metadata[0]; }
    int format(const cpipe_buffer_t* b, int* f) const { return buf->get_format(b, f); }
    int dims(const cpipe_buffer_t* b, uint32_t* w, uint32_t* h) const {
        uint8_t nd = 0;
        uint32_t d[8] = {0};
        const int st = buf->get_dims(b, &nd, d);
        if (st != CPIPE_OK) return st;
        if (nd != 2 || d[0] == 0 || d[1] == 0) return CPIPE_BAD_INDEX;
        *w = d[0];
        *h = d[1];
        return CPIPE_OK;
    }
    const cpipe_metadata_t* metadata(const cpipe_buffer_t* b) const {
        const cpipe_metadata_t* m = nullptr;
        if (buf->get_metadata(b, &m) != CPIPE_OK) return nullptr;
        return m;
    }
    bool blob(const cpipe_metadata_t* m, const char* key, const void** p, size_t* n) const {
        return meta->get_blob(m, key, p, n) == CPIPE_OK;
    }
    bool has_step(const cpipe_metadata_t* m, const char* step) const {
        int b = 0;
        return meta->has_applied_step(m, step, &b) == CPIPE_OK && b != 0;
    }
    bool get_double(const char* key, double* v) const {
        return param && param->get_double && props && param->get_double(props, key, v) == CPIPE_OK;
    }
    double double_or(const char* key, double fallback) const {
        double v;
        return get_double(key, &v) ? v : fallback;
    }
    // ParamUtils.hpp:22-35: clamp after casting, as the reference helpers do.
    float clamped_float(const char* key, float fb, float lo, float hi) const {
        return std::clamp((float)double_or(key, fb), lo, hi);
    }
    int clamped_int(const char* key, int fb, int lo, int hi) const { return std::clamp((int)double_or(key, fb), lo, hi); }
    // ParamUtils.hpp:37-50: the fallback when the suite or the key is missing
    bool bool_or(const char* key, bool fallback) const {
        int v = 0;
        if (!param || !param->get_bool || !props || param->get_bool(props, key, &v) != CPIPE_OK) return fallback;
        return v != 0;
    }
    bool get_string(const char* key, std::string* s) const {
        const char* v = nullptr;
        if (!param || !param->get_enum || !props || param->get_enum(props, key, &v) != CPIPE_OK || !v) return false;
        *s = v;
        return true;
    }
    int submit(const char* aot, const void* blob, size_t n) {
        return compute->submit_halide_with_params(pc->compute, aot, pc->inputs, pc->n_in, pc->outputs, pc->n_out, blob, n);
    }
    int submit_plain(const char* aot) {
        return compute->submit_halide(pc->compute, aot, pc->inputs, pc->n_in, pc->outputs, pc->n_out);
    }
    // Pass-through copy: on the device when the host routes "cpipe_copy" to
    // this library, otherwise through lock_cpu as the reference does
    // (e.g. shading_gainmap.cpp:50-75).
    int copy_through(size_t bytes_per_px) {
        int st = submit("cpipe_copy", nullptr, 0);
        if (st != CPIPE_UNSUPPORTED) return st;
        uint32_t w, h;
        if ((st = dims(in(0), &w, &h)) != CPIPE_OK) return st;
        void* src = nullptr;
        void* dst = nullptr;
        if ((st = buf->lock_cpu(const_cast<cpipe_buffer_t*>(in(0)), CPIPE_CPU_ACCESS_READ, &src)) != CPIPE_OK) return st;
        if ((st = buf->lock_cpu(out(0), CPIPE_CPU_ACCESS_WRITE, &dst)) != CPIPE_OK) {
            buf->unlock_cpu(const_cast<cpipe_buffer_t*>(in(0)));
            return st;
        }
        std::memcpy(dst, src, (size_t)w * h * bytes_per_px);
        buf->unlock_cpu(const_cast<cpipe_buffer_t*>(in(0)));
        st = buf->unlock_cpu(out(0));
        return st != CPIPE_OK ? st : buf->flush_cpu_writes(out(0));
    }
    int step(const char* s) { return mb->add_applied_step(builder(), s); }
};

// nin inputs and one output, all present, with an output metadata builder.
bool n_to_one(const cpipe_process_ctx* pc, size_t nin) {
    if (!pc || pc->n_in != nin || pc->n_out != 1 || (nin > 0 && !pc->inputs) || !pc->outputs || !pc->outputs[0] ||
        !pc->out_metadata || !pc->out_metadata[0])
        return false;
    for (size_t i = 0; i < nin; ++i)
        if (!pc->inputs[i]) return false;
    return true;
}

int check_formats(Ctx& c, int fin, int fout) {
    int a = 0, b = 0;
    int st = c.format(c.in(0), &a);
    if (st == CPIPE_OK) st = c.format(c.out(0), &b);
    if (st != CPIPE_OK) return st;
    if (a != fin || b != fout) return CPIPE_BAD_PRECISION;
    uint32_t w, h;
    return c.dims(c.in(0), &w, &h);
}
// RGBA nodes accept the reference R16G16B16A16_SFLOAT or the FP32 plain form.
int check_rgba(Ctx& c) {
    int a = 0, b = 0;
    int st = c.format(c.in(0), &a);
    if (st == CPIPE_OK) st = c.format(c.out(0), &b);
    if (st != CPIPE_OK) return st;
    if (a != b || (a != CPIPE_FMT_R16G16B16A16_SFLOAT && a != CPIPE_FMT_R32G32B32A32_SFLOAT)) return CPIPE_BAD_PRECISION;
    uint32_t w, h;
    return c.dims(c.in(0), &w, &h);
}
size_t rgba_bytes(Ctx& c) {
    int f = 0;
    c.format(c.in(0), &f);
    return f == CPIPE_FMT_R32G32B32A32_SFLOAT ? 16 : 8;
}

bool calibration(Ctx& c, const cpipe_metadata_t* m, cpipe_calibration_view* cal) {
    return m && c.meta->get_calibration(m, cal) == CPIPE_OK;
}

// ===================================================================== nodes
// precision_convert.cpp:13-96
int node_precision_convert(Ctx& c) {
    std::string target;
    if (!c.get_string("target_format", &target)) return CPIPE_NEED_PARAM;
    int fin = 0, fout = 0;
    int st = c.format(c.in(0), &fin);
    if (st == CPIPE_OK) st = c.format(c.out(0), &fout);
    if (st != CPIPE_OK) return st;
    const bool match = (fout == CPIPE_FMT_R32_SFLOAT && target == "R32_SFLOAT") ||
                       (fout == CPIPE_FMT_R16G16B16A16_SFLOAT && target == "R16G16B16A16_SFLOAT") ||
                       (fout == CPIPE_FMT_R8G8B8A8_UNORM && target == "R8G8B8A8_UNORM") ||
                       (fout == CPIPE_FMT_R16G16B16A16_UNORM && target == "R16G16B16A16_UNORM");
    if (!match) return CPIPE_BAD_PRECISION;
    const char* f = nullptr;
    if (fin == CPIPE_FMT_R16_UINT && target == "R32_SFLOAT") f = "precision_convert_r16u_to_f32";
    else if (fin == CPIPE_FMT_R32_SFLOAT && target == "R16G16B16A16_SFLOAT") f = "precision_convert_f32_to_rgba16f";
    else if (fin == CPIPE_FMT_R16G16B16A16_SFLOAT && target == "R8G8B8A8_UNORM") f = "precision_convert_rgba16f_to_rgba8";
    else if (fin == CPIPE_FMT_R16G16B16A16_SFLOAT && target == "R16G16B16A16_UNORM") f = "precision_convert_rgba16f_to_rgba16u";
    if (!f) return CPIPE_BAD_PRECISION;
    if ((st = c.submit_plain(f)) != CPIPE_OK) return st;
    return c.step("precision_convert");
}

// linearize_dng_lut.cpp:25-79
int node_linearize(Ctx& c) {
    int st = check_formats(c, CPIPE_FMT_R16_UINT, CPIPE_FMT_R32_SFLOAT);
    if (st != CPIPE_OK) return st;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    cpipe_calibration_view cal;
    if (!calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    size_t n = 0;
    if (!cal.has_linearization_table || !cal.get_linearization_table ||
        cal.get_linearization_table(m, 0, &n, nullptr) != CPIPE_OK || n == 0)
        return CPIPE_NEED_METADATA;
    std::vector<unsigned char> blob(sizeof(cpipe_LinearizeParamsHeader) + n * sizeof(uint16_t));
    const cpipe_LinearizeParamsHeader hd{(uint32_t)n};
    std::memcpy(blob.data(), &hd, sizeof(hd));
    if (cal.get_linearization_table(m, n, &n, reinterpret_cast<uint16_t*>(blob.data() + sizeof(hd))) != CPIPE_OK)
        return CPIPE_NEED_METADATA;
    if ((st = c.submit("linearize_dng_lut", blob.data(), blob.size())) != CPIPE_OK) return st;
    return c.step("linearization");
}

// blacklevel_dng_levels.cpp:23-70
int node_blacklevel(Ctx& c) {
    int st = check_formats(c, CPIPE_FMT_R32_SFLOAT, CPIPE_FMT_R32_SFLOAT);
    if (st != CPIPE_OK) return st;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    cpipe_calibration_view cal;
    if (!calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    if (!cal.has_cfa || cal.cfa_repeat[0] != 2 || cal.cfa_repeat[1] != 2 || cal.white_level == 0) return CPIPE_NEED_METADATA;
    cpipe_BlacklevelParams p{};
    std::memcpy(p.black_level, cal.black_level, sizeof(p.black_level));
    p.white_level = cal.white_level;
    std::memcpy(p.cfa_pattern, cal.cfa_pattern, 4);
    if ((st = c.submit("blacklevel_dng_levels", &p, sizeof(p))) != CPIPE_OK) return st;
    return c.step("black_white_scaling");
}

// shading_gainmap.cpp:146-195
int node_gainmap(Ctx& c) {
    int st = check_formats(c, CPIPE_FMT_R32_SFLOAT, CPIPE_FMT_R32_SFLOAT);
    if (st != CPIPE_OK) return st;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    cpipe_calibration_view cal;
    if (!calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    if (!cal.has_cfa) return CPIPE_NEED_METADATA;
    const void* bytes = nullptr;
    size_t n = 0;
    std::vector<cpb::prep::GainMap> maps;
    if (c.blob(m, "com.cpipe.dng.opcode_list_2_bytes", &bytes, &n)) {
        if ((st = cpb::prep::parse_gain_maps(bytes, n, &maps, &c.msg)) != CPIPE_OK) return st;
    }
    if (maps.empty()) {
        if ((st = c.copy_through(4)) != CPIPE_OK) return st;
        return c.step("lens_shading_gainmap");
    }
    std::vector<unsigned char> blob;
    if ((st = cpb::prep::validate_and_pack_gain_maps(maps, cal.cfa_repeat, cal.cfa_pattern, &blob, &c.msg)) != CPIPE_OK)
        return st;
    if ((st = c.submit("lens_shading_gainmap", blob.data(), blob.size())) != CPIPE_OK) return st;
    return c.step("lens_shading_gainmap");
}

// demosaic_{rcd,amaze,bilinear}.cpp (e.g. demosaic_rcd.cpp:20-53), DemosaicCommon.hpp:15-35
int node_demosaic(Ctx& c, const char* aot) {
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    cpipe_calibration_view cal;
    if (!calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    static const uint8_t kSupported[4][4] = {{0, 1, 1, 2}, {2, 1, 1, 0}, {1, 0, 2, 1}, {1, 2, 0, 1}};
    bool ok = cal.has_cfa && cal.cfa_repeat[0] == 2 && cal.cfa_repeat[1] == 2;
    if (ok) {
        ok = false;
        for (const auto& p : kSupported) ok = ok || std::memcmp(p, cal.cfa_pattern, 4) == 0;
    }
    if (!ok) return CPIPE_UNSUPPORTED;
    std::string algorithm = "reference";
    c.get_string("algorithm", &algorithm);
    std::string id = aot;
    if (algorithm == "full" && id != "demosaic_bilinear") id += "_full";
    else if (algorithm != "reference") return CPIPE_BAD_INDEX;
    cpipe_DemosaicParams p{};
    std::memcpy(p.cfa_pattern, cal.cfa_pattern, 4);
    int st = c.submit(id.c_str(), &p, sizeof(p));
    if (st != CPIPE_OK) return st;
    if ((st = c.mb->clear_cfa(c.builder())) != CPIPE_OK) return st;
    return c.step("demosaic");
}

// demosaic_quad_bayer_remosaic.cpp:66-105
int node_qbc(Ctx& c) {
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    cpipe_calibration_view cal;
    if (!calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    static const uint8_t kSonyQbc[16] = {0, 0, 1, 1, 0, 0, 1, 1, 1, 1, 2, 2, 1, 1, 2, 2};
    int st;
    if (cal.has_cfa && cal.cfa_repeat[0] == 2 && cal.cfa_repeat[1] == 2) {
        if ((st = c.copy_through(2)) != CPIPE_OK) return st;
        return c.step("quad_bayer_remosaic");
    }
    if (!(cal.has_cfa && cal.cfa_repeat[0] == 4 && cal.cfa_repeat[1] == 4 && std::memcmp(cal.cfa_pattern, kSonyQbc, 16) == 0))
        return CPIPE_UNSUPPORTED;
    if ((st = c.submit_plain("demosaic_quad_bayer_remosaic")) != CPIPE_OK) return st;
    static const uint8_t kRepeat[2] = {2, 2};
    static const uint8_t kRggb[16] = {0, 1, 1, 2};
    if ((st = c.mb->set_cfa(c.builder(), kRepeat, kRggb)) != CPIPE_OK) return st;
    return c.step("quad_bayer_remosaic");
}

// wb_dual_illuminant.cpp:299-403
// WbMetadata.hpp:265-306 (interpolate_calibration) through the host preparation.
int wb_calibrate(const cpipe_calibration_view& cal, const Vec3& neutral, cpipe_WbParams* p, double* cct) {
    Mat3 cm1, cm2, fm1, fm2;
    std::memcpy(cm1.data(), cal.color_matrix1, sizeof(cm1));
    std::memcpy(cm2.data(), cal.color_matrix2, sizeof(cm2));
    std::memcpy(fm1.data(), cal.forward_matrix1, sizeof(fm1));
    std::memcpy(fm2.data(), cal.forward_matrix2, sizeof(fm2));
    const bool has_fm = cal.has_forward_matrix1 && cal.has_forward_matrix2;
    return cpb::prep::wb_prepare(neutral, cal.has_color_matrix1 ? &cm1 : nullptr, cal.has_color_matrix2 ? &cm2 : nullptr,
                                 has_fm ? &fm1 : nullptr, has_fm ? &fm2 : nullptr, cal.calibration_illuminant1,
                                 cal.calibration_illuminant2, p, cct);
}
int emit_wb_blobs(Ctx& c, const Vec3& neutral, const cpipe_WbParams& p, double cct);
int node_wb(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    cpipe_capture_view cap;
    cpipe_calibration_view cal;
    if (c.meta->get_capture(m, &cap) != CPIPE_OK || !calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    const Vec3 neutral{cap.as_shot_neutral[0], cap.as_shot_neutral[1], cap.as_shot_neutral[2]};
    cpipe_WbParams p{};
    double cct = 0.0;
    if ((st = wb_calibrate(cal, neutral, &p, &cct)) != CPIPE_OK) return st;
    if ((st = c.submit("wb_dual_illuminant", &p, sizeof(p))) != CPIPE_OK) return st;
    if ((st = emit_wb_blobs(c, neutral, p, cct)) != CPIPE_OK) return st;
    return c.step("white_balance");
}

// wb/greyworld_auto.cpp:80-166: checks, the grey-world estimate and apply on
// the GPU through "cpipe_wb_greyworld_auto", then the same calibration and
// metadata as the dual-illuminant node with the estimated neutral.  A host that
// does not route that aot_id gets CPIPE_UNSUPPORTED, as for every other node of
// this library: there is no CPU path.
int node_greyworld(Ctx& c) {
    int a = 0, b = 0;
    int st = c.format(c.in(0), &a);
    if (st == CPIPE_OK) st = c.format(c.out(0), &b);
    if (st != CPIPE_OK) return st;
    if (a != CPIPE_FMT_R16G16B16A16_SFLOAT || b != CPIPE_FMT_R16G16B16A16_SFLOAT) {
        c.msg = "wb.greyworld format mismatch";
        return CPIPE_BAD_PRECISION;
    }
    uint32_t w, h;
    if ((st = c.dims(c.in(0), &w, &h)) != CPIPE_OK) return st;
    (void)w;
    (void)h;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    cpipe_calibration_view cal;
    if (!calibration(c, m, &cal)) return CPIPE_NEED_METADATA;
    float n[3] = {1.0F, 1.0F, 1.0F};
    const cpipe_GreyworldParams gp{(uint64_t)(uintptr_t)n};
    st = c.submit("cpipe_wb_greyworld_auto", &gp, sizeof(gp));
    if (st == CPIPE_UNSUPPORTED && c.msg.empty()) c.msg = "wb.greyworld_auto needs the CUDA filter cpipe_wb_greyworld_auto";
    if (st != CPIPE_OK) return st;
    const Vec3 neutral{n[0], n[1], n[2]};
    cpipe_WbParams p{};
    double cct = 0.0;
    if ((st = wb_calibrate(cal, neutral, &p, &cct)) != CPIPE_OK) return st;
    if ((st = c.mb->set_as_shot_neutral(c.builder(), n)) != CPIPE_OK) return st;
    if ((st = emit_wb_blobs(c, neutral, p, cct)) != CPIPE_OK) return st;
    return c.step("white_balance");
}

// WbMetadata.hpp:308-327: the four white-balance blobs.
int emit_wb_blobs(Ctx& c, const Vec3& neutral, const cpipe_WbParams& p, double cct) {
    int st;
    const float diag[3] = {1.0F / neutral[0], 1.0F / neutral[1], 1.0F / neutral[2]};
    const float cct_f = (float)cct;
    if ((st = c.mb->set_blob(c.builder(), "com.cpipe.wb.camera_diag_f32", diag, sizeof(diag))) != CPIPE_OK) return st;
    if ((st = c.mb->set_blob(c.builder(), "com.cpipe.wb.camera_to_xyz_d50_f32", p.camera_to_xyz_d50, sizeof(float) * 9)) != CPIPE_OK)
        return st;
    if ((st = c.mb->set_blob(c.builder(), "com.cpipe.wb.scene_cct_f32", &cct_f, sizeof(float))) != CPIPE_OK) return st;
    if ((st = c.mb->set_blob(c.builder(), "com.cpipe.wb.dual_illuminant_weight_f32", &p.dual_illuminant_weight,
                             sizeof(float))) != CPIPE_OK)
        return st;
    return CPIPE_OK;
}

// colormatrix_dng_to_working.cpp:99-140
int node_colormatrix(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    const char* role = nullptr;
    if (c.meta->get_cs_role(m, &role) != CPIPE_OK || !role || std::strcmp(role, "raw_camera") != 0 ||
        !c.has_step(m, "white_balance"))
        return CPIPE_NEED_METADATA;
    const void* bytes = nullptr;
    size_t n = 0;
    if (!c.blob(m, "com.cpipe.wb.camera_to_xyz_d50_f32", &bytes, &n) || n != 9 * sizeof(float)) return CPIPE_NEED_METADATA;
    Mat3 cam;
    std::memcpy(cam.data(), bytes, sizeof(cam));
    for (float v : cam)
        if (!std::isfinite(v)) return CPIPE_NEED_METADATA;
    const Mat3 t = cpb::prep::camera_to_rec2020(cam);
    cpipe_ColormatrixParams p{};
    std::memcpy(p.transform, t.data(), sizeof(p.transform));
    if ((st = c.submit("colormatrix_dng_to_working", &p, sizeof(p))) != CPIPE_OK) return st;
    if ((st = c.mb->set_cs_role(c.builder(), "scene_linear_rec2020")) != CPIPE_OK) return st;
    return c.step("color_matrix");
}

// denoise/bm3d.cpp:21-55: sigma from "sigma", else "sigma_override", else the
// NoiseProfile variance at signal 0.25, else 0.03.
float noise_sigma(Ctx& c) {
    double v;
    if (c.get_double("sigma", &v)) return std::clamp((float)v, 0.0F, 0.2F);
    if (c.get_double("sigma_override", &v)) return std::clamp((float)v, 0.0F, 0.2F);
    float sigma = 0.03F;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    cpipe_calibration_view cal;
    size_t n = 0;
    if (m && calibration(c, m, &cal) && cal.get_noise_profile && cal.get_noise_profile(m, 0, &n, nullptr, nullptr) == CPIPE_OK && n) {
        std::vector<float> beta(n), lambda(n);
        if (cal.get_noise_profile(m, n, &n, beta.data(), lambda.data()) == CPIPE_OK) {
            double var = 0.0;
            for (size_t i = 0; i < n; ++i) var += std::max(0.0F, beta[i] + (lambda[i] * 0.25F));
            var /= (double)n;
            sigma = (float)std::sqrt(var);
        }
    }
    return sigma;
}

// denoise/bm3d.cpp:21-105
int node_bm3d(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    double v;
    const float sigma = noise_sigma(c);
    std::string algorithm = "box2x2";
    c.get_string("algorithm", &algorithm);
    if (algorithm == "bm3d") {
        // Extension: the published two-stage BM3D (aot_id denoise_bm3d_spec);
        // "box2x2" (default) is the reference's computation.
        cpipe_Bm3dSpecParams sp{sigma, 2.7F, 2500.0F, 400.0F, 16, 39, 3, 2.0F, 2, 0};
        if (c.get_double("stages", &v)) sp.stages = v < 1.5 ? 1 : 2;
        if ((st = c.submit("denoise_bm3d_spec", &sp, sizeof(sp))) != CPIPE_OK) return st;
        return c.step("denoise.bm3d");
    }
    if (algorithm != "box2x2") return CPIPE_BAD_INDEX;
    const cpipe_Bm3dParams p{sigma};
    if ((st = c.submit("denoise_bm3d_step1", &p, sizeof(p))) != CPIPE_OK) return st;
    return c.step("denoise.bm3d");
}

// denoise/guided_filter.cpp:27-46
int node_guided(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    std::string algorithm = "reference";
    c.get_string("algorithm", &algorithm);
    if (algorithm != "reference" && algorithm != "spec") return CPIPE_BAD_INDEX;
    // Extension: "spec" boxes with the true (2r+1)^2 window (radius 1..16,
    // aot_id denoise_guided_filter_spec); "reference" (default) is the
    // reference's computation, 3x3 or 5x5 whatever the radius.
    const bool spec = algorithm == "spec";
    const cpipe_GuidedFilterParams p{c.clamped_int("radius", 1, 1, spec ? 16 : 32),
                                     c.clamped_float("eps", 0.015F, 0.00001F, 0.1F)};
    if ((st = c.submit(spec ? "denoise_guided_filter_spec" : "denoise_guided_filter", &p, sizeof(p))) != CPIPE_OK)
        return st;
    return c.step("denoise.guided_filter");
}

// denoise/wavelet_bayes_shrink.cpp:25-48
int node_wavelet(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    std::string algorithm = "haar";
    c.get_string("algorithm", &algorithm);
    if (algorithm == "atrous") {
        // Extension: the multi-level a-trous form (aot_id
        // denoise_wavelet_atrous_spec); "haar" (default) is the reference's
        // single 2x2 level on chroma.  Noise sigma as the bm3d node finds it.
        const cpipe_AtrousWaveletParams ap{c.clamped_int("levels", 5, 0, 6), noise_sigma(c),
                                           c.clamped_float("luma_strength", 1.0F, 0.0F, 2.0F),
                                           c.clamped_float("chroma_strength", 1.0F, 0.0F, 2.0F)};
        if ((st = c.submit("denoise_wavelet_atrous_spec", &ap, sizeof(ap))) != CPIPE_OK) return st;
        return c.step("denoise.wavelet_bayes_shrink");
    }
    if (algorithm != "haar") return CPIPE_BAD_INDEX;
    const cpipe_WaveletBayesShrinkParams p{c.clamped_float("chroma_strength", 1.0F, 0.0F, 2.0F)};
    if ((st = c.submit("denoise_wavelet_bayes_shrink", &p, sizeof(p))) != CPIPE_OK) return st;
    return c.step("denoise.wavelet_bayes_shrink");
}

// lens/dng_opcode_list_3.cpp:178-225
int node_opcode3(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    if (!m) return CPIPE_NEED_METADATA;
    const void* bytes = nullptr;
    size_t n = 0;
    std::vector<unsigned char> blob;
    uint32_t count = 0;
    if (c.blob(m, "com.cpipe.dng.opcode_list_3_bytes", &bytes, &n)) {
        if ((st = cpb::prep::parse_and_pack_opcode3(bytes, n, &blob, &count, &c.msg)) != CPIPE_OK) return st;
    }
    if (count == 0) {
        if ((st = c.copy_through(rgba_bytes(c))) != CPIPE_OK) return st;
        return c.step("opcode_list_3");
    }
    if ((st = c.submit("lens_dng_opcode_list_3", blob.data(), blob.size())) != CPIPE_OK) return st;
    return c.step("opcode_list_3");
}

// color/lut3d.cpp:70-104
int node_lut3d(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    std::string path;
    if (!c.get_string("lut_path", &path)) return CPIPE_NEED_PARAM;
    uint32_t size = 0;
    std::vector<float> values;
    if ((st = cpb::prep::load_lut(path, &size, &values, &c.msg)) != CPIPE_OK) return st;
    std::string interp = "tetrahedral";
    c.get_string("interpolation", &interp);
    const cpipe_Lut3dParamHeader hd{size, (uint32_t)values.size(), interp == "trilinear" ? 1U : 0U};
    std::vector<unsigned char> blob(sizeof(hd) + values.size() * sizeof(float));
    std::memcpy(blob.data(), &hd, sizeof(hd));
    std::memcpy(blob.data() + sizeof(hd), values.data(), values.size() * sizeof(float));
    if ((st = c.submit("color_3d_lut", blob.data(), blob.size())) != CPIPE_OK) return st;
    return c.step("color.3d_lut");
}

// tone/filmic_rgb.cpp:22-58
int node_filmic(Ctx& c) {
    int st = check_rgba(c);
    if (st != CPIPE_OK) return st;
    const cpipe_FilmicRgbParams p{c.clamped_float("ev", 0.0F, -2.0F, 2.0F), c.clamped_float("contrast", 1.0F, 0.5F, 2.0F),
                                  c.clamped_float("saturation", 1.0F, 0.0F, 2.0F),
                                  c.clamped_float("highlights", 1.0F, 0.0F, 2.0F),
                                  c.clamped_float("shadows", 1.0F, 0.0F, 2.0F)};
    if ((st = c.submit("tone_filmic_rgb", &p, sizeof(p))) != CPIPE_OK) return st;
    return c.step("tone.filmic_rgb");
}

// tone/mertens_local.cpp:20-101: output and the three inputs RGBA16F with one
// extent, parameters clamped, then the fusion; the step name is the reference's.
int node_mertens(Ctx& c) {
    int f = 0;
    int st = c.format(c.out(0), &f);
    if (st != CPIPE_OK) return st;
    if (f != CPIPE_FMT_R16G16B16A16_SFLOAT) return CPIPE_BAD_PRECISION;
    uint32_t w, h;
    if ((st = c.dims(c.out(0), &w, &h)) != CPIPE_OK) return st;
    for (size_t i = 0; i < 3; ++i) {
        if ((st = c.format(c.in(i), &f)) != CPIPE_OK) return st;
        if (f != CPIPE_FMT_R16G16B16A16_SFLOAT) return CPIPE_BAD_PRECISION;
        uint32_t wi, hi;
        if ((st = c.dims(c.in(i), &wi, &hi)) != CPIPE_OK) return st;
        if (wi != w || hi != h) return CPIPE_BAD_INDEX;
    }
    const cpipe_MertensLocalParams p{c.clamped_float("weight_contrast", 0.0F, 0.0F, 2.0F),
                                     c.clamped_float("weight_saturation", 1.0F, 0.0F, 2.0F),
                                     c.clamped_float("weight_well_exposedness", 1.0F, 0.0F, 2.0F)};
    if ((st = c.submit("tone_mertens_local", &p, sizeof(p))) != CPIPE_OK) return st;
    return c.step("tone_mertens_local");
}

// tone/aces_filmic.cpp:28-46
int node_aces(Ctx& c) {
    const cpipe_AcesFilmicParams p{c.bool_or("toggle", true) ? 1 : 0};
    const int st = c.submit("tone_aces_filmic", &p, sizeof(p));
    if (st != CPIPE_OK) return st;
    return c.step("tone.aces_filmic");
}

// tone/reinhard.cpp:28-47: white_point unset (-1) -> 1e6, else clamped to 0.1..10
int node_reinhard(Ctx& c) {
    const float wp = (float)c.double_or("white_point", -1.0);
    const cpipe_ReinhardParams p{wp < 0.0F ? 1000000.0F : std::clamp(wp, 0.1F, 10.0F)};
    const int st = c.submit("tone_reinhard", &p, sizeof(p));
    if (st != CPIPE_OK) return st;
    return c.step("tone.reinhard");
}

// sharpen/edge_aware_usm.cpp:29-50: parameters clamped as the reference node
// does; the filter checks the buffers.
int node_usm(Ctx& c) {
    const cpipe_EdgeAwareUsmParams p{c.clamped_float("strength", 0.75F, 0.0F, 2.0F), c.clamped_int("radius", 1, 1, 32),
                                     c.clamped_float("threshold", 0.0F, 0.0F, 0.1F)};
    const int st = c.submit("sharpen_edge_aware_usm", &p, sizeof(p));
    if (st != CPIPE_OK) return st;
    return c.step("sharpen.edge_aware_usm");
}

// color/scene_linear_to_display.cpp:31-127: target -> output format and role,
// buffer / metadata checks with the reference's codes, then the encode on this
// library's CUDA filter "cpipe_scene_linear_to_display"; a host that does not
// route it gets CPIPE_UNSUPPORTED (there is no CPU path).
int node_display(Ctx& c) {
    std::string target;
    if (!c.get_string("target", &target)) return CPIPE_NEED_PARAM;
    uint32_t code = 0;
    int want = 0;
    const char* dst = nullptr;
    if (target == "sRGB") {
        code = CPIPE_DISPLAY_SRGB;
        want = CPIPE_FMT_R8G8B8A8_UNORM;
        dst = "output_srgb";
    } else if (target == "BT2020-PQ") {
        code = CPIPE_DISPLAY_BT2020_PQ;
        want = CPIPE_FMT_R16G16B16A16_UNORM;
        dst = "output_pq_rec2020";
    } else if (target == "DisplayP3" || target == "BT2020-HLG") {
        c.msg = "display target reserved for v1.1";
        return CPIPE_UNSUPPORTED;
    } else {
        c.msg = "unknown display target";
        return CPIPE_NEED_PARAM;
    }
    int a = 0, b = 0;
    int st = c.format(c.in(0), &a);
    if (st == CPIPE_OK) st = c.format(c.out(0), &b);
    if (st != CPIPE_OK) return st;
    if (a != CPIPE_FMT_R16G16B16A16_SFLOAT || b != want) {
        c.msg = "scene_linear_to_display format mismatch";
        return CPIPE_BAD_PRECISION;
    }
    uint32_t w0, h0, w1, h1;
    if ((st = c.dims(c.in(0), &w0, &h0)) != CPIPE_OK || (st = c.dims(c.out(0), &w1, &h1)) != CPIPE_OK) return st;
    if (w0 != w1 || h0 != h1) return CPIPE_BAD_INDEX;
    const cpipe_metadata_t* m = c.metadata(c.in(0));
    const char* role = nullptr;
    if (!m || c.meta->get_cs_role(m, &role) != CPIPE_OK || !role || std::strcmp(role, "scene_linear_rec2020") != 0) {
        c.msg = "scene_linear_to_display needs Rec2020 scene linear";
        return CPIPE_NEED_METADATA;
    }
    const cpipe_DisplayParams p{code};
    st = c.submit("cpipe_scene_linear_to_display", &p, sizeof(p));
    if (st == CPIPE_UNSUPPORTED && c.msg.empty())
        c.msg = "scene_linear_to_display needs the CUDA filter cpipe_scene_linear_to_display";
    if (st != CPIPE_OK) return st;
    if ((st = c.mb->set_cs_role(c.builder(), dst)) != CPIPE_OK) return st;
    return c.step("color.scene_linear_to_display");
}

// ------------------------------------------------------------- dispatching
using NodeFn = int (*)(Ctx&);

template <NodeFn F, size_t NIN = 1>
int main_entry(const char* action, cpipe_host_t* host, cpipe_node_t* node, cpipe_props_t* params, void* in_ctx,
               void* out_ctx) {
    (void)node;
    try {
        if (action == nullptr) return CPIPE_BAD_INDEX;
        if (!std::strcmp(action, CPIPE_ACTION_DESCRIBE)) return CPIPE_REPLY_DEFAULT;
        if (!std::strcmp(action, CPIPE_ACTION_CREATE)) {
            if (out_ctx == nullptr) return CPIPE_BAD_INDEX;
            *static_cast<void**>(out_ctx) = new int(0);  // stateless nodes: a token instance
            return CPIPE_OK;
        }
        if (!std::strcmp(action, CPIPE_ACTION_DESTROY)) {
            delete static_cast<int*>(in_ctx);
            return CPIPE_OK;
        }
        if (!std::strcmp(action, CPIPE_ACTION_PREPARE)) return CPIPE_OK;
        if (!std::strcmp(action, CPIPE_ACTION_PROCESS)) {
            if (host == nullptr || host->get_suite == nullptr) return CPIPE_BAD_INDEX;
            auto* pc = static_cast<cpipe_process_ctx*>(in_ctx);
            if (!n_to_one(pc, NIN)) return CPIPE_BAD_INDEX;
            Ctx c{host, nullptr, nullptr, nullptr, nullptr, nullptr, params, pc, {}};
            if (!c.init()) return CPIPE_BAD_INDEX;
            const int st = F(c);
            if (st != CPIPE_OK && !c.msg.empty() && host->log) host->log(host, 2, c.msg.c_str());
            return st;
        }
        return CPIPE_REPLY_DEFAULT;
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}
// nodes/dng_input/dng_input.cpp:17-40: the file at param "path" through
// DngReader::read.  The reference builtin replaces its output's buffer object
// with the reader's; here the host allocates the output (an R16_UINT Image2D
// of the file's extent, else CPIPE_BAD_INDEX), the strip is decoded on the GPU
// straight into it, and the reader's metadata is attached through this
// library's host runtime (another host: CPIPE_UNSUPPORTED).
int node_dng_input(Ctx& c) {
    std::string path;
    if (!c.get_string("path", &path)) {
        c.msg = "dng_input needs a path";
        return CPIPE_NEED_PARAM;
    }
    if (!cpb_is_own_host(c.host)) {
        c.msg = "dng_input writes device buffers of the cpipe_b200 host runtime";
        return CPIPE_UNSUPPORTED;
    }
    std::vector<uint8_t> file;
    {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) {
            c.msg = "failed to open DNG";
            return CPIPE_FAILED;
        }
        uint8_t chunk[1 << 16];
        size_t n;
        while ((n = std::fread(chunk, 1, sizeof(chunk), f)) > 0) file.insert(file.end(), chunk, chunk + n);
        std::fclose(f);
    }
    cpipe_DngInfo info{};
    int st = cpipe_dng_parse(file.data(), file.size(), &info);
    if (st != CPIPE_OK) {
        c.msg = cpipe_cuda_last_error();
        return st == CPIPE_UNSUPPORTED ? CPIPE_FAILED : st;  // DngReader.cpp:192-195
    }
    int fmt = 0;
    uint32_t w = 0, h = 0;
    if ((st = c.format(c.out(0), &fmt)) != CPIPE_OK || (st = c.dims(c.out(0), &w, &h)) != CPIPE_OK) return st;
    if (fmt != CPIPE_FMT_R16_UINT || w != info.width || h != info.height) {
        c.msg = "dng_input output must be an R16_UINT image of the file's extent";
        return CPIPE_BAD_INDEX;
    }
    void* prev = cpipe_cuda_get_stream();
    cpipe_cuda_set_stream(cpb_abi_host_stream(c.host));
    st = cpipe_cuda_dng_decode(file.data(), file.size(), static_cast<uint16_t*>(cpb_buffer_device(c.out(0))),
                               (size_t)w * h * 2, &info);
    cpipe_cuda_set_stream(prev);
    if (st != CPIPE_OK) {
        c.msg = cpipe_cuda_last_error();
        return st;
    }
    return cpb_builder_set_dng(c.builder(), &info, file.data(), file.size());
}

int n_rcd(Ctx& c) { return node_demosaic(c, "demosaic_rcd"); }
int n_amaze(Ctx& c) { return node_demosaic(c, "demosaic_amaze"); }
int n_bilinear(Ctx& c) { return node_demosaic(c, "demosaic_bilinear"); }

// ---------------------------------------------------------------- manifests
// Same ids, versions, ports, metadata requirements and params as the reference
// manifests (src/cpipe/nodes/**/<node>.json); compute names the CUDA device.
#define MANIFEST(id, label, category, in_port, out_port, params, in_role, out_role, chroma, kernels)            \
    "{\"$schema\":\"https://schemas.cpipe.dev/node/v0.2.json\",\"id\":\"" id "\",\"version\":\"1.0.0\","       \
    "\"label\":\"" label "\",\"category\":\"" category "\",\"ports\":[" in_port "," out_port "],"                \
    "\"params\":[" params "],\"compute\":{\"device\":\"CUDA\",\"engine\":\"CUDA\",\"arch\":\"sm_100a\","          \
    "\"kernels\":[" kernels "]},\"color\":{\"input_role\":\"" in_role "\",\"output_role\":\"" out_role          \
    "\",\"respects_chromaticity\":" chroma "}}"
#define PORT(name, kind, ch, prec, meta) \
    "{\"name\":\"" name "\",\"kind\":\"" kind "\",\"caps\":{\"buffer_kind\":\"Image2D\",\"channels\":[" ch "],\"precision\":[" prec "]},\"cardinality\":\"single\",\"metadata\":{" meta "}}"
#define RGBA_IN(name, meta) PORT(name, "in", "\"rgba\"", "\"f16\",\"f32\"", meta)
#define RGBA_OUT(name, step, extra) PORT(name, "out", "\"rgba\"", "\"f16\"", "\"inherits_from\":\"rgb\",\"sets_steps_applied\":[\"" step "\"]" extra)
#define NUM(name, lo, hi, def) "{\"name\":\"" name "\",\"type\":\"number\",\"range\":{\"min\":" lo ",\"max\":" hi "},\"default\":" def "}"

const char kPrecision[] = MANIFEST("com.cpipe.precision_convert", "Precision Convert", "utility",
    PORT("in", "in", "\"r\",\"rgba\"", "\"u16\",\"f32\",\"f16\"", ""),
    PORT("out", "out", "\"r\",\"rgba\"", "\"f32\",\"f16\",\"u8\",\"u16\"", "\"inherits_from\":\"in\",\"sets_steps_applied\":[\"precision_convert\"]"),
    "{\"name\":\"target_format\",\"type\":\"enum\",\"enum_values\":[\"R32_SFLOAT\",\"R16G16B16A16_SFLOAT\",\"R8G8B8A8_UNORM\",\"R16G16B16A16_UNORM\"]}",
    "any", "any", "true", "\"precision_convert\"");
const char kLinearize[] = MANIFEST("com.cpipe.linearize.dng_lut", "DNG Linearization LUT", "raw",
    PORT("raw", "in", "\"r\"", "\"u16\"", "\"requires_fields\":[\"calibration.linearization_table\"]"),
    PORT("bayer", "out", "\"r\"", "\"f32\"", "\"inherits_from\":\"raw\",\"sets_steps_applied\":[\"linearization\"]"),
    "", "raw_camera", "raw_camera", "false", "\"raw_point<linearize>\"");
const char kBlacklevel[] = MANIFEST("com.cpipe.blacklevel.dng_levels", "DNG Black/White Levels", "raw",
    PORT("bayer", "in", "\"r\"", "\"f32\"", "\"requires_steps_applied\":[\"linearization\"],\"requires_fields\":[\"calibration.cfa\",\"calibration.black_level\",\"calibration.white_level\"]"),
    PORT("bayer", "out", "\"r\"", "\"f32\"", "\"inherits_from\":\"bayer\",\"sets_steps_applied\":[\"black_white_scaling\"]"),
    "", "raw_camera", "raw_camera", "false", "\"raw_point<blacklevel>\"");
const char kGainmap[] = MANIFEST("com.cpipe.lens.shading_gainmap", "Lens Shading GainMap", "raw",
    PORT("linear_bayer", "in", "\"r\"", "\"f32\"", "\"requires_fields\":[\"calibration.cfa\"],\"requires_blobs\":[\"com.cpipe.dng.opcode_list_2_bytes\"]"),
    PORT("corrected_bayer", "out", "\"r\"", "\"f32\"", "\"inherits_from\":\"linear_bayer\",\"sets_steps_applied\":[\"lens_shading_gainmap\"]"),
    "", "raw_camera", "raw_camera", "false", "\"raw_point<gainmap>\"");
#define DEMOSAIC_MANIFEST(id, label, params, k) MANIFEST(id, label, "raw",                                           \
    PORT("bayer", "in", "\"r\"", "\"f32\"", "\"requires_steps_applied\":[\"black_white_scaling\"],\"requires_fields\":[\"calibration.cfa\"]"), \
    PORT("rgba", "out", "\"rgba\"", "\"f16\"", "\"inherits_from\":\"bayer\",\"clears_fields\":[\"calibration.cfa\"],\"sets_steps_applied\":[\"demosaic\"]"), \
    params, "raw_camera", "raw_camera", "false", k)
#define DEMOSAIC_ALGORITHM "{\"name\":\"algorithm\",\"type\":\"enum\",\"enum_values\":[\"reference\",\"full\"],\"default\":\"reference\"}"
const char kRcd[] = DEMOSAIC_MANIFEST("com.cpipe.demosaic.rcd", "RCD Demosaic", DEMOSAIC_ALGORITHM,
                                      "\"demosaic_kernel<rcd>\",\"rcd_full_kernel\"");
const char kAmaze[] = DEMOSAIC_MANIFEST("com.cpipe.demosaic.amaze", "AMaZE Demosaic", DEMOSAIC_ALGORITHM,
                                        "\"demosaic_kernel<amaze>\",\"amaze_cd_kernel\",\"amaze_green_kernel\",\"amaze_out_kernel\"");
const char kDngInput[] = "{\"$schema\":\"https://schemas.cpipe.dev/node/v0.2.json\",\"id\":\"com.cpipe.builtin.dng_input\","
    "\"version\":\"1.0.0\",\"label\":\"DNG Input\",\"category\":\"builtin\",\"ports\":["
    PORT("raw", "out", "\"r\"", "\"u16\"", "\"writes_fields\":[\"calibration\",\"capture\",\"cs_role\",\"ext_blobs\"]")
    "],\"params\":[{\"name\":\"path\",\"type\":\"string\",\"required\":true}],"
    "\"compute\":{\"device\":\"CUDA\",\"engine\":\"CUDA\",\"arch\":\"sm_100a\",\"kernels\":[\"dng_words_kernel\",\"dng_packed_kernel\"]},"
    "\"color\":{\"input_role\":\"none\",\"output_role\":\"raw_camera\",\"respects_chromaticity\":false}}";
const char kBilinear[] = DEMOSAIC_MANIFEST("com.cpipe.demosaic.bilinear", "Bilinear Demosaic", "", "\"demosaic_kernel<bilinear>\"");
const char kQbc[] = MANIFEST("com.cpipe.demosaic.quad_bayer_remosaic", "Quad Bayer Remosaic", "raw",
    PORT("qbc", "in", "\"r\"", "\"u16\"", "\"requires_fields\":[\"calibration.cfa\"]"),
    PORT("bayer", "out", "\"r\"", "\"u16\"", "\"inherits_from\":\"qbc\",\"writes_fields\":[\"calibration.cfa\"],\"sets_steps_applied\":[\"quad_bayer_remosaic\"]"),
    "", "raw_camera", "raw_camera", "false", "\"qbc_kernel\"");
const char kWb[] = MANIFEST("com.cpipe.wb.dual_illuminant", "DNG White Balance", "color",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"demosaic\"],\"requires_fields\":[\"capture.as_shot_neutral\",\"calibration.color_matrix1\",\"calibration.color_matrix2\",\"calibration.calibration_illuminant1\",\"calibration.calibration_illuminant2\"]"),
    RGBA_OUT("rgb", "white_balance", ""), "", "raw_camera", "raw_camera", "true", "\"rgba_point<wb>\"");
const char kCm[] = MANIFEST("com.cpipe.colormatrix.dng_to_working", "DNG Color Matrix", "color",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"white_balance\"],\"requires_fields\":[\"cs_role\"],\"requires_blobs\":[\"com.cpipe.wb.camera_to_xyz_d50_f32\"]"),
    RGBA_OUT("rgb", "color_matrix", ",\"writes_fields\":[\"cs_role\"]"), "", "raw_camera", "scene_linear_rec2020", "true",
    "\"rgba_point<colormatrix>\"");
const char kBm3d[] = MANIFEST("com.cpipe.denoise.bm3d", "BM3D Denoise", "denoise",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"color_matrix\"],\"requires_fields\":[\"calibration.noise_profile\"]"),
    RGBA_OUT("rgb", "denoise.bm3d", ""),
    "{\"name\":\"sigma\",\"type\":\"number\",\"range\":{\"min\":0,\"max\":0.2}},{\"name\":\"sigma_override\",\"type\":\"number\",\"range\":{\"min\":0},\"default\":0},"
    "{\"name\":\"algorithm\",\"type\":\"enum\",\"enum_values\":[\"box2x2\",\"bm3d\"],\"default\":\"box2x2\"},"
    NUM("stages", "1", "2", "2"),
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"bm3d_parity_kernel\",\"bm3d_match_kernel\",\"bm3d_filter_kernel\"");
const char kGuided[] = MANIFEST("com.cpipe.denoise.guided_filter", "Guided Filter Denoise", "denoise",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"color_matrix\"]"), RGBA_OUT("rgb", "denoise.guided_filter", ""),
    NUM("radius", "1", "32", "1") "," NUM("eps", "1e-05", "0.1", "0.015") ","
    "{\"name\":\"algorithm\",\"type\":\"enum\",\"enum_values\":[\"reference\",\"spec\"],\"default\":\"reference\"}",
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"guided_kernel\",\"guided_spec_kernel\"");
const char kWavelet[] = MANIFEST("com.cpipe.denoise.wavelet_bayes_shrink", "Wavelet BayesShrink Denoise", "denoise",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"color_matrix\"]"), RGBA_OUT("rgb", "denoise.wavelet_bayes_shrink", ""),
    NUM("chroma_strength", "0", "2", "1") ","
    "{\"name\":\"algorithm\",\"type\":\"enum\",\"enum_values\":[\"haar\",\"atrous\"],\"default\":\"haar\"},"
    NUM("levels", "0", "6", "5") "," NUM("luma_strength", "0", "2", "1") ","
    "{\"name\":\"sigma\",\"type\":\"number\",\"range\":{\"min\":0,\"max\":0.2}}",
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"wavelet_kernel\",\"atrous_level_kernel\"");
const char kOpcode3[] = MANIFEST("com.cpipe.lens.dng_opcode_list_3", "DNG OpcodeList3", "lens",
    PORT("scene_rgb", "in", "\"rgba\"", "\"f16\",\"f32\"", "\"requires_blobs\":[\"com.cpipe.dng.opcode_list_3_bytes\"]"),
    PORT("corrected_rgb", "out", "\"rgba\"", "\"f16\"", "\"inherits_from\":\"scene_rgb\",\"sets_steps_applied\":[\"opcode_list_3\"]"),
    "", "raw_camera", "raw_camera", "true", "\"warp_kernel\",\"vignette_kernel\",\"bad_constant_kernel\",\"bad_list_kernel\",\"trim_kernel\"");
const char kLut[] = MANIFEST("com.cpipe.color.3d_lut", "3D LUT", "color", RGBA_IN("rgb", ""), RGBA_OUT("rgb", "color.3d_lut", ""),
    "{\"name\":\"lut_path\",\"type\":\"string\"},{\"name\":\"interpolation\",\"type\":\"enum\",\"enum_values\":[\"tetrahedral\",\"trilinear\"],\"default\":\"tetrahedral\"}",
    "scene_linear_rec2020", "scene_linear_rec2020", "false", "\"rgba_point<lut3d>\"");
const char kFilmic[] = MANIFEST("com.cpipe.tone.filmic_rgb", "Filmic RGB Tone", "tone",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"denoise.wavelet_bayes_shrink\"]"), RGBA_OUT("rgb", "tone.filmic_rgb", ""),
    NUM("ev", "-2", "2", "0") "," NUM("contrast", "0.5", "2", "1") "," NUM("saturation", "0", "2", "1") ","
    NUM("highlights", "0", "2", "1") "," NUM("shadows", "0", "2", "1"),
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"rgba_point<filmic>\"");

const char kGreyworld[] = MANIFEST("com.cpipe.wb.greyworld_auto", "Grey-world Auto WB", "wb",
    PORT("rgb", "in", "\"rgba\"", "\"f16\"", "\"requires_steps_applied\":[\"demosaic\"],\"requires_fields\":[\"calibration.color_matrix1\",\"calibration.color_matrix2\",\"calibration.calibration_illuminant1\",\"calibration.calibration_illuminant2\"]"),
    PORT("rgb", "out", "\"rgba\"", "\"f16\"", "\"inherits_from\":\"rgb\",\"sets_steps_applied\":[\"white_balance\"],\"writes_fields\":[\"capture.as_shot_neutral\"]"),
    "", "raw_camera", "raw_camera", "true", "\"greyworld_sum_kernel\",\"rgba_point<greyworld>\"");
#define MERTENS_IN(name) PORT(name, "in", "\"rgba\"", "\"f16\"", "\"requires_steps_applied\":[\"denoise.wavelet_bayes_shrink\"]")
const char kMertens[] = MANIFEST("com.cpipe.tone.mertens_local", "Mertens Exposure Fusion", "tone",
    MERTENS_IN("under") "," MERTENS_IN("normal") "," MERTENS_IN("over"),
    PORT("rgb", "out", "\"rgba\"", "\"f16\"", "\"inherits_from\":\"normal\",\"sets_steps_applied\":[\"tone_mertens_local\"]"),
    NUM("weight_contrast", "0", "2", "0") "," NUM("weight_saturation", "0", "2", "1") ","
    NUM("weight_well_exposedness", "0", "2", "1"),
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"mertens_kernel\"");
const char kAces[] = MANIFEST("com.cpipe.tone.aces_filmic", "ACES Filmic Tone", "tone",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"denoise.wavelet_bayes_shrink\"]"), RGBA_OUT("rgb", "tone.aces_filmic", ""),
    "{\"name\":\"toggle\",\"type\":\"bool\",\"default\":true}",
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"rgba_point<aces>\"");
const char kReinhard[] = MANIFEST("com.cpipe.tone.reinhard", "Reinhard Tone", "tone",
    RGBA_IN("rgb", "\"requires_steps_applied\":[\"denoise.wavelet_bayes_shrink\"]"), RGBA_OUT("rgb", "tone.reinhard", ""),
    NUM("white_point", "0.1", "10", "10"),
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"rgba_point<reinhard>\"");
const char kUsm[] = MANIFEST("com.cpipe.sharpen.edge_aware_usm", "Edge-aware USM", "sharpen",
    PORT("rgb", "in", "\"rgba\"", "\"f16\",\"f32\"", "\"requires_steps_applied\":[\"color.3d_lut\"]"),
    PORT("rgb", "out", "\"rgba\"", "\"f16\"", "\"inherits_from\":\"rgb\",\"sets_steps_applied\":[\"sharpen.edge_aware_usm\"]"),
    NUM("strength", "0", "2", "0.75") "," NUM("radius", "1", "32", "1") "," NUM("threshold", "0", "0.1", "0"),
    "scene_linear_rec2020", "scene_linear_rec2020", "true", "\"usm_kernel\"");
const char kDisplay[] = MANIFEST("com.cpipe.color.scene_linear_to_display", "Scene Linear to Display", "color",
    PORT("rgb", "in", "\"rgba\"", "\"f16\"", ""),
    PORT("display", "out", "\"rgba\"", "\"u8\",\"u16\"", "\"inherits_from\":\"rgb\",\"sets_steps_applied\":[\"color.scene_linear_to_display\"]"),
    "{\"name\":\"target\",\"type\":\"enum\",\"enum_values\":[\"sRGB\",\"BT2020-PQ\",\"DisplayP3\",\"BT2020-HLG\"],\"default\":\"sRGB\"}",
    "scene_linear_rec2020", "any", "true", "\"display_kernel\"");

}  // namespace

// Descriptors in the reference registry section (section.hpp:7, registry.hpp:24-31).
#define CPIPE_B200_REGISTER(sym, id, manifest, fn)                                              \
    __attribute__((used, section("cpipe_registry"), aligned(8))) const cpipe_plugin_desc_t sym = \
        {CPIPE_ABI_MAJOR, CPIPE_ABI_MINOR, id, "1.0.0", manifest, &main_entry<fn>};

CPIPE_B200_REGISTER(cpipe_b200_desc_precision, "com.cpipe.precision_convert", kPrecision, node_precision_convert)
CPIPE_B200_REGISTER(cpipe_b200_desc_linearize, "com.cpipe.linearize.dng_lut", kLinearize, node_linearize)
CPIPE_B200_REGISTER(cpipe_b200_desc_blacklevel, "com.cpipe.blacklevel.dng_levels", kBlacklevel, node_blacklevel)
CPIPE_B200_REGISTER(cpipe_b200_desc_gainmap, "com.cpipe.lens.shading_gainmap", kGainmap, node_gainmap)
CPIPE_B200_REGISTER(cpipe_b200_desc_rcd, "com.cpipe.demosaic.rcd", kRcd, n_rcd)
CPIPE_B200_REGISTER(cpipe_b200_desc_amaze, "com.cpipe.demosaic.amaze", kAmaze, n_amaze)
CPIPE_B200_REGISTER(cpipe_b200_desc_bilinear, "com.cpipe.demosaic.bilinear", kBilinear, n_bilinear)
CPIPE_B200_REGISTER(cpipe_b200_desc_qbc, "com.cpipe.demosaic.quad_bayer_remosaic", kQbc, node_qbc)
CPIPE_B200_REGISTER(cpipe_b200_desc_wb, "com.cpipe.wb.dual_illuminant", kWb, node_wb)
CPIPE_B200_REGISTER(cpipe_b200_desc_cm, "com.cpipe.colormatrix.dng_to_working", kCm, node_colormatrix)
CPIPE_B200_REGISTER(cpipe_b200_desc_bm3d, "com.cpipe.denoise.bm3d", kBm3d, node_bm3d)
CPIPE_B200_REGISTER(cpipe_b200_desc_guided, "com.cpipe.denoise.guided_filter", kGuided, node_guided)
CPIPE_B200_REGISTER(cpipe_b200_desc_wavelet, "com.cpipe.denoise.wavelet_bayes_shrink", kWavelet, node_wavelet)
CPIPE_B200_REGISTER(cpipe_b200_desc_opcode3, "com.cpipe.lens.dng_opcode_list_3", kOpcode3, node_opcode3)
CPIPE_B200_REGISTER(cpipe_b200_desc_lut, "com.cpipe.color.3d_lut", kLut, node_lut3d)
CPIPE_B200_REGISTER(cpipe_b200_desc_filmic, "com.cpipe.tone.filmic_rgb", kFilmic, node_filmic)
CPIPE_B200_REGISTER(cpipe_b200_desc_greyworld, "com.cpipe.wb.greyworld_auto", kGreyworld, node_greyworld)
#define CPIPE_B200_REGISTER_N(sym, id, manifest, fn, nin)                                       \
    __attribute__((used, section("cpipe_registry"), aligned(8))) const cpipe_plugin_desc_t sym = \
        {CPIPE_ABI_MAJOR, CPIPE_ABI_MINOR, id, "1.0.0", manifest, &main_entry<fn, nin>};
CPIPE_B200_REGISTER_N(cpipe_b200_desc_mertens, "com.cpipe.tone.mertens_local", kMertens, node_mertens, 3)
CPIPE_B200_REGISTER_N(cpipe_b200_desc_dng_input, "com.cpipe.builtin.dng_input", kDngInput, node_dng_input, 0)
CPIPE_B200_REGISTER(cpipe_b200_desc_aces, "com.cpipe.tone.aces_filmic", kAces, node_aces)
CPIPE_B200_REGISTER(cpipe_b200_desc_reinhard, "com.cpipe.tone.reinhard", kReinhard, node_reinhard)
CPIPE_B200_REGISTER(cpipe_b200_desc_usm, "com.cpipe.sharpen.edge_aware_usm", kUsm, node_usm)
CPIPE_B200_REGISTER(cpipe_b200_desc_display, "com.cpipe.color.scene_linear_to_display", kDisplay, node_display)

extern "C" {
extern const cpipe_plugin_desc_t __start_cpipe_registry[];
extern const cpipe_plugin_desc_t __stop_cpipe_registry[];

const cpipe_plugin_desc_t* cpipe_b200_node_descs(size_t* count) {
    if (count) *count = (size_t)(__stop_cpipe_registry - __start_cpipe_registry);
    return __start_cpipe_registry;
}
const cpipe_plugin_desc_t* cpipe_b200_find_node(const char* node_id) {
    if (!node_id) return nullptr;
    for (const cpipe_plugin_desc_t* d = __start_cpipe_registry; d != __stop_cpipe_registry; ++d)
        if (d->node_id && !std::strcmp(d->node_id, node_id)) return d;
    return nullptr;
}
}
