"""ctypes view of libcpipe_b200.so: the structs of include/cpipe_halide_abi.h,
include/cpipe_b200_params.h and include/cpipe_node_abi.h, and the prototypes of
include/cpipe_b200.h.  Loading fails loudly when the library is missing: there
is no CPU implementation to fall back to."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcpipe_b200.so")

# ---------------------------------------------------------------- status codes
OK, FAILED, REPLY_DEFAULT, OOM, BAD_PRECISION, BAD_INDEX = 0, 1, 2, 3, 4, 5
NEED_PARAM, INTERNAL_ERROR, UNSUPPORTED, NEED_METADATA, NOT_IMPLEMENTED = 6, 7, 8, 9, 100
STATUS_NAMES = {0: "CPIPE_OK", 1: "CPIPE_FAILED", 2: "CPIPE_REPLY_DEFAULT", 3: "CPIPE_OOM",
                4: "CPIPE_BAD_PRECISION", 5: "CPIPE_BAD_INDEX", 6: "CPIPE_NEED_PARAM",
                7: "CPIPE_INTERNAL_ERROR", 8: "CPIPE_UNSUPPORTED", 9: "CPIPE_NEED_METADATA",
                100: "CPIPE_NOT_IMPLEMENTED"}

# ---------------------------------------------------------------- pixel formats
FMT_R16_UINT = 1
FMT_R8G8B8A8_UNORM = 3
FMT_R16G16B16A16_SFLOAT = 6
FMT_R32G32B32A32_SFLOAT = 8
FMT_R32_SFLOAT = 10
FMT_R16G16B16A16_UNORM = 16


class HalideType(C.Structure):
    _fields_ = [("code", C.c_uint8), ("bits", C.c_uint8), ("lanes", C.c_uint16)]


class HalideDim(C.Structure):
    _fields_ = [("min", C.c_int32), ("extent", C.c_int32), ("stride", C.c_int32), ("flags", C.c_uint32)]


class HalideBuffer(C.Structure):
    _fields_ = [("device", C.c_uint64), ("device_interface", C.c_void_p), ("host", C.c_void_p),
                ("flags", C.c_uint64), ("type", HalideType), ("dimensions", C.c_int32),
                ("dim", C.POINTER(HalideDim)), ("padding", C.c_void_p)]


class BlacklevelParams(C.Structure):
    _fields_ = [("black_level", C.c_float * 4), ("white_level", C.c_uint32), ("cfa_pattern", C.c_uint8 * 4)]


class DemosaicParams(C.Structure):
    _fields_ = [("cfa_pattern", C.c_uint8 * 4)]


class WbParams(C.Structure):
    _fields_ = [("as_shot_neutral", C.c_float * 3), ("camera_to_xyz_d50", C.c_float * 9),
                ("scene_cct", C.c_float), ("dual_illuminant_weight", C.c_float)]


class ColormatrixParams(C.Structure):
    _fields_ = [("transform", C.c_float * 9)]


class GainMapDispatchHeader(C.Structure):
    _fields_ = [("map_count", C.c_uint32), ("cfa_repeat", C.c_uint8 * 2), ("cfa_pattern", C.c_uint8 * 16)]


class GainMapDispatchPlane(C.Structure):
    _fields_ = [("top", C.c_uint32), ("left", C.c_uint32), ("bottom", C.c_uint32), ("right", C.c_uint32),
                ("plane", C.c_uint32), ("planes", C.c_uint32), ("map_points_v", C.c_uint32),
                ("map_points_h", C.c_uint32), ("map_spacing_v", C.c_double), ("map_spacing_h", C.c_double),
                ("map_origin_v", C.c_double), ("map_origin_h", C.c_double), ("gain_offset", C.c_uint32),
                ("gain_count", C.c_uint32)]


class Opcode3DispatchHeader(C.Structure):
    _fields_ = [("opcode_count", C.c_uint32), ("reserved", C.c_uint32)]


class Opcode3WarpCoefficient(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("kr0", "kr1", "kr2", "kr3", "kt0", "kt1")]


class Opcode3DispatchRecord(C.Structure):
    _fields_ = [("id", C.c_uint32), ("optional", C.c_uint32), ("coefficient_count", C.c_uint32),
                ("coefficients", Opcode3WarpCoefficient * 4), ("cx_hat", C.c_double), ("cy_hat", C.c_double),
                ("vignette_k", C.c_double * 5), ("vignette_cx_hat", C.c_double), ("vignette_cy_hat", C.c_double),
                ("constant", C.c_uint32), ("bayer_phase", C.c_uint32), ("point_offset", C.c_uint32),
                ("point_count", C.c_uint32), ("rect_offset", C.c_uint32), ("rect_count", C.c_uint32),
                ("top", C.c_uint32), ("left", C.c_uint32), ("bottom", C.c_uint32), ("right", C.c_uint32)]


class Lut3dParamHeader(C.Structure):
    _fields_ = [("size", C.c_uint32), ("value_count", C.c_uint32), ("interpolation", C.c_uint32)]


class Bm3dParams(C.Structure):
    _fields_ = [("sigma", C.c_float)]


class Bm3dSpecParams(C.Structure):
    """cpipe_Bm3dSpecParams (two-stage colour BM3D, aot_id denoise_bm3d_spec)."""
    _fields_ = [("sigma", C.c_float), ("lambda3d", C.c_float), ("tau_match1", C.c_float),
                ("tau_match2", C.c_float), ("n2", C.c_int32), ("ns", C.c_int32), ("nstep", C.c_int32),
                ("kaiser_beta", C.c_float), ("stages", C.c_int32), ("transform", C.c_int32)]


class GuidedFilterParams(C.Structure):
    _fields_ = [("radius", C.c_int32), ("eps", C.c_float)]


class WaveletBayesShrinkParams(C.Structure):
    _fields_ = [("chroma_strength", C.c_float)]


class AtrousWaveletParams(C.Structure):
    """cpipe_AtrousWaveletParams (a-trous wavelet denoiser, aot_id denoise_wavelet_atrous_spec)."""
    _fields_ = [("levels", C.c_int32), ("sigma", C.c_float), ("luma_strength", C.c_float),
                ("chroma_strength", C.c_float)]


class FilmicRgbParams(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("ev", "contrast", "saturation", "highlights", "shadows")]


class GreyworldParams(C.Structure):
    """cpipe_GreyworldParams (aot_id cpipe_wb_greyworld_auto): host address of a float[3] for the neutral."""
    _fields_ = [("neutral_out", C.c_uint64)]


class MertensLocalParams(C.Structure):
    """cpipe_MertensLocalParams (aot_id tone_mertens_local)."""
    _fields_ = [("weight_contrast", C.c_float), ("weight_saturation", C.c_float),
                ("weight_well_exposedness", C.c_float)]


class AcesFilmicParams(C.Structure):
    """cpipe_AcesFilmicParams (aot_id tone_aces_filmic)."""
    _fields_ = [("enabled", C.c_int32)]


class ReinhardParams(C.Structure):
    """cpipe_ReinhardParams (aot_id tone_reinhard)."""
    _fields_ = [("white_point", C.c_float)]


class EdgeAwareUsmParams(C.Structure):
    """cpipe_EdgeAwareUsmParams (aot_id sharpen_edge_aware_usm)."""
    _fields_ = [("strength", C.c_float), ("radius", C.c_int32), ("threshold", C.c_float)]


class DisplayParams(C.Structure):
    """cpipe_DisplayParams (aot_id cpipe_scene_linear_to_display): target 0 sRGB, 1 BT2020-PQ."""
    _fields_ = [("target", C.c_uint32)]


DISPLAY_SRGB, DISPLAY_BT2020_PQ = 0, 1


class DngInfo(C.Structure):
    """include/cpipe_b200_dng.h cpipe_DngInfo."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("bits_per_sample", C.c_uint32),
                ("compression", C.c_uint32), ("strip_offset", C.c_uint32), ("strip_byte_count", C.c_uint32),
                ("orientation", C.c_uint32), ("cfa_repeat", C.c_uint32 * 2), ("cfa_pattern", C.c_uint8 * 16),
                ("black_level", C.c_float * 4), ("white_level", C.c_uint32),
                ("calibration_illuminant", C.c_uint32 * 2), ("has_matrix", C.c_uint32 * 4),
                ("matrix", (C.c_float * 9) * 4), ("as_shot_neutral", C.c_float * 3),
                ("has_active_area", C.c_uint32), ("active_area", C.c_uint32 * 4), ("iso", C.c_int32),
                ("exposure_time_ns", C.c_int64), ("lens_aperture", C.c_float),
                ("lens_focal_length_mm", C.c_float), ("linearization_offset", C.c_uint32),
                ("linearization_count", C.c_uint32), ("opcode_list_offset", C.c_uint32 * 3),
                ("opcode_list_bytes", C.c_uint32 * 3), ("exif_offset", C.c_uint32), ("exif_bytes", C.c_uint32),
                ("xmp_offset", C.c_uint32), ("xmp_bytes", C.c_uint32), ("icc_offset", C.c_uint32),
                ("icc_bytes", C.c_uint32), ("make", C.c_char * 64), ("model", C.c_char * 64),
                ("seg_tiled", C.c_uint32), ("seg_width", C.c_uint32), ("seg_height", C.c_uint32),
                ("seg_count", C.c_uint32), ("seg_offsets_pos", C.c_uint32), ("seg_offsets_type", C.c_uint32),
                ("seg_counts_pos", C.c_uint32), ("seg_counts_type", C.c_uint32)]


class ChainConfig(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("black", BlacklevelParams),
                ("gainmap_blob", C.c_void_p), ("gainmap_blob_size", C.c_size_t), ("demosaic", C.c_int32),
                ("opcode3_blob", C.c_void_p), ("opcode3_blob_size", C.c_size_t),
                ("as_shot_neutral", C.c_float * 3), ("colormatrix", C.c_float * 9), ("bm3d_sigma", C.c_float),
                ("guided_radius", C.c_int32), ("guided_eps", C.c_float), ("wavelet_strength", C.c_float),
                ("filmic", FilmicRgbParams), ("lut_blob", C.c_void_p), ("lut_blob_size", C.c_size_t),
                ("plain_f32", C.c_int32), ("use_graph", C.c_int32), ("denoise_mode", C.c_int32),
                ("bm3d_spec", Bm3dSpecParams), ("surrogate_blob", C.c_void_p), ("surrogate_blob_size", C.c_size_t),
                ("noise_a", C.c_float), ("noise_b", C.c_float), ("stop_after", C.c_int32),
                ("spot_tiles", C.c_int32), ("spot_min_psnr_db", C.c_float), ("quad_bayer", C.c_int32),
                ("guided_spec", C.c_int32), ("atrous_levels", C.c_int32), ("atrous_luma_strength", C.c_float),
                ("sharpen", C.c_int32), ("sharpen_strength", C.c_float), ("sharpen_radius", C.c_int32),
                ("sharpen_threshold", C.c_float), ("display", C.c_int32), ("tone", C.c_int32),
                ("reinhard_white_point", C.c_float)]


MAIN_ENTRY = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)


class PluginDesc(C.Structure):
    _fields_ = [("abi_major", C.c_uint32), ("abi_minor", C.c_uint32), ("node_id", C.c_char_p),
                ("node_version", C.c_char_p), ("manifest_json", C.c_char_p), ("main_entry", MAIN_ENTRY)]


class FilterDesc(C.Structure):
    _fields_ = [("aot_id", C.c_char_p), ("entry", C.c_void_p), ("takes_params", C.c_int)]


PARAM_FILTER = C.CFUNCTYPE(C.c_int, C.POINTER(C.POINTER(HalideBuffer)), C.c_size_t,
                           C.POINTER(C.POINTER(HalideBuffer)), C.c_size_t, C.c_void_p, C.c_size_t)
PLAIN_FILTER = C.CFUNCTYPE(C.c_int, C.POINTER(HalideBuffer), C.POINTER(HalideBuffer))

# Every extern "C" symbol declared in include/cpipe_b200.h.
EXPORTS = [
    "cpipe_cuda_set_stream", "cpipe_cuda_get_stream", "cpipe_cuda_synchronize", "cpipe_cuda_last_error",
    "cpipe_cuda_trim_scratch", "cpipe_cuda_memory_stats",
    "cpipe_cuda_device_count",
    "cpipe_cuda_precision_convert_r16u_to_f32", "cpipe_cuda_precision_convert_f32_to_rgba16f",
    "cpipe_cuda_precision_convert_rgba16f_to_rgba8", "cpipe_cuda_precision_convert_rgba16f_to_rgba16u",
    "cpipe_cuda_demosaic_quad_bayer_remosaic", "cpipe_cuda_linearize_dng_lut", "cpipe_cuda_blacklevel_dng_levels",
    "cpipe_cuda_lens_shading_gainmap", "cpipe_cuda_demosaic_bilinear", "cpipe_cuda_demosaic_rcd",
    "cpipe_cuda_demosaic_amaze", "cpipe_cuda_demosaic_rcd_full", "cpipe_cuda_demosaic_amaze_full",
    "cpipe_cuda_wb_dual_illuminant", "cpipe_cuda_colormatrix_dng_to_working",
    "cpipe_cuda_denoise_bm3d_step1", "cpipe_cuda_denoise_bm3d_step2", "cpipe_cuda_denoise_bm3d_spec",
    "cpipe_cuda_denoise_guided_filter_spec", "cpipe_cuda_denoise_wavelet_atrous_spec",
    "cpipe_cuda_denoise_guided_filter",
    "cpipe_cuda_denoise_wavelet_bayes_shrink", "cpipe_cuda_lens_dng_opcode_list_3", "cpipe_cuda_color_3d_lut",
    "cpipe_cuda_tone_filmic_rgb", "cpipe_cuda_tone_aces_filmic", "cpipe_cuda_tone_reinhard",
    "cpipe_cuda_wb_greyworld_auto", "cpipe_cuda_tone_mertens_local", "cpipe_cuda_selftest_const_division",
    "cpipe_cuda_sharpen_edge_aware_usm", "cpipe_cuda_scene_linear_to_display",
    "cpipe_cuda_copy", "cpipe_cuda_filters", "cpipe_cuda_find_filter",
    "cpipe_cuda_color_3d_lut_noalloc",
    "cpipe_dng_parse", "cpipe_cuda_dng_decode", "cpipe_cuda_dng_unpack", "cpipe_cuda_lj92_decode",
    "cpipe_cuda_lj92_last_stats",
    "cpipe_b200_node_descs", "cpipe_b200_find_node",
    "cpipe_cuda_scene_raw", "cpipe_cuda_scene_raw_cfa", "cpipe_surrogate_blob_size", "cpipe_surrogate_create", "cpipe_surrogate_destroy", "cpipe_surrogate_export",
    "cpipe_surrogate_denoise", "cpipe_surrogate_set_engine", "cpipe_surrogate_check", "cpipe_surrogate_profile", "cpipe_surrogate_train_step", "cpipe_surrogate_gradients",
    "cpipe_b200_wb_prepare", "cpipe_b200_colormatrix_compose", "cpipe_b200_pack_gain_maps",
    "cpipe_b200_pack_opcode_list_3", "cpipe_b200_load_lut",
    "cpipe_b200_host_create", "cpipe_b200_host_destroy", "cpipe_b200_host_abi", "cpipe_b200_host_set_memory_cap",
    "cpipe_b200_buffer_create", "cpipe_b200_buffer_destroy", "cpipe_b200_buffer_upload",
    "cpipe_b200_buffer_download", "cpipe_b200_buffer_device_ptr", "cpipe_b200_buffer_abi", "cpipe_b200_buffer_format",
    "cpipe_b200_buffer_set_cfa", "cpipe_b200_buffer_set_levels", "cpipe_b200_buffer_set_matrix",
    "cpipe_b200_buffer_set_illuminants", "cpipe_b200_buffer_set_linearization_table",
    "cpipe_b200_buffer_set_noise_profile", "cpipe_b200_buffer_set_as_shot_neutral", "cpipe_b200_buffer_set_cs_role",
    "cpipe_b200_buffer_add_applied_step", "cpipe_b200_buffer_set_blob", "cpipe_b200_buffer_has_applied_step",
    "cpipe_b200_buffer_cs_role", "cpipe_b200_buffer_get_blob", "cpipe_b200_buffer_get_cfa",
    "cpipe_b200_params_create", "cpipe_b200_params_destroy", "cpipe_b200_params_set_double",
    "cpipe_b200_params_set_string", "cpipe_b200_params_set_bool", "cpipe_b200_run_node",
    "cpipe_b200_host_last_error",
    "cpipe_b200_pipeline_load", "cpipe_b200_pipeline_destroy", "cpipe_b200_pipeline_last_error",
    "cpipe_b200_pipeline_node_count", "cpipe_b200_pipeline_node_id", "cpipe_b200_pipeline_node_type",
    "cpipe_b200_pipeline_memory_plan", "cpipe_b200_pipeline_run",
    "cpipe_cuda_chain_create", "cpipe_cuda_chain_destroy", "cpipe_cuda_chain_output_bytes", "cpipe_cuda_chain_run",
    "cpipe_cuda_chain_run_host", "cpipe_cuda_chain_run_host_frames", "cpipe_cuda_pinned_alloc", "cpipe_cuda_pinned_free",
    "cpipe_cuda_batch_create", "cpipe_cuda_batch_destroy", "cpipe_cuda_batch_run", "cpipe_cuda_batch_autotune",
    "cpipe_cuda_batch_frame_chain", "cpipe_cuda_batch_schedule", "cpipe_cuda_batch_frame_times", "cpipe_cuda_chain_set_profiling", "cpipe_cuda_chain_profile", "cpipe_cuda_chain_denoise_stats", "cpipe_cuda_set_device", "cpipe_cuda_device_alloc",
    "cpipe_cuda_device_free", "cpipe_cuda_memcpy_h2d", "cpipe_cuda_memcpy_d2h", "cpipe_cuda_memcpy_d2d_async", "cpipe_cuda_count_nonfinite",
    "cpipe_cuda_stream_create",
    "cpipe_cuda_stream_destroy", "cpipe_cuda_stream_synchronize", "cpipe_cuda_event_create",
    "cpipe_cuda_event_destroy", "cpipe_cuda_event_record", "cpipe_cuda_event_elapsed_ms",
]

_lib = None


def lib():
    """Load libcpipe_b200.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m cpipe_b200.build` "
            "(the cpipe B200 nodes have no CPU implementation)")
    L = C.CDLL(LIB_PATH)
    vp, sz, i32, u32, cp = C.c_void_p, C.c_size_t, C.c_int, C.c_uint32, C.c_char_p
    sigs = {
        "cpipe_cuda_set_stream": (i32, [vp]), "cpipe_cuda_get_stream": (vp, []),
        "cpipe_cuda_synchronize": (i32, []), "cpipe_cuda_trim_scratch": (i32, []), "cpipe_cuda_last_error": (cp, []), "cpipe_cuda_device_count": (i32, []),
        "cpipe_cuda_filters": (C.POINTER(FilterDesc), [C.POINTER(sz)]),
        "cpipe_cuda_find_filter": (C.POINTER(FilterDesc), [cp]),
        "cpipe_b200_node_descs": (C.POINTER(PluginDesc), [C.POINTER(sz)]),
        "cpipe_b200_find_node": (C.POINTER(PluginDesc), [cp]),
        "cpipe_b200_host_create": (vp, []), "cpipe_b200_host_destroy": (None, [vp]),
        "cpipe_b200_host_abi": (vp, [vp]), "cpipe_b200_host_set_memory_cap": (i32, [vp, C.c_uint64]),
        "cpipe_b200_buffer_create": (vp, [vp, i32, u32, u32]), "cpipe_b200_buffer_destroy": (None, [vp]),
        "cpipe_b200_buffer_upload": (i32, [vp, vp, sz]), "cpipe_b200_buffer_download": (i32, [vp, vp, sz]),
        "cpipe_b200_buffer_device_ptr": (vp, [vp]), "cpipe_b200_buffer_abi": (vp, [vp]),
        "cpipe_b200_buffer_set_cfa": (i32, [vp, vp, vp]), "cpipe_b200_buffer_set_levels": (i32, [vp, vp, u32]),
        "cpipe_b200_buffer_set_matrix": (i32, [vp, i32, vp]),
        "cpipe_b200_buffer_set_illuminants": (i32, [vp, C.c_uint16, C.c_uint16]),
        "cpipe_b200_buffer_set_linearization_table": (i32, [vp, vp, sz]),
        "cpipe_b200_buffer_set_noise_profile": (i32, [vp, vp, vp, sz]),
        "cpipe_b200_buffer_set_as_shot_neutral": (i32, [vp, vp]),
        "cpipe_b200_buffer_set_cs_role": (i32, [vp, cp]), "cpipe_b200_buffer_add_applied_step": (i32, [vp, cp]),
        "cpipe_b200_buffer_set_blob": (i32, [vp, cp, vp, sz]),
        "cpipe_b200_buffer_has_applied_step": (i32, [vp, cp]), "cpipe_b200_buffer_cs_role": (cp, [vp]),
        "cpipe_b200_buffer_get_blob": (i32, [vp, cp, C.POINTER(vp), C.POINTER(sz)]),
        "cpipe_b200_buffer_get_cfa": (i32, [vp, C.POINTER(i32), vp, vp]),
        "cpipe_b200_params_create": (vp, []), "cpipe_b200_params_destroy": (None, [vp]),
        "cpipe_b200_params_set_double": (i32, [vp, cp, C.c_double]),
        "cpipe_b200_params_set_string": (i32, [vp, cp, cp]), "cpipe_b200_params_set_bool": (i32, [vp, cp, i32]),
        "cpipe_b200_run_node": (i32, [vp, cp, vp, C.POINTER(vp), sz, C.POINTER(vp), sz]),
        "cpipe_b200_host_last_error": (cp, [vp]),
        "cpipe_b200_pipeline_load": (vp, [vp, cp, sz, cp, C.POINTER(i32)]),
        "cpipe_b200_pipeline_destroy": (None, [vp]), "cpipe_b200_pipeline_last_error": (cp, [vp]),
        "cpipe_b200_pipeline_node_count": (sz, [vp]), "cpipe_b200_pipeline_node_id": (cp, [vp, sz]),
        "cpipe_b200_pipeline_node_type": (cp, [vp, sz]),
        "cpipe_b200_pipeline_memory_plan": (i32, [vp, u32, u32, C.POINTER(C.c_uint64), C.POINTER(u32)]),
        "cpipe_b200_pipeline_run": (i32, [vp, vp, C.POINTER(vp)]), "cpipe_b200_buffer_format": (i32, [vp]),
        "cpipe_cuda_memory_stats": (i32, [vp, vp, vp, vp]),
        "cpipe_b200_wb_prepare": (i32, [vp, vp, vp, vp, vp, C.c_uint16, C.c_uint16, vp, C.POINTER(C.c_double)]),
        "cpipe_b200_colormatrix_compose": (i32, [vp, vp]),
        "cpipe_b200_pack_gain_maps": (i32, [vp, sz, vp, vp, vp, C.POINTER(sz)]),
        "cpipe_b200_pack_opcode_list_3": (i32, [vp, sz, vp, C.POINTER(sz), C.POINTER(u32)]),
        "cpipe_b200_load_lut": (i32, [cp, C.POINTER(u32), vp, sz]),
        "cpipe_cuda_chain_create": (vp, [C.POINTER(ChainConfig), C.POINTER(i32)]),
        "cpipe_cuda_chain_destroy": (None, [vp]), "cpipe_cuda_chain_output_bytes": (sz, [vp]),
        "cpipe_cuda_selftest_const_division": (i32, [C.c_float, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "cpipe_dng_parse": (i32, [vp, sz, C.POINTER(DngInfo)]),
        "cpipe_cuda_dng_decode": (i32, [vp, sz, vp, sz, C.POINTER(DngInfo)]),
        "cpipe_cuda_dng_unpack": (i32, [vp, sz, u32, u32, u32, vp]),
        "cpipe_cuda_lj92_decode": (i32, [vp, vp, u32, u32, u32, u32, u32, u32, vp]),
        "cpipe_cuda_lj92_last_stats": (i32, [C.POINTER(C.c_uint64), u32]),
        "cpipe_cuda_chain_run": (i32, [vp, vp, vp, vp]), "cpipe_cuda_chain_run_host": (i32, [vp, vp, vp, vp]),
        "cpipe_cuda_chain_run_host_frames": (i32, [vp, vp, vp, i32, vp]),
        "cpipe_cuda_pinned_alloc": (i32, [sz, C.POINTER(vp)]), "cpipe_cuda_pinned_free": (None, [vp]),
        "cpipe_cuda_chain_set_profiling": (i32, [vp, i32]),
        "cpipe_cuda_batch_create": (vp, [vp, sz, C.POINTER(i32)]), "cpipe_cuda_batch_destroy": (None, [vp]),
        "cpipe_cuda_batch_run": (i32, [vp, vp, vp, vp]), "cpipe_cuda_batch_autotune": (i32, [vp, vp, vp, vp, vp]),
        "cpipe_cuda_batch_frame_chain": (vp, [vp, sz]),
        "cpipe_cuda_batch_schedule": (i32, [vp, vp, C.POINTER(i32)]),
        "cpipe_cuda_batch_frame_times": (i32, [vp, vp, vp, sz]),
        "cpipe_cuda_chain_profile": (i32, [vp, C.POINTER(C.c_double), C.POINTER(i32)]),
        "cpipe_cuda_chain_denoise_stats": (i32, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_float)]),
        "cpipe_cuda_set_device": (i32, [i32]), "cpipe_cuda_device_alloc": (i32, [sz, C.POINTER(vp)]),
        "cpipe_cuda_device_free": (None, [vp]), "cpipe_cuda_memcpy_h2d": (i32, [vp, vp, sz]),
        "cpipe_cuda_memcpy_d2h": (i32, [vp, vp, sz]), "cpipe_cuda_memcpy_d2d_async": (i32, [vp, vp, sz, vp]),
        "cpipe_cuda_count_nonfinite": (i32, [vp, sz, i32, C.POINTER(C.c_uint64), vp]), "cpipe_cuda_stream_create": (i32, [C.POINTER(vp)]),
        "cpipe_cuda_stream_destroy": (None, [vp]), "cpipe_cuda_stream_synchronize": (i32, [vp]),
        "cpipe_cuda_event_create": (i32, [C.POINTER(vp)]), "cpipe_cuda_event_destroy": (None, [vp]),
        "cpipe_cuda_event_record": (i32, [vp, vp]),
        "cpipe_cuda_event_elapsed_ms": (i32, [vp, vp, C.POINTER(C.c_float)]),
        "cpipe_cuda_scene_raw": (i32, [vp, i32, i32, C.c_uint64, i32, i32, C.c_float, C.c_float, vp, i32, vp]),
        "cpipe_cuda_scene_raw_cfa": (i32, [vp, i32, i32, C.c_uint64, i32, i32, C.c_float, C.c_float, vp, i32, i32,
                                           vp]),
        "cpipe_surrogate_blob_size": (sz, []), "cpipe_surrogate_create": (vp, [vp, sz, C.POINTER(i32)]),
        "cpipe_surrogate_destroy": (None, [vp]), "cpipe_surrogate_export": (i32, [vp, vp, sz]),
        "cpipe_surrogate_denoise": (i32, [vp, vp, vp, i32, i32, i32, i32, vp, vp]),
        "cpipe_surrogate_profile": (i32, [vp, vp, vp, i32, i32, i32, i32, vp, vp, vp]),
        "cpipe_surrogate_set_engine": (i32, [vp, i32]), "cpipe_surrogate_check": (i32, [vp]),
        "cpipe_surrogate_train_step": (i32, [vp, vp, vp, vp, i32, i32, i32, C.c_float, i32, C.POINTER(C.c_float),
                                             vp]),
        "cpipe_surrogate_gradients": (i32, [vp, vp, sz]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L
