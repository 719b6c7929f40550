/* libcpipe_b200: B200 (sm_100a) CUDA implementation of the cpipe raw->linear
 * node chain, behind the reference's own plugin and filter interfaces.
 *
 * Three layers, each a drop-in at the boundary a reference integration binds:
 *
 *  1. Filter seam -- one function per reference aot_id with the reference's
 *     filter signatures (src/cpipe/runtime/HalideFilterRegistry.hpp:18-21):
 *       HalideParamFilterEntry  int(halide_buffer_t* const*, size_t,
 *                                   halide_buffer_t* const*, size_t,
 *                                   const void* param_blob, size_t blob_size)
 *       HalideFilterEntry       int(halide_buffer_t* input, halide_buffer_t* output)
 *     A reference runtime registers them per aot_id with
 *     ComputeContext::register_halide_[param_]filter (ComputeContext.cpp:16-23).
 *     Param blobs are the reference PODs (cpipe_b200_params.h).  A buffer whose
 *     `device` field is non-zero is CUDA device memory processed in place,
 *     asynchronously on the thread's current stream; any other buffer is staged
 *     through device memory and the call returns when the host buffer holds the
 *     result.  Return values are cpipe_status_t codes with the reference's
 *     meaning; CUDA failures are CPIPE_INTERNAL_ERROR (message in
 *     cpipe_cuda_last_error()).  There is no CPU path.
 *
 *  2. Node plugins -- one cpipe_plugin_desc_t per reference node id, placed in
 *     the ELF section `cpipe_registry` (reference include/cpipe/sdk/registry.hpp:17-32)
 *     and also listed by cpipe_b200_node_descs().  Their main_entry does the
 *     reference node's host-side work (metadata checks, WB CCT search,
 *     colormatrix composition, OpcodeList2/3 parsing, .cube loading) and submits
 *     the CUDA filter through the host's compute suite.
 *
 *  3. A small host runtime (cpipe_b200_host_*) implementing the reference host
 *     suites over device-resident buffers, used by tests, benchmarks and hosts
 *     without their own runtime; and the fused chain (cpipe_cuda_chain_*).
 */
#ifndef CPIPE_B200_H
#define CPIPE_B200_H

#include <stddef.h>
#include <stdint.h>

#include "cpipe_b200_params.h"
#include "cpipe_halide_abi.h"
#include "cpipe_node_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------- stream / status */
/* Stream used by filter calls made from this thread (a cudaStream_t; NULL = legacy default stream). */
int cpipe_cuda_set_stream(void* cuda_stream);
void* cpipe_cuda_get_stream(void);
int cpipe_cuda_synchronize(void);
/* The filters draw their per-call device scratch from a memory pool of the
 * library's own, one per device, which keeps what it has reserved between
 * calls; this waits for the device and returns that memory.  (No reference
 * counterpart: the reference's filters run on the CPU.) */
int cpipe_cuda_trim_scratch(void);
/* Memory figures of the current device, for callers that budget device memory:
 * bytes the scratch pool above has reserved and has handed out, the device's
 * free bytes (cudaMemGetInfo), and the number of prepared tables (linearize,
 * GainMap, LUT) the library keeps.  Any pointer may be NULL.  (No reference
 * counterpart.) */
int cpipe_cuda_memory_stats(uint64_t* scratch_reserved, uint64_t* scratch_used, uint64_t* device_free,
                            uint64_t* prepared_tables);
const char* cpipe_cuda_last_error(void);
int cpipe_cuda_device_count(void);

/* ------------------------------------------------------------------ filter seam */
/* precision_convert_generator.cpp:31-124, registered in precision_convert_dispatch.cpp */
int cpipe_cuda_precision_convert_r16u_to_f32(halide_buffer_t* input, halide_buffer_t* output);
int cpipe_cuda_precision_convert_f32_to_rgba16f(halide_buffer_t* input, halide_buffer_t* output);
int cpipe_cuda_precision_convert_rgba16f_to_rgba8(halide_buffer_t* input, halide_buffer_t* output);
int cpipe_cuda_precision_convert_rgba16f_to_rgba16u(halide_buffer_t* input, halide_buffer_t* output);
/* demosaic_quad_bayer_remosaic_dispatch.cpp:6-8 */
int cpipe_cuda_demosaic_quad_bayer_remosaic(halide_buffer_t* input, halide_buffer_t* output);

#define CPIPE_CUDA_PARAM_FILTER(name)                                                         \
    int name(halide_buffer_t* const* inputs, size_t n_inputs, halide_buffer_t* const* outputs, \
             size_t n_outputs, const void* param_blob, size_t param_blob_size)
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_linearize_dng_lut);          /* linearize_dng_lut_dispatch.cpp:17-51 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_blacklevel_dng_levels);      /* blacklevel_dng_levels_dispatch.cpp:16-47 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_lens_shading_gainmap);       /* shading_gainmap_dispatch.cpp:73-133 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_demosaic_bilinear);          /* demosaic_bilinear_dispatch.cpp */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_demosaic_rcd);               /* demosaic_rcd_dispatch.cpp:19-38 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_demosaic_amaze);
/* Full-form RCD and AMaZE (aot_ids "demosaic_rcd_full", "demosaic_amaze_full";
 * node parameter algorithm = "full" of com.cpipe.demosaic.rcd / .amaze): the
 * published algorithms the reference's reduced 5x5 stencils are named after
 * (demosaic_rcd_generator.cpp:8-77, demosaic_amaze_generator.cpp:8-79 are the
 * nodes they stand beside; no reference filter counterpart).  Same buffers and
 * blob as the reference demosaic filters; 2x2 Bayer patterns only
 * (otherwise CPIPE_UNSUPPORTED). */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_demosaic_rcd_full);
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_demosaic_amaze_full);             /* demosaic_amaze_dispatch.cpp */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_wb_dual_illuminant);         /* wb_dual_illuminant_dispatch.cpp:16-48 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_colormatrix_dng_to_working); /* colormatrix_dng_to_working_dispatch.cpp:17-62 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_bm3d_step1);         /* bm3d_dispatch.cpp:19-30 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_bm3d_step2);         /* bm3d_dispatch.cpp:32-43 */
/* Two-stage colour BM3D (aot_id "denoise_bm3d_spec", blob cpipe_Bm3dSpecParams):
 * the published algorithm the reference's denoise.bm3d node is named after; the
 * node selects it with param algorithm = "bm3d".  No reference filter
 * counterpart (the reference's bm3d_step1 is a 2x2 box blend). */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_bm3d_spec);
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_guided_filter);      /* guided_filter_dispatch.cpp */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_wavelet_bayes_shrink); /* wavelet_bayes_shrink_dispatch.cpp */
/* Guided filter with a true (2r+1)^2 box (aot_id "denoise_guided_filter_spec",
 * blob cpipe_GuidedFilterParams, radius 1..16): the reference's
 * guided_filter formula (guided_filter_generator.cpp:45-85) without its
 * clamp of every radius above 1 to a 5x5 box.  The guided_filter node selects
 * it with param algorithm = "spec". */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_guided_filter_spec);
/* Multi-level a-trous wavelet denoiser (aot_id "denoise_wavelet_atrous_spec",
 * blob cpipe_AtrousWaveletParams); the wavelet_bayes_shrink node selects it
 * with param algorithm = "atrous".  No reference filter counterpart (the
 * reference's node is one 2x2 Haar level on chroma). */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_denoise_wavelet_atrous_spec);
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_lens_dng_opcode_list_3);     /* dng_opcode_list_3_dispatch.cpp:333-398 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_color_3d_lut);               /* lut3d_dispatch.cpp:20-60 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_tone_filmic_rgb);            /* filmic_rgb_dispatch.cpp:22-36 */
/* wb.greyworld_auto (aot_id "cpipe_wb_greyworld_auto", blob
 * cpipe_GreyworldParams; RGBA16F in and out): the grey-world neutral from
 * exact per-channel sums of the frame, then v / neutral per RGB channel.
 * Replaces the CPU loops of the reference node (greyworld_auto.cpp:44-77);
 * no reference filter counterpart.  CPIPE_NEED_METADATA when a channel sum is
 * not positive or a value is not finite, as the reference node. */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_wb_greyworld_auto);
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_tone_aces_filmic);           /* aces_filmic_dispatch.cpp:17-31 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_tone_reinhard);              /* reinhard_dispatch.cpp:16-29 */
/* Three inputs (under, normal, over), one output. */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_tone_mertens_local);         /* mertens_local_dispatch.cpp:18-37 */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_sharpen_edge_aware_usm);     /* edge_aware_usm_dispatch.cpp:18-31 */
/* Scene-linear Rec.2020 to display encode (aot_id "cpipe_scene_linear_to_display",
 * blob cpipe_DisplayParams; RGBA16F in, RGBA8 unorm out for sRGB, RGBA16
 * unorm with 10-bit codes in the top bits for BT2020-PQ).  Replaces the OCIO
 * CPU processor the reference node runs through its host
 * (scene_linear_to_display.cpp:114-121, HostContext.cpp:956-983, the
 * transforms of share/cpipe/ocio/v0.2/config.ocio); no reference filter
 * counterpart. */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_scene_linear_to_display);
/* Device copy for pass-through cases (aot_id "cpipe_copy"); replaces the lock_cpu
 * memcpy of e.g. shading_gainmap.cpp:50-75.  No reference filter counterpart. */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_copy);

/* Allocation-free 3D LUT filter: the same arguments and result as
 * cpipe_cuda_color_3d_lut, for callers that cannot allocate device memory while
 * they run (a frame loop with a fixed latency budget, where an allocator call
 * may block on the device, or a host that fixes each plugin's device memory at
 * start-up).  It has no counterpart in the reference: the LUT goes into a fixed
 * 3.3 MB device array every GPU holds while the library is loaded, so the LUT
 * edge length is at most 65 (larger: CPIPE_BAD_INDEX with a message), input and
 * output must be device buffers (host buffers: CPIPE_UNSUPPORTED), and calls
 * that overlap on the GPU race on that one array (calls in order on one stream
 * are safe).  The first call on a device looks up the array's device address;
 * make it before any stream capture on that device.  The LUT is copied from the
 * blob with cudaMemcpyAsync on the call's stream: from pageable host memory
 * that copy first waits for the work already queued on the stream, so the call
 * returns only after it; a page-locked blob avoids the wait and must stay
 * unchanged until the stream reaches the copy.  Frames of any height are
 * covered (the grid's rows step through the frame). */
CPIPE_CUDA_PARAM_FILTER(cpipe_cuda_color_3d_lut_noalloc);

/* Registration table: entry is a HalideParamFilterEntry when takes_params != 0,
 * else a HalideFilterEntry. */
typedef struct {
    const char* aot_id;
    void* entry;
    int takes_params;
} cpipe_cuda_filter_desc;
const cpipe_cuda_filter_desc* cpipe_cuda_filters(size_t* count);
const cpipe_cuda_filter_desc* cpipe_cuda_find_filter(const char* aot_id);

/* ----------------------------------------------------------------- node plugins */
/* Every node descriptor of this library (the same records are in `cpipe_registry`). */
const cpipe_plugin_desc_t* cpipe_b200_node_descs(size_t* count);
const cpipe_plugin_desc_t* cpipe_b200_find_node(const char* node_id);

/* ---------------------------------------------------- host-side parameter prep */
/* Dual-illuminant WB: CCT search + matrix blend (wb_dual_illuminant.cpp:79-282,352-367).
 * fm1/fm2 may be NULL (ColorMatrix blend inverted instead). */
int cpipe_b200_wb_prepare(const float neutral[3], const float cm1[9], const float cm2[9], const float* fm1,
                          const float* fm2, uint16_t illuminant1, uint16_t illuminant2, cpipe_WbParams* out,
                          double* scene_cct);
/* XYZ(D65)->Rec.2020 * Bradford D50->D65 * camera->XYZ(D50) (colormatrix_dng_to_working.cpp:20-28,125). */
int cpipe_b200_colormatrix_compose(const float camera_to_xyz_d50[9], float out[9]);
/* OpcodeList2 GainMap parse + pack (OpcodeList2.cpp:94-176, shading_gainmap.cpp:80-137).
 * *blob_size: capacity in, bytes needed out. */
int cpipe_b200_pack_gain_maps(const void* opcode_list_2, size_t n, const uint8_t cfa_repeat[2],
                              const uint8_t cfa_pattern[16], void* blob, size_t* blob_size);
/* OpcodeList3 parse + pack (OpcodeList3.cpp:83-296, dng_opcode_list_3.cpp:75-168). */
int cpipe_b200_pack_opcode_list_3(const void* opcode_list_3, size_t n, void* blob, size_t* blob_size,
                                  uint32_t* opcode_count);
/* .cube / .spi3d loader (Cube3dLutLoader.cpp:57-204); values NULL queries *size. */
int cpipe_b200_load_lut(const char* path, uint32_t* size, float* values, size_t capacity);

/* ----------------------------------------------------------------- host runtime */
typedef struct cpipe_b200_host cpipe_b200_host;
typedef struct cpipe_b200_buffer cpipe_b200_buffer;
typedef struct cpipe_b200_params cpipe_b200_params;

cpipe_b200_host* cpipe_b200_host_create(void);
void cpipe_b200_host_destroy(cpipe_b200_host* host);
cpipe_host_t* cpipe_b200_host_abi(cpipe_b200_host* host);
/* Device allocation cap for buffers and scratch of this host (0 = none);
 * allocations past it fail with CPIPE_OOM (reference Pipeline.cpp:587-592). */
int cpipe_b200_host_set_memory_cap(cpipe_b200_host* host, uint64_t bytes);

/* Image2D buffer in device memory; format is a CPIPE_FMT_* value. */
cpipe_b200_buffer* cpipe_b200_buffer_create(cpipe_b200_host* host, int format, uint32_t width, uint32_t height);
void cpipe_b200_buffer_destroy(cpipe_b200_buffer* buffer);
int cpipe_b200_buffer_upload(cpipe_b200_buffer* buffer, const void* host_data, size_t bytes);
int cpipe_b200_buffer_download(cpipe_b200_buffer* buffer, void* host_data, size_t bytes);
void* cpipe_b200_buffer_device_ptr(cpipe_b200_buffer* buffer);
/* The buffer's CPIPE_FMT_* value (0 for NULL). */
int cpipe_b200_buffer_format(const cpipe_b200_buffer* buffer);
const cpipe_buffer_t* cpipe_b200_buffer_abi(cpipe_b200_buffer* buffer);

/* Buffer metadata (what the reference BufferMetadata carries for this path). */
int cpipe_b200_buffer_set_cfa(cpipe_b200_buffer* b, const uint8_t repeat[2], const uint8_t pattern[16]);
int cpipe_b200_buffer_set_levels(cpipe_b200_buffer* b, const float black[4], uint32_t white);
int cpipe_b200_buffer_set_matrix(cpipe_b200_buffer* b, int which, const float m[9]); /* 1,2 color; 3,4 forward */
int cpipe_b200_buffer_set_illuminants(cpipe_b200_buffer* b, uint16_t illuminant1, uint16_t illuminant2);
int cpipe_b200_buffer_set_linearization_table(cpipe_b200_buffer* b, const uint16_t* values, size_t n);
int cpipe_b200_buffer_set_noise_profile(cpipe_b200_buffer* b, const float* beta, const float* lambda, size_t n);
int cpipe_b200_buffer_set_as_shot_neutral(cpipe_b200_buffer* b, const float rgb[3]);
int cpipe_b200_buffer_set_cs_role(cpipe_b200_buffer* b, const char* role);
int cpipe_b200_buffer_add_applied_step(cpipe_b200_buffer* b, const char* step);
int cpipe_b200_buffer_set_blob(cpipe_b200_buffer* b, const char* key, const void* data, size_t size);
int cpipe_b200_buffer_has_applied_step(cpipe_b200_buffer* b, const char* step);
const char* cpipe_b200_buffer_cs_role(cpipe_b200_buffer* b);
int cpipe_b200_buffer_get_blob(cpipe_b200_buffer* b, const char* key, const void** data, size_t* size);
int cpipe_b200_buffer_get_cfa(cpipe_b200_buffer* b, int* has_cfa, uint8_t repeat[2], uint8_t pattern[16]);

cpipe_b200_params* cpipe_b200_params_create(void);
void cpipe_b200_params_destroy(cpipe_b200_params* p);
int cpipe_b200_params_set_double(cpipe_b200_params* p, const char* key, double value);
int cpipe_b200_params_set_string(cpipe_b200_params* p, const char* key, const char* value);
int cpipe_b200_params_set_bool(cpipe_b200_params* p, const char* key, int value);

/* create -> process -> destroy one node on the host's stream, then freeze the
 * metadata builder into each output (reference Pipeline.cpp:704-787 per node).
 * Synchronises before returning. */
int cpipe_b200_run_node(cpipe_b200_host* host, const char* node_id, const cpipe_b200_params* params,
                        cpipe_b200_buffer* const* inputs, size_t n_in, cpipe_b200_buffer* const* outputs,
                        size_t n_out);
const char* cpipe_b200_host_last_error(cpipe_b200_host* host);

/* ---------------------------------------------------------- pipeline runner */
/* A pipeline document (*.cpipe.json, schema v0.4) planned once and run on
 * device buffers: replaces Pipeline::load + Pipeline::run_bound
 * (src/cpipe/runtime/Pipeline.cpp:368-601, 629-792) with the same load-time
 * checks and status codes (version / schema: CPIPE_FAILED; reserved or
 * unknown node type, bad param, dangling edge: CPIPE_BAD_INDEX; cycle:
 * CPIPE_FAILED; missing step or colour-role mismatch: CPIPE_NEED_METADATA;
 * implicit precision_convert insertion as PrecisionPlanner::auto_insert, else
 * CPIPE_BAD_PRECISION), the memory plan of MemoryPlanner::plan_graph
 * (MemoryPlanner.cpp:188-219) kept as device slots between runs, and one
 * host synchronisation per run.  until: NULL, or a node id whose ancestors and
 * itself are the nodes planned (a document's device prefix).  host may be NULL
 * for planning only (load checks, node order, memory plan; run refuses).  After
 * a failed load, cpipe_b200_pipeline_last_error(NULL) gives this thread's
 * message. */
typedef struct cpipe_b200_pipeline cpipe_b200_pipeline;
cpipe_b200_pipeline* cpipe_b200_pipeline_load(cpipe_b200_host* host, const char* json, size_t json_bytes,
                                              const char* until, int* status);
void cpipe_b200_pipeline_destroy(cpipe_b200_pipeline* p);
const char* cpipe_b200_pipeline_last_error(const cpipe_b200_pipeline* p);
/* Planned nodes in execution order, implicit precision converts included. */
size_t cpipe_b200_pipeline_node_count(const cpipe_b200_pipeline* p);
const char* cpipe_b200_pipeline_node_id(const cpipe_b200_pipeline* p, size_t i);
const char* cpipe_b200_pipeline_node_type(const cpipe_b200_pipeline* p, size_t i);
/* Memory plan for a w x h input: peak bytes (input + slots) and slot count. */
int cpipe_b200_pipeline_memory_plan(cpipe_b200_pipeline* p, uint32_t w, uint32_t h, uint64_t* peak_bytes,
                                    uint32_t* slots);
/* Runs the plan on `input` (a buffer of this host in the input port's format).
 * *output: the last node's buffer, owned by the pipeline and valid until the
 * next run or destroy (its device memory is a planner slot).  A peak above the
 * host's memory cap is CPIPE_OOM (reference Pipeline.cpp:587-592). */
int cpipe_b200_pipeline_run(cpipe_b200_pipeline* p, cpipe_b200_buffer* input, cpipe_b200_buffer** output);

/* ---------------------------------------------------------------- fused chain */
/* The raw->linear node sequence of the reference's classic pipeline
 * (examples/pipelines/full-classic-pipeline.cpipe.json, nodes lin..lut):
 *   precision_convert(r16u->f32) -> blacklevel -> GainMap -> demosaic ->
 *   OpcodeList3 -> WB -> colormatrix -> BM3D -> guided -> wavelet -> filmic -> 3D LUT
 * with every parameter already resolved by the nodes' host-side preparation
 * (the same blobs the filters take).  Output: RGBA16F (or RGBA f32 when
 * plain_f32), identical to running the nodes one by one. */
typedef struct {
    int32_t width, height;
    cpipe_BlacklevelParams black;       /* levels and the 2x2 CFA pattern */
    const void* gainmap_blob;           /* GainMap dispatch blob, or NULL for none */
    size_t gainmap_blob_size;
    int32_t demosaic;                   /* 0 bilinear, 1 RCD, 2 AMaZE */
    const void* opcode3_blob;           /* OpcodeList3 dispatch blob, or NULL */
    size_t opcode3_blob_size;
    float as_shot_neutral[3];           /* WB divisor */
    float colormatrix[9];               /* camera -> Rec.2020 */
    float bm3d_sigma;
    int32_t guided_radius;              /* 0: no guided node */
    float guided_eps;
    float wavelet_strength;             /* < 0: no wavelet node */
    cpipe_FilmicRgbParams filmic;
    const void* lut_blob;               /* Lut3dParamHeader + values, or NULL */
    size_t lut_blob_size;
    int32_t plain_f32;                  /* 1: FP32 plain form (no f16 rounding between nodes) */
    int32_t use_graph;                  /* 1: replay a captured CUDA graph per (input, output) pair */
    /* Denoiser in the BM3D slot: 0 = the reference's denoise.bm3d computation
     * (2x2 box blend, bm3d_sigma); 1 = two-stage BM3D (bm3d_spec; its sigma 0
     * means bm3d_sigma); 2 = learned surrogate (surrogate_blob). */
    int32_t denoise_mode;
    cpipe_Bm3dSpecParams bm3d_spec;
    const void* surrogate_blob;
    size_t surrogate_blob_size;
    float noise_a, noise_b;             /* noise model var = a*x + b (the surrogate's noise-map input) */
    int32_t stop_after;                 /* 0: whole chain; 1: output the colormatrix result (the
                                           denoiser's input); 2: output the denoiser's result */
    /* denoise_mode 2 spot check: every frame, two-stage BM3D on spot_tiles (<= 16)
     * stratified 256x256 tiles of the denoiser's input; if any tile of the
     * surrogate's output is below spot_min_psnr_db against it (peak 1), the
     * whole frame is denoised by BM3D instead.  Decided on the device (no host
     * synchronisation); 0 tiles: no check. */
    int32_t spot_tiles;
    float spot_min_psnr_db;
    /* 1: the raw input is a Sony Quad-Bayer mosaic (4x4 CFA repeat); the chain
     * starts with demosaic.quad_bayer_remosaic to an RGGB Bayer frame (then
     * `black.cfa_pattern` must be RGGB). */
    int32_t quad_bayer;
    /* Spec-mode denoisers ahead of the tone stage (extensions; 0 = the
     * reference's computation): guided_spec = 1 boxes with the true
     * (2 guided_radius + 1)^2 window (guided_radius 1..16; filter
     * denoise_guided_filter_spec); atrous_levels 1..6 replaces the wavelet
     * node's 2x2 Haar by the a-trous form with that many levels (filter
     * denoise_wavelet_atrous_spec; noise sigma bm3d_sigma, chroma strength
     * wavelet_strength when >= 0 else 1, luma strength atrous_luma_strength). */
    int32_t guided_spec;
    int32_t atrous_levels;
    float atrous_luma_strength;
    /* Finishing stages after the LUT, as the reference's example pipeline
     * continues (sharpen, display): sharpen = 1 runs sharpen.edge_aware_usm
     * (sharpen_strength / _radius / _threshold as that node's params);
     * display 1 = sRGB (RGBA8 unorm output, 4 bytes per pixel), 2 = BT2020-PQ
     * (RGBA16 unorm output, 10-bit codes in the top bits), 0 = none (RGBA16F
     * output).  Both need the f16 form and stop_after 0; with both, one kernel
     * sharpens and encodes. */
    int32_t sharpen;
    float sharpen_strength;
    int32_t sharpen_radius;
    float sharpen_threshold;
    int32_t display;
    /* Tone node in the tone stage: 0 = tone.filmic_rgb (`filmic` params),
     * 1 = tone.aces_filmic, 2 = tone.reinhard (reinhard_white_point < 0: the
     * node's unset value 1e6; else clamped to 0.1..10). */
    int32_t tone;
    float reinhard_white_point;
} cpipe_cuda_chain_config;

typedef struct cpipe_cuda_chain cpipe_cuda_chain;
/* Allocates the chain's device tables and two intermediate frames. */
cpipe_cuda_chain* cpipe_cuda_chain_create(const cpipe_cuda_chain_config* cfg, int* status);
void cpipe_cuda_chain_destroy(cpipe_cuda_chain* chain);
size_t cpipe_cuda_chain_output_bytes(const cpipe_cuda_chain* chain);
/* Device pointers (dense rows); asynchronous on `stream` (a cudaStream_t). */
int cpipe_cuda_chain_run(cpipe_cuda_chain* chain, const void* d_raw_u16, void* d_out, void* stream);
/* Host pointers: H2D of the raw frame, the chain, D2H of the result; returns after the copy-out. */
int cpipe_cuda_chain_run_host(cpipe_cuda_chain* chain, const uint16_t* h_raw, void* h_out, void* stream);
/* n frames from host memory, pipelined: frame i's upload and download overlap
 * the chain of its neighbours (two device frames each way, copy streams of the
 * chain's own); h_outs[i] receives frame i's result, the same bytes run_host
 * gives.  Returns after every frame is back.  Pinned host buffers let the
 * copies run asynchronously.  (The reference's filters take one frame per
 * call, HalideFilterRegistry.hpp:18-21; this is the batched form of run_host.) */
int cpipe_cuda_chain_run_host_frames(cpipe_cuda_chain* chain, const uint16_t* const* h_raws, void* const* h_outs,
                                     int n, void* stream);
/* Per-stage timing: while enabled, each run records CUDA events around its
 * stages (and bypasses the graph); chain_profile sums the stage times of the
 * runs recorded since the last call: [0] raw_to_rgba, [1] warp_wb_cm,
 * [2] the denoiser of denoise_mode 1 or 2 (0 in mode 0), [3] denoise_tone. */
int cpipe_cuda_chain_set_profiling(cpipe_cuda_chain* chain, int enable);
int cpipe_cuda_chain_profile(cpipe_cuda_chain* chain, double ms_per_stage[4], int* frames);
/* Spot-check counters since creation (denoise_mode 2): frames checked, frames
 * that fell back to BM3D, and the lowest tile PSNR seen (dB).  Waits for the
 * device. */
int cpipe_cuda_chain_denoise_stats(cpipe_cuda_chain* chain, uint32_t* frames, uint32_t* fallbacks,
                                   float* worst_tile_psnr_db);
/* Seeded synthetic raw frame on the device (uint16, width x height): linear
 * gradients, `rects` (<= 64) rectangles of uniform reflectance, a zone plate,
 * 2x2 CFA mosaic, Gaussian-form noise var = a*x + b, `bits`-bit values above
 * `black`.  Counter-based (Philox4x32-10), so a seed gives the same frame on
 * every launch.  No reference counterpart (training data and benchmarks). */
int cpipe_cuda_scene_raw(void* d_out, int width, int height, uint64_t seed, int bits, int black, float noise_a,
                         float noise_b, const uint8_t cfa[4], int rects, void* stream);
/* The same with a cfa_repeat x cfa_repeat pattern (2: Bayer, 4: Quad Bayer). */
int cpipe_cuda_scene_raw_cfa(void* d_out, int width, int height, uint64_t seed, int bits, int black, float noise_a,
                             float noise_b, const uint8_t* cfa, int cfa_repeat, int rects, void* stream);

/* ---------------------------------------------------------- learned surrogate */
/* A residual convolutional denoiser that stands in for BM3D (weights:
 * cpipe_SurrogateHeader + FP32 parameters, see cpipe_b200_params.h), with its
 * own forward and training kernels.  No reference counterpart: the reference's
 * AI denoise node is planned but not implemented.  Frames are dense RGBA
 * device buffers [n][height][width][4] (binary16 when f16, training: binary16);
 * noise_ab holds n host-side (a, b) pairs of the noise model var = a*x + b that
 * the network's noise-map input is computed from. */
typedef struct cpipe_surrogate cpipe_surrogate;
size_t cpipe_surrogate_blob_size(void);
cpipe_surrogate* cpipe_surrogate_create(const void* blob, size_t blob_size, int* status);
void cpipe_surrogate_destroy(cpipe_surrogate* s);
/* Current (trained) weights in the blob format. */
int cpipe_surrogate_export(const cpipe_surrogate* s, void* blob, size_t blob_size);
int cpipe_surrogate_denoise(cpipe_surrogate* s, const void* d_in, void* d_out, int n, int width, int height, int f16,
                            const float* noise_ab, void* stream);
/* Inference engine: 1 = tcgen05 kernels (default where the driver provides the
 * tensor-map encoder), 0 = the mma.sync kernels the training uses. */
int cpipe_surrogate_set_engine(cpipe_surrogate* s, int engine);
/* Waits for the device; CPIPE_INTERNAL_ERROR (with a message) when a bounded
 * wait inside a tcgen05 kernel ran out since creation. */
int cpipe_surrogate_check(cpipe_surrogate* s);
/* One denoise with CUDA events between its kernels: ms[0] the input map,
 * ms[1 + l] layer l (l = 0..7).  Waits for the stream. */
int cpipe_surrogate_profile(cpipe_surrogate* s, const void* d_in, void* d_out, int n, int width, int height, int f16,
                            const float* noise_ab, float ms[9], void* stream);
/* One step on a batch: forward, mean-squared-error loss against the target,
 * backward; with update != 0 also an Adam step (lr).  *loss (optional) gets
 * the batch loss (the call then waits for the stream). */
int cpipe_surrogate_train_step(cpipe_surrogate* s, const void* d_noisy, const void* d_target, const float* noise_ab,
                               int n, int width, int height, float lr, int update, float* loss, void* stream);
/* Gradients of the last train_step, in blob parameter order. */
int cpipe_surrogate_gradients(const cpipe_surrogate* s, float* grad, size_t count);

/* ----------------------------------------------------------- batched form */
/* Up to 64 frames of any size, CFA (Bayer, or Quad Bayer with quad_bayer = 1),
 * bit depth and noise through the chain (binary16 between nodes, the
 * reference's denoise.bm3d) in one launch per stage: persistent kernels walk a
 * queue of (frame, tile) work items.  The frames share the demosaic, the guided
 * radius class and the warp form.  run() replays one CUDA graph for a given set
 * of input / output pointers.  autotune() times candidate persistent grid sizes
 * per stage on the given frames and keeps the fastest (per_sm_out: CTAs per SM
 * chosen for the three stages). */
typedef struct cpipe_cuda_batch cpipe_cuda_batch;
cpipe_cuda_batch* cpipe_cuda_batch_create(const cpipe_cuda_chain_config* cfgs, size_t n, int* status);
void cpipe_cuda_batch_destroy(cpipe_cuda_batch* batch);
int cpipe_cuda_batch_run(cpipe_cuda_batch* batch, const void* const* d_raw, void* const* d_out, void* stream);
int cpipe_cuda_batch_autotune(cpipe_cuda_batch* batch, const void* const* d_raw, void* const* d_out, void* stream,
                              int per_sm_out[3]);
/* Frame i's single-frame chain (the same node parameters; for per-frame runs). */
cpipe_cuda_chain* cpipe_cuda_batch_frame_chain(cpipe_cuda_batch* batch, size_t i);
/* The schedule in use: persistent CTAs per SM of the three stages (0: one
 * work item per CTA, a grid of all the stage's items) and the rows of a
 * stage-2 work item (128 pixels wide); both set by cpipe_cuda_batch_autotune. */
int cpipe_cuda_batch_schedule(cpipe_cuda_batch* batch, int per_sm[3], int* rows_per_item);
/* Completion time of each frame in the last cpipe_cuda_batch_run on `stream`,
 * in ms after the run's first kernel started: the device clock is read when the
 * last stage-3 work item of the frame finishes (its latency inside the batched
 * launch).  Waits for the stream; n >= the batch's frame count. */
int cpipe_cuda_batch_frame_times(cpipe_cuda_batch* batch, void* stream, float* ms, size_t n);

/* Self-test of the division by a fixed divisor the kernels use in place of
 * IEEE division (Markstein's method, nodes.cuh const_div): compares it with
 * IEEE division on every binary32 in its range for `divisor`; no reference
 * counterpart. */
int cpipe_cuda_selftest_const_division(float divisor, uint64_t* mismatches, uint64_t* checked);

/* Device memory, streams and events for callers without their own CUDA runtime. */
int cpipe_cuda_set_device(int device);
int cpipe_cuda_device_alloc(size_t bytes, void** out);
void cpipe_cuda_device_free(void* p);
int cpipe_cuda_memcpy_h2d(void* dst, const void* src, size_t bytes);
int cpipe_cuda_memcpy_d2h(void* dst, const void* src, size_t bytes);
int cpipe_cuda_memcpy_d2d_async(void* dst, const void* src, size_t bytes, void* stream);
/* Number of non-finite values among `count` binary16 (f16 != 0) or float32
 * values on the device; waits for the stream. */
int cpipe_cuda_count_nonfinite(const void* d, size_t count, int f16, uint64_t* out, void* stream);
int cpipe_cuda_stream_create(void** out);
void cpipe_cuda_stream_destroy(void* stream);
int cpipe_cuda_stream_synchronize(void* stream);
int cpipe_cuda_event_create(void** out);
void cpipe_cuda_event_destroy(void* event);
int cpipe_cuda_event_record(void* event, void* stream);
int cpipe_cuda_event_elapsed_ms(void* start, void* stop, float* ms);
/* Page-locked host memory for run_host callers. */
int cpipe_cuda_pinned_alloc(size_t bytes, void** out);
void cpipe_cuda_pinned_free(void* p);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CPIPE_B200_H */
