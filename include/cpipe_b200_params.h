/* Parameter blobs passed through `submit_halide_with_params` to each filter.
 *
 * Every struct is byte-compatible with the POD the reference node packs for its
 * filter, so a reference host can hand the same blob to the CUDA filter:
 *   LinearizeParamsHeader .. Opcode3BadRect  src/cpipe/nodes/detail/P1ParamDispatch.hpp:10-104
 *   Lut3dParamHeader                          src/cpipe/nodes/color/Lut3dParams.hpp:10-14
 *   Bm3dParams                                src/cpipe/nodes/denoise/bm3d_dispatch.cpp:12-14
 *   GuidedFilterParams                        src/cpipe/nodes/denoise/guided_filter_dispatch.cpp:13-16
 *   WaveletBayesShrinkParams                  src/cpipe/nodes/denoise/wavelet_bayes_shrink_dispatch.cpp:12-14
 *   FilmicRgbParams                           src/cpipe/nodes/tone/filmic_rgb_dispatch.cpp:12-18
 * The static size checks at the end pin the layouts (x86-64 / aarch64 LP64).
 */
#ifndef CPIPE_B200_PARAMS_H
#define CPIPE_B200_PARAMS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t table_size; /* followed by table_size uint16 entries */
} cpipe_LinearizeParamsHeader;

typedef struct {
    float black_level[4];
    uint32_t white_level;
    uint8_t cfa_pattern[4];
} cpipe_BlacklevelParams;

typedef struct {
    uint8_t cfa_pattern[4];
} cpipe_DemosaicParams;

typedef struct {
    float as_shot_neutral[3];
    float camera_to_xyz_d50[9];
    float scene_cct;
    float dual_illuminant_weight;
} cpipe_WbParams;

typedef struct {
    float transform[9];
} cpipe_ColormatrixParams;

typedef struct {
    uint32_t map_count;
    uint8_t cfa_repeat[2];
    uint8_t cfa_pattern[16];
} cpipe_GainMapDispatchHeader;

typedef struct {
    uint32_t top;
    uint32_t left;
    uint32_t bottom;
    uint32_t right;
    uint32_t plane;
    uint32_t planes;
    uint32_t map_points_v;
    uint32_t map_points_h;
    double map_spacing_v;
    double map_spacing_h;
    double map_origin_v;
    double map_origin_h;
    uint32_t gain_offset;
    uint32_t gain_count;
} cpipe_GainMapDispatchPlane;

typedef struct {
    uint32_t opcode_count;
    uint32_t reserved;
} cpipe_Opcode3DispatchHeader;

typedef struct {
    double kr0;
    double kr1;
    double kr2;
    double kr3;
    double kt0;
    double kt1;
} cpipe_Opcode3WarpCoefficient;

typedef struct {
    uint32_t id;
    uint32_t optional;
    uint32_t coefficient_count;
    cpipe_Opcode3WarpCoefficient coefficients[4];
    double cx_hat;
    double cy_hat;
    double vignette_k[5];
    double vignette_cx_hat;
    double vignette_cy_hat;
    uint32_t constant;
    uint32_t bayer_phase;
    uint32_t point_offset;
    uint32_t point_count;
    uint32_t rect_offset;
    uint32_t rect_count;
    uint32_t top;
    uint32_t left;
    uint32_t bottom;
    uint32_t right;
} cpipe_Opcode3DispatchRecord;

typedef struct {
    uint32_t row;
    uint32_t column;
} cpipe_Opcode3BadPoint;

typedef struct {
    uint32_t top;
    uint32_t left;
    uint32_t bottom;
    uint32_t right;
} cpipe_Opcode3BadRect;

/* Opcode ids as packed into cpipe_Opcode3DispatchRecord::id
 * (reference src/cpipe/nodes/lens/dng_opcode_list_3_dispatch.cpp:26-31). */
enum {
    CPIPE_OPCODE3_UNKNOWN = 0,
    CPIPE_OPCODE3_WARP_RECTILINEAR = 1,
    CPIPE_OPCODE3_FIX_VIGNETTE_RADIAL = 3,
    CPIPE_OPCODE3_FIX_BAD_PIXELS_CONSTANT = 4,
    CPIPE_OPCODE3_FIX_BAD_PIXELS_LIST = 5,
    CPIPE_OPCODE3_TRIM_BOUNDS = 6
};

typedef struct {
    uint32_t size;
    uint32_t value_count;
    uint32_t interpolation; /* 0 tetrahedral, 1 trilinear */
} cpipe_Lut3dParamHeader;

typedef struct {
    float sigma;
} cpipe_Bm3dParams;

typedef struct {
    int32_t radius;
    float eps;
} cpipe_GuidedFilterParams;

typedef struct {
    float chroma_strength;
} cpipe_WaveletBayesShrinkParams;

/* Multi-level a-trous wavelet denoiser ("spec mode"; aot_id
 * denoise_wavelet_atrous_spec).  The reference's denoise.wavelet_bayes_shrink
 * node is a single-level 2x2 Haar chroma shrink
 * (nodes/denoise/wavelet_bayes_shrink_generator.cpp:57-86); this is the
 * undecimated form that the node is named after, on the node's own colour
 * space (Y = (r+2g+b)/4, Co = r-b, Cg = g-(r+b)/2): B3-spline a-trous
 * decomposition (Starck, Murtagh, "Image restoration with noise suppression
 * using the wavelet transform", A&A 288, 1994), per band soft thresholds of
 * BayesShrink form (Chang, Yu, Vetterli, IEEE TIP 9(9), 2000),
 * T = sigma_n^2 / sigma_x.  There is no reference counterpart. */
typedef struct {
    int32_t levels;         /* detail levels, 0..6 (5); 0 copies */
    float sigma;            /* noise standard deviation per RGB channel (linear units) */
    float luma_strength;    /* threshold scale on Y (1); 0 leaves Y unchanged */
    float chroma_strength;  /* threshold scale on Co and Cg (1) */
} cpipe_AtrousWaveletParams;

typedef struct {
    float ev;
    float contrast;
    float saturation;
    float highlights;
    float shadows;
} cpipe_FilmicRgbParams;

/* wb.greyworld_auto on the GPU (aot_id "cpipe_wb_greyworld_auto").
 * neutral_out: host address of a float[3] that receives the estimated neutral
 * (R/G, 1, B/G) the node then writes into the metadata. */
typedef struct {
    uint64_t neutral_out;
} cpipe_GreyworldParams;

/* tone.mertens_local (nodes/tone/mertens_local_dispatch.cpp:12-16). */
typedef struct {
    float weight_contrast;          /* 0..2 (node default 0) */
    float weight_saturation;        /* 0..2 (1) */
    float weight_well_exposedness;  /* 0..2 (1) */
} cpipe_MertensLocalParams;

/* tone.aces_filmic (nodes/tone/aces_filmic_dispatch.cpp:13-15). */
typedef struct {
    int32_t enabled;   /* 0: pass-through */
} cpipe_AcesFilmicParams;

/* tone.reinhard (nodes/tone/reinhard_dispatch.cpp:12-14). */
typedef struct {
    float white_point; /* the node sends 1e6 when its param is unset, else clamp(0.1, 10) */
} cpipe_ReinhardParams;

/* sharpen.edge_aware_usm (nodes/sharpen/edge_aware_usm_dispatch.cpp:12-16). */
typedef struct {
    float strength;    /* 0..2 (node default 0.75) */
    int32_t radius;    /* <= 1: 3x3 mean, else 5x5 mean */
    float threshold;   /* |v - blur| below this leaves v unchanged */
} cpipe_EdgeAwareUsmParams;

/* color.scene_linear_to_display (nodes/color/scene_linear_to_display.cpp:31-50):
 * target 0 = "sRGB" (R8G8B8A8_UNORM output), 1 = "BT2020-PQ"
 * (R16G16B16A16_UNORM output, 10-bit codes in the top bits). */
typedef struct {
    uint32_t target;
} cpipe_DisplayParams;
#define CPIPE_DISPLAY_SRGB 0U
#define CPIPE_DISPLAY_BT2020_PQ 1U

/* Two-stage colour BM3D ("spec mode"; aot_id denoise_bm3d_spec).  The
 * reference's denoise.bm3d node computes a 2x2 box blend
 * (nodes/denoise/bm3d_step1_generator.cpp:33-61); this is the published
 * algorithm it is named after: Dabov, Foi, Katkovnik, Egiazarian, "Image
 * denoising by sparse 3D transform-domain collaborative filtering", IEEE TIP
 * 16(8), 2007, in its colour form (grouping on luminance, ICIP 2007), with
 * the parameter values of Lebrun, "An analysis and implementation of the BM3D
 * image denoising method", IPOL 2012.  Blocks are 8x8; matching uses the
 * 8-bit-quantised luminance mean; thresholds are mean squared 8-bit
 * differences per pixel.  There is no reference counterpart. */
typedef struct {
    float sigma;        /* noise standard deviation per RGB channel (linear units); <= 0 copies */
    float lambda3d;     /* hard-threshold factor (2.7) */
    float tau_match1;   /* step-1 match threshold, mean squared 8-bit difference (2500, <= 16000) */
    float tau_match2;   /* step-2 match threshold (400, <= 16000) */
    int32_t n2;         /* maximum blocks per stack: 1, 2, 4, 8 or 16 */
    int32_t ns;         /* search window edge, odd, 1..45 (39) */
    int32_t nstep;      /* reference-block step, 1..8 (3) */
    float kaiser_beta;  /* aggregation window parameter (2.0) */
    int32_t stages;     /* 1 = hard threshold only, 2 = hard threshold then Wiener */
    int32_t transform;  /* 0 = DCT/Haar on the tensor cores (FP16 hi/lo split products, FP32
                           accumulation); 1 = FP32 on the CUDA cores.  Same definition.
                           2 = screening form: tensor cores with single FP16 products (about
                           2^-11 relative per product), for checks that need BM3D's output
                           to a few 1e-4 rather than to FP32 accuracy. */
} cpipe_Bm3dSpecParams;

/* Learned surrogate denoiser weights (no reference counterpart: the
 * reference's AI denoise node is planned but not implemented).  A residual
 * network of `layers` 3x3 convolutions, zero padded, ReLU after every layer but
 * the last; input = R, G, B and the noise map sigma/0.03 with
 * sigma = sqrt(max(0, noise_b + noise_a * max(L, 0))), L = (R+G+B)/3; output =
 * input RGB + the last layer's 3 channels.  The blob is this header followed,
 * per layer l, by float weights[cout][cin][3][3] then float bias[cout]
 * (cin = in_channels for l = 0 else channels; cout = out_channels for the last
 * layer else channels), little endian. */
typedef struct {
    char magic[4];          /* "CPSN" */
    uint32_t version;       /* 1 */
    uint32_t layers;        /* 8 */
    uint32_t channels;      /* 32 */
    uint32_t in_channels;   /* 4 */
    uint32_t out_channels;  /* 3 */
    uint32_t reserved[2];   /* 0 */
} cpipe_SurrogateHeader;

#if defined(__cplusplus)
#define CPIPE_STATIC_ASSERT static_assert
#else
#define CPIPE_STATIC_ASSERT _Static_assert
#endif
CPIPE_STATIC_ASSERT(sizeof(cpipe_BlacklevelParams) == 24, "BlacklevelParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_WbParams) == 56, "WbParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_GainMapDispatchHeader) == 24, "GainMapDispatchHeader layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_GainMapDispatchPlane) == 72, "GainMapDispatchPlane layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_Opcode3DispatchRecord) == 320, "Opcode3DispatchRecord layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_Lut3dParamHeader) == 12, "Lut3dParamHeader layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_Bm3dSpecParams) == 40, "Bm3dSpecParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_SurrogateHeader) == 32, "SurrogateHeader layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_AtrousWaveletParams) == 16, "AtrousWaveletParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_EdgeAwareUsmParams) == 12, "EdgeAwareUsmParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_AcesFilmicParams) == 4, "AcesFilmicParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_MertensLocalParams) == 12, "MertensLocalParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_GreyworldParams) == 8, "GreyworldParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_ReinhardParams) == 4, "ReinhardParams layout");
CPIPE_STATIC_ASSERT(sizeof(cpipe_DisplayParams) == 4, "DisplayParams layout");

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CPIPE_B200_PARAMS_H */
