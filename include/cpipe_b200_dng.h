/* DNG ingest: host TIFF/DNG tag parse and GPU unpack of the CFA strip into an
 * R16_UINT plane in device memory.
 *
 * Replaces the reference's ingest pair:
 *   - cpipe::ingest::dng_opcode::OpcodeListParser::parse
 *     (src/cpipe/ingest/dng_opcode/OpcodeListParser.cpp:330-515), whose
 *     ParsedDngMetadata (include/cpipe/ingest/dng_opcode/OpcodeList.hpp:15-40)
 *     cpipe_DngInfo flattens into plain fields and file byte ranges;
 *   - cpipe::ingest::dng::DngReader::read
 *     (src/cpipe/ingest/dng/DngReader.cpp:190-232), which the
 *     com.cpipe.builtin.dng_input node calls
 *     (src/cpipe/nodes/dng_input/dng_input.cpp:27-38).
 *
 * Status codes are the reference's cpipe_status_t values (cpipe_node_abi.h).
 * The message of the last failure is read with cpipe_cuda_last_error(). */
#ifndef CPIPE_B200_DNG_H
#define CPIPE_B200_DNG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cpipe_DngInfo {
    uint32_t width, height;            /* ImageWidth / ImageLength */
    uint32_t bits_per_sample;          /* BitsPerSample (1..16) */
    uint32_t compression;              /* Compression (1 = none; 1 when the tag is absent) */
    uint32_t strip_offset;             /* first StripOffsets value */
    uint32_t strip_byte_count;         /* first StripByteCounts value */
    uint32_t orientation;              /* Orientation; 0 when the tag is absent */
    uint32_t cfa_repeat[2];            /* CFARepeatPatternDim (2x2 or 4x4) */
    uint8_t cfa_pattern[16];           /* CFAPattern, row-major, repeat[0] * repeat[1] entries */
    float black_level[4];              /* first four BlackLevel values, 0 past the tag's count */
    uint32_t white_level;              /* WhiteLevel (SHORT / LONG); 0 when absent */
    uint32_t calibration_illuminant[2];
    uint32_t has_matrix[4];            /* ColorMatrix1, ColorMatrix2, ForwardMatrix1, ForwardMatrix2 present */
    float matrix[4][9];                /* in the same order, row-major, 0 past the tag's count */
    float as_shot_neutral[3];
    uint32_t has_active_area;
    uint32_t active_area[4];           /* x, y, width, height (from the tag's top, left, bottom, right) */
    int32_t iso;                       /* ISOSpeedRatings (IFD0, then the Exif IFD) */
    int64_t exposure_time_ns;          /* ExposureTime * 1e9 in binary32, truncated */
    float lens_aperture, lens_focal_length_mm;
    /* Byte ranges of variable-length values inside the file (offset, bytes);
     * bytes = 0 when the tag is absent.  linearization holds SHORT entries. */
    uint32_t linearization_offset, linearization_count;
    uint32_t opcode_list_offset[3], opcode_list_bytes[3];
    uint32_t exif_offset, exif_bytes;  /* the Exif IFD's entry table (2 + 12 n + 4 bytes) */
    uint32_t xmp_offset, xmp_bytes, icc_offset, icc_bytes;
    char make[64], model[64];          /* NUL-terminated, truncated to 63 characters */
    /* Raw data segments: the tiles (TileWidth / TileLength / TileOffsets /
     * TileByteCounts) when the file has them, else the strips (RowsPerStrip,
     * StripOffsets, StripByteCounts).  seg_width x seg_height per segment,
     * seg_count segments in row-major order; the offset and byte-count arrays
     * sit at the given file offsets with the given TIFF types (3 SHORT,
     * 4 LONG).  A Compression 7 file has one lossless JPEG stream per segment. */
    uint32_t seg_tiled, seg_width, seg_height, seg_count;
    uint32_t seg_offsets_pos, seg_offsets_type, seg_counts_pos, seg_counts_type;
} cpipe_DngInfo;

/* Parse IFD0 of a little-endian DNG held in host memory.  CPIPE_OK, or
 * CPIPE_FAILED (bad header, bad IFD table, missing raw fields), or
 * CPIPE_UNSUPPORTED (not a single-plane CFA, CFA repeat other than 2x2 / 4x4,
 * missing CFA pattern), exactly as OpcodeListParser::parse decides.  One
 * extension for files that parse rejects: when IFD0 is not a single-plane CFA
 * image (a preview), the first full-resolution single-plane CFA SubIFD
 * supplies the image tags, IFD0 the camera tags.  Host only: needs no GPU. */
int cpipe_dng_parse(const uint8_t* file, size_t file_bytes, cpipe_DngInfo* info);

/* DngReader::read over a file image in host memory: parse (CPIPE_UNSUPPORTED
 * becomes CPIPE_FAILED, as the reader maps it), copy the raw data to the
 * device and decode it into `d_raw` (width x height R16_UINT, row pitch width,
 * at least width * height * 2 bytes) on the library's current stream.
 * Compression 1: the uncompressed strip (cpipe_cuda_dng_unpack).  Compression
 * 7: the lossless JPEG segments (tiles or strips) through
 * cpipe_cuda_lj92_decode, where the reference reader calls LibRaw
 * (DngReader.cpp:113-124); a stream that does not decode is CPIPE_FAILED.
 * Other compressions: CPIPE_UNSUPPORTED.  `info` may be NULL. */
int cpipe_cuda_dng_decode(const uint8_t* file, size_t file_bytes, uint16_t* d_raw, size_t raw_bytes,
                          cpipe_DngInfo* info);

/* The unpack alone, from a strip already in device memory (16-byte aligned):
 *   bits == 16, or strip_bytes >= width * height * 2: little-endian 16-bit
 *     words, the first min(strip_bytes, width * height * 2) bytes copied and
 *     the rest of the plane zero (DngReader.cpp:145-164);
 *   bits 1..15 otherwise: samples packed most-significant bit first, each row
 *     starting on a byte boundary (DNG 1.4 uncompressed layout); bits past the
 *     strip read as zero. */
int cpipe_cuda_dng_unpack(const uint8_t* d_strip, size_t strip_bytes, uint32_t width, uint32_t height,
                          uint32_t bits, uint16_t* d_raw);

/* Lossless JPEG (ITU-T T.81 process 14; DNG Compression 7) segments held in
 * host memory, decoded on the GPU into `d_raw` (width x height R16_UINT): one
 * stream per segment, segments row-major, `across` per row, each
 * seg_w x seg_h samples filled row after row from the JPEG lines (X * Nf
 * samples each) and cropped at the image edges.  Headers are parsed on the
 * host (SOF3, DHT, DRI, SOS; 1-4 components, predictors 1-7, restart
 * intervals, point transform).  Segments without restart intervals are
 * decoded in parallel within each stream (1024-bit chunks decoded
 * speculatively and chained by warps; predictor 1 reconstructed by prefix
 * sums); segments with restart intervals by one GPU thread each.
 * CPIPE_FAILED with a message when a header is malformed or a stream does not
 * decode (it never reads past its segment).  No reference counterpart: the
 * reference decodes these through LibRaw. */
int cpipe_cuda_lj92_decode(const uint8_t* const* streams, const size_t* stream_bytes, uint32_t count, uint32_t across,
                           uint32_t seg_w, uint32_t seg_h, uint32_t width, uint32_t height, uint16_t* d_raw);

/* Figures of the process's last successful lossless-JPEG decode, the first
 * min(count, 9) of: [0] stream chunks of the parallel path, [1] segments on
 * the parallel path, [2] on the sequential path, [3] chunks the group walks
 * decoded again (no speculative path started at the exact state), [4] groups
 * whose entry the segment walks did not find, [5] chunks those walks decoded
 * again, [6] chunks the write walks decoded again, [7] bits decoded again,
 * [8] the longest such decode in bits.  CPIPE_BAD_INDEX when figures is NULL
 * and count is not 0. */
int cpipe_cuda_lj92_last_stats(uint64_t* figures, uint32_t count);

#ifdef __cplusplus
}
#endif

#endif
