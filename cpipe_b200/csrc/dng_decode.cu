// GPU unpack of a DNG's uncompressed CFA strip into an R16_UINT plane, and the
// DngReader::read entry point over a file image in host memory
// (src/cpipe/ingest/dng/DngReader.cpp:190-232).
//
// Layout in HBM: the strip bytes, copied as they sit in the file to a scratch
// buffer (16-byte aligned); the output plane, width x height uint16 with row
// pitch width.  Both kernels are streaming copies: the 16-bit form moves 2
// bytes in and 2 out per sample, the packed form `bits`/8 in and 2 out.
#include <cstdint>
#include <cstring>

#include <vector>

#include "../../include/cpipe_b200_dng.h"
#include "filters_impl.h"

namespace cpb {
namespace {

constexpr int kUnpackThreads = 256;

// 16-bit words: thread i writes output bytes [16 i, 16 i + 16).  Bytes below
// `copy` come from the strip, the rest are zero (the reference copies
// min(expected, strip bytes) into a zeroed plane).
template <bool kVec>
__global__ void __launch_bounds__(kUnpackThreads) dng_words_kernel(const uint8_t* __restrict__ strip, uint64_t copy,
                                                                   uint8_t* __restrict__ out, uint64_t out_bytes) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i * 16 < out_bytes; i += stride) {
        const uint64_t b0 = i * 16;
        if (kVec && b0 + 16 <= copy && b0 + 16 <= out_bytes) {
            *reinterpret_cast<uint4*>(out + b0) = __ldg(reinterpret_cast<const uint4*>(strip + b0));
            continue;
        }
        const uint64_t end = b0 + 16 < out_bytes ? b0 + 16 : out_bytes;
        for (uint64_t b = b0; b < end; ++b) out[b] = b < copy ? strip[b] : (uint8_t)0;
    }
}

// Packed samples, most-significant bit first, rows starting on byte
// boundaries.  Thread (y, g) writes samples [8 g, 8 g + 8) of row y, which
// start at bit 8 g * bits = byte g * bits of the row: no group straddles a
// byte it shares with another group.  Bytes at or past `avail` read as zero.
// kWords: the group's bytes come in as aligned 32-bit words (the strip is
// 4-byte aligned), funnel-shifted to the group's first byte; otherwise byte
// by byte.
template <int kBits, bool kWords>
__global__ void __launch_bounds__(kUnpackThreads) dng_packed_kernel(const uint8_t* __restrict__ strip, uint64_t avail,
                                                                    uint32_t w, uint32_t h, uint64_t row_bytes,
                                                                    uint16_t* __restrict__ out, bool vec_store) {
    const uint32_t groups = (w + 7) / 8;
    const uint64_t total = (uint64_t)groups * h;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const uint32_t y = (uint32_t)(t / groups);
        const uint32_t g = (uint32_t)(t - (uint64_t)y * groups);
        const uint64_t base = (uint64_t)y * row_bytes + (uint64_t)g * kBits;
        // Up to 8 * 16 = 128 bits: hi holds the first 64, lo the rest.
        uint64_t hi = 0, lo = 0;
        if constexpr (kWords) {
            constexpr int kAligned = (kBits + 3) / 4;  // little-endian words from `base`
            const uint64_t start = base & ~3ull;
            const uint32_t sh = 8u * (uint32_t)(base & 3);
            uint32_t raw[kAligned + 1];
#pragma unroll
            for (int i = 0; i <= kAligned; ++i) {
                const uint64_t a = start + 4ull * i;
                if (a + 4 <= avail) {
                    raw[i] = __ldg(reinterpret_cast<const uint32_t*>(strip + a));
                } else {
                    uint32_t v = 0;
                    for (int k = 0; k < 4; ++k)
                        if (a + k < avail) v |= (uint32_t)__ldg(strip + a + k) << (8 * k);
                    raw[i] = v;
                }
            }
            uint32_t wd[4] = {0, 0, 0, 0};  // bytes base .. base + 15, big-endian per word
#pragma unroll
            for (int i = 0; i < kAligned; ++i) wd[i] = __byte_perm(__funnelshift_r(raw[i], raw[i + 1], sh), 0, 0x0123);
            hi = ((uint64_t)wd[0] << 32) | wd[1];
            lo = ((uint64_t)wd[2] << 32) | wd[3];
        } else {
#pragma unroll
            for (int k = 0; k < kBits; ++k) {
                const uint64_t b = base + k;
                const uint64_t v = b < avail ? (uint64_t)__ldg(strip + b) : 0ull;
                if (k < 8) hi |= v << ((56 - 8 * k) & 63);
                else lo |= v << ((120 - 8 * k) & 63);
            }
        }
        uint16_t s[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int bit = j * kBits;  // first bit of sample j within the group
            uint64_t v;
            if (bit + kBits <= 64) {
                v = hi >> (64 - bit - kBits);
            } else if (bit >= 64) {
                v = lo >> (128 - bit - kBits);
            } else {
                const int in_lo = bit + kBits - 64;  // bits taken from lo
                v = (hi << in_lo) | (lo >> (64 - in_lo));
            }
            s[j] = (uint16_t)(v & ((1u << kBits) - 1u));
        }
        uint16_t* row = out + (uint64_t)y * w;
        const uint32_t x0 = g * 8;
        if (vec_store && x0 + 8 <= w) {
            uint4 q;
            q.x = (uint32_t)s[0] | ((uint32_t)s[1] << 16);
            q.y = (uint32_t)s[2] | ((uint32_t)s[3] << 16);
            q.z = (uint32_t)s[4] | ((uint32_t)s[5] << 16);
            q.w = (uint32_t)s[6] | ((uint32_t)s[7] << 16);
            *reinterpret_cast<uint4*>(row + x0) = q;
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (x0 + j < w) row[x0 + j] = s[j];
        }
    }
}

int grid_for(uint64_t units) {
    const uint64_t per = (uint64_t)kUnpackThreads;
    uint64_t blocks = (units + per - 1) / per;
    const uint64_t cap = 148ull * 16;
    if (blocks > cap) blocks = cap;
    return blocks == 0 ? 1 : (int)blocks;
}

template <int kBits>
void launch_packed(const uint8_t* strip, uint64_t avail, uint32_t w, uint32_t h, uint64_t row_bytes, uint16_t* out,
                   bool vec, cudaStream_t st) {
    const uint64_t units = (uint64_t)((w + 7) / 8) * h;
    if ((uintptr_t)strip % 4 == 0)
        dng_packed_kernel<kBits, true><<<grid_for(units), kUnpackThreads, 0, st>>>(strip, avail, w, h, row_bytes, out, vec);
    else
        dng_packed_kernel<kBits, false><<<grid_for(units), kUnpackThreads, 0, st>>>(strip, avail, w, h, row_bytes, out, vec);
}

int unpack(const uint8_t* d_strip, uint64_t strip_bytes, uint32_t w, uint32_t h, uint32_t bits, uint16_t* d_raw,
           cudaStream_t st) {
    if (bits < 1 || bits > 16) {
        set_error("%s", "BitsPerSample outside 1..16");
        return CPIPE_UNSUPPORTED;
    }
    const uint64_t plane = (uint64_t)w * h * 2;
    if (bits == 16 || strip_bytes >= plane) {
        const uint64_t copy = strip_bytes < plane ? strip_bytes : plane;
        const bool vec = ((uintptr_t)d_strip % 16 == 0) && ((uintptr_t)d_raw % 16 == 0);
        const int grid = grid_for((plane + 15) / 16);
        if (vec) dng_words_kernel<true><<<grid, kUnpackThreads, 0, st>>>(d_strip, copy, (uint8_t*)d_raw, plane);
        else dng_words_kernel<false><<<grid, kUnpackThreads, 0, st>>>(d_strip, copy, (uint8_t*)d_raw, plane);
        return cuda_status(cudaGetLastError(), "dng unpack launch");
    }
    const uint64_t row_bytes = ((uint64_t)w * bits + 7) / 8;
    const bool vec = ((uintptr_t)d_raw % 16 == 0) && (w % 8 == 0);
    switch (bits) {
#define CPB_DNG_BITS(B) \
    case B: launch_packed<B>(d_strip, strip_bytes, w, h, row_bytes, d_raw, vec, st); break;
        CPB_DNG_BITS(1) CPB_DNG_BITS(2) CPB_DNG_BITS(3) CPB_DNG_BITS(4) CPB_DNG_BITS(5)
        CPB_DNG_BITS(6) CPB_DNG_BITS(7) CPB_DNG_BITS(8) CPB_DNG_BITS(9) CPB_DNG_BITS(10)
        CPB_DNG_BITS(11) CPB_DNG_BITS(12) CPB_DNG_BITS(13) CPB_DNG_BITS(14) CPB_DNG_BITS(15)
#undef CPB_DNG_BITS
        default:
            set_error("%s", "BitsPerSample outside 1..16");
            return CPIPE_UNSUPPORTED;
    }
    return cuda_status(cudaGetLastError(), "dng unpack launch");
}

}  // namespace
}  // namespace cpb

extern "C" int cpipe_cuda_dng_unpack(const uint8_t* d_strip, size_t strip_bytes, uint32_t width, uint32_t height,
                                     uint32_t bits, uint16_t* d_raw) {
    using namespace cpb;
    if (d_raw == nullptr || (d_strip == nullptr && strip_bytes != 0) || width == 0 || height == 0) {
        set_error("%s", "dng unpack: null buffer or empty extent");
        return CPIPE_BAD_INDEX;
    }
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    return unpack(d_strip, strip_bytes, width, height, bits, d_raw, current_stream());
}

extern "C" int cpipe_cuda_dng_decode(const uint8_t* file, size_t file_bytes, uint16_t* d_raw, size_t raw_bytes,
                                     cpipe_DngInfo* info) {
    using namespace cpb;
    cpipe_DngInfo local;
    cpipe_DngInfo* d = info ? info : &local;
    int st = cpipe_dng_parse(file, file_bytes, d);
    if (st == CPIPE_UNSUPPORTED) return CPIPE_FAILED;  // DngReader.cpp:192-195
    if (st != CPIPE_OK) return st;
    if (d->compression == 7) {
        // Lossless JPEG segments (the reference reader hands these to LibRaw).
        const uint64_t plane7 = (uint64_t)d->width * d->height * 2;
        if (d_raw == nullptr || raw_bytes < plane7) {
            set_error("%s", "dng decode: output plane smaller than width * height * 2 bytes");
            return CPIPE_BAD_INDEX;
        }
        if (d->seg_count == 0) {
            set_error("%s", "compressed DNG without raw data segments");
            return CPIPE_FAILED;
        }
        auto value = [&](uint32_t pos, uint32_t type, uint32_t i, uint64_t* v) {
            const uint64_t sz = type == 3 ? 2 : 4, at = (uint64_t)pos + sz * i;
            if (at + sz > file_bytes) return false;
            const uint8_t* q = file + at;
            *v = type == 3 ? (uint64_t)(q[0] | (q[1] << 8))
                           : (uint64_t)q[0] | ((uint64_t)q[1] << 8) | ((uint64_t)q[2] << 16) | ((uint64_t)q[3] << 24);
            return true;
        };
        std::vector<const uint8_t*> streams(d->seg_count);
        std::vector<size_t> sizes(d->seg_count);
        for (uint32_t i = 0; i < d->seg_count; ++i) {
            uint64_t off = 0, cnt = 0;
            if (!value(d->seg_offsets_pos, d->seg_offsets_type, i, &off) ||
                !value(d->seg_counts_pos, d->seg_counts_type, i, &cnt) || off > file_bytes || cnt > file_bytes - off) {
                set_error("%s", "compressed DNG segment lies outside the file");
                return CPIPE_FAILED;
            }
            streams[i] = file + off;
            sizes[i] = (size_t)cnt;
        }
        const uint32_t across = d->seg_tiled ? (d->width + d->seg_width - 1) / d->seg_width : 1;
        st = lj92_decode(streams.data(), sizes.data(), d->seg_count, across, d->seg_width, d->seg_height, d->width,
                         d->height, d_raw);
        return st == CPIPE_UNSUPPORTED ? CPIPE_FAILED : st;
    }
    if (d->compression != 1) {
        set_error("%s", "DNG compression other than none (1) and lossless JPEG (7)");
        return CPIPE_UNSUPPORTED;
    }
    // The strip must lie inside the file (DngReader.cpp:151-154).
    if (d->strip_offset > file_bytes || d->strip_byte_count > file_bytes - d->strip_offset) {
        set_error("%s", "failed to decode DNG RAW16 payload");
        return CPIPE_FAILED;
    }
    const uint64_t plane = (uint64_t)d->width * d->height * 2;
    if (d_raw == nullptr || raw_bytes < plane) {
        set_error("%s", "dng decode: output plane smaller than width * height * 2 bytes");
        return CPIPE_BAD_INDEX;
    }
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    void* d_strip = nullptr;
    st = call.alloc(((uint64_t)d->strip_byte_count + 15) / 16 * 16, &d_strip);
    if (st == CPIPE_OK)
        st = cuda_status(cudaMemcpyAsync(d_strip, file + d->strip_offset, d->strip_byte_count,
                                         cudaMemcpyHostToDevice, call.stream),
                         "dng strip upload");
    if (st == CPIPE_OK)
        st = unpack((const uint8_t*)d_strip, d->strip_byte_count, d->width, d->height, d->bits_per_sample, d_raw,
                    call.stream);
    return call.finish(st);
}
