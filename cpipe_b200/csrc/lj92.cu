// Lossless JPEG (ITU-T T.81 process 14), the codec of DNG Compression 7, on
// the GPU: cpipe_cuda_lj92_decode, and the Compression 7 branch of
// cpipe_cuda_dng_decode.  The reference decodes these files through LibRaw
// (DngReader.cpp:113-124), which is not part of the reference tree; this is an
// implementation of the published standard.
//
// Host: each segment's marker stream is parsed (SOF3 frame, DHT tables, DRI,
// SOS scan; APPn / COM skipped), its Huffman tables turned into canonical
// decoding arrays (T.81 F.2.2.3) plus a 9-bit lookahead table, and the
// entropy-coded bytes of all segments copied to the device in one block.
// Device: one thread per segment walks its entropy-coded bytes with a 64-bit
// bit buffer (0xFF00 unstuffed; a marker ends the data, zeros follow), decodes
// the category and extra bits of every sample (EXTEND, SSSS = 16 -> 32768),
// predicts it (T.81 H.1.2.1: 2^(P-Pt-1) at the scan's and every restart
// interval's first sample, Ra on that line, Rb in the first column, predictor
// 1-7 elsewhere, from two line buffers of its own), and writes the sample,
// shifted left by Pt, to its place in the segment raster: JPEG lines of X * Nf
// samples fill the seg_w x seg_h raster row after row, cropped at the image.
// Every loop is bounded by the frame's sample count and every read by the
// segment's end; a code longer than 16 bits, or a missing restart marker,
// marks the segment failed.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "../../include/cpipe_b200_dng.h"
#include "filters_impl.h"

namespace cpb {
namespace {

struct HuffDev {
    int32_t maxcode[17];  // [l]: largest code of length l, -1 when none
    int32_t valoff[17];   // [l]: index of the first symbol of length l minus the first code of length l
    uint8_t vals[20];
    uint16_t fast[512];   // 9-bit lookahead: (length << 8) | symbol; 0 when the code is longer than 9 bits
};

struct SegDev {
    uint64_t off;   // entropy-coded data in the device block
    uint64_t len;
    uint32_t X, Y, nf, p, ps, pt, ri;
    uint32_t table[4];
    uint32_t x0, y0;
    uint64_t rowbuf;  // u16 index of the segment's two line buffers
};

constexpr int kLjThreads = 64;

__device__ __forceinline__ int lj_predict(const uint16_t* cur, const uint16_t* prev, int x, int c, int nf, int ps,
                                          bool first_line) {
    if (first_line) return cur[(x - 1) * nf + c];  // x > 0 here
    if (x == 0) return prev[c];
    const int ra = cur[(x - 1) * nf + c], rb = prev[x * nf + c], rc = prev[(x - 1) * nf + c];
    switch (ps) {
        case 1: return ra;
        case 2: return rb;
        case 3: return rc;
        case 4: return ra + rb - rc;
        case 5: return ra + ((rb - rc) >> 1);
        case 6: return rb + ((ra - rc) >> 1);
        default: return (ra + rb) >> 1;
    }
}

__global__ void __launch_bounds__(kLjThreads) lj92_kernel(const uint8_t* __restrict__ data, const SegDev* __restrict__ segs,
                                                          int nseg, const HuffDev* __restrict__ tables,
                                                          uint16_t* __restrict__ rowbufs, uint16_t* __restrict__ out,
                                                          int width, int height, int seg_w, int seg_h,
                                                          int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseg) return;
    const SegDev s = segs[i];
    const uint8_t* p = data + s.off;
    const uint8_t* const end = p + s.len;
    uint64_t acc = 0;
    int nbits = 0;
    bool marker = false;
    auto refill = [&]() {
        while (nbits <= 56) {
            uint32_t b = 0;
            if (!marker && p < end) {
                b = *p;
                if (b == 0xFF) {
                    const uint32_t nx = p + 1 < end ? p[1] : 0xD9;
                    if (nx == 0) {
                        p += 2;
                    } else {
                        marker = true;  // the data ends at a marker; zeros follow
                        b = 0;
                    }
                } else {
                    ++p;
                }
            }
            acc |= (uint64_t)b << (56 - nbits);
            nbits += 8;
        }
    };
    const int W = (int)(s.X * s.nf);
    uint16_t* rows = rowbufs + s.rowbuf;
    const int dflt = 1 << (s.p - s.pt - 1);
    int err = 0, tr = 0, tc = 0, first_line_y = 0;
    long long mcu = 0;
    bool reset = true;
    for (int y = 0; y < (int)s.Y && !err; ++y) {
        uint16_t* cur = rows + (size_t)(y & 1) * W;
        const uint16_t* prev = rows + (size_t)((y & 1) ^ 1) * W;
        for (int x = 0; x < (int)s.X && !err; ++x) {
            if (s.ri && mcu && mcu % s.ri == 0) {
                acc = 0;
                nbits = 0;
                marker = false;
                if (p + 1 < end && p[0] == 0xFF && (p[1] & 0xF8) == 0xD0) p += 2;
                else err = 2;
                first_line_y = y;
                reset = true;
            }
            for (int c = 0; c < (int)s.nf && !err; ++c) {
                refill();
                const HuffDev* t = tables + s.table[c];
                const uint32_t look = (uint32_t)(acc >> 55);
                const uint32_t f = t->fast[look];
                int len, sym;
                if (f) {
                    len = (int)(f >> 8);
                    sym = (int)(f & 0xFF);
                } else {
                    len = 10;
                    int code = (int)(acc >> 54);
                    while (len <= 16 && code > t->maxcode[len]) {
                        ++len;
                        code = (int)(acc >> (64 - len));
                    }
                    if (len > 16) {
                        err = 1;
                        break;
                    }
                    sym = t->vals[t->valoff[len] + code];
                }
                acc <<= len;
                nbits -= len;
                int diff = 0;
                if (sym == 16) {
                    diff = 32768;
                } else if (sym > 0) {
                    const int v = (int)(acc >> (64 - sym));
                    acc <<= sym;
                    nbits -= sym;
                    diff = v < (1 << (sym - 1)) ? v - (1 << sym) + 1 : v;
                }
                const int pred = reset ? dflt : lj_predict(cur, prev, x, c, (int)s.nf, (int)s.ps, y == first_line_y);
                const uint16_t v = (uint16_t)((pred + diff) & 0xFFFF);
                cur[x * s.nf + c] = v;
                if (tr < seg_h) {
                    const int gx = (int)s.x0 + tc, gy = (int)s.y0 + tr;
                    if (gx < width && gy < height) out[(size_t)gy * width + gx] = (uint16_t)(v << s.pt);
                }
                if (++tc == seg_w) {
                    tc = 0;
                    ++tr;
                }
            }
            reset = false;
            ++mcu;
        }
    }
    status[i] = err;
}

uint32_t be16(const uint8_t* q) { return ((uint32_t)q[0] << 8) | q[1]; }

// One segment's markers up to its scan: frame, tables, restart interval.
int parse_segment(const uint8_t* s, size_t n, SegDev* seg, std::vector<HuffDev>* tables, std::string* err) {
    if (n < 4 || s[0] != 0xFF || s[1] != 0xD8) {
        *err = "lossless JPEG stream without SOI";
        return CPIPE_FAILED;
    }
    size_t pos = 2;
    int local[4] = {-1, -1, -1, -1};
    bool have_frame = false;
    uint32_t ids[4] = {0, 0, 0, 0};
    *seg = SegDev{};
    while (pos + 4 <= n) {
        if (s[pos] != 0xFF) {
            *err = "lossless JPEG marker expected";
            return CPIPE_FAILED;
        }
        const uint32_t m = s[pos + 1];
        if (m == 0xFF) {  // fill byte
            ++pos;
            continue;
        }
        const uint32_t len = be16(s + pos + 2);
        if (len < 2 || pos + 2 + len > n) {
            *err = "lossless JPEG segment runs past its data";
            return CPIPE_FAILED;
        }
        const uint8_t* b = s + pos + 4;
        const uint32_t bl = len - 2;
        if (m == 0xC4) {  // DHT
            uint32_t q = 0;
            while (q + 17 <= bl) {
                const uint32_t tc = b[q] >> 4, th = b[q] & 0x0F;
                uint32_t total = 0;
                for (int l = 0; l < 16; ++l) total += b[q + 1 + l];
                if (tc != 0 || th > 3 || total > 17 || q + 17 + total > bl) {
                    *err = "lossless JPEG Huffman table is not a lossless (class 0) table of at most 17 symbols";
                    return CPIPE_FAILED;
                }
                HuffDev h;
                std::memset(&h, 0, sizeof(h));
                int code = 0, k = 0;
                for (int l = 1; l <= 16; ++l) {
                    const int cnt = b[q + l];
                    h.maxcode[l] = -1;
                    if (cnt) {
                        h.valoff[l] = k - code;
                        for (int j = 0; j < cnt; ++j, ++code, ++k) {
                            const uint8_t sym = b[q + 17 + k];
                            if (sym > 16) {
                                *err = "lossless JPEG Huffman symbol above 16";
                                return CPIPE_FAILED;
                            }
                            h.vals[k] = sym;
                            if (l <= 9)
                                for (int e = code << (9 - l); e < (code + 1) << (9 - l); ++e)
                                    h.fast[e] = (uint16_t)((l << 8) | sym);
                        }
                        h.maxcode[l] = code - 1;
                    }
                    if (code > (1 << l)) {
                        *err = "lossless JPEG Huffman table over-subscribed";
                        return CPIPE_FAILED;
                    }
                    code <<= 1;
                }
                local[th] = (int)tables->size();
                tables->push_back(h);
                q += 17 + total;
            }
        } else if (m == 0xC3) {  // SOF3
            if (bl < 6) {
                *err = "short SOF3";
                return CPIPE_FAILED;
            }
            seg->p = b[0];
            seg->Y = be16(b + 1);
            seg->X = be16(b + 3);
            seg->nf = b[5];
            if (seg->p < 2 || seg->p > 16 || seg->Y == 0 || seg->X == 0 || seg->nf < 1 || seg->nf > 4 ||
                bl < 6 + 3 * seg->nf) {
                *err = "lossless JPEG frame header out of range";
                return CPIPE_FAILED;
            }
            for (uint32_t c = 0; c < seg->nf; ++c) ids[c] = b[6 + 3 * c];
            have_frame = true;
        } else if (m == 0xC0 || m == 0xC1 || m == 0xC2 || (m >= 0xC5 && m <= 0xCF && m != 0xC8 && m != 0xCC)) {
            *err = "not a lossless Huffman JPEG (SOF3) stream";
            return CPIPE_UNSUPPORTED;
        } else if (m == 0xDD) {  // DRI
            if (bl < 2) {
                *err = "short DRI";
                return CPIPE_FAILED;
            }
            seg->ri = be16(b);
        } else if (m == 0xDA) {  // SOS
            if (!have_frame || bl < 1 || b[0] != seg->nf || bl < 1 + 2 * seg->nf + 3) {
                *err = "lossless JPEG scan must carry every frame component";
                return CPIPE_FAILED;
            }
            for (uint32_t c = 0; c < seg->nf; ++c) {
                const uint32_t cid = b[1 + 2 * c], td = b[2 + 2 * c] >> 4;
                if (cid != ids[c] || td > 3 || local[td] < 0) {
                    *err = "lossless JPEG scan names a missing table or component";
                    return CPIPE_FAILED;
                }
                seg->table[c] = (uint32_t)local[td];
            }
            seg->ps = b[1 + 2 * seg->nf];
            seg->pt = b[3 + 2 * seg->nf] & 0x0F;
            if (seg->ps < 1 || seg->ps > 7 || seg->pt >= seg->p) {
                *err = "lossless JPEG predictor or point transform out of range";
                return CPIPE_FAILED;
            }
            seg->off = pos + 2 + len;  // relative to the stream; rebased by the caller
            seg->len = n - seg->off;
            return CPIPE_OK;
        }
        pos += 2 + len;
    }
    *err = "lossless JPEG stream without a scan";
    return CPIPE_FAILED;
}

}  // namespace

int lj92_decode(const uint8_t* const* streams, const size_t* bytes, uint32_t count, uint32_t across, uint32_t seg_w,
                uint32_t seg_h, uint32_t width, uint32_t height, uint16_t* d_raw) {
    if (!streams || !bytes || count == 0 || across == 0 || seg_w == 0 || seg_h == 0 || width == 0 || height == 0 ||
        !d_raw) {
        set_error("%s", "lj92 decode: empty or null argument");
        return CPIPE_BAD_INDEX;
    }
    std::vector<SegDev> segs(count);
    std::vector<HuffDev> tables;
    std::vector<uint8_t> block;
    uint64_t rows = 0;
    for (uint32_t i = 0; i < count; ++i) {
        std::string err;
        if (!streams[i]) {
            set_error("%s", "lj92 decode: null stream");
            return CPIPE_BAD_INDEX;
        }
        const int st = parse_segment(streams[i], bytes[i], &segs[i], &tables, &err);
        if (st != CPIPE_OK) {
            set_error("%s", err.c_str());
            return st;
        }
        if ((uint64_t)segs[i].X * segs[i].nf * segs[i].Y > (uint64_t)seg_w * seg_h) {
            set_error("%s", "lossless JPEG frame holds more samples than its segment");
            return CPIPE_FAILED;
        }
        const uint64_t start = segs[i].off;
        segs[i].off = block.size();
        block.insert(block.end(), streams[i] + start, streams[i] + bytes[i]);
        segs[i].x0 = (i % across) * seg_w;
        segs[i].y0 = (i / across) * seg_h;
        segs[i].rowbuf = rows;
        rows += 2ull * segs[i].X * segs[i].nf;
    }
    block.resize(block.size() + 16, 0);
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    void *d_block = nullptr, *d_segs = nullptr, *d_tables = nullptr, *d_rows = nullptr, *d_status = nullptr;
    int st = call.upload(block.data(), block.size(), &d_block);
    if (st == CPIPE_OK) st = call.upload(segs.data(), segs.size() * sizeof(SegDev), &d_segs);
    if (st == CPIPE_OK) st = call.upload(tables.data(), tables.size() * sizeof(HuffDev), &d_tables);
    if (st == CPIPE_OK) st = call.alloc(rows * sizeof(uint16_t), &d_rows);
    if (st == CPIPE_OK) st = call.alloc(count * sizeof(int), &d_status);
    if (st == CPIPE_OK)
        st = cuda_status(cudaMemsetAsync(d_raw, 0, (size_t)width * height * 2, call.stream), "lj92 clear");
    if (st != CPIPE_OK) return call.finish(st);
    lj92_kernel<<<(count + kLjThreads - 1) / kLjThreads, kLjThreads, 0, call.stream>>>(
        static_cast<const uint8_t*>(d_block), static_cast<const SegDev*>(d_segs), (int)count,
        static_cast<const HuffDev*>(d_tables), static_cast<uint16_t*>(d_rows), d_raw, (int)width, (int)height,
        (int)seg_w, (int)seg_h, static_cast<int*>(d_status));
    std::vector<int> status(count, 0);
    st = cuda_status(cudaGetLastError(), "lj92 launch");
    if (st == CPIPE_OK)
        st = cuda_status(cudaMemcpyAsync(status.data(), d_status, count * sizeof(int), cudaMemcpyDeviceToHost, call.stream),
                         "lj92 status");
    if (st == CPIPE_OK) st = cuda_status(cudaStreamSynchronize(call.stream), "lj92 decode");
    if (st == CPIPE_OK)
        for (uint32_t i = 0; i < count; ++i)
            if (status[i]) {
                set_error("%s", status[i] == 2 ? "lossless JPEG restart marker missing"
                                               : "lossless JPEG stream does not decode");
                st = CPIPE_FAILED;
                break;
            }
    return call.finish(st);
}

}  // namespace cpb

extern "C" int cpipe_cuda_lj92_decode(const uint8_t* const* streams, const size_t* stream_bytes, uint32_t count,
                                      uint32_t across, uint32_t seg_w, uint32_t seg_h, uint32_t width, uint32_t height,
                                      uint16_t* d_raw) {
    try {
        return cpb::lj92_decode(streams, stream_bytes, count, across, seg_w, seg_h, width, height, d_raw);
    } catch (...) {
        return CPIPE_INTERNAL_ERROR;
    }
}
