// Lossless JPEG (ITU-T T.81 process 14), the codec of DNG Compression 7, on
// the GPU: cpipe_cuda_lj92_decode, and the Compression 7 branch of
// cpipe_cuda_dng_decode.  The reference decodes these files through LibRaw
// (DngReader.cpp:113-124), which is not part of the reference tree; this is an
// implementation of the published standard.
//
// Host: each segment's marker stream is parsed (SOF3 frame, DHT tables, DRI,
// SOS scan; APPn / COM skipped), its Huffman tables deduplicated and turned
// into canonical decoding arrays (T.81 F.2.2.3) plus a 12-bit lookahead table,
// and the entropy-coded bytes of all segments copied to the device in one
// block (straight from the caller's memory when the segments lie together, as
// they do in a DNG file).
//
// Device, segments without restart intervals (the DNG case), in parallel:
//  1. unstuff: per 4 KB block, the first marker of each segment (0xFF followed
//     by anything but 0x00 ends the entropy-coded data) and the stuffed 0x00
//     bytes; per segment, the blocks' output offsets; per block, the kept bytes
//     compacted into a 16-byte aligned, zero-padded bit stream;
//  2. candidates: the stream is cut into chunks of kChunkBits bits.  A thread
//     per chunk decodes from kOverlapBits before its chunk and records where
//     that path first reaches a sample boundary inside the chunk (its start
//     state: bit position and component phase), where it leaves the chunk and
//     how many samples lie between; with different tables per component, also
//     the path from that start one phase on.  Huffman codes resynchronise, so
//     one of these is almost always the true path.  The lead is long because
//     high-entropy data resynchronise slowly: with an optimal table for 10-bit
//     noise the codes are 1-3 bits ahead of 9-10 raw bits, and a path one
//     component off under different tables soon parts again.  Within a CTA, in
//     two rounds, each chunk also takes a path from every exit of the chunk
//     before that starts none of its own, so only runs of failures miss;
//  3. walks: a warp per group of 32 chunks chains the chunks from its first
//     chunk's lead path and next-phase path (lane j takes the path whose start
//     is lane j-1's exit; a chunk with no matching path is decoded again from
//     the exact state), then a warp per segment chains the groups from the
//     stream's start (walking a group's chunks itself where neither entry was
//     the true one), giving every group its exact entry state and first
//     sample;
//  4. write: a warp per group chains its chunks once more from the exact entry,
//     scans the counts, and every lane decodes its chunk from its exact start,
//     storing each sample's difference (EXTEND, SSSS = 16 -> 32768); an invalid
//     code (longer than 16 bits) before the frame's last sample fails the
//     segment; a stream that ends early reads zeros past its data, as a
//     sequential decoder does;
//  5. reconstruct: predictor 1 (the DNG case) is two prefix sums modulo 2^16 --
//     down the first column from 2^(P-Pt-1), then along each JPEG line -- a
//     warp per line; predictors 2-7 walk each segment in one thread.  Samples
//     fill the seg_w x seg_h raster row after row from the JPEG lines of X * Nf
//     samples, shifted left by Pt and cropped at the image.
// Segments with restart intervals (and very large segments) take a sequential
// decoder, one thread per segment, with the same semantics: the data of each
// interval ends at a marker, zeros follow, and the next restart marker must
// stand where the interval's data ends.  Every loop is bounded by the frame's
// sample count or its segment's bit length, and every read by the segment's
// end.
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "../../include/cpipe_b200_dng.h"
#include "filters_impl.h"

namespace cpb {
namespace {

constexpr int kLutBits = 12;
constexpr int kLut = 1 << kLutBits;
constexpr uint32_t kChunkBits = 1024;   // bits of stream per chunk
constexpr uint32_t kOverlapBits = 1536;  // bits decoded ahead of a chunk to synchronise
constexpr int kChunksPerCta = 256;      // one chunk per thread; 8 groups of 32
constexpr int kCands = 4;  // paths kept per chunk: lead, next phase, two from the exits of the chunk before
constexpr int kGroupEntries = 2;  // group walks from a chunk group's lead path and its next-phase path
constexpr int kStageWords = 8576;       // >= skewed words a CTA stages: (256 x 1024 + 1536 + 192) / 32 + 2 + skew
constexpr int kScanBytes = 4096;        // unstuff block: 256 threads x 16 bytes
constexpr uint64_t kMaxParallelBytes = 1ull << 27;
constexpr uint64_t kMaxParallelSamples = 1ull << 27;

struct LjTab {
    uint16_t lut[kLut];   // symbol | code length << 5 | (code + extra bits) << 9 for codes of at most
                          // kLutBits bits; 0 for longer ones
    int32_t maxcode[18];  // [l]: largest code of length l (1..16), -1 when none
    int32_t valoff[17];   // [l]: index of the first symbol of length l minus the first code of length l
    uint8_t vals[20];
};

struct SegDev {
    uint64_t off;    // entropy-coded (stuffed) bytes in the upload block
    uint64_t len;
    uint64_t uoff;   // unstuffed stream (16-byte aligned) in the parallel path's buffer
    uint64_t sbase;  // first sample in the difference buffer
    uint64_t rowbuf; // u16 index of the sequential decoders' two line buffers
    uint32_t X, Y, nf, p, ps, pt, ri;
    uint32_t tids;   // table of component c in bits 8c..8c+7
    uint32_t shared; // every component uses one table
    uint32_t x0, y0;
    uint32_t nchunk; // chunks reserved: ceil(8 len / kChunkBits), at least 1
    uint32_t chunk0, group0, blk0, line0;
};

// A decode path through one chunk: start state (first sample boundary at or
// after the chunk's first bit), exit state (first one at or after its end),
// samples in between.  meta: start phase | exit phase << 2 | valid << 4.
struct LjCand {
    uint32_t s, e, n, meta;
};
// A path through a group of chunks from one of its first chunk's paths
// (entry state, exit state, samples).
struct LjGroup {
    uint32_t s, e, n, meta;
};
// Device counters of one decode (diagnostics): chunks decoded again by the
// group, segment and write walks, groups whose entry the segment walk did not
// find, bits decoded again, the longest such decode.
enum { kStatGroup, kStatGroupMiss, kStatSeg, kStatWrite, kStatBits, kStatLongest, kStats };

struct CtaDesc {
    uint32_t seg, c0;  // segment, first chunk (or line) of the CTA within it
};

__device__ __forceinline__ uint32_t lj_tid(uint32_t tids, uint32_t ph) { return (tids >> (8 * ph)) & 0xFF; }

// Most-significant-bit-first reader of an unstuffed stream of 32-bit words
// [0, hi); words past it read as zero.  STAGED: words lo .. hi-1 held in
// shared memory, already in big-endian order, word lo + r at r + r / 32 (one
// skew word per 32 so that lanes reading chunks 32 words apart hit different
// banks); otherwise the global stream.  After refill() the buffer holds at
// least 33 bits, enough for one code and its extra bits.
template <bool STAGED>
struct LjBits {
    const uint32_t* w;
    uint32_t lo, hi, next;
    int nb;
    uint64_t buf;
    uint4 q;         // global reader: the 16-byte line holding words qb .. qb+3 (the stream is 16-byte aligned
    uint32_t qb;     // and zero-padded to a whole line past its end)
    __device__ __forceinline__ uint32_t word(uint32_t i) {
        if (i >= hi) return 0u;
        if (STAGED) {
            const uint32_t r = i - lo;
            return w[r + (r >> 5)];
        }
        if ((i & ~3u) != qb) {
            qb = i & ~3u;
            q = __ldg(reinterpret_cast<const uint4*>(w + qb));
        }
        const uint32_t v = (i & 2u) ? ((i & 1u) ? q.w : q.z) : ((i & 1u) ? q.y : q.x);
        return __byte_perm(v, 0, 0x0123);
    }
    __device__ __forceinline__ void refill() {
        buf |= (uint64_t)word(next) << (32 - nb);
        nb += 32;
        ++next;
    }
    __device__ __forceinline__ void init(const uint32_t* words, uint32_t first, uint32_t end, uint32_t pos) {
        w = words;
        lo = first;
        hi = end;
        qb = 0xFFFFFFFFu;
        next = pos >> 5;
        buf = 0;
        nb = 0;
        refill();
        refill();
        buf <<= (pos & 31);
        nb -= (int)(pos & 31);
    }
    __device__ __forceinline__ uint32_t pos() const { return next * 32u - (uint32_t)nb; }
};

// One sample's difference, with the lookahead table `lut` and, for codes
// longer than kLutBits, the canonical arrays of `tab`.  False on an invalid
// code, after which the reader has consumed one bit (a deterministic step, so
// paths from a wrong start still move on; on the true path it fails the
// segment).
template <class Bits>
__device__ __forceinline__ bool lj_sym(Bits& br, const uint16_t* lut, const LjTab* tab, int& diff) {
    if (br.nb <= 32) br.refill();
    const uint32_t f = lut[(uint32_t)(br.buf >> (64 - kLutBits))];
    int len, sym;
    if (f) {
        len = (int)((f >> 5) & 15u);
        sym = (int)(f & 31u);
    } else {
        len = kLutBits + 1;
        int code = (int)(br.buf >> (64 - len));
        while (len <= 16 && code > tab->maxcode[len]) {
            ++len;
            code = (int)(br.buf >> (64 - len));
        }
        if (len > 16) {
            br.buf <<= 1;
            br.nb -= 1;
            return false;
        }
        sym = tab->vals[tab->valoff[len] + code];
    }
    br.buf <<= len;
    br.nb -= len;
    if (sym == 0) {
        diff = 0;
    } else if (sym == 16) {
        diff = 32768;
    } else {
        const int v = (int)(br.buf >> (64 - sym));
        br.buf <<= sym;
        br.nb -= sym;
        diff = v < (1 << (sym - 1)) ? v - (1 << sym) + 1 : v;
    }
    return true;
}

// The segment's decoding context on the device.
struct LjCtx {
    const uint32_t* words;  // global stream
    uint32_t nw;            // its words
    const uint32_t* sw;     // staged words lo .. hi-1 (kernels that stage)
    uint32_t lo, hi;
    uint32_t bits;          // stream length in bits (8 x unstuffed bytes)
    uint32_t last;          // last live chunk: the one holding the stream's final bit (0 for an empty stream)
    const uint16_t* lut;    // kLut entries per component phase (shared memory)
    const LjTab* tabs;
    uint32_t tids, nf;
    bool shared;
    __device__ __forceinline__ uint32_t step(uint32_t ph) const { return shared ? 0u : (ph + 1 == nf ? 0u : ph + 1); }
    __device__ __forceinline__ uint32_t cs(uint32_t c) const { return c * kChunkBits; }
    __device__ __forceinline__ uint32_t ce(uint32_t c) const { return c >= last ? bits : (c + 1) * kChunkBits; }
    template <bool STAGED>
    __device__ __forceinline__ void open(LjBits<STAGED>& br, uint32_t pos) const {
        if (STAGED) br.init(sw, lo, hi, pos);
        else br.init(words, 0, nw, pos);
    }
};

template <class Bits>
__device__ __forceinline__ bool lj_next(const LjCtx& x, Bits& br, uint32_t ph, int& diff) {
    const uint32_t tp = x.shared ? 0u : ph;
    return lj_sym(br, x.lut + tp * kLut, x.tabs + lj_tid(x.tids, tp), diff);
}

// Skips one sample's code and extra bits (counting paths need no values).
// False on an invalid code, after which one bit is consumed, as in lj_sym.
template <class Bits>
__device__ __forceinline__ bool lj_skip(Bits& br, const uint16_t* lut, const LjTab* tab) {
    if (br.nb <= 32) br.refill();
    const uint32_t f = lut[(uint32_t)(br.buf >> (64 - kLutBits))];
    int total;
    if (f) {
        total = (int)(f >> 9);
    } else {
        int len = kLutBits + 1;
        int code = (int)(br.buf >> (64 - len));
        while (len <= 16 && code > tab->maxcode[len]) {
            ++len;
            code = (int)(br.buf >> (64 - len));
        }
        if (len > 16) {
            br.buf <<= 1;
            br.nb -= 1;
            return false;
        }
        const int sym = tab->vals[tab->valoff[len] + code];
        total = len + (sym < 16 ? sym : 0);
    }
    br.buf <<= total;
    br.nb -= total;
    return true;
}

// From (pos, ph): to the first sample boundary at or after cs (the start
// state), then to the first at or after ce (the exit), counting samples.
// SHARED: one table, the phase stays 0.
template <bool STAGED, bool SHARED>
__device__ __forceinline__ LjCand lj_path_t(const LjCtx& x, uint32_t pos, uint32_t ph, uint32_t cs, uint32_t ce) {
    LjBits<STAGED> br;
    x.open(br, pos);
    const LjTab* tab0 = x.tabs + lj_tid(x.tids, 0);
    while (br.pos() < cs) {
        if (SHARED) {
            lj_skip(br, x.lut, tab0);
        } else if (lj_skip(br, x.lut + ph * kLut, x.tabs + lj_tid(x.tids, ph))) {
            ph = ph + 1 == x.nf ? 0u : ph + 1;
        }
    }
    LjCand c;
    c.s = br.pos();
    const uint32_t sp = ph;
    uint32_t n = 0;
    while (br.pos() < ce) {
        if (SHARED) {
            n += lj_skip(br, x.lut, tab0);
        } else if (lj_skip(br, x.lut + ph * kLut, x.tabs + lj_tid(x.tids, ph))) {
            ph = ph + 1 == x.nf ? 0u : ph + 1;
            ++n;
        }
    }
    c.e = br.pos();
    c.n = n;
    c.meta = sp | (ph << 2) | 16u;
    return c;
}

template <bool STAGED>
__device__ __forceinline__ LjCand lj_path(const LjCtx& x, uint32_t pos, uint32_t ph, uint32_t cs, uint32_t ce) {
    return x.shared ? lj_path_t<STAGED, true>(x, pos, 0, cs, ce) : lj_path_t<STAGED, false>(x, pos, ph, cs, ce);
}

// The lookahead tables of the segment's phases into shared memory, 16 bytes a
// load with eight loads in flight per thread.
__device__ __forceinline__ void stage_luts(uint16_t* lut, const LjTab* tabs, const SegDev& s) {
    constexpr uint32_t kVec = kLut / 8;  // uint4 per table
    const uint32_t phases = s.shared ? 1u : s.nf;
    uint4* dst = reinterpret_cast<uint4*>(lut);
    for (uint32_t i0 = threadIdx.x; i0 < phases * kVec; i0 += 8 * blockDim.x) {
        uint4 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            if (i < phases * kVec)
                v[k] = __ldg(reinterpret_cast<const uint4*>(tabs[lj_tid(s.tids, i / kVec)].lut) + i % kVec);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            if (i < phases * kVec) dst[i] = v[k];
        }
    }
}

__device__ __forceinline__ LjCtx make_ctx(const SegDev& s, const uint8_t* ubuf, uint32_t ulen, const uint16_t* lut,
                                          const LjTab* tabs) {
    LjCtx x;
    x.words = reinterpret_cast<const uint32_t*>(ubuf + s.uoff);
    x.nw = (ulen + 3) / 4;
    x.sw = nullptr;
    x.lo = 0;
    x.hi = 0;
    x.bits = ulen * 8;
    x.last = x.bits ? (x.bits - 1) / kChunkBits : 0;
    if (x.last >= s.nchunk) x.last = s.nchunk - 1;  // cannot happen: the unstuffed stream is not longer
    x.lut = lut;
    x.tabs = tabs;
    x.tids = s.tids;
    x.nf = s.nf;
    x.shared = s.shared != 0;
    return x;
}

// Words a CTA over chunks c0 .. c0 + kChunksPerCta - 1 reads: from its first
// chunk's lead to past its last live chunk's exit and the reader's lookahead.
__device__ __forceinline__ void stage_range(const LjCtx& x, uint32_t c0, uint32_t* lo, uint32_t* hi) {
    const uint32_t cs0 = x.cs(c0), lead = kOverlapBits;
    *lo = (cs0 > lead ? cs0 - lead : 0) >> 5;
    const uint32_t cl = min(c0 + kChunksPerCta - 1, x.last);
    *hi = min(x.nw, (x.ce(cl) + 192) / 32 + 1);
    if (*hi < *lo) *hi = *lo;
}

// Byte-swapped, skewed copy of words lo .. hi-1 into shared memory.
__device__ __forceinline__ void stage_words(uint32_t* sw, const LjCtx& x, uint32_t lo, uint32_t hi) {
    for (uint32_t r = threadIdx.x; r < hi - lo; r += blockDim.x)
        sw[r + (r >> 5)] = __byte_perm(__ldg(x.words + lo + r), 0, 0x0123);
}

// ---------------------------------------------------------------- unstuffing
struct ScanBlk {
    uint32_t seg, start;  // segment, first stuffed byte of the block within it
};

// Per block: the first marker (0xFF followed by a non-zero byte, or 0xFF as
// the segment's last byte) into seg_end[seg] (atomic min, preset to the
// segment's length), and the number of stuffed 0x00 bytes into blk_stuff.
__global__ void __launch_bounds__(256) lj_mark_kernel(const uint8_t* __restrict__ block, const SegDev* __restrict__ segs,
                                                      const ScanBlk* __restrict__ blks, uint32_t* __restrict__ seg_end,
                                                      uint32_t* __restrict__ blk_stuff) {
    __shared__ uint8_t sb[kScanBytes + 2];
    __shared__ uint32_t red_min[8], red_cnt[8];
    const ScanBlk b = blks[blockIdx.x];
    const SegDev& s = segs[b.seg];
    const uint8_t* src = block + s.off;
    const uint32_t len = (uint32_t)s.len;
    const uint32_t n = min((uint32_t)kScanBytes, len - b.start);
    // sb[k] = byte start + k - 1, k = 0 .. n + 1 (zero outside the segment)
    for (uint32_t k = threadIdx.x; k < n + 2; k += blockDim.x) {
        const int64_t at = (int64_t)b.start + k - 1;
        sb[k] = (at >= 0 && at < (int64_t)len) ? src[at] : 0;
    }
    __syncthreads();
    uint32_t first = 0xFFFFFFFFu, cnt = 0;
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const uint32_t pos = b.start + k;
        const uint32_t v = sb[k + 1], prev = sb[k];
        const uint32_t nx = pos + 1 < len ? sb[k + 2] : 0xD9u;
        if (v == 0xFF && nx != 0) first = min(first, pos);
        if (v == 0 && prev == 0xFF && pos > 0) ++cnt;
    }
    for (int o = 16; o; o >>= 1) {
        first = min(first, __shfl_xor_sync(0xFFFFFFFFu, first, o));
        cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red_min[threadIdx.x >> 5] = first;
        red_cnt[threadIdx.x >> 5] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
            first = min(first, red_min[i]);
            cnt += red_cnt[i];
        }
        if (first != 0xFFFFFFFFu) atomicMin(&seg_end[b.seg], first);
        blk_stuff[blockIdx.x] = cnt;
    }
}

// Per segment: each block's first output byte (kept bytes of the blocks
// before it; exact for every block that starts before the first marker).
__global__ void lj_offsets_kernel(const SegDev* __restrict__ segs, const uint32_t* __restrict__ par, int npar,
                                  const uint32_t* __restrict__ blk_stuff, uint32_t* __restrict__ blk_off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npar) return;
    const SegDev s = segs[par[i]];
    const uint32_t nblk = (uint32_t)((s.len + kScanBytes - 1) / kScanBytes);
    uint32_t acc = 0;
    for (uint32_t k = 0; k < nblk; ++k) {
        blk_off[s.blk0 + k] = acc;
        const uint32_t n = min((uint64_t)kScanBytes, s.len - (uint64_t)k * kScanBytes);
        acc += n - blk_stuff[s.blk0 + k];
    }
}

// Per block: bytes before the segment's first marker that are not stuffed
// 0x00s, compacted to ubuf + uoff + blk_off; ulen[seg] = the kept length.
__global__ void __launch_bounds__(256) lj_pack_kernel(const uint8_t* __restrict__ block, const SegDev* __restrict__ segs,
                                                      const ScanBlk* __restrict__ blks,
                                                      const uint32_t* __restrict__ seg_end,
                                                      const uint32_t* __restrict__ blk_off, uint8_t* __restrict__ ubuf,
                                                      uint32_t* __restrict__ ulen) {
    __shared__ uint8_t sb[kScanBytes + 1];
    __shared__ uint8_t so[kScanBytes];
    __shared__ uint32_t warp_sum[8];
    const ScanBlk b = blks[blockIdx.x];
    const SegDev& s = segs[b.seg];
    const uint32_t end = seg_end[b.seg];
    if (b.start >= end) return;
    const uint8_t* src = block + s.off;
    const uint32_t n = min((uint32_t)kScanBytes, end - b.start);
    for (uint32_t k = threadIdx.x; k < n + 1; k += blockDim.x) {
        const int64_t at = (int64_t)b.start + k - 1;
        sb[k] = at >= 0 ? src[at] : 0;
    }
    __syncthreads();
    // thread t: bytes 16t .. 16t+15 of the block
    const uint32_t k0 = threadIdx.x * 16;
    uint32_t keep = 0, cnt = 0;
    for (uint32_t k = 0; k < 16; ++k) {
        const uint32_t kk = k0 + k;
        const bool kept = kk < n && !(sb[kk + 1] == 0 && sb[kk] == 0xFF && b.start + kk > 0);
        keep |= (uint32_t)kept << k;
        cnt += kept;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        if (w < warp) before += warp_sum[w];
        total += warp_sum[w];
    }
    uint32_t at = before + inc - cnt;
    for (uint32_t k = 0; k < 16; ++k)
        if (keep >> k & 1) so[at++] = sb[k0 + k + 1];
    __syncthreads();
    uint8_t* dst = ubuf + s.uoff + blk_off[blockIdx.x];
    for (uint32_t k = threadIdx.x; k < total; k += blockDim.x) dst[k] = so[k];
    if (threadIdx.x == 0) atomicMax(&ulen[b.seg], blk_off[blockIdx.x] + total);
}

// ------------------------------------------------------ candidates and walks
// Shared memory of the staging kernels: the lookahead tables of the
// segment's phases, then its staged words.
__device__ __forceinline__ LjCtx open_cta(const SegDev& s, const uint8_t* ubuf, uint32_t ulen, const LjTab* tabs,
                                          uint32_t c0, uint32_t* smem) {
    uint16_t* lut = reinterpret_cast<uint16_t*>(smem);
    uint32_t* sw = smem + (s.shared ? 1u : s.nf) * (kLut / 2);  // after the phases' tables
    stage_luts(lut, tabs, s);
    LjCtx x = make_ctx(s, ubuf, ulen, lut, tabs);
    stage_range(x, c0, &x.lo, &x.hi);
    stage_words(sw, x, x.lo, x.hi);
    x.sw = sw;
    __syncthreads();
    return x;
}

extern __shared__ uint4 lj_dyn_smem[];

__global__ void __launch_bounds__(kChunksPerCta) lj_cand_kernel(const SegDev* __restrict__ segs,
                                                                const CtaDesc* __restrict__ ctas,
                                                                const LjTab* __restrict__ tabs,
                                                                const uint8_t* __restrict__ ubuf,
                                                                const uint32_t* __restrict__ ulen,
                                                                LjCand* __restrict__ cand) {
    const CtaDesc d = ctas[blockIdx.x];
    const SegDev s = segs[d.seg];
    uint32_t* smem = reinterpret_cast<uint32_t*>(lj_dyn_smem);
    const LjCtx x = open_cta(s, ubuf, ulen[d.seg], tabs, d.c0, smem);
    // this CTA's first paths, after the tables and the staged words
    LjCand* first = reinterpret_cast<LjCand*>(smem + (s.shared ? 1u : s.nf) * (kLut / 2) + kStageWords);
    const uint32_t c = d.c0 + threadIdx.x;
    const bool live = c < s.nchunk && c <= x.last;
    const LjCand none = {0, 0, 0, 0};
    const uint32_t cs = x.cs(c), ce = live ? x.ce(c) : cs;
    LjCand p0 = none, p1 = none;
    if (live) {
        // the stream's start is exact; elsewhere a lead of kOverlapBits
        p0 = lj_path<true>(x, c == 0 ? 0 : (cs > kOverlapBits ? cs - kOverlapBits : 0), 0, cs, ce);
        // Different tables per component: the same start one phase on.  Where
        // the tables give the codes in play the same lengths (a flat stretch, a
        // padded tile edge) a path can sit on the true boundaries one
        // component off for any length.
        if (c > 0 && !x.shared) p1 = lj_path<true>(x, p0.s, ((p0.meta & 3u) + 1) % x.nf, cs, ce);
    }
    first[2 * threadIdx.x] = p0;
    first[2 * threadIdx.x + 1] = p1;
    __syncthreads();
    // Where a path of the chunk before leaves at a state that starts none of
    // this chunk's paths, one more path from that exact state: the walks then
    // miss only where neighbouring chunks both failed to synchronise.
    LjCand f0 = none, f1 = none;
    if (live && c > 0 && threadIdx.x > 0)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const LjCand q = first[2 * (threadIdx.x - 1) + j];
            const uint32_t ep = (q.meta >> 2) & 3u;
            auto starts = [&](const LjCand& r) { return (r.meta & 16u) && r.s == q.e && (r.meta & 3u) == ep; };
            if ((q.meta & 16u) && !starts(p0) && !starts(p1) && !starts(f0)) {
                const LjCand r = lj_path<true>(x, q.e, ep, cs, ce);
                if (f0.meta & 16u) f1 = r;
                else f0 = r;
            }
        }
    // A second round over the paths the first one added, for runs of two
    // chunks that did not synchronise.
    __syncthreads();
    first[2 * threadIdx.x] = f0;
    first[2 * threadIdx.x + 1] = f1;
    __syncthreads();
    if (live && c > 0 && threadIdx.x > 0 && !(f1.meta & 16u))
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const LjCand q = first[2 * (threadIdx.x - 1) + j];
            const uint32_t ep = (q.meta >> 2) & 3u;
            auto starts = [&](const LjCand& r) { return (r.meta & 16u) && r.s == q.e && (r.meta & 3u) == ep; };
            if ((q.meta & 16u) && !(f1.meta & 16u) && !starts(p0) && !starts(p1) && !starts(f0)) {
                const LjCand r = lj_path<true>(x, q.e, ep, cs, ce);
                if (f0.meta & 16u) f1 = r;
                else f0 = r;
            }
        }
    if (c >= s.nchunk) return;
    LjCand* out = cand + (size_t)(s.chunk0 + c) * kCands;
    out[0] = p0;
    out[1] = p1;
    out[2] = f0;
    out[3] = f1;
}

// Chains chunks gc0 .. gc0 + glive - 1 (lane j holds chunk gc0 + j's
// candidates in c) from state (pos, ph), warp-collectively: lane j takes the
// candidate that starts at lane j-1's exit, or decodes its chunk again from
// that exact state (or, with give_up, the walk returns false there).  On
// return (pos, ph) is the group's exit, `total` has grown by its samples, and
// lane j holds its chunk's exact start and count.
template <bool STAGED>
__device__ bool lj_walk(const LjCtx& x, const LjCand (&c)[kCands], uint32_t gc0, uint32_t glive, uint32_t& pos,
                        uint32_t& ph, uint32_t& my_pos, uint32_t& my_ph, uint32_t& my_n, uint32_t& total,
                        unsigned long long* stats, int which, bool give_up = false) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t j = 0; j < glive; ++j) {
        uint32_t e = 0, ep = 0, n = 0;
        bool hit = false;
        if (lane == j) {
#pragma unroll
            for (int k = 0; k < kCands; ++k)
                if (!hit && (c[k].meta & 16u) && c[k].s == pos && (c[k].meta & 3u) == ph) {
                    hit = true;
                    e = c[k].e;
                    ep = (c[k].meta >> 2) & 3u;
                    n = c[k].n;
                }
            if (!hit && !give_up) {
                const uint32_t cc = gc0 + j;
                const LjCand r = lj_path<STAGED>(x, pos, ph, x.cs(cc), x.ce(cc));
                e = r.e;
                ep = (r.meta >> 2) & 3u;
                n = r.n;
                atomicAdd(stats + which, 1ull);
                atomicAdd(stats + kStatBits, (unsigned long long)(r.e - pos));
                atomicMax(stats + kStatLongest, (unsigned long long)(r.e - pos));
            }
            my_pos = pos;
            my_ph = ph;
            my_n = n;
        }
        if (give_up && !__shfl_sync(0xFFFFFFFFu, hit, j)) return false;
        pos = __shfl_sync(0xFFFFFFFFu, e, j);
        ph = __shfl_sync(0xFFFFFFFFu, ep, j);
        total += __shfl_sync(0xFFFFFFFFu, n, j);
    }
    return true;
}

__device__ __forceinline__ void load_cands(const LjCand* __restrict__ cand, const SegDev& s, uint32_t gc0,
                                           uint32_t glive, LjCand (&c)[kCands]) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kCands; ++k) c[k] = LjCand{0, 0, 0, 0};
    if (lane < glive) {
        const LjCand* p = cand + (size_t)(s.chunk0 + gc0 + lane) * kCands;
#pragma unroll
        for (int k = 0; k < kCands; ++k) c[k] = p[k];
    }
}

// A warp per group of 32 chunks: the group's paths from the lead path of its
// first chunk and from that path's next-phase start.  When the true entry is
// neither (a chunk that did not synchronise) the segment walk chains that
// group's chunks itself.
__global__ void __launch_bounds__(kChunksPerCta) lj_group_kernel(const SegDev* __restrict__ segs,
                                                                 const CtaDesc* __restrict__ ctas,
                                                                 const LjTab* __restrict__ tabs,
                                                                 const uint8_t* __restrict__ ubuf,
                                                                 const uint32_t* __restrict__ ulen,
                                                                 const LjCand* __restrict__ cand,
                                                                 LjGroup* __restrict__ groups,
                                                                 unsigned long long* stats) {
    __shared__ __align__(16) uint16_t lut[4 * kLut];
    const CtaDesc d = ctas[blockIdx.x];
    const SegDev s = segs[d.seg];
    stage_luts(lut, tabs, s);
    __syncthreads();
    const LjCtx x = make_ctx(s, ubuf, ulen[d.seg], lut, tabs);
    const uint32_t gc0 = d.c0 + (threadIdx.x >> 5) * 32;
    if (gc0 >= s.nchunk) return;  // warp-uniform
    LjGroup* out = groups + (size_t)(s.group0 + gc0 / 32) * kGroupEntries;
    const uint32_t lane = threadIdx.x & 31;
    if (gc0 > x.last) {
        if (lane < kGroupEntries) out[lane] = LjGroup{0, 0, 0, 0};
        return;
    }
    const uint32_t glive = min(32u, x.last + 1 - gc0);
    LjCand c[kCands];
    load_cands(cand, s, gc0, glive, c);
#pragma unroll
#pragma unroll
    for (int k = 0; k < kGroupEntries; ++k) {
        const uint32_t meta = __shfl_sync(0xFFFFFFFFu, c[k].meta, 0);
        LjGroup g = {0, 0, 0, 0};
        if (meta & 16u) {
            uint32_t pos = __shfl_sync(0xFFFFFFFFu, c[k].s, 0), ph = meta & 3u;
            const uint32_t s0 = pos, p0 = ph;
            uint32_t mp = 0, mph = 0, mn = 0, total = 0;
            // the lead path's walk decodes missing chunks again; the other
            // phase's walk gives up at its first miss
            if (lj_walk<false>(x, c, gc0, glive, pos, ph, mp, mph, mn, total, stats, kStatGroup, k > 0))
                g = LjGroup{s0, pos, total, p0 | (ph << 2) | 16u};
        }
        if (lane == 0) out[k] = g;
    }
}

// A warp per segment: chains the groups from the stream's start; gentry[g] =
// (entry bit position, entry phase, first sample).
__global__ void __launch_bounds__(32) lj_seg_kernel(const SegDev* __restrict__ segs, const uint32_t* __restrict__ par,
                                                    const LjTab* __restrict__ tabs, const uint8_t* __restrict__ ubuf,
                                                    const uint32_t* __restrict__ ulen, const LjCand* __restrict__ cand,
                                                    const LjGroup* __restrict__ groups, uint4* __restrict__ gentry,
                                                    unsigned long long* stats) {
    __shared__ __align__(16) uint16_t lut[4 * kLut];
    const uint32_t seg = par[blockIdx.x];
    const SegDev s = segs[seg];
    stage_luts(lut, tabs, s);
    __syncthreads();
    const LjCtx x = make_ctx(s, ubuf, ulen[seg], lut, tabs);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t ngl = x.last / 32 + 1;
    uint32_t pos = 0, ph = 0, off = 0;
    for (uint32_t gb = 0; gb < ngl; gb += 32) {
        LjGroup e[kGroupEntries];
#pragma unroll
        for (int k = 0; k < kGroupEntries; ++k)
            e[k] = gb + lane < ngl ? groups[(size_t)(s.group0 + gb + lane) * kGroupEntries + k] : LjGroup{0, 0, 0, 0};
        const uint32_t nb = min(32u, ngl - gb);
        for (uint32_t j = 0; j < nb; ++j) {
            uint32_t hit = 0, ex = 0, exp = 0, n = 0;
            if (lane == j)
#pragma unroll
                for (int k = 0; k < kGroupEntries; ++k)
                    if (!hit && (e[k].meta & 16u) && e[k].s == pos && (e[k].meta & 3u) == ph) {
                        hit = 1;
                        ex = e[k].e;
                        exp = (e[k].meta >> 2) & 3u;
                        n = e[k].n;
                    }
            if (lane == 0) gentry[s.group0 + gb + j] = make_uint4(pos, ph, off, 0);
            if (__shfl_sync(0xFFFFFFFFu, hit, j)) {
                pos = __shfl_sync(0xFFFFFFFFu, ex, j);
                ph = __shfl_sync(0xFFFFFFFFu, exp, j);
                off += __shfl_sync(0xFFFFFFFFu, n, j);
            } else {
                const uint32_t gc0 = (gb + j) * 32, glive = min(32u, x.last + 1 - gc0);
                LjCand c[kCands];
                load_cands(cand, s, gc0, glive, c);
                uint32_t mp = 0, mph = 0, mn = 0;
                if (lane == 0) atomicAdd(stats + kStatGroupMiss, 1ull);
                lj_walk<false>(x, c, gc0, glive, pos, ph, mp, mph, mn, off, stats, kStatSeg);
            }
        }
    }
}

// A warp per group: each lane decodes its chunk from its exact start and
// stores the samples' differences (mod 2^16) in segment order.
__global__ void __launch_bounds__(kChunksPerCta) lj_write_kernel(const SegDev* __restrict__ segs,
                                                                 const CtaDesc* __restrict__ ctas,
                                                                 const LjTab* __restrict__ tabs,
                                                                 const uint8_t* __restrict__ ubuf,
                                                                 const uint32_t* __restrict__ ulen,
                                                                 const LjCand* __restrict__ cand,
                                                                 const uint4* __restrict__ gentry,
                                                                 uint16_t* __restrict__ dbuf, int* __restrict__ status,
                                                                 unsigned long long* stats) {
    const CtaDesc d = ctas[blockIdx.x];
    const SegDev s = segs[d.seg];
    const LjCtx x = open_cta(s, ubuf, ulen[d.seg], tabs, d.c0, reinterpret_cast<uint32_t*>(lj_dyn_smem));
    const uint32_t gc0 = d.c0 + (threadIdx.x >> 5) * 32;
    if (gc0 >= s.nchunk || gc0 > x.last) return;  // warp-uniform
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t glive = min(32u, x.last + 1 - gc0);
    const uint4 ge = gentry[s.group0 + gc0 / 32];
    LjCand c[kCands];
    load_cands(cand, s, gc0, glive, c);
    uint32_t pos = ge.x, ph = ge.y, total = 0, my_pos = 0, my_ph = 0, my_n = 0;
    lj_walk<true>(x, c, gc0, glive, pos, ph, my_pos, my_ph, my_n, total, stats, kStatWrite);
    uint32_t inc = lane < glive ? my_n : 0;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= (uint32_t)o) inc += v;
    }
    if (lane >= glive) return;
    const uint32_t samples = s.X * s.Y * s.nf;
    const uint32_t t0 = ge.z + inc - my_n;
    // the stream's last chunk goes on (through zeros past a short stream) to the frame's last sample
    const uint32_t lim = gc0 + lane == x.last ? samples : min(t0 + my_n, samples);
    if (t0 >= lim) return;
    LjBits<true> br;
    x.open(br, my_pos);
    uint16_t* o = dbuf + s.sbase;  // 8-byte aligned: segments start on a multiple of 4 samples
    uint32_t p = my_ph, t = t0;
    int diff;
    // single samples up to a multiple of 4, then 4 per 8-byte store, then the rest
    for (; t < lim && (t & 3u); ++t, p = x.step(p)) {
        if (!lj_next(x, br, p, diff)) {
            status[d.seg] = 1;
            return;
        }
        o[t] = (uint16_t)diff;
    }
    for (; t + 4 <= lim; t += 4) {
        uint64_t four = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k, p = x.step(p)) {
            if (!lj_next(x, br, p, diff)) {
                status[d.seg] = 1;
                return;
            }
            four |= (uint64_t)(uint16_t)diff << (16 * k);
        }
        *reinterpret_cast<uint64_t*>(o + t) = four;
    }
    for (; t < lim; ++t, p = x.step(p)) {
        if (!lj_next(x, br, p, diff)) {
            status[d.seg] = 1;
            return;
        }
        o[t] = (uint16_t)diff;
    }
}

// ------------------------------------------------------------ reconstruction
__device__ __forceinline__ void lj_put(const SegDev& s, uint32_t tr, uint32_t tc, uint32_t v, uint16_t* __restrict__ out,
                                       int width, int height, int seg_h) {
    if (tr >= (uint32_t)seg_h) return;
    const uint32_t gx = s.x0 + tc, gy = s.y0 + tr;
    if (gx < (uint32_t)width && gy < (uint32_t)height) out[(size_t)gy * width + gx] = (uint16_t)(v << s.pt);
}

// Sample t of a segment (in decoding order) to its place in the raster.
__device__ __forceinline__ void lj_store(const SegDev& s, uint32_t t, uint32_t v, uint16_t* __restrict__ out, int width,
                                         int height, int seg_w, int seg_h) {
    const uint32_t tr = t / (uint32_t)seg_w;
    lj_put(s, tr, t - tr * (uint32_t)seg_w, v, out, width, height, seg_h);
}

// Predictor 1, first column: C[y][c] = 2^(P-Pt-1) + the first-column
// differences of lines 0..y (mod 2^16).  A warp per segment.
__global__ void __launch_bounds__(32) lj_col_kernel(const SegDev* __restrict__ segs, const uint32_t* __restrict__ par,
                                                    const uint16_t* __restrict__ dbuf, uint16_t* __restrict__ cbuf) {
    const SegDev s = segs[par[blockIdx.x]];
    if (s.ps != 1) return;
    const uint32_t lane = threadIdx.x & 31, W = s.X * s.nf;
    const uint32_t dflt = 1u << (s.p - s.pt - 1);
    uint32_t carry[4] = {dflt, dflt, dflt, dflt};
    for (uint32_t y0 = 0; y0 < s.Y; y0 += 32) {
        const uint32_t y = y0 + lane;
        uint32_t v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = (y < s.Y && (uint32_t)c < s.nf) ? dbuf[s.sbase + (size_t)y * W + c] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, v[c], o);
                if (lane >= (uint32_t)o) v[c] += u;
            }
        if (y < s.Y) {
            ushort4 r;
            r.x = (uint16_t)(carry[0] + v[0]);
            r.y = (uint16_t)(carry[1] + v[1]);
            r.z = (uint16_t)(carry[2] + v[2]);
            r.w = (uint16_t)(carry[3] + v[3]);
            reinterpret_cast<ushort4*>(cbuf)[s.line0 + y] = r;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) carry[c] += __shfl_sync(0xFFFFFFFFu, v[c], 31);
    }
}

// Predictor 1, along each JPEG line: sample (y, x, c) = C[y][c] + the
// differences at x' = 1..x (mod 2^16).  A warp per line, 8 lines per CTA.
__global__ void __launch_bounds__(256) lj_line_kernel(const SegDev* __restrict__ segs, const CtaDesc* __restrict__ lines,
                                                      const uint16_t* __restrict__ dbuf,
                                                      const uint16_t* __restrict__ cbuf, uint16_t* __restrict__ out,
                                                      int width, int height, int seg_w, int seg_h) {
    const CtaDesc d = lines[blockIdx.x];
    const SegDev s = segs[d.seg];
    const uint32_t y = d.c0 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (y >= s.Y) return;
    const uint32_t W = s.X * s.nf, nf = s.nf;
    const bool rows_match = W == (uint32_t)seg_w;  // JPEG line y is raster row y
    const uint16_t* row = dbuf + s.sbase + (size_t)y * W;
    const ushort4 cy = reinterpret_cast<const ushort4*>(cbuf)[s.line0 + y];
    uint32_t carry[4] = {cy.x, cy.y, cy.z, cy.w};
    for (uint32_t xb = 0; xb < s.X; xb += 32) {
        const uint32_t x = xb + lane;
        uint32_t v[4] = {0, 0, 0, 0};
        if (x < s.X && x > 0)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if ((uint32_t)c < nf) v[c] = row[x * nf + c];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if ((uint32_t)c >= nf) break;  // uniform
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, v[c], o);
                if (lane >= (uint32_t)o) v[c] += u;
            }
        }
        if (x < s.X)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if ((uint32_t)c < nf) {
                    const uint32_t val = (carry[c] + v[c]) & 0xFFFFu;
                    if (rows_match) lj_put(s, y, x * nf + c, val, out, width, height, seg_h);
                    else lj_store(s, y * W + x * nf + c, val, out, width, height, seg_w, seg_h);
                }
#pragma unroll
        for (int c = 0; c < 4; ++c) carry[c] += __shfl_sync(0xFFFFFFFFu, v[c], 31);
    }
}

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

// Predictors 2-7 (no restart intervals): one thread walks a segment's
// differences with two line buffers.
__global__ void lj_recon_serial_kernel(const SegDev* __restrict__ segs, const uint32_t* __restrict__ par, int npar,
                                       const uint16_t* __restrict__ dbuf, uint16_t* __restrict__ rowbufs,
                                       uint16_t* __restrict__ out, int width, int height, int seg_w, int seg_h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npar) return;
    const SegDev s = segs[par[i]];
    if (s.ps == 1) return;
    const int W = (int)(s.X * s.nf), nf = (int)s.nf;
    uint16_t* rows = rowbufs + s.rowbuf;
    const uint16_t* dif = dbuf + s.sbase;
    const int dflt = 1 << (s.p - s.pt - 1);
    uint32_t t = 0;
    for (int y = 0; y < (int)s.Y; ++y) {
        uint16_t* cur = rows + (size_t)(y & 1) * W;
        const uint16_t* prev = rows + (size_t)((y & 1) ^ 1) * W;
        for (int x = 0; x < (int)s.X; ++x)
            for (int c = 0; c < nf; ++c, ++t) {
                const int pred = (y == 0 && x == 0) ? dflt : lj_predict(cur, prev, x, c, nf, (int)s.ps, y == 0);
                const uint16_t v = (uint16_t)((pred + dif[t]) & 0xFFFF);
                cur[x * nf + c] = v;
                lj_store(s, t, v, out, width, height, seg_w, seg_h);
            }
    }
}

// ------------------------------------------------------ sequential decoder
// Segments with restart intervals (or too large for the parallel path): one
// thread per segment reads the stuffed bytes directly with a 64-bit buffer
// (0xFF00 unstuffed; a marker ends the data, zeros follow), decodes, predicts
// (H.1.2.1 with the scan's and every interval's first sample reset, Ra on that
// line) and stores.  At each restart the reader must stand at RSTm.
__global__ void __launch_bounds__(32) lj_serial_kernel(const uint8_t* __restrict__ data,
                                                       const SegDev* __restrict__ segs, const uint32_t* __restrict__ ser,
                                                       int nser, const LjTab* __restrict__ tables,
                                                       uint16_t* __restrict__ rowbufs, uint16_t* __restrict__ out,
                                                       int width, int height, int seg_w, int seg_h,
                                                       int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nser) return;
    const uint32_t si = ser[i];
    const SegDev s = segs[si];
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
    int err = 0, first_line_y = 0;
    uint32_t t = 0;
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
            for (int c = 0; c < (int)s.nf && !err; ++c, ++t) {
                refill();
                const LjTab* tb = tables + lj_tid(s.tids, (uint32_t)c);
                const uint32_t f = tb->lut[(uint32_t)(acc >> (64 - kLutBits))];
                int len, sym;
                if (f) {
                    len = (int)((f >> 5) & 15u);
                    sym = (int)(f & 31u);
                } else {
                    len = kLutBits + 1;
                    int code = (int)(acc >> (64 - len));
                    while (len <= 16 && code > tb->maxcode[len]) {
                        ++len;
                        code = (int)(acc >> (64 - len));
                    }
                    if (len > 16) {
                        err = 1;
                        break;
                    }
                    sym = tb->vals[tb->valoff[len] + code];
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
                lj_store(s, t, v, out, width, height, seg_w, seg_h);
            }
            reset = false;
            ++mcu;
        }
    }
    status[si] = err;
}

// ----------------------------------------------------------------- host side
uint32_t be16(const uint8_t* q) { return ((uint32_t)q[0] << 8) | q[1]; }

// Canonical decoding arrays and the lookahead table of one DHT table.
int build_table(const uint8_t* counts, const uint8_t* vals, LjTab* h, std::string* err) {
    std::memset(h, 0, sizeof(*h));
    int code = 0, k = 0;
    for (int l = 1; l <= 16; ++l) {
        const int cnt = counts[l - 1];
        h->maxcode[l] = -1;
        if (cnt) {
            h->valoff[l] = k - code;
            for (int j = 0; j < cnt; ++j, ++code, ++k) {
                if (code >= (1 << l)) {
                    *err = "lossless JPEG Huffman table over-subscribed";
                    return CPIPE_FAILED;
                }
                const uint8_t sym = vals[k];
                if (sym > 16) {
                    *err = "lossless JPEG Huffman symbol above 16";
                    return CPIPE_FAILED;
                }
                h->vals[k] = sym;
                if (l <= kLutBits)
                    for (int e = code << (kLutBits - l); e < (code + 1) << (kLutBits - l); ++e)
                        h->lut[e] = (uint16_t)(sym | (l << 5) | ((l + (sym < 16 ? sym : 0)) << 9));
            }
            h->maxcode[l] = code - 1;
        }
        code <<= 1;
    }
    return CPIPE_OK;
}

// One segment's markers up to its scan: frame, tables (deduplicated across
// segments by content), restart interval.
int parse_segment(const uint8_t* s, size_t n, SegDev* seg, std::vector<LjTab>* tables,
                  std::map<std::string, int>* known, std::string* err) {
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
                const std::string key(reinterpret_cast<const char*>(b + q + 1), 16 + total);
                auto it = known->find(key);
                if (it == known->end()) {
                    LjTab h;
                    const int st = build_table(b + q + 1, b + q + 17, &h, err);
                    if (st != CPIPE_OK) return st;
                    if (tables->size() >= 255) {
                        *err = "more than 255 distinct lossless JPEG Huffman tables";
                        return CPIPE_UNSUPPORTED;
                    }
                    it = known->emplace(key, (int)tables->size()).first;
                    tables->push_back(h);
                }
                local[th] = it->second;
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
            bool same = true;
            for (uint32_t c = 0; c < seg->nf; ++c) {
                const uint32_t cid = b[1 + 2 * c], td = b[2 + 2 * c] >> 4;
                if (cid != ids[c] || td > 3 || local[td] < 0) {
                    *err = "lossless JPEG scan names a missing table or component";
                    return CPIPE_FAILED;
                }
                seg->tids |= (uint32_t)local[td] << (8 * c);
                same = same && local[td] == (int)(seg->tids & 0xFF);
            }
            seg->shared = same ? 1u : 0u;
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

struct LjStats {
    uint64_t figures[9] = {};  // chunks, parallel and sequential segments, then the device counters
};
std::mutex g_lj_mu;
LjStats g_lj_last;

}  // namespace

int lj92_decode(const uint8_t* const* streams, const size_t* bytes, uint32_t count, uint32_t across, uint32_t seg_w,
                uint32_t seg_h, uint32_t width, uint32_t height, uint16_t* d_raw) {
    if (!streams || !bytes || count == 0 || across == 0 || seg_w == 0 || seg_h == 0 || width == 0 || height == 0 ||
        !d_raw) {
        set_error("%s", "lj92 decode: empty or null argument");
        return CPIPE_BAD_INDEX;
    }
    std::vector<SegDev> segs(count);
    std::vector<LjTab> tables;
    std::map<std::string, int> known;
    std::vector<const uint8_t*> data(count);
    uint64_t rows = 0, sum = 0;
    const uint8_t *lo = nullptr, *hi = nullptr;
    for (uint32_t i = 0; i < count; ++i) {
        std::string err;
        if (!streams[i]) {
            set_error("%s", "lj92 decode: null stream");
            return CPIPE_BAD_INDEX;
        }
        const int st = parse_segment(streams[i], bytes[i], &segs[i], &tables, &known, &err);
        if (st != CPIPE_OK) {
            set_error("%s", err.c_str());
            return st;
        }
        SegDev& s = segs[i];
        if ((uint64_t)s.X * s.nf * s.Y > (uint64_t)seg_w * seg_h) {
            set_error("%s", "lossless JPEG frame holds more samples than its segment");
            return CPIPE_FAILED;
        }
        data[i] = streams[i] + s.off;
        lo = (!lo || data[i] < lo) ? data[i] : lo;
        hi = (!hi || data[i] + s.len > hi) ? data[i] + s.len : hi;
        sum += s.len;
        s.x0 = (i % across) * seg_w;
        s.y0 = (i / across) * seg_h;
        s.rowbuf = rows;
        rows += 2ull * s.X * s.nf;
    }
    // The entropy-coded bytes in one device block: the caller's span when the
    // segments lie together (a DNG file), else packed on the host.
    std::vector<uint8_t> packed;
    const uint8_t* src = lo;
    uint64_t src_bytes = (uint64_t)(hi - lo);
    if (src_bytes > sum + sum / 4 + (1u << 20)) {
        packed.reserve(sum);
        for (uint32_t i = 0; i < count; ++i) {
            const uint64_t at = packed.size();
            packed.insert(packed.end(), data[i], data[i] + segs[i].len);
            segs[i].off = at;
        }
        src = packed.data();
        src_bytes = packed.size();
    } else {
        for (uint32_t i = 0; i < count; ++i) segs[i].off = (uint64_t)(data[i] - lo);
    }
    // Plan: parallel segments (no restart intervals, bounded size) and the rest.
    std::vector<uint32_t> par, ser, seg_end;
    std::vector<CtaDesc> ctas, lines;
    std::vector<ScanBlk> blks;
    uint64_t ubytes = 0, samples = 0, chunks = 0, groups = 0, nlines = 0;
    bool any_serial_recon = false;
    uint32_t max_phases = 1;
    for (uint32_t i = 0; i < count; ++i) {
        SegDev& s = segs[i];
        const uint64_t n = (uint64_t)s.X * s.Y * s.nf;
        if (s.ri != 0 || s.len >= kMaxParallelBytes || n >= kMaxParallelSamples) {
            ser.push_back(i);
            continue;
        }
        par.push_back(i);
        max_phases = std::max(max_phases, s.shared ? 1u : s.nf);
        s.uoff = ubytes;
        ubytes += (s.len + 15) / 16 * 16 + 16;
        s.sbase = samples;
        samples += (n + 3) / 4 * 4;
        s.nchunk = (uint32_t)std::max<uint64_t>(1, (8 * s.len + kChunkBits - 1) / kChunkBits);
        s.chunk0 = (uint32_t)chunks;
        chunks += s.nchunk;
        s.group0 = (uint32_t)groups;
        groups += (s.nchunk + 31) / 32;
        s.blk0 = (uint32_t)blks.size();
        for (uint64_t b = 0; b < s.len; b += kScanBytes) blks.push_back(ScanBlk{i, (uint32_t)b});
        s.line0 = (uint32_t)nlines;
        nlines += s.Y;
        for (uint32_t c = 0; c < s.nchunk; c += kChunksPerCta) ctas.push_back(CtaDesc{i, c});
        if (s.ps == 1)
            for (uint32_t y = 0; y < s.Y; y += 8) lines.push_back(CtaDesc{i, y});
        else
            any_serial_recon = true;
    }
    seg_end.resize(count);
    for (uint32_t i = 0; i < count; ++i) seg_end[i] = (uint32_t)std::min<uint64_t>(segs[i].len, 0xFFFFFFFFu);
    if (!device_ready()) return CPIPE_INTERNAL_ERROR;
    Call call;
    void *d_block = nullptr, *d_segs = nullptr, *d_tables = nullptr, *d_rows = nullptr, *d_status = nullptr;
    void *d_stats = nullptr;
    int st = call.alloc(src_bytes + 16, &d_block);
    if (st == CPIPE_OK && src_bytes)
        st = cuda_status(cudaMemcpyAsync(d_block, src, src_bytes, cudaMemcpyHostToDevice, call.stream), "lj92 upload");
    if (st == CPIPE_OK) st = call.upload(segs.data(), segs.size() * sizeof(SegDev), &d_segs);
    if (st == CPIPE_OK) st = call.upload(tables.data(), tables.size() * sizeof(LjTab), &d_tables);
    if (st == CPIPE_OK) st = call.alloc(rows * sizeof(uint16_t), &d_rows);
    if (st == CPIPE_OK) st = call.alloc(count * sizeof(int), &d_status);
    if (st == CPIPE_OK) st = call.alloc(kStats * sizeof(unsigned long long), &d_stats);
    if (st == CPIPE_OK) st = cuda_status(cudaMemsetAsync(d_status, 0, count * sizeof(int), call.stream), "lj92 clear");
    if (st == CPIPE_OK)
        st = cuda_status(cudaMemsetAsync(d_stats, 0, kStats * sizeof(unsigned long long), call.stream), "lj92 clear");
    if (st == CPIPE_OK)
        st = cuda_status(cudaMemsetAsync(d_raw, 0, (size_t)width * height * 2, call.stream), "lj92 clear");
    if (st != CPIPE_OK) return call.finish(st);
    const auto* blk = static_cast<const uint8_t*>(d_block);
    const auto* dsegs = static_cast<const SegDev*>(d_segs);
    const auto* dtabs = static_cast<const LjTab*>(d_tables);
    auto* drows = static_cast<uint16_t*>(d_rows);
    auto* dstatus = static_cast<int*>(d_status);
    auto* dstats = static_cast<unsigned long long*>(d_stats);
    const int W = (int)width, H = (int)height, SW = (int)seg_w, SH = (int)seg_h;
    if (!par.empty()) {
        void *d_par = nullptr, *d_ctas = nullptr, *d_lines = nullptr, *d_blks = nullptr, *d_end = nullptr;
        void *d_stuff = nullptr, *d_boff = nullptr, *d_ulen = nullptr, *d_ubuf = nullptr, *d_cand = nullptr;
        void *d_groups = nullptr, *d_gentry = nullptr, *d_dbuf = nullptr, *d_cbuf = nullptr;
        const size_t nb = blks.size();
        st = call.upload(par.data(), par.size() * 4, &d_par);
        if (st == CPIPE_OK) st = call.upload(ctas.data(), ctas.size() * sizeof(CtaDesc), &d_ctas);
        if (st == CPIPE_OK && !lines.empty()) st = call.upload(lines.data(), lines.size() * sizeof(CtaDesc), &d_lines);
        if (st == CPIPE_OK && nb) st = call.upload(blks.data(), nb * sizeof(ScanBlk), &d_blks);
        if (st == CPIPE_OK) st = call.upload(seg_end.data(), count * 4, &d_end);
        if (st == CPIPE_OK) st = call.alloc(nb * 4, &d_stuff);
        if (st == CPIPE_OK) st = call.alloc(nb * 4, &d_boff);
        if (st == CPIPE_OK) st = call.alloc(count * 4, &d_ulen);
        if (st == CPIPE_OK) st = call.alloc(ubytes, &d_ubuf);
        if (st == CPIPE_OK) st = call.alloc(chunks * kCands * sizeof(LjCand), &d_cand);
        if (st == CPIPE_OK) st = call.alloc(groups * kGroupEntries * sizeof(LjGroup), &d_groups);
        if (st == CPIPE_OK) st = call.alloc(groups * sizeof(uint4), &d_gentry);
        if (st == CPIPE_OK) st = call.alloc(samples * 2, &d_dbuf);
        if (st == CPIPE_OK) st = call.alloc(nlines * 8, &d_cbuf);
        if (st == CPIPE_OK) st = cuda_status(cudaMemsetAsync(d_ulen, 0, count * 4, call.stream), "lj92 clear");
        if (st == CPIPE_OK) st = cuda_status(cudaMemsetAsync(d_ubuf, 0, ubytes, call.stream), "lj92 clear");
        if (st != CPIPE_OK) return call.finish(st);
        const auto* dpar = static_cast<const uint32_t*>(d_par);
        const auto* dctas = static_cast<const CtaDesc*>(d_ctas);
        auto* ulen = static_cast<uint32_t*>(d_ulen);
        auto* ubuf = static_cast<uint8_t*>(d_ubuf);
        auto* cand = static_cast<LjCand*>(d_cand);
        auto* grp = static_cast<LjGroup*>(d_groups);
        auto* gentry = static_cast<uint4*>(d_gentry);
        auto* dbuf = static_cast<uint16_t*>(d_dbuf);
        auto* cbuf = static_cast<uint16_t*>(d_cbuf);
        const int npar = (int)par.size(), nctas = (int)ctas.size();
        if (nb) {
            lj_mark_kernel<<<(unsigned)nb, 256, 0, call.stream>>>(blk, dsegs, static_cast<const ScanBlk*>(d_blks),
                                                                  static_cast<uint32_t*>(d_end),
                                                                  static_cast<uint32_t*>(d_stuff));
            lj_offsets_kernel<<<(npar + 127) / 128, 128, 0, call.stream>>>(
                dsegs, dpar, npar, static_cast<const uint32_t*>(d_stuff), static_cast<uint32_t*>(d_boff));
            lj_pack_kernel<<<(unsigned)nb, 256, 0, call.stream>>>(blk, dsegs, static_cast<const ScanBlk*>(d_blks),
                                                                  static_cast<const uint32_t*>(d_end),
                                                                  static_cast<const uint32_t*>(d_boff), ubuf, ulen);
        }
        // per call: the attribute belongs to the current device
        const int most = 4 * kLut * 2 + kStageWords * 4 + kChunksPerCta * 2 * (int)sizeof(LjCand);
        const bool attrs =
            cudaFuncSetAttribute(lj_cand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, most) == cudaSuccess &&
            cudaFuncSetAttribute(lj_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, most) == cudaSuccess;
        if (!attrs) {
            cudaGetLastError();
            set_error("%s", "lj92: shared memory attribute refused");
            return call.finish(CPIPE_INTERNAL_ERROR);
        }
        const size_t smem = (size_t)max_phases * kLut * 2 + kStageWords * 4;
        lj_cand_kernel<<<nctas, kChunksPerCta, smem + kChunksPerCta * 2 * sizeof(LjCand), call.stream>>>(
            dsegs, dctas, dtabs, ubuf, ulen, cand);
        lj_group_kernel<<<nctas, kChunksPerCta, 0, call.stream>>>(dsegs, dctas, dtabs, ubuf, ulen, cand, grp,
                                                                  dstats);
        lj_seg_kernel<<<npar, 32, 0, call.stream>>>(dsegs, dpar, dtabs, ubuf, ulen, cand, grp, gentry, dstats);
        lj_write_kernel<<<nctas, kChunksPerCta, smem, call.stream>>>(dsegs, dctas, dtabs, ubuf, ulen, cand, gentry, dbuf,
                                                                  dstatus, dstats);
        if (!lines.empty()) {
            lj_col_kernel<<<npar, 32, 0, call.stream>>>(dsegs, dpar, dbuf, cbuf);
            lj_line_kernel<<<(unsigned)lines.size(), 256, 0, call.stream>>>(
                dsegs, static_cast<const CtaDesc*>(d_lines), dbuf, cbuf, d_raw, W, H, SW, SH);
        }
        if (any_serial_recon)
            lj_recon_serial_kernel<<<(npar + 31) / 32, 32, 0, call.stream>>>(dsegs, dpar, npar, dbuf, drows, d_raw, W,
                                                                             H, SW, SH);
        st = cuda_status(cudaGetLastError(), "lj92 launch");
        if (st != CPIPE_OK) return call.finish(st);
    }
    if (!ser.empty()) {
        void* d_ser = nullptr;
        st = call.upload(ser.data(), ser.size() * 4, &d_ser);
        if (st != CPIPE_OK) return call.finish(st);
        const int nser = (int)ser.size();
        lj_serial_kernel<<<(nser + 31) / 32, 32, 0, call.stream>>>(blk, dsegs, static_cast<const uint32_t*>(d_ser), nser,
                                                                   dtabs, drows, d_raw, W, H, SW, SH, dstatus);
        st = cuda_status(cudaGetLastError(), "lj92 launch");
        if (st != CPIPE_OK) return call.finish(st);
    }
    std::vector<int> status(count, 0);
    unsigned long long counters[kStats] = {};
    st = cuda_status(cudaMemcpyAsync(status.data(), d_status, count * sizeof(int), cudaMemcpyDeviceToHost, call.stream),
                     "lj92 status");
    if (st == CPIPE_OK)
        st = cuda_status(cudaMemcpyAsync(counters, d_stats, sizeof(counters), cudaMemcpyDeviceToHost, call.stream),
                         "lj92 status");
    if (st == CPIPE_OK) st = cuda_status(cudaStreamSynchronize(call.stream), "lj92 decode");
    if (st == CPIPE_OK) {
        std::lock_guard<std::mutex> g(g_lj_mu);
        g_lj_last.figures[0] = chunks;
        g_lj_last.figures[1] = par.size();
        g_lj_last.figures[2] = ser.size();
        for (int k = 0; k < kStats; ++k) g_lj_last.figures[3 + k] = counters[k];
    }
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

extern "C" int cpipe_cuda_lj92_last_stats(uint64_t* figures, uint32_t count) {
    if (!figures && count) return CPIPE_BAD_INDEX;
    std::lock_guard<std::mutex> g(cpb::g_lj_mu);
    for (uint32_t k = 0; k < count && k < 9; ++k) figures[k] = cpb::g_lj_last.figures[k];
    return CPIPE_OK;
}
