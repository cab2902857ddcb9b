// lj92.cu -- lossless JPEG (ITU T.81 process 14) tiles of a 16-bit CFA image
// on the device: the DNG export's compression 7 (examples/prr2dng/lj92.rs,
// the tile cut of examples/prr2dng/dng.rs:95-125), byte for byte.
//
// One CTA of 1024 threads per tile. A tile T sensels square is coded as a
// JPEG image T/2 wide with two interleaved components, each sample
// predicted from the one two columns to its left (same Bayer colour), the
// one above for a row's first two, 32768 for the first. Passes:
//   1. the tile's prediction differences go to shared memory; each thread
//      takes a run of consecutive samples in coding order and counts their
//      magnitude categories (warp sums, then 17 shared bins). In whole
//      256-square tiles a thread loads its own run with 16-byte loads and
//      counts as it goes; other tiles are read row by row, edges repeated;
//   2. one warp builds the tile's optimal Huffman table (Annex K.2 with a
//      reserved all-ones code, lengths limited to 16, canonical codes);
//   3. each thread's bits follow from its category counts; a block scan
//      gives every thread its bit offset in the tile's stream;
//   4. each thread packs its bits, most significant first, into 32-bit
//      words of a per-tile scratch stream (whole words stored, the shared
//      first and last words OR-ed); the last byte is padded with ones;
//   5. the stream is copied into the differences' shared memory when it
//      fits; each warp takes a run of its words, a lane a word at a time,
//      and counts their 0xFF bytes, which gives the stream's size;
//   6. a warp's decoupled look-back over the tiles (claimed in launch
//      order) gives the stream's offset in the output, and the CTA writes
//      the markers, the table and the stream there, each 0xFF followed by
//      a stuffed 0x00.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/prr.h"
#include "context.h"
#include "kernels.h"

namespace prr {
namespace {

constexpr int kLjThreads = 1024;
constexpr int kLjMaxTile = 256;
// SOI 2, SOF3 16, DHT 21 + its values (17 at most), SOS 12.
constexpr int kLjHeaderMax = 51 + 17;

struct Lj92Desc {
    const uint16_t* image;
    uint64_t stride;
    uint32_t width, height, tile, across, ntiles;
    uint32_t pad_even;             // streams placed at even offsets, a 0 byte after odd ones (TIFF chunks)
    uint32_t* words;               // per tile: word_cap words of bit stream
    uint64_t word_cap;
    uint8_t* out;                  // the streams back to back
    uint64_t out_cap;
    uint64_t* offsets;             // ntiles + 1: each stream's offset, then the end
    uint32_t* sizes;               // per tile: its stream's bytes
    unsigned long long* lookback;  // per tile: state << 62 | bytes (aggregate or inclusive prefix)
    uint32_t* counter;             // tiles claimed, in launch order
    uint32_t* error;               // 1: a look-back wait gave up; 2: out_cap too small
};

constexpr unsigned long long kAggregate = 1ull << 62, kInclusive = 2ull << 62, kValueMask = (1ull << 62) - 1;
constexpr uint32_t kLookbackSpins = 1u << 22;  // with a 64 ns sleep: about a quarter of a second

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Decoupled look-back by one warp: publish this tile's size, then sum the
// sizes of the tiles before it back to the nearest published inclusive
// prefix, 32 tiles a step (lane l reads tile base - l), and publish this
// tile's inclusive prefix. Tiles are claimed in launch order, so every tile
// before this one belongs to a CTA that is running or done; the wait is
// bounded all the same. Every lane returns the exclusive prefix, or ~0 if
// the wait gave up.
__device__ unsigned long long lookback_warp(const Lj92Desc& d, uint32_t tile, unsigned long long slot,
                                            uint32_t lane) {
    if (tile == 0) {
        if (lane == 0) st_release(d.lookback, kInclusive | slot);
        return 0;
    }
    if (lane == 0) st_release(d.lookback + tile, kAggregate | slot);
    unsigned long long excl = 0;
    int64_t base = int64_t(tile) - 1;
    uint32_t spins = 0;
    for (;;) {
        const int64_t j = base - int64_t(lane);
        // Before tile 0 there is nothing to add: an inclusive prefix of 0.
        const unsigned long long v = j >= 0 ? ld_acquire(d.lookback + j) : kInclusive;
        const unsigned long long state = v & ~kValueMask;
        const uint32_t inc = __ballot_sync(0xFFFFFFFFu, state == kInclusive);
        const uint32_t unpublished = __ballot_sync(0xFFFFFFFFu, state == 0);
        // The lanes up to the nearest inclusive prefix (all 32 without one).
        const uint32_t need = inc ? (inc ^ (inc - 1)) : 0xFFFFFFFFu;
        if (unpublished & need) {
            if (++spins > kLookbackSpins) {
                // Give up, and still publish, so that the tiles after this
                // one do not wait too; the call reports the failure.
                if (lane == 0) st_release(d.lookback + tile, kInclusive | slot);
                return ~0ull;
            }
            __nanosleep(64);
            continue;
        }
        unsigned long long part = ((need >> lane) & 1u) ? (v & kValueMask) : 0ull;
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
        excl += part;
        if (inc) break;
        base -= 32;
    }
    if (lane == 0) st_release(d.lookback + tile, kInclusive | (excl + slot));
    return excl;
}

__device__ __forceinline__ uint32_t clamp_edge(uint32_t i, uint32_t n) { return i < n ? i : n - 2 + (i - n) % 2; }

__device__ __forceinline__ uint32_t category(int32_t d) {
    const uint32_t a = uint32_t(d < 0 ? -d : d);
    return 32 - __clz(a);  // __clz(0) = 32
}

struct HuffTable {
    uint8_t counts[16];
    uint8_t values[17];
    uint32_t nvalues;
    uint16_t code[17];
    uint8_t length[17];
};

// HuffmanTable::optimal (lj92.rs:96-202) by one warp: lane v holds symbol v
// (categories 0-16, and 17, the reserved symbol of frequency 1). The two
// least frequent trees come from two minimum reductions over a key that
// orders by frequency, then by the larger symbol (the crate's tie rule); a
// merge lengthens the codes of both trees' symbols (each lane carries the
// symbol that holds its tree's frequency). The code-length limit, the value
// order and the canonical codes follow with ballots and shuffles. A tile's
// frequencies total at most 65536 + 1, so a key (frequency << 8 | 255 - v)
// fits in 32 bits.
__device__ void build_table(const uint32_t* histogram, HuffTable& t, uint32_t lane) {
    constexpr uint32_t kAll = 0xFFFFFFFFu, kNone = 0xFFFFFFFFu;
    uint32_t f = lane < 17 ? histogram[lane] : (lane == 17 ? 1u : 0u);
    uint32_t label = lane, size = 0;
    for (;;) {
        const uint32_t key = f > 0 ? (f << 8) | (255u - lane) : kNone;
        const uint32_t k1 = __reduce_min_sync(kAll, key);
        const uint32_t v1 = 255u - (k1 & 255u);
        const uint32_t k2 = __reduce_min_sync(kAll, lane == v1 ? kNone : key);
        if (k2 == kNone) break;
        const uint32_t v2 = 255u - (k2 & 255u);
        if (lane == v1) f += k2 >> 8;
        if (lane == v2) f = 0;
        if (label == v1 || label == v2) size++;
        if (label == v2) label = v1;
    }
    // bits[i] in lane i: the symbols of code size i (at most 17 with 18
    // symbols).
    uint32_t bits = 0;
    for (uint32_t i = 1; i < 32; i++) {
        const uint32_t c = __popc(__ballot_sync(kAll, lane < 18 && size == i));
        if (lane == i) bits = c;
    }
    // Lengths limited to 16 (Figure K.3); only size 17 can exceed it.
    for (;;) {
        if (__shfl_sync(kAll, bits, 17) == 0) break;
        const uint32_t m = __ballot_sync(kAll, lane <= 15 && bits > 0);
        if (m == 0) break;  // a code of 15 bits or less always exists
        const uint32_t j = 31 - __clz(m);
        if (lane == 17) bits -= 2;
        if (lane == 16) bits += 1;
        if (lane == j + 1) bits += 2;
        if (lane == j) bits -= 1;
    }
    {
        // The reserved symbol's code, the longest, is not used.
        const uint32_t m = __ballot_sync(kAll, lane >= 1 && lane <= 16 && bits > 0);
        if (m && lane == 31 - __clz(m)) bits -= 1;
    }
    // HUFFVAL: used categories by (unlimited) code size, then value.
    const bool used = lane < 17 && size > 0;
    const uint32_t used_mask = __ballot_sync(kAll, used);
    uint32_t rank = 0;
    for (uint32_t u = 0; u < 17; u++) {
        const uint32_t su = __shfl_sync(kAll, size, u);
        if (((used_mask >> u) & 1u) && (su < size || (su == size && u < lane))) rank++;
    }
    if (used) t.values[rank] = uint8_t(lane);
    if (lane == 0) t.nvalues = uint32_t(__popc(used_mask));
    const uint32_t cnt = (lane >= 1 && lane <= 16) ? bits : 0u;
    if (lane >= 1 && lane <= 16) t.counts[lane - 1] = uint8_t(cnt);
    // Canonical codes: the first code of length L is the sum over m < L of
    // counts(m) << (L - m); a value's code is that plus its place among the
    // values of its length.
    uint32_t cum = cnt;  // inclusive scan of the counts over the lengths
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kAll, cum, o);
        if (lane >= o) cum += y;
    }
    uint32_t first = 0;
    for (uint32_t m = 1; m < 16; m++) {
        const uint32_t cm = __shfl_sync(kAll, cnt, m);
        if (m < lane) first += cm << (lane - m);
    }
    uint32_t code = 0, length = 0;
    for (uint32_t len = 1; len <= 16; len++) {
        const uint32_t upto = __shfl_sync(kAll, cum, len), before = __shfl_sync(kAll, cum, len - 1);
        const uint32_t start = __shfl_sync(kAll, first, len);
        if (used && length == 0 && upto > rank) {
            length = len;
            code = start + (rank - before);
        }
    }
    if (lane < 17) {
        t.code[lane] = uint16_t(code);
        t.length[lane] = uint8_t(length);
    }
}

// Exclusive block scan of one 64-bit value per thread; `total` gets the sum.
__device__ uint64_t block_scan(uint64_t v, uint64_t* warp_sums, uint64_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t s = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;  // inclusive
    }
    __syncthreads();
    total = warp_sums[31];
    const uint64_t before = warp == 0 ? 0 : warp_sums[warp - 1];
    const uint64_t r = before + x - v;
    __syncthreads();  // warp_sums is reused by the next scan
    return r;
}

__device__ __forceinline__ void put_be16(uint8_t* p, uint32_t v) {
    p[0] = uint8_t(v >> 8);
    p[1] = uint8_t(v);
}

// The markers before the entropy-coded segment (lj92.rs:24-52); their length.
__device__ uint32_t write_header(uint8_t* o, const HuffTable& t, uint32_t tile) {
    uint32_t n = 0;
    o[n++] = 0xFF, o[n++] = 0xD8;                 // SOI
    o[n++] = 0xFF, o[n++] = 0xC3;                 // SOF3
    put_be16(o + n, 8 + 3 * 2), n += 2;
    o[n++] = 16;
    put_be16(o + n, tile), n += 2;                // height
    put_be16(o + n, tile / 2), n += 2;            // width in two-component pixels
    o[n++] = 2;
    for (uint32_t id = 0; id < 2; id++) o[n++] = uint8_t(id), o[n++] = 0x11, o[n++] = 0;
    o[n++] = 0xFF, o[n++] = 0xC4;                 // DHT
    put_be16(o + n, 2 + 1 + 16 + t.nvalues), n += 2;
    o[n++] = 0;
    for (int k = 0; k < 16; k++) o[n++] = t.counts[k];
    for (uint32_t k = 0; k < t.nvalues; k++) o[n++] = t.values[k];
    o[n++] = 0xFF, o[n++] = 0xDA;                 // SOS
    put_be16(o + n, 6 + 2 * 2), n += 2;
    o[n++] = 2;
    for (uint32_t id = 0; id < 2; id++) o[n++] = uint8_t(id), o[n++] = 0;
    o[n++] = 1, o[n++] = 0, o[n++] = 0;           // predictor 1, no point transform
    return n;
}

// Shared-memory layout of a tile's prediction differences: thread t's run
// of `per` consecutive samples (in coding order) is column t of a per x
// kLjPitch array of int16, so that the threads of a warp reading the i-th
// sample of their runs read consecutive halfwords, and the staging writes
// (a warp's 32 consecutive samples: 32 rows of one column) fall in 32
// different banks (the pitch is an odd number of words).
constexpr uint32_t kLjPitch = kLjThreads + 2;

// Tile geometry: compile-time for the DNG tile (256: every division a
// shift), run-time for other sizes.
template <uint32_t TT>
struct Geometry {
    uint32_t T, per;
    __device__ Geometry(uint32_t t) : T(TT ? TT : t), per(TT ? TT * TT / kLjThreads : (t * t + kLjThreads - 1) / kLjThreads) {}
    __device__ __forceinline__ uint32_t row(uint32_t s) const { return s / T; }
    __device__ __forceinline__ uint32_t col(uint32_t s) const { return s % T; }
    __device__ __forceinline__ uint32_t index(uint32_t s) const { return (s % per) * kLjPitch + s / per; }
};

// Packed per-thread counts of the 17 categories: eight 8-bit fields a word
// (a thread's run is at most 64 samples), categories 0-7, 8-15, 16.
struct Counts {
    uint64_t lo = 0, hi = 0;
    uint32_t top = 0;
    __device__ __forceinline__ void add(uint32_t c) {
        const uint64_t one = uint64_t(1) << (8 * (c & 7));
        lo += c < 8 ? one : 0;
        hi += (c >= 8 && c < 16) ? one : 0;
        top += c == 16;
    }
    __device__ __forceinline__ uint32_t get(int k) const {
        return k < 8 ? uint32_t(lo >> (8 * k)) & 0xFF : (k < 16 ? uint32_t(hi >> (8 * (k - 8))) & 0xFF : top);
    }
};

template <uint32_t TT>
__global__ void __launch_bounds__(kLjThreads, 1) k_lj92_encode(Lj92Desc d) {
    extern __shared__ int16_t diffs[];
    __shared__ uint32_t hist[17];
    __shared__ HuffTable table;
    __shared__ uint64_t warp_sums[32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_offset;
    const Geometry<TT> g(d.tile);
    const uint32_t T = g.T, n = T * T, per = g.per;
    if (threadIdx.x == 0) s_tile = atomicAdd(d.counter, 1u);
    if (threadIdx.x < 17) hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t tile_index = s_tile;
    const uint32_t left = tile_index % d.across * T, top = tile_index / d.across * T;
    const uint32_t s0 = min(n, threadIdx.x * per), s1 = min(n, s0 + per);
    const uint32_t run = s1 - s0;
    const uint32_t col_t = threadIdx.x;  // this thread's column of `diffs`

    // 0. The tile's differences (edges repeated as dng::tile does): each
    // sample less the one two to its left (same Bayer colour), the one above
    // for a row's first two, 32768 for the tile's first; modulo 2^16,
    // centred on 0. 1. Each thread's counts of their categories, and the
    // tile's histogram.
    Counts counts;
    const bool whole = TT == 256 && left + T <= d.width && top + T <= d.height &&
                       (reinterpret_cast<uintptr_t>(d.image) & 15) == 0 && (d.stride & 7) == 0;
    if (whole) {
        // A 256-square tile inside the picture, rows 16-byte aligned: thread
        // t loads its own run (row t / 4 of the tile, columns (t % 4) * 64
        // on) with 16-byte loads and counts its categories as it goes.
        const uint32_t r = threadIdx.x >> 2, c0 = (threadIdx.x & 3) * 64;
        const uint16_t* row = d.image + uint64_t(top + r) * d.stride + left;
        uint32_t p0 = 32768u, p1 = 32768u;  // the predictions of the next even and odd samples
        if (c0 > 0 || r > 0) {
            const uint32_t two = __ldg(reinterpret_cast<const uint32_t*>(c0 > 0 ? row + c0 - 2 : row - d.stride));
            p0 = two & 0xFFFFu;
            p1 = two >> 16;
        }
        const uint4* v = reinterpret_cast<const uint4*>(row + c0);
#pragma unroll
        for (uint32_t q = 0; q < 8; q++) {
            const uint4 w = __ldg(v + q);
            const uint32_t pairs[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (uint32_t h = 0; h < 4; h++) {
                const uint32_t a = pairs[h] & 0xFFFFu, b = pairs[h] >> 16;
                const int16_t da = int16_t(uint16_t(a - p0)), db = int16_t(uint16_t(b - p1));
                const uint32_t i = 8 * q + 2 * h;
                diffs[i * kLjPitch + col_t] = da;
                diffs[(i + 1) * kLjPitch + col_t] = db;
                counts.add(category(da));
                counts.add(category(db));
                p0 = a;
                p1 = b;
            }
        }
    } else {
        // Any tile: coalesced loads in coding order, edges clamped.
        for (uint32_t s = threadIdx.x; s < n; s += kLjThreads) {
            const uint32_t r = g.row(s), c = g.col(s);
            const uint16_t* row = d.image + uint64_t(clamp_edge(top + r, d.height)) * d.stride;
            const uint32_t x = __ldg(row + clamp_edge(left + c, d.width));
            uint32_t p;
            if (c >= 2)
                p = __ldg(row + clamp_edge(left + c - 2, d.width));
            else if (r > 0)
                p = __ldg(d.image + uint64_t(clamp_edge(top + r - 1, d.height)) * d.stride + clamp_edge(left + c, d.width));
            else
                p = 32768u;
            diffs[g.index(s)] = int16_t(uint16_t(x - p));
        }
        __syncthreads();
        for (uint32_t i = 0; i < run; i++) counts.add(category(diffs[i * kLjPitch + col_t]));
    }
#pragma unroll
    for (int k = 0; k < 17; k++) {
        const uint32_t sum = __reduce_add_sync(0xFFFFFFFFu, counts.get(k));
        if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&hist[k], sum);
    }
    __syncthreads();

    // 2. The table.
    if (threadIdx.x < 32) build_table(hist, table, threadIdx.x);
    __syncthreads();

    // 3. Bit offsets: this thread's bits from its category counts (each
    // sample costs its category's code length, plus c extra bits for
    // categories 1-15).
    uint64_t mine = 0;
#pragma unroll
    for (int k = 0; k < 17; k++) mine += uint64_t(counts.get(k)) * (table.length[k] + ((k > 0 && k < 16) ? k : 0));
    uint64_t total_bits = 0;
    const uint64_t b0 = block_scan(mine, warp_sums, total_bits);
    uint32_t* words = d.words + uint64_t(tile_index) * d.word_cap;
    const uint64_t nwords = (total_bits + 31) / 32;
    for (uint64_t w = threadIdx.x; w < nwords; w += kLjThreads) words[w] = 0;
    __syncthreads();

    // 4. Pack the bits: whole words stored, the first (when it starts
    // inside a word) and the last OR-ed, since a neighbour shares them.
    {
        uint64_t w = b0 / 32;
        const uint32_t lead = uint32_t(b0 % 32);
        uint64_t acc = 0;
        uint32_t pending = lead;
        bool first = true;
        for (uint32_t i = 0; i < run; i++) {
            const int32_t diff = diffs[i * kLjPitch + col_t];
            const uint32_t c = category(diff);
            uint32_t len = table.length[c];
            uint64_t bits = table.code[c];
            if (c > 0 && c < 16) {
                // Negative differences go as d - 1 in c bits.
                const uint32_t extra = uint32_t(diff < 0 ? diff - 1 : diff) & ((1u << c) - 1);
                bits = (bits << c) | extra;
                len += c;
            }
            acc = (acc << len) | bits;
            pending += len;
            if (pending >= 32) {
                pending -= 32;
                const uint32_t word = uint32_t(acc >> pending);
                if (first && lead > 0)
                    atomicOr(words + w, word);
                else
                    words[w] = word;
                first = false;
                w++;
                acc &= (uint64_t(1) << pending) - 1;
            }
        }
        if (pending > 0 && run > 0) atomicOr(words + w, uint32_t(acc << (32 - pending)));
    }
    __syncthreads();
    if (threadIdx.x == 0 && (total_bits & 7)) {
        // Pad the last byte with one bits (lj92.rs:239-245).
        const uint32_t used = uint32_t(total_bits % 32), pad = 8 - uint32_t(total_bits & 7);
        words[total_bits / 32] |= ((1u << pad) - 1) << (32 - used - pad);
    }
    __syncthreads();
    // The differences are no longer needed: a stream that fits in their
    // shared memory is copied there once (coalesced), and the two passes
    // below read it from there instead of from L2.
    const uint32_t* src = words;
    if (nwords <= uint64_t(per) * kLjPitch / 2) {
        uint32_t* staged = reinterpret_cast<uint32_t*>(diffs);
        for (uint64_t w = threadIdx.x; w < nwords; w += kLjThreads) staged[w] = words[w];
        src = staged;
        __syncthreads();
    }

    // 5. Byte stuffing: warp k takes words [k R, (k + 1) R) of the stream,
    // 32 at a time (a lane a word), counts their 0xFF bytes; the warps'
    // counts are scanned once, which gives the stream's size and (by the
    // look-back) its place in the output; each lane then writes its bytes,
    // every 0xFF followed by a 0x00, at the place the counts before it give.
    const uint32_t hdr = 51 + table.nvalues;
    const uint64_t nbytes = (total_bits + 7) / 8;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t R = (nwords + 31) / 32;
    const uint64_t wb = min(nwords, uint64_t(warp) * R), we = min(nwords, wb + R);
    auto word_ff = [&](uint64_t w, uint32_t& word, uint32_t& nb) -> uint32_t {
        word = src[w];
        const uint64_t left_bytes = nbytes - 4 * w;  // bytes of this word in the stream
        nb = left_bytes < 4 ? uint32_t(left_bytes) : 4u;
        uint32_t ff = 0;
        for (uint32_t k = 0; k < nb; k++) ff += ((word >> (24 - 8 * k)) & 0xFF) == 0xFF;
        return ff;
    };
    uint32_t ff = 0;
    for (uint64_t w = wb + lane; w < we; w += 32) {
        uint32_t word, nb;
        ff += word_ff(w, word, nb);
    }
    ff = __reduce_add_sync(0xFFFFFFFFu, ff);
    uint64_t total_ff = 0;
    uint64_t carry = block_scan(lane == 0 ? ff : 0, warp_sums, total_ff);
    carry = __shfl_sync(0xFFFFFFFFu, carry, 0);
    const uint64_t size = hdr + nbytes + total_ff + 2;
    const uint64_t slot = size + (d.pad_even ? (size & 1) : 0);
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) d.sizes[tile_index] = uint32_t(size);
        unsigned long long off = lookback_warp(d, tile_index, slot, threadIdx.x);
        if (threadIdx.x == 0) {
            if (off == ~0ull) {
                atomicOr(d.error, 1u);
            } else {
                d.offsets[tile_index] = off;
                if (tile_index == d.ntiles - 1) d.offsets[d.ntiles] = off + slot;
                if (off + slot > d.out_cap) {
                    atomicOr(d.error, 2u);
                    off = ~0ull;
                }
            }
            s_offset = off;
        }
    }
    __syncthreads();
    if (s_offset == ~0ull) return;
    uint8_t* out = d.out + s_offset;
    for (uint64_t base = wb; base < we; base += 32) {
        const uint64_t w = base + lane;
        uint32_t word = 0, nb = 0, f = 0;
        if (w < we) f = word_ff(w, word, nb);
        uint32_t incl = f;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= uint32_t(o)) incl += y;
        }
        if (w < we) {
            uint64_t o = hdr + 4 * w + carry + (incl - f);
            for (uint32_t k = 0; k < nb; k++) {
                const uint8_t byte = uint8_t(word >> (24 - 8 * k));
                out[o++] = byte;
                if (byte == 0xFF) out[o++] = 0;
            }
        }
        carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (threadIdx.x == 0) {
        write_header(out, table, T);
        const uint64_t end = hdr + nbytes + total_ff;
        out[end] = 0xFF;  // EOI
        out[end + 1] = 0xD9;
        if (slot > size) out[size] = 0;  // the TIFF chunk's pad byte
    }
}

}  // namespace

// Worst-case stream bytes of one tile: markers, 31 bits a sample, every
// byte stuffed, EOI.
uint64_t lj92_tile_bound(uint32_t tile) {
    const uint64_t bits = uint64_t(tile) * tile * 31;
    return (uint64_t(kLjHeaderMax) + 2 * ((bits + 7) / 8) + 2 + 15) & ~uint64_t(15);
}

int lj92_encode(prr_ctx* c, const uint16_t* image, uint32_t width, uint32_t height, uint64_t stride, uint32_t tile,
                uint8_t* out, uint64_t out_cap, uint64_t* dev_offsets, uint32_t* dev_sizes, uint32_t* dev_error,
                bool pad_even) {
    if (!image || !out || !dev_offsets || !dev_sizes || !dev_error || width < 2 || height < 2 || stride < width || tile < 2 ||
        tile > kLjMaxTile || (tile & 1))
        return PRR_ERR_INVALID;
    const uint32_t across = (width + tile - 1) / tile, down = (height + tile - 1) / tile;
    const uint32_t ntiles = across * down;
    const uint64_t word_cap = (uint64_t(tile) * tile * 31 + 31) / 32 + 2;
    PRR_TRY(c->cuda(c->lj_words.ensure(size_t(ntiles) * word_cap)));
    // Look-back words (one per tile), then the claim counter.
    PRR_TRY(c->cuda(c->lj_lookback.ensure(size_t(ntiles) + 1)));
    PRR_TRY(c->cuda(cudaMemsetAsync(c->lj_lookback.p, 0, (size_t(ntiles) + 1) * sizeof(unsigned long long),
                                    c->stream)));
    PRR_TRY(c->cuda(cudaMemsetAsync(dev_error, 0, sizeof(uint32_t), c->stream)));
    Lj92Desc d{};
    d.image = image;
    d.stride = stride;
    d.width = width;
    d.height = height;
    d.tile = tile;
    d.across = across;
    d.ntiles = ntiles;
    d.pad_even = pad_even ? 1u : 0u;
    d.words = c->lj_words.p;
    d.word_cap = word_cap;
    d.out = out;
    d.out_cap = out_cap;
    d.offsets = dev_offsets;
    d.sizes = dev_sizes;
    d.lookback = c->lj_lookback.p;
    d.counter = reinterpret_cast<uint32_t*>(c->lj_lookback.p + ntiles);
    d.error = dev_error;
    const uint32_t per = (tile * tile + kLjThreads - 1) / kLjThreads;
    const size_t smem = size_t(per) * kLjPitch * sizeof(int16_t);
    auto kernel = tile == 256 ? k_lj92_encode<256> : k_lj92_encode<0>;
    PRR_TRY(c->cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))));
    kernel<<<ntiles, kLjThreads, smem, c->stream>>>(d);
    count_launch();
    return c->cuda(cudaGetLastError());
}

}  // namespace prr

using namespace prr;

namespace {

uint32_t tiles_of(uint32_t width, uint32_t height, uint32_t tile) {
    return ((width + tile - 1) / tile) * ((height + tile - 1) / tile);
}

// Encode into the context's packed buffer and bring the offsets and sizes
// to its pinned buffers (the streams stay on the device); *ntiles_out gets
// the tile count.
int encode_on_device(prr_ctx* c, const uint16_t* image, uint32_t width, uint32_t height, uint64_t stride,
                     uint32_t tile, bool pad_even, uint32_t* ntiles_out) {
    if (width < 2 || height < 2 || tile < 2 || tile > 256 || (tile & 1)) return PRR_ERR_INVALID;
    const uint32_t ntiles = tiles_of(width, height, tile);
    const uint64_t cap = uint64_t(ntiles) * lj92_tile_bound(tile);
    PRR_TRY(c->cuda(c->lj_out.ensure(cap)));
    // offsets (ntiles + 1), then sizes (ntiles, as u32 pairs), then the error word
    const size_t words = size_t(ntiles) + 1 + (size_t(ntiles) + 1) / 2 + 1;
    PRR_TRY(c->cuda(c->lj_offsets.ensure(words)));
    PRR_TRY(c->cuda(c->lj_hoffsets.ensure(words)));
    uint64_t* offsets = c->lj_offsets.p;
    uint32_t* sizes = reinterpret_cast<uint32_t*>(offsets + ntiles + 1);
    uint32_t* error = reinterpret_cast<uint32_t*>(offsets + words - 1);
    PRR_TRY(lj92_encode(c, image, width, height, stride, tile, c->lj_out.p, cap, offsets, sizes, error, pad_even));
    PRR_TRY(c->cuda(cudaMemcpyAsync(c->lj_hoffsets.p, offsets, words * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                    c->stream)));
    PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
    const uint32_t err = *reinterpret_cast<const uint32_t*>(c->lj_hoffsets.p + words - 1);
    if (err & 1) {
        c->last_error = "a tile encoder's wait for the tiles before it gave up";
        return PRR_ERR_TIMEOUT;
    }
    if (err) return PRR_ERR_BUFFER;
    *ntiles_out = ntiles;
    return PRR_OK;
}

const uint32_t* host_sizes(prr_ctx* c, uint32_t ntiles) {
    return reinterpret_cast<const uint32_t*>(c->lj_hoffsets.p + ntiles + 1);
}

// A frame's DNG file, ready to be copied out: the bytes before the image
// data, and where the data is on the device.
struct Prepared {
    std::vector<uint8_t> prefix;
    const uint16_t* image = nullptr;  // uncompressed: the visible samples' rows
    uint64_t stride = 0;
    uint32_t width = 0, height = 0;
    bool tiles = false;  // the streams in the context's packed buffer
    uint64_t data = 0;   // image data bytes
    size_t len() const { return prefix.size() + data; }
};

int dng_prepare(prr_ctx* c, const prr_header* h, const uint16_t* dev_samples, int samples, int compression,
                const prr_dng_clip* clip, Prepared& p) {
    if (samples != PRR_DNG_CODE_VALUES && samples != PRR_DNG_LINEAR) return PRR_ERR_INVALID;
    if (compression != PRR_DNG_UNCOMPRESSED && compression != PRR_DNG_LJ92) return PRR_ERR_INVALID;
    p.width = h->width;
    p.height = h->height;
    p.image = dev_samples;
    p.stride = (uint64_t(p.width) + 15) & ~uint64_t(15);  // the decoded frame's coded width
    if (samples == PRR_DNG_LINEAR) {
        const size_t n = size_t(p.width) * p.height;
        PRR_TRY(c->cuda(c->lin.ensure(std::max<size_t>(n, 1))));
        PRR_TRY(prr_linearize(c, h, dev_samples, c->lin.p, n));
        p.image = c->lin.p;
        p.stride = p.width;
    }
    if (compression == PRR_DNG_UNCOMPRESSED) {
        p.data = uint64_t(p.width) * p.height * 2;
        if (p.data > 0xFFFFFFFFull) return PRR_ERR_INVALID;
        return dng_prefix(h, clip, samples, compression, {uint32_t(p.data)}, p.prefix);
    }
    uint32_t ntiles = 0;
    PRR_TRY(encode_on_device(c, p.image, p.width, p.height, p.stride, 256, true, &ntiles));
    const uint32_t* sz = host_sizes(c, ntiles);
    PRR_TRY(dng_prefix(h, clip, samples, compression, std::vector<uint32_t>(sz, sz + ntiles), p.prefix));
    p.tiles = true;
    p.data = c->lj_hoffsets.p[ntiles];  // the streams, each padded to an even length
    return PRR_OK;
}

int dng_emit(prr_ctx* c, const Prepared& p, uint8_t* dst) {
    std::memcpy(dst, p.prefix.data(), p.prefix.size());
    uint8_t* data = dst + p.prefix.size();
    if (p.tiles) {
        PRR_TRY(c->cuda(cudaMemcpyAsync(data, c->lj_out.p, p.data, cudaMemcpyDeviceToHost, c->stream)));
    } else if (p.data > 0) {
        PRR_TRY(c->cuda(cudaMemcpy2DAsync(data, size_t(p.width) * 2, p.image, size_t(p.stride) * 2,
                                          size_t(p.width) * 2, p.height, cudaMemcpyDeviceToHost, c->stream)));
    }
    return c->cuda(cudaStreamSynchronize(c->stream));
}

}  // namespace

extern "C" {

uint64_t prr_lj92_tile_bound(uint32_t tile) { return tile >= 2 && tile <= 256 ? lj92_tile_bound(tile) : 0; }

int prr_lj92_encode(prr_ctx* c, const uint16_t* dev_image, uint32_t width, uint32_t height, uint64_t stride,
                    uint32_t tile, uint8_t* dev_out, uint64_t out_cap, uint64_t* dev_offsets) {
    if (!c || !dev_image || !dev_out || !dev_offsets) return PRR_ERR_INVALID;
    if (width < 2 || height < 2 || tile < 2 || tile > 256 || (tile & 1)) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    const uint32_t ntiles = tiles_of(width, height, tile);
    if (out_cap < uint64_t(ntiles) * lj92_tile_bound(tile)) return PRR_ERR_BUFFER;
    PRR_TRY(c->cuda(c->lj_flag.ensure(size_t(ntiles) + 1)));
    return lj92_encode(c, dev_image, width, height, stride, tile, dev_out, out_cap, dev_offsets, c->lj_flag.p + 1,
                       c->lj_flag.p, false);
}

int prr_lj92_encode_host(prr_ctx* c, const uint16_t* dev_image, uint32_t width, uint32_t height, uint64_t stride,
                         uint32_t tile, uint8_t* out, size_t cap, uint64_t* offsets, size_t* total) {
    if (!c || !dev_image || !offsets || !total) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    uint32_t ntiles = 0;
    PRR_TRY(encode_on_device(c, dev_image, width, height, stride, tile, false, &ntiles));
    std::memcpy(offsets, c->lj_hoffsets.p, (ntiles + 1) * sizeof(uint64_t));
    *total = size_t(offsets[ntiles]);
    if (*total > cap || (!out && *total > 0)) return PRR_ERR_BUFFER;
    PRR_TRY(c->cuda(cudaMemcpyAsync(out, c->lj_out.p, *total, cudaMemcpyDeviceToHost, c->stream)));
    return c->cuda(cudaStreamSynchronize(c->stream));
}

int prr_dng_write(prr_ctx* c, const prr_header* h, const uint16_t* dev_samples, int samples, int compression,
                  const prr_dng_clip* clip, prr_dng_file** out) {
    if (!c || !h || !dev_samples || !out) return PRR_ERR_INVALID;
    *out = nullptr;
    PRR_TRY(c->use_device());
    Prepared p;
    PRR_TRY(dng_prepare(c, h, dev_samples, samples, compression, clip, p));
    prr_dng_file* f = nullptr;
    try {
        f = dng_file_new(p.len());
    } catch (const std::bad_alloc&) {
        return PRR_ERR_NO_MEMORY;
    }
    const int rc = dng_emit(c, p, dng_file_bytes(f));
    if (rc != PRR_OK) {
        prr_dng_free(f);
        return rc;
    }
    *out = f;
    return PRR_OK;
}

int prr_dng_write_into(prr_ctx* c, const prr_header* h, const uint16_t* dev_samples, int samples, int compression,
                       const prr_dng_clip* clip, uint8_t* out, size_t cap, size_t* len) {
    if (!c || !h || !dev_samples || !len) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    Prepared p;
    PRR_TRY(dng_prepare(c, h, dev_samples, samples, compression, clip, p));
    *len = p.len();
    if (!out || cap < p.len()) return PRR_ERR_BUFFER;
    return dng_emit(c, p, out);
}

}  // extern "C"
