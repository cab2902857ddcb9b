// decode.cu -- ProRes RAW frame decoding on sm_100a.
//
// Two launches per frame:
//  1. k_tile_index: one CTA walks the tile size table (src/decoder.rs:104-116)
//     with a block-wide prefix scan, giving every tile's byte offset, the
//     first tile that reaches past the packet (Error::TileOutOfBounds) and
//     ParsedFrame::max_qscale (the byte after every tile start).
//  2. k_decode_full / k_decode_reduced: one CTA per (tile row, 256-sensel
//     segment). Tiles are powers of two of 16-sensel columns placed at
//     multiples of their width, so every tile lies inside one segment. The
//     CTA parses its tiles' headers (Tile::parse, src/tile.rs:126-153),
//     entropy-decodes each component stream on its own thread straight into
//     shared memory (dequantized as it is stored), runs the inverse transform
//     in shared memory and writes whole rows of its segment with 16-byte
//     stores. Coefficients never reach HBM. Squares of skipped tiles are
//     written as 0, so the output needs no clearing.

#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"

namespace prr {

namespace {

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v, uint32_t lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= uint32_t(o)) v += n;
    }
    return v;
}
__device__ __forceinline__ uint64_t warp_incl_scan_u64(uint64_t v, uint32_t lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t n = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= uint32_t(o)) v += n;
    }
    return v;
}

// Tile j of a tile row: first 16-sensel column and log2 block count
// (TileGrid::row, src/tile.rs:79-101, in closed form).
__device__ __forceinline__ void tile_geom(uint32_t j, uint32_t columns, uint32_t a, uint32_t& x,
                                          uint32_t& log2) {
    const uint32_t full = columns >> a;
    if (j < full) {
        x = j << a;
        log2 = a;
        return;
    }
    uint32_t k = j - full;
    const uint32_t rem = columns & ((1u << a) - 1);
    x = full << a;
    log2 = 0;
    for (int e = int(a) - 1; e >= 0; e--) {
        if (rem & (1u << e)) {
            if (k == 0) {
                log2 = uint32_t(e);
                return;
            }
            k--;
            x += 1u << e;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_tile_index(FrameDesc d, uint32_t* __restrict__ tile_off,
                                                     prr_dev_status* __restrict__ st) {
    __shared__ uint64_t warp_tot[32];
    __shared__ uint32_t red_max[32], red_min[32];
    const uint32_t T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t n = d.ntiles;
    const uint32_t chunk = (n + T - 1) / T;
    const uint32_t i0 = min(tid * chunk, n), i1 = min(i0 + chunk, n);
    uint64_t local = 0;
    for (uint32_t i = i0; i < i1; i++) local += be16_at(d.words, d.table_off + 2 * i);
    const uint64_t incl = warp_incl_scan_u64(local, lane);
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = T / 32;
        uint64_t v = lane < nw ? warp_tot[lane] : 0;
        const uint64_t wi = warp_incl_scan_u64(v, lane);
        if (lane < nw) warp_tot[lane] = wi - v;
    }
    __syncthreads();
    uint64_t off = uint64_t(d.table_off) + 2ull * n + warp_tot[warp] + (incl - local);
    uint32_t maxq = 0, oob = NO_TILE;
    for (uint32_t i = i0; i < i1; i++) {
        const uint32_t size = be16_at(d.words, d.table_off + 2 * i);
        // The byte after the tile start, even for a tile too short to hold
        // it (src/decoder.rs:109-110).
        if (off + 1 < d.len) maxq = max(maxq, byte_at(d.words, uint32_t(off + 1)));
        if (off + size > d.len) oob = min(oob, i);
        tile_off[i] = uint32_t(off < 0xFFFFFFFFull ? off : 0xFFFFFFFFull);
        off += size;
    }
    if (i1 == n && i0 < n) tile_off[n] = uint32_t(off < 0xFFFFFFFFull ? off : 0xFFFFFFFFull);
    // Block reductions: largest qscale byte, first out-of-bounds tile.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        maxq = max(maxq, __shfl_xor_sync(0xFFFFFFFFu, maxq, o));
        oob = min(oob, __shfl_xor_sync(0xFFFFFFFFu, oob, o));
    }
    if (lane == 0) {
        red_max[warp] = maxq;
        red_min[warp] = oob;
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = T / 32;
        maxq = lane < nw ? red_max[lane] : 0;
        oob = lane < nw ? red_min[lane] : NO_TILE;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            maxq = max(maxq, __shfl_xor_sync(0xFFFFFFFFu, maxq, o));
            oob = min(oob, __shfl_xor_sync(0xFFFFFFFFu, oob, o));
        }
        if (lane == 0) {
            st->oob_tile = oob;
            st->max_qscale = maxq;
            st->n_skipped = 0;
            st->error = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Segment decode, shared by the full and reduced kernels.

constexpr int kThreads = 256;
constexpr int kCoefStride = 72;   // int16 per block: 16-byte aligned rows, conflict-free loads
constexpr int kRowStride = 65;    // 32-bit words per block in the row buffer

struct SegTile {
    uint32_t soff[4], slen[4];
    uint32_t x_rel;  // first square relative to the segment
    uint32_t log2;
    uint32_t qscale;
    uint32_t valid;
};

struct SegShared {
    CodeTables T;
    SegTile tiles[16];
    uint8_t sq_valid[16];
    uint8_t qmat[64];
    uint32_t ntiles;
    __align__(16) int16_t coef[64 * kCoefStride];  // [square * 4 + stream][72]
    __align__(16) uint32_t rowbuf[64 * kRowStride];  // row-pass output, f32 or int32 bits
};

// Parse this segment's tiles and zero the coefficient buffer. `streams_mask`
// selects the streams to be decoded; returns the number of 16-sensel columns
// (squares) of the segment.
__device__ __forceinline__ uint32_t seg_setup(SegShared& S, const FrameDesc& d,
                                              const uint32_t* __restrict__ tile_off,
                                              prr_dev_status* st, uint32_t* skipped,
                                              uint32_t seg, uint32_t trow) {
    const uint32_t tid = threadIdx.x;
    load_tables(&S.T);
    if (tid < 16) reinterpret_cast<uint32_t*>(S.qmat)[tid] = reinterpret_cast<const uint32_t*>(d.qmat)[tid];
    {
        uint4* c = reinterpret_cast<uint4*>(S.coef);
        for (uint32_t i = tid; i < 64 * kCoefStride * 2 / 16; i += kThreads) c[i] = make_uint4(0, 0, 0, 0);
    }
    const uint32_t sq0 = seg * 16;
    const uint32_t nsq = min(16u, d.columns - sq0);
    if (tid < 32) {
        const uint32_t a = d.alignment;
        const uint32_t fullsq = (d.columns >> a) << a;
        const uint32_t j0 = sq0 < fullsq ? (sq0 >> a) : (d.columns >> a);
        const uint32_t j = j0 + tid;
        uint32_t x = 0, log2 = 0;
        bool here = false;
        if (tid < 16 && j < d.tiles_per_row) {
            tile_geom(j, d.columns, a, x, log2);
            here = x < sq0 + nsq;
        }
        const uint32_t count = __popc(__ballot_sync(0xFFFFFFFFu, here));
        if (tid == 0) S.ntiles = count;
        if (here) {
            SegTile t;
            const uint32_t idx = trow * d.tiles_per_row + j;
            const uint32_t off = tile_off[idx];
            const uint32_t end = tile_off[idx + 1];
            const bool in_bounds = off <= end && end <= d.len;
            const uint32_t size = end - off;
            bool valid = false;
            if (in_bounds && size >= 8) {
                const uint32_t header_len = byte_at(d.words, off) >> 3;
                const uint32_t qscale = byte_at(d.words, off + 1);
                const uint32_t s0 = be16_at(d.words, off + 2);
                const uint32_t s1 = be16_at(d.words, off + 4);
                const uint32_t s2 = be16_at(d.words, off + 6);
                const uint32_t used = header_len + s0 + s1 + s2;
                valid = header_len >= 8 && qscale != 0 && s0 != 0 && s1 != 0 && s2 != 0 && used < size;
                t.qscale = qscale;
                t.soff[0] = off + header_len;
                t.soff[1] = t.soff[0] + s0;
                t.soff[2] = t.soff[1] + s1;
                t.soff[3] = t.soff[2] + s2;
                t.slen[0] = s0;
                t.slen[1] = s1;
                t.slen[2] = s2;
                t.slen[3] = size - used;
            }
            if (in_bounds && !valid) {
                const uint32_t k = atomicAdd(&st->n_skipped, 1u);
                skipped[k] = idx;
            }
            t.x_rel = x - sq0;
            t.log2 = log2;
            t.valid = valid ? 1u : 0u;
            S.tiles[tid] = t;
            for (uint32_t q = 0; q < (1u << log2); q++) S.sq_valid[t.x_rel + q] = valid ? 1 : 0;
        }
    }
    __syncthreads();
    return nsq;
}

// Entropy-decode stream (tile, s) of the segment into shared memory,
// dequantized (src/decoder.rs:283-284, src/idct.rs:41-43).
__device__ __forceinline__ void seg_decode_stream(SegShared& S, const FrameDesc& d, uint32_t tile,
                                                  uint32_t s, uint32_t log2_coefs,
                                                  prr_dev_status* st) {
    const SegTile& t = S.tiles[tile];
    if (!t.valid) return;
    const uint32_t qscale = t.qscale;
    const uint32_t lc = log2_coefs;
    const uint32_t hl = lc >> 1;
    int16_t* base = S.coef + (t.x_rel * 4 + s) * kCoefStride;
    const uint8_t* qm = S.qmat;
    auto store = [&](uint32_t idx, int16_t v) {
        const uint32_t b = idx >> lc;
        const uint32_t p = idx & ((1u << lc) - 1);
        const uint32_t qi = ((p >> hl) << 3) | (p & ((1u << hl) - 1));
        base[b * 4 * kCoefStride + p] = dequantize(v, int32_t(qm[qi]) * int32_t(qscale));
    };
    if (!decode_component(d.words, t.soff[s], t.slen[s], t.log2, lc, S.T, store))
        atomicOr(&st->error, 1u);
}

template <int IDCT>
__global__ void __launch_bounds__(kThreads) k_decode_full(FrameDesc d, const uint32_t* __restrict__ tile_off,
                                                         prr_dev_status* __restrict__ st,
                                                         uint32_t* __restrict__ skipped,
                                                         uint16_t* __restrict__ out) {
    __shared__ SegShared S;
    const uint32_t tid = threadIdx.x;
    const uint32_t seg = blockIdx.x, trow = blockIdx.y;
    const uint32_t nsq = seg_setup(S, d, tile_off, st, skipped, seg, trow);
    // Entropy decoding: one thread per component stream.
    if (tid < 4 * S.ntiles) seg_decode_stream(S, d, tid >> 2, tid & 3, 6, st);
    __syncthreads();
    // Row pass: task = row * 64 + block; a warp shares one row (and its
    // table set), 32 blocks side by side.
    for (uint32_t task = tid; task < 512; task += kThreads) {
        const uint32_t row = task >> 6, blk = task & 63, sq = blk >> 2;
        if (sq >= nsq || !S.sq_valid[sq]) continue;
        const uint4 raw = *reinterpret_cast<const uint4*>(S.coef + blk * kCoefStride + row * 8);
        const int16_t* x = reinterpret_cast<const int16_t*>(&raw);
        uint32_t* dst = S.rowbuf + blk * kRowStride + row * 8;
        if (IDCT == PRR_IDCT_APPLE) {
            float y[8];
            apple_row(x, int(row), y);
#pragma unroll
            for (int k = 0; k < 8; k++) dst[k] = __float_as_uint(y[k]);
        } else {
            int32_t y[8];
            ffmpeg_row(x, y);
#pragma unroll
            for (int k = 0; k < 8; k++) dst[k] = uint32_t(y[k]);
        }
    }
    __syncthreads();
    // Column pass, writing code values onto the Bayer phase of each stream
    // (src/decoder.rs:293-303) in a [16 rows][256 sensels] staging tile that
    // reuses the coefficient buffer.
    uint16_t* stage = reinterpret_cast<uint16_t*>(S.coef);
    __syncthreads();
    uint16_t vals[2][8];
    uint32_t tasks[2];
    int ntask = 0;
    for (uint32_t task = tid; task < 512; task += kThreads) {
        const uint32_t col = task >> 6, blk = task & 63, sq = blk >> 2;
        tasks[ntask] = task;
        if (sq < nsq && S.sq_valid[sq]) {
            const uint32_t* src = S.rowbuf + blk * kRowStride + col;
            if (IDCT == PRR_IDCT_APPLE) {
                float r[8];
#pragma unroll
                for (int i = 0; i < 8; i++) r[i] = __uint_as_float(src[i * 8]);
                apple_col(r, vals[ntask]);
            } else {
                int32_t r[8];
#pragma unroll
                for (int i = 0; i < 8; i++) r[i] = int32_t(src[i * 8]);
                ffmpeg_col(r, vals[ntask]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) vals[ntask][i] = 0;
        }
        ntask++;
    }
    // The staging tile aliases the coefficients, which the row pass has
    // consumed: every thread is past it once this barrier is crossed.
    __syncthreads();
    for (int k = 0; k < ntask; k++) {
        const uint32_t task = tasks[k];
        const uint32_t col = task >> 6, blk = task & 63, sq = blk >> 2, s = blk & 3;
        if (sq >= nsq) continue;
        const uint32_t pr = d.phase[s] >> 1, pc = d.phase[s] & 1;
#pragma unroll
        for (int i = 0; i < 8; i++) stage[(2 * i + pr) * 256 + sq * 16 + 2 * col + pc] = vals[k][i];
    }
    __syncthreads();
    // Whole rows of the segment, 16 bytes at a time.
    const uint32_t vec_per_row = nsq * 2;
    for (uint32_t t = tid; t < 16 * vec_per_row; t += kThreads) {
        const uint32_t r = t / vec_per_row, k = t - r * vec_per_row;
        const uint4 v = *reinterpret_cast<const uint4*>(stage + r * 256 + k * 8);
        uint16_t* dst = out + size_t(trow * 16 + r) * d.coded_w + seg * 256 + k * 8;
        *reinterpret_cast<uint4*>(dst) = v;
    }
}

// Reduced-resolution decode (src/reduced.rs:217-273): red from stream 3,
// green from stream 0 (averaged with stream 1 for Greens::Average), blue
// from stream 2, through the 8x8, 4x4 or 2x2 transform and the curve.
template <int SHIFT>
__global__ void __launch_bounds__(kThreads) k_decode_reduced(FrameDesc d, int greens,
                                                            const uint32_t* __restrict__ tile_off,
                                                            prr_dev_status* __restrict__ st,
                                                            uint32_t* __restrict__ skipped,
                                                            uint16_t* __restrict__ out) {
    __shared__ SegShared S;
    __shared__ uint32_t c0[8], cd[8];
    constexpr uint32_t LC = SHIFT == 1 ? 6 : (SHIFT == 2 ? 4 : 2);
    constexpr uint32_t SIDE = 16 >> SHIFT;  // output pixels per square side
    const uint32_t tid = threadIdx.x;
    const uint32_t seg = blockIdx.x, trow = blockIdx.y;
    if (tid < 8) {
        c0[tid] = d.curve_c0[tid];
        cd[tid] = d.curve_delta[tid];
    }
    const uint32_t nsq = seg_setup(S, d, tile_off, st, skipped, seg, trow);
    {
        const uint32_t s = tid & 3;
        if (tid < 4 * S.ntiles && (s != 1 || greens)) seg_decode_stream(S, d, tid >> 2, s, LC, st);
    }
    __syncthreads();
    // Code values per block in `vals` ([block][64] u16), aliasing the row
    // buffer's tail is not possible, so they reuse the coefficient buffer
    // after the row pass.
    uint16_t* vals = reinterpret_cast<uint16_t*>(S.coef);
    if (SHIFT == 1) {
        for (uint32_t task = tid; task < 512; task += kThreads) {
            const uint32_t row = task >> 6, blk = task & 63, sq = blk >> 2;
            if (sq >= nsq || !S.sq_valid[sq]) continue;
            const uint4 raw = *reinterpret_cast<const uint4*>(S.coef + blk * kCoefStride + row * 8);
            float y[8];
            apple_row(reinterpret_cast<const int16_t*>(&raw), int(row), y);
#pragma unroll
            for (int k = 0; k < 8; k++) S.rowbuf[blk * kRowStride + row * 8 + k] = __float_as_uint(y[k]);
        }
        __syncthreads();
        for (uint32_t task = tid; task < 512; task += kThreads) {
            const uint32_t col = task >> 6, blk = task & 63, sq = blk >> 2;
            if (sq >= nsq || !S.sq_valid[sq]) continue;
            float r[8];
#pragma unroll
            for (int i = 0; i < 8; i++) r[i] = __uint_as_float(S.rowbuf[blk * kRowStride + i * 8 + col]);
            uint16_t v[8];
            apple_col(r, v);
#pragma unroll
            for (int i = 0; i < 8; i++) S.rowbuf[blk * kRowStride + i * 8 + col] = v[i];
        }
        __syncthreads();
        for (uint32_t i = tid; i < 64 * 64; i += kThreads)
            vals[i] = uint16_t(S.rowbuf[(i >> 6) * kRowStride + (i & 63)]);
    } else if (SHIFT == 2) {
        for (uint32_t task = tid; task < 256; task += kThreads) {
            const uint32_t row = task >> 6, blk = task & 63, sq = blk >> 2;
            if (sq >= nsq || !S.sq_valid[sq]) continue;
            const uint2 raw = *reinterpret_cast<const uint2*>(S.coef + blk * kCoefStride + row * 4);
            float y[4];
            apple_row4(reinterpret_cast<const int16_t*>(&raw), int(row), y);
#pragma unroll
            for (int k = 0; k < 4; k++) S.rowbuf[blk * kRowStride + row * 4 + k] = __float_as_uint(y[k]);
        }
        __syncthreads();
        for (uint32_t task = tid; task < 256; task += kThreads) {
            const uint32_t col = task >> 6, blk = task & 63, sq = blk >> 2;
            if (sq >= nsq || !S.sq_valid[sq]) continue;
            float r[4];
#pragma unroll
            for (int i = 0; i < 4; i++) r[i] = __uint_as_float(S.rowbuf[blk * kRowStride + i * 4 + col]);
            uint16_t v[4];
            apple_col4(r, v);
#pragma unroll
            for (int i = 0; i < 4; i++) S.rowbuf[blk * kRowStride + i * 4 + col] = v[i];
        }
        __syncthreads();
        for (uint32_t i = tid; i < 64 * 16; i += kThreads)
            vals[(i >> 4) * 64 + (i & 15)] = uint16_t(S.rowbuf[(i >> 4) * kRowStride + (i & 15)]);
    } else {
        for (uint32_t blk = tid; blk < 64; blk += kThreads) {
            const uint32_t sq = blk >> 2;
            if (sq >= nsq || !S.sq_valid[sq]) continue;
            const int16_t* c = S.coef + blk * kCoefStride;
            uint16_t v[4];
            apple_2x2(c[0], c[1], c[2], c[3], v);
#pragma unroll
            for (int i = 0; i < 4; i++) S.rowbuf[blk * kRowStride + i] = v[i];
        }
        __syncthreads();
        for (uint32_t i = tid; i < 64 * 4; i += kThreads)
            vals[(i >> 2) * 64 + (i & 3)] = uint16_t(S.rowbuf[(i >> 2) * kRowStride + (i & 3)]);
    }
    __syncthreads();
    // Linearize, average the greens, interleave RGB (src/reduced.rs:256-270).
    const uint32_t stride = d.coded_w >> SHIFT;
    const uint32_t npx = nsq * SIDE;
    for (uint32_t t = tid; t < SIDE * npx; t += kThreads) {
        const uint32_t i = t / npx, px = t - i * npx;
        const uint32_t sq = px / SIDE, j = px - sq * SIDE;
        uint16_t rgb[3] = {0, 0, 0};
        if (S.sq_valid[sq]) {
            const uint32_t at = i * SIDE + j;
            rgb[0] = uint16_t(curve_apply(c0, cd, vals[(sq * 4 + 3) * 64 + at]));
            uint32_t g = curve_apply(c0, cd, vals[(sq * 4 + 0) * 64 + at]);
            if (greens) g = (g + curve_apply(c0, cd, vals[(sq * 4 + 1) * 64 + at]) + 1) >> 1;
            rgb[1] = uint16_t(g);
            rgb[2] = uint16_t(curve_apply(c0, cd, vals[(sq * 4 + 2) * 64 + at]));
        }
        uint16_t* dst = out + (size_t(trow * SIDE + i) * stride + seg * 16 * SIDE + px) * 3;
        dst[0] = rgb[0];
        dst[1] = rgb[1];
        dst[2] = rgb[2];
    }
}

// ---------------------------------------------------------------------------
// Diagnostics: transforms of raw blocks, entropy decode of raw streams.
__global__ void k_transform_blocks(int kind, const int16_t* __restrict__ coefs,
                                   const int16_t* __restrict__ q, uint16_t* __restrict__ out, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int16_t* qq = q + 64 * i;
    if (kind == 0 || kind == 1) {
        const int16_t* c = coefs + 64 * i;
        int16_t dq[64];
        for (int k = 0; k < 64; k++) dq[k] = dequantize(c[k], qq[k]);
        uint16_t* o = out + 64 * i;
        if (kind == 0) {
            float rows[8][8];
            for (int r = 0; r < 8; r++) apple_row(dq + 8 * r, r, rows[r]);
            for (int col = 0; col < 8; col++) {
                float cc[8];
                uint16_t v[8];
                for (int r = 0; r < 8; r++) cc[r] = rows[r][col];
                apple_col(cc, v);
                for (int r = 0; r < 8; r++) o[8 * r + col] = v[r];
            }
        } else {
            int32_t rows[8][8];
            for (int r = 0; r < 8; r++) ffmpeg_row(dq + 8 * r, rows[r]);
            for (int col = 0; col < 8; col++) {
                int32_t cc[8];
                uint16_t v[8];
                for (int r = 0; r < 8; r++) cc[r] = rows[r][col];
                ffmpeg_col(cc, v);
                for (int r = 0; r < 8; r++) o[8 * r + col] = v[r];
            }
        }
    } else if (kind == 2) {
        const int16_t* c = coefs + 16 * i;
        int16_t dq[16];
        for (int r = 0; r < 4; r++)
            for (int k = 0; k < 4; k++) dq[4 * r + k] = dequantize(c[4 * r + k], qq[8 * r + k]);
        float rows[4][4];
        for (int r = 0; r < 4; r++) apple_row4(dq + 4 * r, r, rows[r]);
        uint16_t* o = out + 16 * i;
        for (int col = 0; col < 4; col++) {
            float cc[4];
            uint16_t v[4];
            for (int r = 0; r < 4; r++) cc[r] = rows[r][col];
            apple_col4(cc, v);
            for (int r = 0; r < 4; r++) o[4 * r + col] = v[r];
        }
    } else {
        const int16_t* c = coefs + 4 * i;
        apple_2x2(dequantize(c[0], qq[0]), dequantize(c[1], qq[1]), dequantize(c[2], qq[8]),
                  dequantize(c[3], qq[9]), out + 4 * i);
    }
}

__global__ void k_decode_components(const uint32_t* __restrict__ words, const uint32_t* __restrict__ off,
                                    const uint32_t* __restrict__ len, size_t n, int log2_blocks,
                                    int log2_coefs, int16_t* __restrict__ coefs) {
    __shared__ CodeTables T;
    load_tables(&T);
    __syncthreads();
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t codes = 1u << (log2_blocks + log2_coefs);
    int16_t* dst = coefs + i * codes;
    for (uint32_t k = 0; k < codes; k++) dst[k] = 0;
    decode_component(words, off[i], len[i], uint32_t(log2_blocks), uint32_t(log2_coefs), T,
                     [&](uint32_t idx, int16_t v) { dst[idx] = v; });
}

// ---------------------------------------------------------------------------
// Launchers.

FrameDesc make_frame_desc(const prr_frame_info& info, const uint8_t* dev_packet) {
    FrameDesc d{};
    d.words = reinterpret_cast<const uint32_t*>(dev_packet);
    d.len = uint32_t(info.packet_len);
    d.table_off = uint32_t(info.table_offset);
    d.ntiles = info.ntiles;
    d.tiles_per_row = info.tiles_per_row;
    d.tile_rows = info.tile_rows;
    d.columns = info.coded_width / 16;
    d.alignment = info.header.alignment;
    d.coded_w = info.coded_width;
    d.segs_per_row = (d.columns + 15) / 16;
    // Stream s lands on phase (1-r, c), (r, 1-c), (1-r, 1-c), (r, c) for the
    // red sensel at (r, c) (src/header.rs:64-82).
    const uint32_t p = info.header.bayer_pattern & 3;
    const uint32_t r = (p == 2 || p == 3) ? 1 : 0, c = (p == 1 || p == 3) ? 1 : 0;
    d.phase[0] = ((1 - r) << 1) | c;
    d.phase[1] = (r << 1) | (1 - c);
    d.phase[2] = ((1 - r) << 1) | (1 - c);
    d.phase[3] = (r << 1) | c;
    for (int s = 0; s < 8; s++) {
        const uint32_t c0 = info.header.curve[s];
        const uint32_t c1 = s < 7 ? info.header.curve[s + 1] : 65536u;
        d.curve_c0[s] = c0;
        d.curve_delta[s] = (c1 - c0) & 0xFFFF;
    }
    for (int i = 0; i < 64; i++) d.qmat[i] = info.header.quant_matrix[i];
    return d;
}

cudaError_t launch_tile_index(const FrameDesc& d, uint32_t* tile_off, prr_dev_status* st, cudaStream_t s) {
    k_tile_index<<<1, 1024, 0, s>>>(d, tile_off, st);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_full(const FrameDesc& d, int idct, const uint32_t* tile_off, prr_dev_status* st,
                               uint32_t* skipped, uint16_t* out, cudaStream_t s) {
    dim3 grid(d.segs_per_row, d.tile_rows);
    if (idct == PRR_IDCT_FFMPEG)
        k_decode_full<PRR_IDCT_FFMPEG><<<grid, kThreads, 0, s>>>(d, tile_off, st, skipped, out);
    else
        k_decode_full<PRR_IDCT_APPLE><<<grid, kThreads, 0, s>>>(d, tile_off, st, skipped, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_reduced(const FrameDesc& d, int shift, int greens, const uint32_t* tile_off,
                                  prr_dev_status* st, uint32_t* skipped, uint16_t* out, cudaStream_t s) {
    dim3 grid(d.segs_per_row, d.tile_rows);
    if (shift == 1)
        k_decode_reduced<1><<<grid, kThreads, 0, s>>>(d, greens, tile_off, st, skipped, out);
    else if (shift == 2)
        k_decode_reduced<2><<<grid, kThreads, 0, s>>>(d, greens, tile_off, st, skipped, out);
    else
        k_decode_reduced<3><<<grid, kThreads, 0, s>>>(d, greens, tile_off, st, skipped, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_transform_blocks(int kind, const int16_t* coefs, const int16_t* q, uint16_t* out,
                                    size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = unsigned((n + 127) / 128);
    k_transform_blocks<<<blocks, 128, 0, s>>>(kind, coefs, q, out, n);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_components(const uint8_t* packet, const uint32_t* off, const uint32_t* len,
                                     size_t n, int log2_blocks, int log2_coefs, int16_t* coefs,
                                     cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = unsigned((n + 63) / 64);
    k_decode_components<<<blocks, 64, 0, s>>>(reinterpret_cast<const uint32_t*>(packet), off, len, n,
                                              log2_blocks, log2_coefs, coefs);
    count_launch();
    return cudaGetLastError();
}

}  // namespace prr
