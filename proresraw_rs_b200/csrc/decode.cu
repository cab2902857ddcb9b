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

#include <algorithm>
#include <cstddef>

#include "device_common.cuh"
#include "kernels.h"

namespace prr {

namespace {

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
__device__ __forceinline__ void tile_index_body(const FrameDesc& d, uint32_t* __restrict__ tile_off,
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

__global__ void __launch_bounds__(1024) k_tile_index(FrameDesc d, uint32_t* __restrict__ tile_off,
                                                     prr_dev_status* __restrict__ st) {
    tile_index_body(d, tile_off, st);
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
    uint32_t first_j;  // index within the tile row of the segment's first tile
    uint32_t sq0;      // first 16-sensel column of the segment
    uint32_t c0[8], cd[8];  // linearization curve (reduced decode)
    __align__(16) int16_t coef[64 * kCoefStride];  // [square * 4 + stream][72]
    __align__(16) uint32_t rowbuf[64 * kRowStride];  // row-pass output, f32 or int32 bits
};

// First entry of the (position, value) list of stream s of the tile whose
// first square is column `sq_x` of tile row `trow`: the tile's squares own
// 4 << log2_coefs entries each, so every tile's four lists are disjoint.
__device__ __forceinline__ uint32_t stream_list_base(const FrameDesc& d, uint32_t trow, uint32_t sq_x,
                                                     uint32_t log2, uint32_t s, uint32_t lc) {
    return ((trow * d.columns + sq_x) * 4 + (s << log2)) << lc;
}

// Parse this segment's tiles and zero the coefficient buffer; returns the
// number of 16-sensel columns (squares) of the segment. A CTA that keeps
// its code tables across segments passes load_code_tables = false.
__device__ __forceinline__ uint32_t seg_setup(SegShared& S, const FrameDesc& d,
                                              const uint32_t* __restrict__ tile_off,
                                              prr_dev_status* st, uint32_t* skipped,
                                              uint32_t seg, uint32_t trow, bool load_code_tables = true) {
    const uint32_t tid = threadIdx.x;
    if (load_code_tables) load_tables(&S.T);
    if (tid < 16) reinterpret_cast<uint32_t*>(S.qmat)[tid] = reinterpret_cast<const uint32_t*>(d.qmat)[tid];
    if (tid < 8) {
        S.c0[tid] = d.curve_c0[tid];
        S.cd[tid] = d.curve_delta[tid];
    }
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
        if (tid == 0) {
            S.ntiles = count;
            S.first_j = j0;
            S.sq0 = sq0;
        }
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
    bool revisited = false;
    if (!decode_component(GlobalWords{d.words}, t.soff[s], t.slen[s], t.log2, lc, S.T, store, revisited) && st)
        atomicOr(&st->error, 1u);
}

// Fill the segment's shared coefficients from the lists k_entropy wrote:
// one warp per stream, lanes over the list's (position, value) entries.
// A stream whose zero run wrapped back over stored positions may hold a
// position twice; it is replayed in order by one lane so the later value
// wins, as on the host. COHERENT reads the counts and lists through L2 only,
// for lists another CTA wrote during the same launch.
template <bool COHERENT = false>
__device__ __forceinline__ void seg_scatter(SegShared& S, const FrameDesc& d, uint32_t trow,
                                            uint32_t log2_coefs, bool second_green, prr_dev_status* st) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lc = log2_coefs;
    const uint32_t first_tile = trow * d.tiles_per_row + S.first_j;
    for (uint32_t k = warp; k < 4 * S.ntiles; k += kThreads / 32) {
        const uint32_t t = k >> 2, s = k & 3;
        const SegTile& tl = S.tiles[t];
        if (!tl.valid || (s == 1 && !second_green)) continue;
        const uint32_t g = (first_tile + t) * 4 + s;
        const uint32_t cnt = COHERENT ? __ldcg(d.counts + g) : d.counts[g];
        const uint32_t n = cnt & 0x7FFFFFFFu;
        const uint32_t* list = d.pairs + stream_list_base(d, trow, tl.x_rel + S.sq0, tl.log2, s, lc);
        int16_t* base = S.coef + (tl.x_rel * 4 + s) * kCoefStride;
        // Entry: interleaved position n << 16 | raw 16-bit value. Placement
        // (src/coefficients.rs:86-88) and dequantization (src/idct.rs:41-43)
        // happen here, off the entropy decoder's serial chain.
        const uint8_t* scan = lc == 6 ? S.T.scan : (lc == 4 ? S.T.scan4 : S.T.scan2);
        const uint32_t hl = lc >> 1, mask = (1u << tl.log2) - 1;
        const int32_t qscale = int32_t(tl.qscale);
        auto put = [&](uint32_t e) {
            const uint32_t nn = e >> 16;
            const uint32_t p = scan[nn >> tl.log2];
            const uint32_t qi = ((p >> hl) << 3) | (p & ((1u << hl) - 1));
            base[(nn & mask) * 4 * kCoefStride + p] =
                dequantize(int16_t(e & 0xFFFF), int32_t(S.qmat[qi]) * qscale);
        };
        if (cnt >> 31) {
            // Positions revisited (and possibly more entries than the list
            // holds): decode the stream again here, in order.
            if (lane == 0) seg_decode_stream(S, d, t, s, lc, st);
        } else {
            for (uint32_t i = lane; i < n; i += 32) put(COHERENT ? __ldcg(list + i) : __ldg(list + i));
        }
    }
}

// Full-resolution decode of segment `seg` of tile row `trow` (the CTA's
// work in k_decode_full and the batch kernel). PERSIST: the CTA keeps its
// code tables and the lists come from the same launch.
template <int IDCT, bool SPLIT, bool PERSIST>
__device__ __forceinline__ void full_segment(SegShared& S, const FrameDesc& d, uint32_t seg, uint32_t trow,
                                             const uint32_t* __restrict__ tile_off, prr_dev_status* st,
                                             uint32_t* skipped, uint16_t* __restrict__ out) {
    const uint32_t tid = threadIdx.x;
    const uint32_t nsq = seg_setup(S, d, tile_off, st, skipped, seg, trow, !PERSIST);
    if (SPLIT) {
        seg_scatter<PERSIST>(S, d, trow, 6, true, st);
    } else {
        // Entropy decoding in the CTA: one thread per component stream.
        if (tid < 4 * S.ntiles) seg_decode_stream(S, d, tid >> 2, tid & 3, 6, st);
    }
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
        // In the batch kernel the outputs are not read again soon: streaming
        // stores (evict first) keep L2 for the coefficient lists the other
        // segments read back. The single-frame decode keeps them cached for
        // the develop that follows.
        if (PERSIST)
            __stcs(reinterpret_cast<uint4*>(dst), v);
        else
            *reinterpret_cast<uint4*>(dst) = v;
    }
}

template <int IDCT, bool SPLIT>
__global__ void __launch_bounds__(kThreads) k_decode_full(FrameDesc d, const uint32_t* __restrict__ tile_off,
                                                         prr_dev_status* __restrict__ st,
                                                         uint32_t* __restrict__ skipped,
                                                         uint16_t* __restrict__ out) {
    __shared__ SegShared S;
    full_segment<IDCT, SPLIT, false>(S, d, blockIdx.x, blockIdx.y, tile_off, st, skipped, out);
}

// Reduced-resolution decode (src/reduced.rs:217-273): red from stream 3,
// green from stream 0 (averaged with stream 1 for Greens::Average), blue
// from stream 2, through the 8x8, 4x4 or 2x2 transform and the curve.
template <int SHIFT, bool SPLIT, bool PERSIST>
__device__ __forceinline__ void reduced_segment(SegShared& S, const FrameDesc& d, int greens, uint32_t seg,
                                                uint32_t trow, const uint32_t* __restrict__ tile_off,
                                                prr_dev_status* st, uint32_t* skipped,
                                                uint16_t* __restrict__ out) {
    constexpr uint32_t LC = SHIFT == 1 ? 6 : (SHIFT == 2 ? 4 : 2);
    constexpr uint32_t SIDE = 16 >> SHIFT;  // output pixels per square side
    const uint32_t tid = threadIdx.x;
    const uint32_t* c0 = S.c0;
    const uint32_t* cd = S.cd;
    const uint32_t nsq = seg_setup(S, d, tile_off, st, skipped, seg, trow, !PERSIST);
    if (SPLIT) {
        seg_scatter<PERSIST>(S, d, trow, LC, greens != 0, st);
    } else {
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
        if (PERSIST) {
            __stcs(dst, rgb[0]);
            __stcs(dst + 1, rgb[1]);
            __stcs(dst + 2, rgb[2]);
        } else {
            dst[0] = rgb[0];
            dst[1] = rgb[1];
            dst[2] = rgb[2];
        }
    }
}

template <int SHIFT, bool SPLIT>
__global__ void __launch_bounds__(kThreads) k_decode_reduced(FrameDesc d, int greens,
                                                            const uint32_t* __restrict__ tile_off,
                                                            prr_dev_status* __restrict__ st,
                                                            uint32_t* __restrict__ skipped,
                                                            uint16_t* __restrict__ out) {
    __shared__ SegShared S;
    reduced_segment<SHIFT, SPLIT, false>(S, d, greens, blockIdx.x, blockIdx.y, tile_off, st, skipped, out);
}

// ---------------------------------------------------------------------------
// Entropy decoding apart from the transform: one thread per component
// stream, streams in frame order (tile-major), so a warp decodes the 32
// streams of 8 neighbouring tiles side by side. Each thread parses its tile's
// header (Tile::parse, src/tile.rs:126-153) and appends every coefficient
// its stream stores as an (interleaved position n << 16 | raw 16-bit value)
// entry to its stream's list, four entries per 16-byte store; counts[g]
// gets the entry count. Placement and dequantization are left to the
// transform kernel so that the serial symbol chain stays short. A stream
// whose zero run wrapped back over stored positions (malformed input only)
// gets bit 31 instead and is decoded again, in order, by the transform
// kernel; its list is never written past its capacity. Invalid tiles are
// left to the transform kernel, which records them.
//
// The symbol loop is decode_component_reduced (src/coefficients.rs:37-146)
// as a state machine, one symbol per iteration; the codebook lookups of all
// states are issued together and the state's own update picks its result.
// The 25 distinct codebook parameter sets of the format (src/codebook.rs:25-55).
// The entropy kernel names a codebook by its index here.
constexpr int kCodebooks = 25;
__constant__ uint16_t c_cb_params[kCodebooks] = {0x2BC, 0x064, 0x010, 0x021, 0x032, 0x033, 0x044,
                                                 0x076, 0x031, 0x000, 0x211, 0x111, 0x222, 0x122,
                                                 0x233, 0x133, 0x244, 0x355, 0x166, 0x200, 0x100,
                                                 0x011, 0x022, 0x042, 0x433};
constexpr uint32_t kIdFirstDc = 0, kIdDcReset = 1, kIdAcInitial = 8, kIdRnInitial = 9, kIdLnInitial = 23;

// Codeword decoding by table. For a view p with lz leading zeros, codeword()
// (src/bits.rs:116-134) is value = base + ((p << sh1) >> sh2) with a shift of
// 32 giving 0, and a length, all fixed by (codebook, lz):
//   Rice (lz <= s):  base = lz << r, sh1 = (lz + 1) & 31, sh2 = 32 - r,
//                    length r + 1 + lz;
//   exp-Golomb:      base = ((s + 1) << r) - (1 << e), sh1 = 0,
//                    sh2 = (32 - length) & 31, length 2 lz - s + e,
// in wrapping u32 arithmetic, over-long codewords included. One shared
// load replaces the arithmetic of the symbol loop's critical chain.
struct EntropyTables {
    uint2 cw[kCodebooks * 32];  // x: base, y: length | sh1 << 8 | sh2 << 16
    // Next codebook indices after an AC symbol v, at [min(v, 94)]: AC table
    // (bits 0-7, index min(v, 94)), LN (bits 8-15, min(v, 14)), RN (bits
    // 16-23, min(v, 27)) -- one lookup for the three tables.
    uint32_t nx[95];
    uint8_t dc[16];  // next DC codebook index, by clamped magnitude
};

__device__ __forceinline__ void build_entropy_tables(EntropyTables& E, const CodeTables& T) {
    auto id_of = [](uint32_t params) {
        uint32_t id = 0;
        for (int k = 0; k < kCodebooks; k++)
            if (c_cb_params[k] == params) id = uint32_t(k);
        return id;
    };
    for (uint32_t i = threadIdx.x; i < kCodebooks * 32; i += blockDim.x) {
        const uint32_t p = c_cb_params[i >> 5], lz = i & 31;
        const uint32_t s = p >> 8, e = (p >> 4) & 15, r = p & 15;
        uint32_t base, len, sh1, sh2;
        if (lz <= s) {
            base = lz << r;
            len = r + 1 + lz;
            sh1 = (lz + 1) & 31;
            sh2 = 32 - r;
        } else {
            len = 2 * lz - s + e;
            base = ((s + 1) << r) - (1u << e);
            sh1 = 0;
            sh2 = (32u - len) & 31;
        }
        E.cw[i] = make_uint2(base, len | (sh1 << 8) | (sh2 << 16));
    }
    for (uint32_t i = threadIdx.x; i < 95; i += blockDim.x)
        E.nx[i] = id_of(T.ac[i]) | (id_of(T.ln[min(i, 14u)]) << 8) | (id_of(T.rn[min(i, 27u)]) << 16);
    for (uint32_t i = threadIdx.x; i < 13; i += blockDim.x) E.dc[i] = uint8_t(id_of(T.dc[i]));
}

// Big-endian words of the packet for the entropy kernel: from global memory
// (swapped at load), or from the CTA's stage, swapped once when staged.
// Both are indexed by the packet's word index.
struct PacketWords {
    const uint32_t* w;
    __device__ __forceinline__ uint32_t be(uint32_t i) const { return bswap32(__ldg(w + i)); }
};
struct StagedWords {
    const uint32_t* w;
    uint32_t base;
    __device__ __forceinline__ uint32_t be(uint32_t i) const { return w[i - base]; }
};

// The bit reader of src/bits.rs:17-112 with a refill that every lane runs
// on every symbol, so that the refills of different lanes do not split the
// warp. BitReader::next_word returns whole aligned words while four bytes
// remain, then the partial tail, then zeros: here the tail is read once at
// set-up, so a refill is one aligned word (or the tail, or 0) selected by the
// byte position. It is ORed into the window only when the count of bits
// below the view goes negative, exactly as consume() does. Loads may touch
// the word after the stream's last byte, which both word sources provide
// (padded packet, padded stage).
template <class Src>
struct LeanReader {
    Src src;
    uint32_t pos, end, words_end, tail;
    uint64_t window;
    int32_t extra;

    // n = min(4, end - p) bytes at byte p, big-endian, zero-filled (set-up only).
    __device__ __forceinline__ uint32_t word_at(uint32_t p) const {
        const uint32_t k = p >> 2;
        const uint32_t hi = src.be(k), lo = src.be(k + 1);
        const uint32_t w = __funnelshift_l(lo, hi, (p & 3) * 8);
        const uint32_t n = min(4u, end - min(p, end));
        return n == 0 ? 0u : (w & (0xFFFFFFFFu << (32 - 8 * n)));
    }

    __device__ __forceinline__ void init(const Src& s, uint32_t off, uint32_t len) {
        // BitReader::new (src/bits.rs:44-76).
        src = s;
        end = off + len;
        uint32_t remaining = len;
        const uint32_t first = word_at(off);
        const uint32_t took = min(4u, remaining);
        pos = off + took;
        remaining -= took;
        uint32_t low = 0;
        extra = 0;
        const uint32_t to_boundary = (4 - (pos & 3)) & 3;
        if (to_boundary != 0 && to_boundary <= remaining) {
            low = word_at(pos) & (0xFFFFFFFFu << (32 - 8 * to_boundary));
            pos += to_boundary;
            remaining -= to_boundary;
            extra = int32_t(8 * to_boundary);
        }
        // Whole words while pos < words_end (pos is then 4-aligned), then
        // the tail of end - words_end < 4 bytes, then zeros.
        words_end = pos + 4 * (remaining / 4);
        tail = word_at(words_end);
        window = (uint64_t(first) << 32) | uint64_t(low);
    }

    __device__ __forceinline__ uint32_t top() const { return uint32_t(window >> 32); }

    // BitReader::consume (src/bits.rs:97-105).
    __device__ __forceinline__ void consume(uint32_t n) {
        const bool whole = pos < words_end;
        const uint32_t ww = src.be(pos >> 2);  // independent of n: issued early
        const uint32_t w = whole ? ww : (pos < end ? tail : 0u);
        const uint32_t adv = whole ? 4u : end - pos;
        window <<= (n & 63);
        extra = int32_t(uint32_t(extra) - n);
        const bool refill = extra < 0;
        const uint32_t shift = uint32_t(-int32_t(int8_t(extra))) & 63;
        window |= refill ? (uint64_t(w) << shift) : 0ull;
        pos += refill ? adv : 0u;
        extra += refill ? 32 : 0;
    }
};

// codeword() through the table: value, and the length in `len`.
__device__ __forceinline__ uint32_t table_codeword(const EntropyTables& E, uint32_t top, uint32_t cb,
                                                   uint32_t& len) {
    const uint2 ce = E.cw[(cb << 5) | __clz(top)];
    len = ce.y & 0xFF;
    return ce.x + __funnelshift_rc(top << ((ce.y >> 8) & 0xFF), 0u, ce.y >> 16);
}

template <uint32_t LC, class Src>
__device__ __forceinline__ uint32_t entropy_events(const Src& src, uint32_t off, uint32_t len,
                                                   uint32_t log2_blocks, const EntropyTables& T, uint32_t* list,
                                                   bool& revisited, bool& ok) {
    const uint32_t blocks = 1u << log2_blocks;
    const uint32_t codes = blocks << LC;
    LeanReader<Src> r;
    r.init(src, off, len);
    uint32_t cnt = 0, e0 = 0, e1 = 0, e2 = 0, e3 = 0;
    // Append the coefficient at interleaved position n (DCs are 0..blocks-1).
    auto append = [&](uint32_t n, uint32_t value) {
        e0 = e1;
        e1 = e2;
        e2 = e3;
        e3 = (n << 16) | (value & 0xFFFF);
        if ((cnt & 3) == 3) *reinterpret_cast<uint4*>(list + cnt - 3) = make_uint4(e0, e1, e2, e3);
        cnt++;
    };
    bool live = r.top() != 0;
    // DC: the sign-folded first value, then deltas with a running sign
    // (src/coefficients.rs:59-82).
    if (live) {
        uint32_t l;
        const uint32_t v = table_codeword(T, r.top(), kIdFirstDc, l);
        r.consume(l);
        const uint32_t odd = v & 1;
        int32_t dc = int32_t((((odd + v) >> 1) ^ (0u - odd)) + odd);
        append(0, uint32_t(dc));
        uint32_t dc_cb = kIdDcReset, sign = 0;
        for (uint32_t block = 1; block < blocks; block++) {
            if (r.top() == 0) {
                live = false;
                break;
            }
            const uint32_t s = table_codeword(T, r.top(), dc_cb, l);
            sign ^= s & 1;
            const uint32_t magnitude = ((s & 1) + s) >> 1;
            const int32_t delta = int32_t(((0u - sign) ^ magnitude) + sign);
            dc_cb = T.dc[min(magnitude, 12u)];
            sign = delta < 0 ? 1u : 0u;
            r.consume(l);
            dc = int32_t(uint32_t(dc) + uint32_t(delta));
            append(block, uint32_t(dc));
        }
    }
    // AC (src/coefficients.rs:105-145) as four states, updated with selects
    // so that lanes in different states run the same instructions: the
    // length of a non-zero run, a level inside the run, a zero run, the level
    // after a zero run.
    enum : uint32_t { RUN_LENGTH = 0, ZEROS = 1, LEVELS = 2, LEVEL = 3 };
    uint32_t state = RUN_LENGTH, cb = kIdLnInitial;
    uint32_t ac_cb = kIdAcInitial, rn_cb = kIdRnInitial, ln_cb = kIdLnInitial;
    uint32_t n = blocks, run = 0;
    uint32_t budget = 64u * (8u * len + 64u) + 4u * codes;
    while (live) {
        const uint32_t top = r.top();
        if (top == 0) break;  // end of component
        if (budget-- == 0) {
            ok = false;
            break;
        }
        uint32_t l;
        const uint32_t v = table_codeword(T, top, cb, l);
        const bool is_level = state >= LEVELS;
        const bool negative = int32_t(top << (l & 31)) < 0;
        r.consume(l + (is_level ? 1u : 0u));
        const uint32_t nx = T.nx[min(v, 94u)];
        const uint32_t ac_next = nx & 0xFF, ln_next = (nx >> 8) & 0xFF, rn_next = nx >> 16;
        if (is_level) {
            const uint32_t mag = (v + 1) & 0xFFFF;
            if (cnt < codes) append(n, negative ? (0u - mag) : mag);
        }
        const bool rl = state == RUN_LENGTH, zr = state == ZEROS, l1 = state == LEVEL;
        // A zero run is zeros + 1 long and wraps like the crate's u32.
        const uint32_t n_new = zr ? n + 1 + v : n + (is_level ? 1u : 0u);
        revisited |= zr && n_new < n;
        n = n_new;
        ac_cb = is_level ? ac_next : ac_cb;
        ln_cb = l1 ? ln_next : ln_cb;
        rn_cb = zr ? rn_next : rn_cb;
        run = rl ? v : (state == LEVELS ? run - 1 : run);
        if ((zr || is_level) && n >= codes) break;
        state = rl ? (v > 0 ? LEVELS : ZEROS) : zr ? LEVEL : l1 ? RUN_LENGTH : (run == 0 ? ZEROS : LEVELS);
        cb = state >= LEVELS ? ac_cb : (state == RUN_LENGTH ? ln_cb : rn_cb);
    }
    // Entries still in registers: the last cnt & 3 of e1..e3.
    const uint32_t rem = cnt & 3;
    if (rem >= 1) list[cnt - rem] = rem == 3 ? e1 : (rem == 2 ? e2 : e3);
    if (rem >= 2) list[cnt - rem + 1] = rem == 3 ? e2 : e3;
    if (rem >= 3) list[cnt - rem + 2] = e3;
    return cnt;
}

// Bytes of packet a k_entropy CTA stages in shared memory: its 32 tiles are
// contiguous in the packet, and a span this size covers tiles of up to 1 KB
// on average. Larger spans are read from global memory instead.
constexpr uint32_t kStageBytes = 32 * 1024;

// One component stream of a chunk: where its bytes and its list are.
struct StreamJob {
    bool valid;
    uint32_t g, s, trow, x, log2, soff, slen;
};

// Stream g of the frame (tile g / 4, component g % 4): Tile::parse
// (src/tile.rs:126-153) of its tile's header and the stream's span; not
// valid when there is nothing to decode (past the last tile, a second green
// a reduced decode does not average, an invalid tile -- left to the
// transform kernel, which records it).
template <uint32_t LC>
__device__ __forceinline__ StreamJob stream_job(const FrameDesc& d, int greens, const uint32_t* __restrict__ tile_off,
                                                uint32_t g) {
    StreamJob j{};
    j.g = g;
    if (g >= 4 * d.ntiles) return j;
    const uint32_t tile = g >> 2, s = g & 3;
    if (LC != 6 && s == 1 && !greens) return j;  // a reduced decode reads the second green only to average
    j.s = s;
    j.trow = tile / d.tiles_per_row;
    const uint32_t col = tile - j.trow * d.tiles_per_row;
    tile_geom(col, d.columns, d.alignment, j.x, j.log2);
    const uint32_t off = tile_off[tile], end = tile_off[tile + 1];
    if (!(off <= end && end <= d.len) || end - off < 8) return j;
    const uint32_t size = end - off;
    const uint32_t header_len = byte_at(d.words, off) >> 3;
    const uint32_t qscale = byte_at(d.words, off + 1);
    const uint32_t s0 = be16_at(d.words, off + 2), s1 = be16_at(d.words, off + 4), s2 = be16_at(d.words, off + 6);
    const uint32_t used = header_len + s0 + s1 + s2;
    if (!(header_len >= 8 && qscale != 0 && s0 != 0 && s1 != 0 && s2 != 0 && used < size)) return j;
    j.soff = off + header_len + (s > 0 ? s0 : 0) + (s > 1 ? s1 : 0) + (s > 2 ? s2 : 0);
    j.slen = s == 0 ? s0 : s == 1 ? s1 : s == 2 ? s2 : size - used;
    j.valid = true;
    return j;
}

// Entropy-decode the streams of tiles [chunk * 32, ...) of a frame, one
// stream per thread of a 128-thread CTA. `stage` holds stage_bytes + 16
// bytes of shared memory; the chunk's packet span is copied there when it
// fits. `keys` holds 128 words of shared memory. Ends with the CTA's threads
// at different points (no barrier).
template <uint32_t LC>
__device__ __forceinline__ void entropy_chunk(const EntropyTables& T, uint32_t* stage, uint32_t stage_bytes,
                                              uint32_t* keys, const FrameDesc& d, int greens,
                                              const uint32_t* __restrict__ tile_off, prr_dev_status* st,
                                              uint32_t chunk) {
    // The chunk's tiles [t0, t1) occupy bytes [tile_off[t0], tile_off[t1]).
    const uint32_t t0 = chunk * (blockDim.x / 4);
    const uint32_t t1 = min(t0 + blockDim.x / 4, d.ntiles);
    const uint32_t hi = min(tile_off[t1], d.len);
    const uint32_t lo = min(tile_off[t0], hi);
    const uint32_t base = lo & ~15u, top = (hi + 15) & ~15u;  // within the padded packet buffer
    const bool staged = top - base <= stage_bytes;
    if (staged) {
        const uint4* src = reinterpret_cast<const uint4*>(d.words) + base / 16;
        uint4* dst = reinterpret_cast<uint4*>(stage);
        for (uint32_t i = threadIdx.x; i < (top - base) / 16; i += blockDim.x) {
            const uint4 v = __ldg(src + i);
            dst[i] = make_uint4(bswap32(v.x), bswap32(v.y), bswap32(v.z), bswap32(v.w));
        }
    }
    // Threads take the chunk's streams in order of length (the shortest
    // first), so that the streams of a warp end at about the same time: the
    // kernel issues fewer warp instructions for the same symbols, which
    // leaves more issue slots to the kernels beside it. Key: length << 7 |
    // stream (128 streams a CTA), streams with nothing to decode last.
    const StreamJob mine = stream_job<LC>(d, greens, tile_off, chunk * blockDim.x + threadIdx.x);
    keys[threadIdx.x] = (mine.valid ? min(mine.slen, 0xFFFFFEu) : 0xFFFFFFu) << 7 | threadIdx.x;
    __syncthreads();
    for (uint32_t k = 2; k <= 128; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const uint32_t i = threadIdx.x, l = i ^ j;
            if (l > i) {
                const uint32_t a = keys[i], b = keys[l];
                if ((a > b) == ((i & k) == 0)) {
                    keys[i] = b;
                    keys[l] = a;
                }
            }
            __syncthreads();
        }
    }
    const uint32_t pick = keys[threadIdx.x] & 127u;
    const StreamJob job = pick == threadIdx.x ? mine : stream_job<LC>(d, greens, tile_off, chunk * blockDim.x + pick);
    if (!job.valid) return;
    uint32_t* list = d.pairs + stream_list_base(d, job.trow, job.x, job.log2, job.s, LC);
    bool revisited = false, ok = true;
    const uint32_t cnt =
        staged ? entropy_events<LC>(StagedWords{stage, base >> 2}, job.soff, job.slen, job.log2, T, list, revisited, ok)
               : entropy_events<LC>(PacketWords{d.words}, job.soff, job.slen, job.log2, T, list, revisited, ok);
    if (!ok) atomicOr(&st->error, 1u);
    d.counts[job.g] = revisited ? 0x80000000u : cnt;
}

template <uint32_t LC>
__global__ void __launch_bounds__(128) k_entropy(FrameDesc d, int greens, const uint32_t* __restrict__ tile_off,
                                                 prr_dev_status* __restrict__ st) {
    __shared__ CodeTables CT;
    __shared__ EntropyTables T;
    __shared__ __align__(16) uint32_t stage[kStageBytes / 4 + 4];  // + the word after the last byte
    __shared__ uint32_t keys[128];
    load_tables(&CT);
    __syncthreads();
    build_entropy_tables(T, CT);
    entropy_chunk<LC>(T, stage, kStageBytes, keys, d, greens, tile_off, st, blockIdx.x);
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
    bool revisited = false;
    decode_component(GlobalWords{words}, off[i], len[i], uint32_t(log2_blocks), uint32_t(log2_coefs), T,
                     [&](uint32_t idx, int16_t v) { dst[idx] = v; }, revisited);
}

// The frame decode's entropy decoder (entropy_events, the one k_entropy and
// the batch kernel run) on raw streams, so that the crate's component
// known-answer tests reach it directly. Thread i decodes stream i into its
// (position, value) list at lists + i * codes, from the packet in global
// memory or, with `staged` and when the CTA's streams span at most
// kStageBytes, from a shared-memory stage as k_entropy does; then it replays
// the list in order into dense coefficients (placement of
// src/coefficients.rs:86-88), later entries overwriting earlier ones, and
// writes flags[i] = entry count | bit 30 when the symbol budget ran out |
// bit 31 when a zero run wrapped back over stored positions.
template <uint32_t LC>
__global__ void __launch_bounds__(128) k_decode_components_events(const uint32_t* __restrict__ words,
                                                                  const uint32_t* __restrict__ off,
                                                                  const uint32_t* __restrict__ len, size_t n,
                                                                  uint32_t log2_blocks, int staged,
                                                                  uint32_t* __restrict__ lists,
                                                                  int16_t* __restrict__ coefs,
                                                                  uint32_t* __restrict__ flags) {
    __shared__ CodeTables CT;
    __shared__ EntropyTables T;
    __shared__ __align__(16) uint32_t stage[kStageBytes / 4 + 4];  // + the word after the last byte
    __shared__ uint32_t s_lo, s_hi;
    load_tables(&CT);
    if (threadIdx.x == 0) {
        s_lo = 0xFFFFFFFFu;
        s_hi = 0;
    }
    __syncthreads();
    build_entropy_tables(T, CT);
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool mine = i < n;
    const uint32_t o = mine ? off[i] : 0, l = mine ? len[i] : 0;
    if (mine) {
        atomicMin(&s_lo, o);
        atomicMax(&s_hi, o + l);
    }
    __syncthreads();
    const uint32_t base = s_lo & ~15u, top = (s_hi + 15) & ~15u;
    const bool use_stage = staged && s_lo <= s_hi && top - base <= kStageBytes;
    if (use_stage) {
        const uint4* src = reinterpret_cast<const uint4*>(words) + base / 16;
        uint4* dst = reinterpret_cast<uint4*>(stage);
        for (uint32_t k = threadIdx.x; k < (top - base) / 16; k += blockDim.x) {
            const uint4 v = __ldg(src + k);
            dst[k] = make_uint4(bswap32(v.x), bswap32(v.y), bswap32(v.z), bswap32(v.w));
        }
    }
    __syncthreads();
    if (!mine) return;
    const uint32_t codes = 1u << (log2_blocks + LC);
    uint32_t* list = lists + i * codes;
    bool revisited = false, ok = true;
    const uint32_t cnt =
        use_stage ? entropy_events<LC>(StagedWords{stage, base >> 2}, o, l, log2_blocks, T, list, revisited, ok)
                  : entropy_events<LC>(PacketWords{words}, o, l, log2_blocks, T, list, revisited, ok);
    int16_t* dst = coefs + i * codes;
    for (uint32_t k = 0; k < codes; k++) dst[k] = 0;
    const uint8_t* scan = LC == 6 ? CT.scan : (LC == 4 ? CT.scan4 : CT.scan2);
    const uint32_t mask = (1u << log2_blocks) - 1;
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t e = list[k], nn = e >> 16;
        dst[((nn & mask) << LC) + scan[nn >> log2_blocks]] = int16_t(e & 0xFFFF);
    }
    flags[i] = cnt | (ok ? 0u : 0x40000000u) | (revisited ? 0x80000000u : 0u);
}

// ---------------------------------------------------------------------------
// Batch decode: one CTA per frame for the tile offsets, then one persistent
// launch for the entropy chunks and transform segments of all frames.

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait until *flag == want, for at most ~limit_ns (and a fixed number of
// polls); false when the limit ran out.
__device__ __forceinline__ bool wait_flag(const uint32_t* flag, uint32_t want, uint64_t limit_ns) {
    if (ld_acquire_gpu(flag) == want) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < (1u << 26); it++) {
        __nanosleep(128);
        if (ld_acquire_gpu(flag) == want) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

constexpr uint64_t kChunkWaitNs = 2000000000ull;  // 2 s

__global__ void __launch_bounds__(1024) k_batch_tile_index(BatchDesc b) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.q->head = 0;
        b.q->error = 0;
        b.q->epoch = b.q->epoch + 1;
    }
    if (blockIdx.x >= b.hdr->nframes) return;
    const BatchFrame& F = b.frames[blockIdx.x];
    tile_index_body(F.d, F.tile_off, F.st);
}

// Last frame whose first item of the kind is <= key (frames without items
// of the kind share their successor's first item and are passed over).
__device__ __forceinline__ uint32_t batch_frame_of(const BatchDesc& b, uint32_t nframes, uint32_t key,
                                                  bool entropy) {
    uint32_t lo = 0, hi = nframes;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t begin = entropy ? b.frames[mid].ent_begin : b.frames[mid].seg_begin;
        if (begin <= key)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// The batch kernel's work items as separate functions, so that each gets
// the registers it needs on its own instead of the sum of all of them.
// An entropy item of the batch kernel: the S x blockDim.x streams of
// S x blockDim.x / 4 consecutive tiles (S = streams per thread, 1, 2 or 4).
// The item's packet span is staged when it fits; the streams are sorted by
// byte length (bitonic) and the sorted list is cut into pairs of the i-th
// shortest and i-th longest, which the threads take in turn, so every lane
// has about the same number of symbols to decode and the CTA's warps reach
// the item's closing barrier together.
template <uint32_t LC>
__device__ __noinline__ void batch_entropy(const EntropyTables& T, uint32_t* stage, uint32_t stage_bytes,
                                           const FrameDesc& d, int greens, const uint32_t* tile_off,
                                           prr_dev_status* st, uint32_t item, uint32_t* keys, uint32_t spt) {
    const uint32_t n = spt * blockDim.x;  // streams of the item (a power of two, at most 1024)
    const uint32_t g0 = item * n;
    const uint32_t t0 = g0 / 4;
    const uint32_t t1 = min(t0 + n / 4, d.ntiles);
    const uint32_t hi = min(tile_off[t1], d.len);
    const uint32_t lo = min(tile_off[t0], hi);
    const uint32_t base = lo & ~15u, top = (hi + 15) & ~15u;  // within the padded packet buffer
    const bool staged = top - base <= stage_bytes;
    if (staged) {
        const uint4* src = reinterpret_cast<const uint4*>(d.words) + base / 16;
        uint4* dst = reinterpret_cast<uint4*>(stage);
        for (uint32_t i = threadIdx.x; i < (top - base) / 16; i += blockDim.x) {
            const uint4 v = __ldg(src + i);
            dst[i] = make_uint4(bswap32(v.x), bswap32(v.y), bswap32(v.z), bswap32(v.w));
        }
    }
    for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
        const StreamJob jb = stream_job<LC>(d, greens, tile_off, g0 + e);
        keys[e] = (jb.valid ? (min(jb.slen, 0x3FFFFFu) << 10) : 0u) | e;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= n; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
                const uint32_t p = e ^ j;
                if (p > e) {
                    const uint32_t a = keys[e], b = keys[p];
                    if ((a > b) == ((e & k) == 0)) {
                        keys[e] = b;
                        keys[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // Sorted positions of this thread's streams: one (S = 1), or the pairs
    // (k, n - 1 - k) for k = i, i + blockDim.x, ...
    const uint32_t i = threadIdx.x;
#pragma unroll 1
    for (uint32_t q = 0; q < spt; q++) {
        const uint32_t k = i + (q >> 1) * blockDim.x;
        const uint32_t pos = spt == 1 ? i : ((q & 1) ? n - 1 - k : k);
        const StreamJob jb = stream_job<LC>(d, greens, tile_off, g0 + (keys[pos] & 1023));
        if (!jb.valid) continue;
        uint32_t* list = d.pairs + stream_list_base(d, jb.trow, jb.x, jb.log2, jb.s, LC);
        bool revisited = false, ok = true;
        const uint32_t cnt =
            staged ? entropy_events<LC>(StagedWords{stage, base >> 2}, jb.soff, jb.slen, jb.log2, T, list, revisited,
                                        ok)
                   : entropy_events<LC>(PacketWords{d.words}, jb.soff, jb.slen, jb.log2, T, list, revisited, ok);
        if (!ok) atomicOr(&st->error, 1u);
        d.counts[jb.g] = revisited ? 0x80000000u : cnt;
    }
}
template <int IDCT>
__device__ __noinline__ void batch_full(SegShared& S, const FrameDesc& d, uint32_t seg, uint32_t trow,
                                        const uint32_t* tile_off, prr_dev_status* st, uint32_t* skipped,
                                        uint16_t* out) {
    full_segment<IDCT, true, true>(S, d, seg, trow, tile_off, st, skipped, out);
}
template <int SHIFT>
__device__ __noinline__ void batch_reduced(SegShared& S, const FrameDesc& d, int greens, uint32_t seg,
                                           uint32_t trow, const uint32_t* tile_off, prr_dev_status* st,
                                           uint32_t* skipped, uint16_t* out) {
    reduced_segment<SHIFT, true, true>(S, d, greens, seg, trow, tile_off, st, skipped, out);
}

// The work items are claimed in order, so every chunk has been claimed by a
// running CTA before any segment is: the waits of a segment always end,
// whatever the grid size. The code tables and the codeword table are built
// once per CTA. The packet stage of a chunk aliases the segment buffers.
__global__ void __launch_bounds__(kBatchThreads, 4) k_batch_decode(BatchDesc b) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    SegShared& S = *reinterpret_cast<SegShared*>(dyn_smem);
    uint32_t* stage = reinterpret_cast<uint32_t*>(S.coef);
    __shared__ EntropyTables T;
    __shared__ FrameDesc fd;
    __shared__ uint32_t s_item, s_frame, s_epoch, s_ok;
    __shared__ uint32_t keys[kBatchMaxStreamsPerThread * kBatchThreads];  // the entropy items' stream order
    const uint32_t tid = threadIdx.x;
    load_tables(&S.T);
    if (tid == 0) s_epoch = b.q->epoch;
    __syncthreads();
    build_entropy_tables(T, S.T);
    const uint32_t nframes = b.hdr->nframes, ent_items = b.hdr->ent_items;
    const uint32_t total = ent_items + b.hdr->seg_items;
    const uint32_t drop_item = b.hdr->drop_item;
    const uint32_t spt = (b.hdr->streams_per_thread == 1 || b.hdr->streams_per_thread == 4) ? b.hdr->streams_per_thread
                                                                                          : 2u;
    const uint32_t tiles_per_item = batch_tiles_per_item(spt);
    const uint64_t wait_ns = b.hdr->wait_limit_us ? uint64_t(b.hdr->wait_limit_us) * 1000u : kChunkWaitNs;
    for (;;) {
        __syncthreads();  // the previous item's shared memory is no longer read
        if (tid == 0) {
            const uint32_t item = atomicAdd(&b.q->head, 1u);
            s_item = item;
            if (item < total) {
                const bool ent = item < ent_items;
                s_frame = batch_frame_of(b, nframes, ent ? item : item - ent_items, ent);
            }
        }
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total) break;
        const BatchFrame& F = b.frames[s_frame];
        for (uint32_t i = tid; i < sizeof(FrameDesc) / 4; i += kBatchThreads)
            reinterpret_cast<uint32_t*>(&fd)[i] = reinterpret_cast<const uint32_t*>(&F.d)[i];
        const uint32_t shift = F.shift, lc = F.lc, greens = F.greens;
        // A test can name one chunk that is claimed and then abandoned, as a
        // CTA that died would leave it: its flag is never set, and the
        // segments that wait for it give up after wait_ns.
        if (item == drop_item && item < ent_items) continue;
        if (item < ent_items) {
            __syncthreads();
            const uint32_t chunk = item - F.ent_begin;
            if (lc == 6)
                batch_entropy<6>(T, stage, b.stage_bytes, fd, greens, F.tile_off, F.st, chunk, keys, spt);
            else if (lc == 4)
                batch_entropy<4>(T, stage, b.stage_bytes, fd, greens, F.tile_off, F.st, chunk, keys, spt);
            else
                batch_entropy<2>(T, stage, b.stage_bytes, fd, greens, F.tile_off, F.st, chunk, keys, spt);
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                st_release_gpu(b.flags + item, s_epoch);
            }
            continue;
        }
        const uint32_t local = item - ent_items - F.seg_begin;
        const uint32_t trow = local / F.d.segs_per_row, seg = local - trow * F.d.segs_per_row;
        if (tid == 0) {
            // The segment's tiles lie among the 16 tiles of the row from its
            // first one (seg_setup's j0); wait for the chunks holding them.
            const uint32_t a = F.d.alignment, cols = F.d.columns, sq0 = seg * 16;
            const uint32_t fullsq = (cols >> a) << a;
            const uint32_t j0 = sq0 < fullsq ? (sq0 >> a) : (cols >> a);
            const uint32_t first = trow * F.d.tiles_per_row + j0;
            const uint32_t last = trow * F.d.tiles_per_row + min(j0 + 15, F.d.tiles_per_row - 1);
            bool ok = true;
            for (uint32_t c = first / tiles_per_item; ok && c <= last / tiles_per_item; c++)
                ok = wait_flag(b.flags + F.ent_begin + c, s_epoch, wait_ns);
            if (!ok) {
                atomicOr(&b.q->error, 1u);
                atomicOr(&F.st->error, 2u);
            }
            s_ok = ok ? 1u : 0u;
        }
        __syncthreads();
        if (!s_ok) continue;  // the segment is left unwritten; the frame reports the timeout
        if (shift == 0) {
            if (F.idct == PRR_IDCT_FFMPEG)
                batch_full<PRR_IDCT_FFMPEG>(S, fd, seg, trow, F.tile_off, F.st, F.skipped, F.out);
            else
                batch_full<PRR_IDCT_APPLE>(S, fd, seg, trow, F.tile_off, F.st, F.skipped, F.out);
        } else if (shift == 1) {
            batch_reduced<1>(S, fd, int(greens), seg, trow, F.tile_off, F.st, F.skipped, F.out);
        } else if (shift == 2) {
            batch_reduced<2>(S, fd, int(greens), seg, trow, F.tile_off, F.st, F.skipped, F.out);
        } else {
            batch_reduced<3>(S, fd, int(greens), seg, trow, F.tile_off, F.st, F.skipped, F.out);
        }
    }
}

size_t batch_smem_bytes(uint32_t stage_bytes) {
    const size_t stage_end = offsetof(SegShared, coef) + size_t(stage_bytes) + 16;
    return std::max(sizeof(SegShared), (stage_end + 15) & ~size_t(15));
}

// Allow the largest stage on the current device (once per device, before
// any capture).
cudaError_t batch_prepare_device() {
    return cudaFuncSetAttribute(k_batch_decode, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(batch_smem_bytes(kBatchMaxStageBytes)));
}

cudaError_t batch_max_ctas_per_sm(uint32_t stage_bytes, int* ctas) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, k_batch_decode, kBatchThreads,
                                                         batch_smem_bytes(stage_bytes));
}

cudaError_t launch_batch_tile_index(const BatchDesc& b, uint32_t grid, cudaStream_t s) {
    k_batch_tile_index<<<std::max(grid, 1u), 1024, 0, s>>>(b);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_batch_decode(const BatchDesc& b, uint32_t ctas, cudaStream_t s) {
    if (b.stage_bytes > kBatchMaxStageBytes || (b.stage_bytes & 15) != 0) return cudaErrorInvalidValue;
    k_batch_decode<<<std::max(ctas, 1u), kBatchThreads, batch_smem_bytes(b.stage_bytes), s>>>(b);
    count_launch();
    return cudaGetLastError();
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

DecodeScratch decode_scratch_layout(uint32_t ntiles, uint32_t coded_w, uint32_t coded_h) {
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    DecodeScratch l;
    l.tile_off = 0;
    l.counts = up(4 * (size_t(ntiles) + 1));
    l.pairs = l.counts + up(16 * size_t(ntiles));
    l.total = l.pairs + up(4 * size_t(coded_w) * coded_h);
    return l;
}

// The split path launches k_entropy first (128 threads per CTA: 32 tiles'
// streams), then the transform kernel; the fused path only the latter.
static cudaError_t launch_entropy(const FrameDesc& d, uint32_t lc, int greens, const uint32_t* tile_off,
                                  prr_dev_status* st, cudaStream_t s) {
    const unsigned blocks = unsigned((4 * size_t(d.ntiles) + 127) / 128);
    if (lc == 6)
        k_entropy<6><<<blocks, 128, 0, s>>>(d, greens, tile_off, st);
    else if (lc == 4)
        k_entropy<4><<<blocks, 128, 0, s>>>(d, greens, tile_off, st);
    else
        k_entropy<2><<<blocks, 128, 0, s>>>(d, greens, tile_off, st);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_full(const FrameDesc& d, int idct, const uint32_t* tile_off, prr_dev_status* st,
                               uint32_t* skipped, uint16_t* out, cudaStream_t s) {
    dim3 grid(d.segs_per_row, d.tile_rows);
    const bool split = d.pairs != nullptr;
    if (split) {
        const cudaError_t e = launch_entropy(d, 6, 1, tile_off, st, s);
        if (e != cudaSuccess) return e;
    }
    if (idct == PRR_IDCT_FFMPEG) {
        if (split)
            k_decode_full<PRR_IDCT_FFMPEG, true><<<grid, kThreads, 0, s>>>(d, tile_off, st, skipped, out);
        else
            k_decode_full<PRR_IDCT_FFMPEG, false><<<grid, kThreads, 0, s>>>(d, tile_off, st, skipped, out);
    } else {
        if (split)
            k_decode_full<PRR_IDCT_APPLE, true><<<grid, kThreads, 0, s>>>(d, tile_off, st, skipped, out);
        else
            k_decode_full<PRR_IDCT_APPLE, false><<<grid, kThreads, 0, s>>>(d, tile_off, st, skipped, out);
    }
    count_launch();
    return cudaGetLastError();
}

template <int SHIFT>
static void launch_reduced_t(const FrameDesc& d, int greens, const uint32_t* tile_off, prr_dev_status* st,
                             uint32_t* skipped, uint16_t* out, cudaStream_t s) {
    dim3 grid(d.segs_per_row, d.tile_rows);
    if (d.pairs != nullptr)
        k_decode_reduced<SHIFT, true><<<grid, kThreads, 0, s>>>(d, greens, tile_off, st, skipped, out);
    else
        k_decode_reduced<SHIFT, false><<<grid, kThreads, 0, s>>>(d, greens, tile_off, st, skipped, out);
}

cudaError_t launch_decode_reduced(const FrameDesc& d, int shift, int greens, const uint32_t* tile_off,
                                  prr_dev_status* st, uint32_t* skipped, uint16_t* out, cudaStream_t s) {
    if (d.pairs != nullptr) {
        const uint32_t lc = shift == 1 ? 6 : (shift == 2 ? 4 : 2);
        const cudaError_t e = launch_entropy(d, lc, greens, tile_off, st, s);
        if (e != cudaSuccess) return e;
    }
    if (shift == 1)
        launch_reduced_t<1>(d, greens, tile_off, st, skipped, out, s);
    else if (shift == 2)
        launch_reduced_t<2>(d, greens, tile_off, st, skipped, out, s);
    else
        launch_reduced_t<3>(d, greens, tile_off, st, skipped, out, s);
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

cudaError_t launch_decode_components_events(const uint8_t* packet, const uint32_t* off, const uint32_t* len,
                                            size_t n, int log2_blocks, int log2_coefs, int staged,
                                            uint32_t* lists, int16_t* coefs, uint32_t* flags, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = unsigned((n + 127) / 128);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(packet);
    const uint32_t lb = uint32_t(log2_blocks);
    if (log2_coefs == 6)
        k_decode_components_events<6><<<blocks, 128, 0, s>>>(w, off, len, n, lb, staged, lists, coefs, flags);
    else if (log2_coefs == 4)
        k_decode_components_events<4><<<blocks, 128, 0, s>>>(w, off, len, n, lb, staged, lists, coefs, flags);
    else
        k_decode_components_events<2><<<blocks, 128, 0, s>>>(w, off, len, n, lb, staged, lists, coefs, flags);
    count_launch();
    return cudaGetLastError();
}

}  // namespace prr
