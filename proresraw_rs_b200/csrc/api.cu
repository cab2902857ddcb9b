// api.cu -- host side of libprr.so: header and frame parsing, the context
// (device, stream, scratch) and the C-ABI entry points of include/prr.h.
//
// The host parses what the crate parses before any tile is touched
// (src/decoder.rs:45-103, src/header.rs:156-246): the frame prefix, the
// header and the bounds of the tile size table. The per-tile walk (offsets,
// TileOutOfBounds, max_qscale) runs on the device (k_tile_index).

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/prr.h"
#include "context.h"
#include "kernels.h"

namespace prr {

static std::atomic<uint64_t> g_launches{0};
void count_launch(uint32_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

constexpr size_t PREFIX_LEN = 10;
constexpr size_t FIXED_BODY_LEN = 70;
constexpr uint16_t MIN_HEADER_SIZE = 72;
constexpr uint16_t DEFAULT_CURVE[8] = {0, 512, 1024, 2048, 4096, 8192, 16384, 32768};

inline uint16_t be16(const uint8_t* p) { return uint16_t(p[0] << 8 | p[1]); }
inline uint32_t be32(const uint8_t* p) {
    return uint32_t(p[0]) << 24 | uint32_t(p[1]) << 16 | uint32_t(p[2]) << 8 | p[3];
}
inline float bef32(const uint8_t* p) {
    const uint32_t u = be32(p);
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

int fail(prr_error* e, int code) {
    if (e) {
        std::memset(e, 0, sizeof(*e));
        e->code = code;
    }
    return code;
}
int truncated(prr_error* e, const char* what, size_t needed, size_t available) {
    fail(e, PRR_ERR_TRUNCATED);
    if (e) {
        std::strncpy(e->what, what, sizeof(e->what) - 1);
        e->needed = needed;
        e->available = available;
    }
    return PRR_ERR_TRUNCATED;
}

// FrameHeader::parse, src/header.rs:156-246.
int parse_body(const uint8_t* body, size_t n, prr_header* h, prr_error* err) {
    if (n < FIXED_BODY_LEN) return truncated(err, "frame header", FIXED_BODY_LEN, n);
    std::memset(h, 0, sizeof(*h));
    h->version = body[1];
    if (h->version > 1) {
        fail(err, PRR_ERR_UNSUPPORTED_VERSION);
        if (err) err->value = h->version;
        return PRR_ERR_UNSUPPORTED_VERSION;
    }
    std::memcpy(h->vendor, body + 2, 4);
    h->width = be16(body + 6);
    h->height = be16(body + 8);
    if (h->width == 0 || h->height == 0 || (h->width & 1) || (h->height & 1)) {
        fail(err, PRR_ERR_BAD_DIMENSIONS);
        if (err) {
            err->width = h->width;
            err->height = h->height;
        }
        return PRR_ERR_BAD_DIMENSIONS;
    }
    std::memcpy(h->crop, body + 10, 4);
    h->bayer_pattern = uint8_t(be16(body + 14) & 3);
    h->white_level = uint16_t(be16(body + 16) + 256);
    h->wb_red = bef32(body + 18);
    h->wb_blue = bef32(body + 22);
    for (int i = 0; i < 9; i++) h->color_matrix[i] = bef32(body + 26 + 4 * i);
    h->gain = bef32(body + 62);
    h->wb_cct = be16(body + 66);
    h->flags = be16(body + 68);
    h->alignment = uint8_t((h->flags >> 1) & 7);
    if (h->alignment > 4) {
        fail(err, PRR_ERR_BAD_ALIGNMENT);
        if (err) err->value = h->alignment;
        return PRR_ERR_BAD_ALIGNMENT;
    }
    size_t pos = FIXED_BODY_LEN;
    std::fill(h->quant_matrix, h->quant_matrix + 64, uint8_t(1));
    if (h->flags & 1) {
        if (pos + 64 > n) return truncated(err, "quantization matrix", pos + 64, n);
        std::memcpy(h->quant_matrix, body + pos, 64);
        pos += 64;
        for (int i = 0; i < 64; i++) {
            if (h->quant_matrix[i] < 1 || h->quant_matrix[i] > 63) {
                fail(err, PRR_ERR_BAD_QUANT_MATRIX);
                if (err) {
                    err->index = uint64_t(i);
                    err->value = h->quant_matrix[i];
                }
                return PRR_ERR_BAD_QUANT_MATRIX;
            }
        }
    }
    if ((h->flags >> 4) & 1) {
        if (pos + 16 > n) return truncated(err, "linearization curve", pos + 16, n);
        uint16_t pts[8];
        for (int i = 0; i < 8; i++) pts[i] = be16(body + pos + 2 * i);
        if (h->version == 0) return fail(err, PRR_ERR_UNEXPECTED_CURVE);
        for (int i = 0; i < 7; i++) {
            if (pts[i] >= pts[i + 1]) {
                fail(err, PRR_ERR_BAD_CURVE);
                if (err) std::memcpy(err->curve, pts, sizeof(pts));
                return PRR_ERR_BAD_CURVE;
            }
        }
        std::memcpy(h->curve, pts, sizeof(pts));
    } else {
        std::memcpy(h->curve, DEFAULT_CURVE, sizeof(DEFAULT_CURVE));
    }
    return PRR_OK;
}

// TileGrid (src/tile.rs:46-71).
void grid_dims(const prr_header& h, uint32_t& tiles_per_row, uint32_t& rows) {
    const uint32_t columns = (uint32_t(h.width) + 15) / 16;
    rows = (uint32_t(h.height) + 15) / 16;
    const uint32_t a = h.alignment;
    tiles_per_row = (columns >> a) + uint32_t(__builtin_popcount(columns & ((1u << a) - 1)));
}

bool is_pinned(const void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

}  // namespace
}  // namespace prr

using namespace prr;

extern "C" {

const char* prr_status_string(int s) {
    switch (s) {
        case PRR_OK: return "ok";
        case PRR_ERR_TRUNCATED: return "truncated";
        case PRR_ERR_FRAME_SIZE_MISMATCH: return "frame size mismatch";
        case PRR_ERR_BAD_QUANT_MATRIX: return "bad quantization matrix";
        case PRR_ERR_BAD_CURVE: return "bad linearization curve";
        case PRR_ERR_UNEXPECTED_CURVE: return "version 0 header carries a linearization curve";
        case PRR_ERR_BAD_TAG: return "bad frame tag";
        case PRR_ERR_HEADER_TOO_SHORT: return "frame header too short";
        case PRR_ERR_UNSUPPORTED_VERSION: return "unsupported bitstream version";
        case PRR_ERR_BAD_DIMENSIONS: return "bad dimensions";
        case PRR_ERR_BAD_ALIGNMENT: return "bad tile alignment";
        case PRR_ERR_TILE_OUT_OF_BOUNDS: return "tile out of bounds";
        case PRR_ERR_BAD_TILE_HEADER: return "bad tile header";
        case PRR_ERR_BUFFER: return "output buffer has the wrong size";
        case PRR_ERR_CUDA: return "CUDA error";
        case PRR_ERR_TIMEOUT: return "device loop bound reached";
        case PRR_ERR_INVALID: return "invalid argument";
        case PRR_ERR_NO_MEMORY: return "out of memory";
        case PRR_ERR_SCRATCH_LIMIT: return "frame exceeds the fixed scratch of the no-alloc decode";
        default: return "unknown status";
    }
}

int prr_ctx_create(int device, void* stream, prr_ctx** out) {
    if (!out) return PRR_ERR_INVALID;
    *out = nullptr;
    prr_ctx* c = new prr_ctx;
    c->device = device;
    if (c->use_device() != PRR_OK) {
        delete c;
        return PRR_ERR_CUDA;
    }
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return PRR_ERR_CUDA;
        }
        c->own_stream = true;
    }
    if (c->status.ensure(1) != cudaSuccess || c->hstatus.ensure(1) != cudaSuccess) {
        if (c->own_stream) cudaStreamDestroy(c->stream);
        delete c;
        return PRR_ERR_CUDA;
    }
    *out = c;
    return PRR_OK;
}

void prr_ctx_destroy(prr_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->pkt.release();
    c->hpkt.release();
    c->scratch.release();
    c->skipped.release();
    c->status.release();
    c->hstatus.release();
    c->hskipped.release();
    c->samples.release();
    c->planes.release();
    c->lj_words.release();
    c->lj_lookback.release();
    c->lj_out.release();
    c->lj_offsets.release();
    c->lj_flag.release();
    c->lj_hout.release();
    c->lj_hoffsets.release();
    c->lin.release();
    batch_state_destroy(c->batch);
    c->batch = nullptr;
    learned_state_destroy(c->learned);
    c->learned = nullptr;
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

void* prr_ctx_stream(prr_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int prr_sync(prr_ctx* c) {
    if (!c) return PRR_ERR_INVALID;
    return c->cuda(cudaStreamSynchronize(c->stream));
}

const char* prr_last_error_string(prr_ctx* c) { return c ? c->last_error.c_str() : ""; }

size_t prr_padded_packet_bytes(size_t len) { return ((len + 15) & ~size_t(15)) + 16; }

uint64_t prr_kernel_launches(void) { return g_launches.load(); }

int prr_header_len(const uint8_t* pkt, size_t len, size_t* out, prr_error* err) {
    // src/decoder.rs:58-73
    if (len < PREFIX_LEN) return truncated(err, "frame prefix", PREFIX_LEN, len);
    if (std::memcmp(pkt + 4, "prrf", 4) != 0) {
        fail(err, PRR_ERR_BAD_TAG);
        if (err) std::memcpy(err->tag, pkt + 4, 4);
        return PRR_ERR_BAD_TAG;
    }
    const uint16_t hs = be16(pkt + 8);
    if (hs < MIN_HEADER_SIZE) {
        fail(err, PRR_ERR_HEADER_TOO_SHORT);
        if (err) err->value = hs;
        return PRR_ERR_HEADER_TOO_SHORT;
    }
    if (out) *out = PREFIX_LEN + size_t(hs) - 2;
    return PRR_OK;
}

int prr_parse_header(const uint8_t* pkt, size_t len, prr_header* out, prr_error* err) {
    // src/decoder.rs:45-53
    size_t body_end = 0;
    PRR_TRY(prr_header_len(pkt, len, &body_end, err));
    if (body_end > len) return truncated(err, "frame header", body_end, len);
    prr_header h;
    PRR_TRY(parse_body(pkt + PREFIX_LEN, body_end - PREFIX_LEN, &h, err));
    if (out) *out = h;
    return PRR_OK;
}

int prr_frame_info_parse(const uint8_t* pkt, size_t len, prr_frame_info* out, prr_error* err) {
    // src/decoder.rs:76-103
    if (len < PREFIX_LEN) return truncated(err, "frame prefix", PREFIX_LEN, len);
    const uint32_t declared = be32(pkt);
    if (declared == 0 || size_t(declared) > len) {
        fail(err, PRR_ERR_FRAME_SIZE_MISMATCH);
        if (err) {
            err->declared = declared;
            err->actual = len;
        }
        return PRR_ERR_FRAME_SIZE_MISMATCH;
    }
    if (len > 0xFFFFFFF0ull) return fail(err, PRR_ERR_INVALID);
    size_t body_end = 0;
    PRR_TRY(prr_header_len(pkt, len, &body_end, err));
    prr_frame_info f;
    std::memset(&f, 0, sizeof(f));
    PRR_TRY(prr_parse_header(pkt, len, &f.header, err));
    grid_dims(f.header, f.tiles_per_row, f.tile_rows);
    f.ntiles = f.tiles_per_row * f.tile_rows;
    const size_t table_end = body_end + 2 * size_t(f.ntiles);
    if (table_end > len) return truncated(err, "tile size table", table_end, len);
    f.packet_len = len;
    f.table_offset = body_end;
    f.coded_width = (uint32_t(f.header.width) + 15) & ~15u;
    f.coded_height = (uint32_t(f.header.height) + 15) & ~15u;
    if (out) *out = f;
    return PRR_OK;
}

int prr_parse_frame(const uint8_t* pkt, size_t len, prr_frame_info* out, uint8_t* max_qscale,
                    prr_error* err) {
    // src/decoder.rs:104-116, walked on the host.
    prr_frame_info f;
    PRR_TRY(prr_frame_info_parse(pkt, len, &f, err));
    size_t offset = f.table_offset + 2 * size_t(f.ntiles);
    uint8_t maxq = 0;
    for (uint32_t i = 0; i < f.ntiles; i++) {
        const size_t size = be16(pkt + f.table_offset + 2 * size_t(i));
        if (offset + 1 < len) maxq = std::max(maxq, pkt[offset + 1]);
        if (offset + size > len) {
            fail(err, PRR_ERR_TILE_OUT_OF_BOUNDS);
            if (err) err->index = i;
            return PRR_ERR_TILE_OUT_OF_BOUNDS;
        }
        offset += size;
    }
    if (out) *out = f;
    if (max_qscale) *max_qscale = maxq;
    return PRR_OK;
}

size_t prr_decode_scratch_bytes(const prr_frame_info* info) {
    return info ? decode_scratch_layout(info->ntiles, info->coded_width, info->coded_height).total : 0;
}

}  // extern "C"

namespace {

// Upload a host packet into the context's padded device staging buffer.
int upload_packet(prr_ctx* c, const uint8_t* packet, size_t len, const uint8_t** dev) {
    const size_t padded = prr_padded_packet_bytes(len);
    PRR_TRY(c->cuda(c->pkt.ensure(padded)));
    if (is_pinned(packet)) {
        PRR_TRY(c->cuda(cudaMemcpyAsync(c->pkt.p, packet, len, cudaMemcpyHostToDevice, c->stream)));
    } else {
        // Stage through pinned memory; wait for the previous upload that
        // may still read the staging buffer.
        PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
        PRR_TRY(c->cuda(c->hpkt.ensure(padded)));
        std::memcpy(c->hpkt.p, packet, len);
        PRR_TRY(c->cuda(cudaMemcpyAsync(c->pkt.p, c->hpkt.p, len, cudaMemcpyHostToDevice, c->stream)));
    }
    *dev = c->pkt.p;
    return PRR_OK;
}

// Wait for a decode, then report its device status like parse_frame and
// decode_frame report theirs.
int finish_decode(prr_ctx* c, const prr_frame_info& f, prr_decode_result* res, prr_error* err) {
    PRR_TRY(c->cuda(cudaMemcpyAsync(c->hstatus.p, c->status.p, sizeof(prr_dev_status),
                                    cudaMemcpyDeviceToHost, c->stream)));
    PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
    const prr_dev_status st = *c->hstatus.p;
    if (st.oob_tile != NO_TILE) {
        fail(err, PRR_ERR_TILE_OUT_OF_BOUNDS);
        if (err) err->index = st.oob_tile;
        return PRR_ERR_TILE_OUT_OF_BOUNDS;
    }
    if (st.error) return fail(err, PRR_ERR_TIMEOUT);
    if (res) {
        res->header = f.header;
        res->max_qscale = uint8_t(st.max_qscale);
        res->n_skipped = st.n_skipped;
        if (st.n_skipped > 0 && res->skipped && res->skipped_cap > 0) {
            PRR_TRY(c->cuda(c->hskipped.ensure(st.n_skipped)));
            PRR_TRY(c->cuda(cudaMemcpyAsync(c->hskipped.p, c->skipped.p, st.n_skipped * sizeof(uint32_t),
                                            cudaMemcpyDeviceToHost, c->stream)));
            PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
            std::sort(c->hskipped.p, c->hskipped.p + st.n_skipped);
            const size_t n = std::min<size_t>(st.n_skipped, res->skipped_cap);
            for (size_t i = 0; i < n; i++) res->skipped[i] = c->hskipped.p[i];
        }
    }
    return PRR_OK;
}

// Enqueue a frame decode: the tile-offset scan, the entropy kernel and the
// transform kernel, with the scratch laid out by decode_scratch_layout.
int launch_frame(prr_ctx* c, const prr_frame_info& f, const uint8_t* dev_pkt, bool reduced, int idct,
                 int scale, int greens, uint16_t* dev_out, prr_dev_status* st, uint32_t* skipped,
                 uint8_t* scratch) {
    const DecodeScratch l = decode_scratch_layout(f.ntiles, f.coded_width, f.coded_height);
    FrameDesc d = make_frame_desc(f, dev_pkt);
    uint32_t* tile_off = reinterpret_cast<uint32_t*>(scratch + l.tile_off);
    d.counts = reinterpret_cast<uint32_t*>(scratch + l.counts);
    d.pairs = reinterpret_cast<uint32_t*>(scratch + l.pairs);
    PRR_TRY(c->cuda(launch_tile_index(d, tile_off, st, c->stream)));
    if (reduced) return c->cuda(launch_decode_reduced(d, scale, greens, tile_off, st, skipped, dev_out, c->stream));
    return c->cuda(launch_decode_full(d, idct, tile_off, st, skipped, dev_out, c->stream));
}

int decode_common(prr_ctx* c, const uint8_t* packet, size_t len, bool reduced, int idct, int scale,
                  int greens, uint16_t* dev_out, size_t out_len, prr_decode_result* res,
                  prr_error* err) {
    if (!c || !packet || !dev_out) return fail(err, PRR_ERR_INVALID);
    PRR_TRY(c->use_device());
    prr_frame_info f;
    PRR_TRY(prr_frame_info_parse(packet, len, &f, err));
    if (reduced) {
        if (scale < 1 || scale > 3 || greens < 0 || greens > 1) return fail(err, PRR_ERR_INVALID);
        const size_t want = 3 * size_t(f.coded_width >> scale) * (f.coded_height >> scale);
        if (out_len != want) return fail(err, PRR_ERR_BUFFER);
    } else {
        if (idct != PRR_IDCT_APPLE && idct != PRR_IDCT_FFMPEG) return fail(err, PRR_ERR_INVALID);
        if (out_len != size_t(f.coded_width) * f.coded_height) return fail(err, PRR_ERR_BUFFER);
    }
    const uint8_t* dev_pkt = nullptr;
    PRR_TRY(upload_packet(c, packet, len, &dev_pkt));
    const size_t scratch_bytes = prr_decode_scratch_bytes(&f);
    PRR_TRY(c->cuda(c->scratch.ensure(scratch_bytes)));
    PRR_TRY(c->cuda(c->skipped.ensure(f.ntiles)));
    PRR_TRY(launch_frame(c, f, dev_pkt, reduced, idct, scale, greens, dev_out, c->status.p, c->skipped.p,
                         c->scratch.p));
    return finish_decode(c, f, res, err);
}

int decode_async_common(prr_ctx* c, const prr_frame_info* info, const uint8_t* dev_packet, bool reduced,
                        int idct, int scale, int greens, uint16_t* dev_out, prr_dev_status* st,
                        uint32_t* skipped, void* scratch, size_t scratch_bytes) {
    if (!c || !info || !dev_packet || !dev_out || !st || !skipped || !scratch) return PRR_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(dev_packet) & 3) != 0) return PRR_ERR_INVALID;
    if (scratch_bytes < prr_decode_scratch_bytes(info)) return PRR_ERR_BUFFER;
    if (reduced && (scale < 1 || scale > 3 || greens < 0 || greens > 1)) return PRR_ERR_INVALID;
    if (!reduced && idct != PRR_IDCT_APPLE && idct != PRR_IDCT_FFMPEG) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return launch_frame(c, *info, dev_packet, reduced, idct, scale, greens, dev_out, st, skipped,
                        static_cast<uint8_t*>(scratch));
}

void params_wb(const prr_header* h, uint32_t quantizer, float red, float blue, prr_params* out) {
    // DemosaicParams::with_white_balance, src/demosaic.rs:86-106 (f64 then f32).
    const uint32_t range = uint16_t(h->white_level - 256);
    const double q = double(quantizer);
    const double base = q * q * 5.0 + 64.0 / 3.0;
    const double range2 = double(range) * double(range);
    const float rangef = float(range);
    auto inverse = [](float g) { return g == 0.0f ? 1.0f : 1.0f / g; };
    out->cfa_phase = h->bayer_pattern & 3;
    out->black = 256;
    out->one_over_range = 1.0f / rangef;
    out->noise[0] = float(base / 150994944.0);
    out->noise[1] = float(base / (range2 * 256.0));
    out->noise[2] = float(64.0 / 3.0 / range2);
    out->clip[0] = inverse(red);
    out->clip[1] = inverse(blue);
    out->black_over_range = 256.0f / rangef;
    out->wb[0] = red;
    out->wb[1] = blue;
}

}  // namespace

void prr::output_matrix(const prr_header* h, int exposure, float* m) {
    // src/demosaic.rs:138-153, XYZ_TO_REC2020 from src/demosaic.rs:37-41.
    static const double G[3][3] = {{1.716651187971268, -0.355670783776393, -0.25336628137366},
                                   {-0.666684351832489, 1.616481236634939, 0.015768545813911},
                                   {0.017639857445311, -0.042770613257809, 0.942103121235474}};
    double gain = double(h->gain);
    if (exposure == PRR_EXPOSURE_NORMALIZED) gain = gain * 10.0 / 9.0;
    for (int i = 0; i < 9; i++) {
        const int row = i / 3, col = i % 3;
        const double v = G[row][0] * double(h->color_matrix[col]) + G[row][1] * double(h->color_matrix[3 + col]) +
                         G[row][2] * double(h->color_matrix[6 + col]);
        m[i] = float(v * gain);
    }
}

namespace {

}  // namespace

// Check a develop call's arguments and fill its kernel descriptor.
int prr::build_develop_desc(const prr_header* h, const prr_params* params, int stage, const uint16_t* dev_samples,
                            int layout, float* r, float* g, float* b, size_t out_len, DevelopDesc* out) {
    if (!h || !params || !dev_samples || !r) return PRR_ERR_INVALID;
    if (stage < PRR_STAGE_DEMOSAICED || stage > PRR_STAGE_REC2020) return PRR_ERR_INVALID;
    const size_t n = size_t(h->width) * h->height;
    if (layout == PRR_PLANAR) {
        if (!g || !b) return PRR_ERR_INVALID;
        if (out_len != n) return PRR_ERR_BUFFER;
        if (((reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(g) | reinterpret_cast<uintptr_t>(b)) & 7) != 0)
            return PRR_ERR_INVALID;
    } else if (layout == PRR_INTERLEAVED) {
        if (out_len != 3 * n) return PRR_ERR_BUFFER;
        if ((reinterpret_cast<uintptr_t>(r) & 7) != 0) return PRR_ERR_INVALID;
    } else {
        return PRR_ERR_INVALID;
    }
    // Conversion::new, src/demosaic.rs:286-304.
    prr_params p = *params;
    if (stage == PRR_STAGE_DEMOSAICED) {
        p.wb[0] = p.wb[1] = 1.0f;
        p.clip[0] = p.clip[1] = 1.0f;
    }
    DevelopDesc d{};
    d.codes = dev_samples;
    d.stride = (uint32_t(h->width) + 15) & ~15u;
    d.w = h->width;
    d.h = h->height;
    for (int s = 0; s < 8; s++) {
        const uint32_t c0 = h->curve[s];
        const uint32_t c1 = s < 7 ? h->curve[s + 1] : 65536u;
        d.curve_c0[s] = c0;
        d.curve_delta[s] = (c1 - c0) & 0xFFFF;
    }
    d.cfa = p.cfa_phase & 3;
    d.black = p.black;
    d.one_over_range = p.one_over_range;
    d.green_off = float(p.black) * p.one_over_range;  // src/demosaic.rs:483
    d.chroma_off = p.black_over_range;                // src/demosaic.rs:656
    for (int i = 0; i < 3; i++) d.noise[i] = p.noise[i];
    d.clip[0] = p.clip[0];
    d.clip[1] = p.clip[1];
    d.wb[0] = p.wb[0];
    d.wb[1] = p.wb[1];
    d.has_matrix = stage == PRR_STAGE_REC2020;
    if (d.has_matrix) output_matrix(h, PRR_EXPOSURE_NORMALIZED, d.m);
    d.layout = layout;
    d.r = r;
    d.g = g;
    d.b = b;
    *out = d;
    return PRR_OK;
}

namespace {

uint32_t ceil_log2_u32(uint32_t v) {
    uint32_t k = 0;
    while (k < 32 && (uint64_t(1) << k) < v) k++;
    return k;
}

prr_develop_config default_develop_config() {
    prr_develop_config c{};
    c.tile_w = 32;
    c.tile_h = 32;
    c.ctas_per_sm = 0;
    return c;
}

// The launch shape for a frame: its bucket's config, the context's
// occupancy cap (prr_develop_set_occupancy) over it when set.
void apply_develop_config(const prr_ctx* c, const prr_develop_config& cfg, DevelopDesc* d) {
    d->tile_w = cfg.tile_w;
    d->tile_h = cfg.tile_h;
    d->ctas_per_sm = c->develop_ctas ? c->develop_ctas : cfg.ctas_per_sm;
}

int develop_launch(prr_ctx* c, const prr_header* h, const prr_params* params, int stage,
                   const uint16_t* dev_samples, int layout, float* r, float* g, float* b, size_t out_len,
                   const prr_develop_config* force = nullptr) {
    if (!c) return PRR_ERR_INVALID;
    DevelopDesc d{};
    PRR_TRY(build_develop_desc(h, params, stage, dev_samples, layout, r, g, b, out_len, &d));
    PRR_TRY(c->use_device());
    prr_develop_config cfg = default_develop_config();
    if (force) {
        cfg = *force;
    } else {
        const auto it = c->develop_cfgs.find(prr_develop_bucket(h->width, h->height));
        if (it != c->develop_cfgs.end()) cfg = it->second;
    }
    apply_develop_config(c, cfg, &d);
    return c->cuda(launch_develop(d, c->stream));
}

}  // namespace

extern "C" {

int prr_decode(prr_ctx* c, const uint8_t* packet, size_t len, int idct, uint16_t* dev_samples,
               size_t samples_len, prr_decode_result* res, prr_error* err) {
    return decode_common(c, packet, len, false, idct, 0, 0, dev_samples, samples_len, res, err);
}

int prr_decode_reduced(prr_ctx* c, const uint8_t* packet, size_t len, int scale, int greens,
                       uint16_t* dev_rgb, size_t rgb_len, prr_decode_result* res, prr_error* err) {
    return decode_common(c, packet, len, true, 0, scale, greens, dev_rgb, rgb_len, res, err);
}

int prr_decode_async(prr_ctx* c, const prr_frame_info* info, const uint8_t* dev_packet, int idct,
                     uint16_t* dev_samples, prr_dev_status* st, uint32_t* skipped, void* scratch,
                     size_t scratch_bytes) {
    return decode_async_common(c, info, dev_packet, false, idct, 0, 0, dev_samples, st, skipped, scratch,
                               scratch_bytes);
}

int prr_decode_reduced_async(prr_ctx* c, const prr_frame_info* info, const uint8_t* dev_packet, int scale,
                             int greens, uint16_t* dev_rgb, prr_dev_status* st, uint32_t* skipped,
                             void* scratch, size_t scratch_bytes) {
    return decode_async_common(c, info, dev_packet, true, 0, scale, greens, dev_rgb, st, skipped, scratch,
                               scratch_bytes);
}

int prr_linearize(prr_ctx* c, const prr_header* h, const uint16_t* dev_samples, uint16_t* dev_out,
                  size_t out_len) {
    if (!c || !h || !dev_samples || !dev_out) return PRR_ERR_INVALID;
    if (out_len != size_t(h->width) * h->height) return PRR_ERR_BUFFER;
    PRR_TRY(c->use_device());
    uint32_t c0[8], cd[8];
    for (int s = 0; s < 8; s++) {
        c0[s] = h->curve[s];
        cd[s] = ((s < 7 ? uint32_t(h->curve[s + 1]) : 65536u) - c0[s]) & 0xFFFF;
    }
    const uint32_t stride = (uint32_t(h->width) + 15) & ~15u;
    return c->cuda(launch_linearize(dev_samples, stride, h->width, h->height, c0, cd, dev_out, c->stream));
}

int prr_params_new(const prr_header* h, uint32_t quantizer, prr_params* out) {
    if (!h || !out) return PRR_ERR_INVALID;
    params_wb(h, quantizer, h->wb_red, h->wb_blue, out);
    return PRR_OK;
}

int prr_params_with_white_balance(const prr_header* h, uint32_t quantizer, float red, float blue,
                                  prr_params* out) {
    if (!h || !out) return PRR_ERR_INVALID;
    params_wb(h, quantizer, red, blue, out);
    return PRR_OK;
}

int prr_output_matrix(const prr_header* h, int exposure, float m[9]) {
    if (!h || !m || exposure < 0 || exposure > 1) return PRR_ERR_INVALID;
    output_matrix(h, exposure, m);
    return PRR_OK;
}

int prr_develop(prr_ctx* c, const prr_header* h, const prr_params* params, int stage,
                const uint16_t* dev_samples, int layout, float* r, float* g, float* b, size_t out_len) {
    return develop_launch(c, h, params, stage, dev_samples, layout, r, g, b, out_len);
}

int prr_decode_develop_host(prr_ctx* c, const uint8_t* packet, size_t len, int idct, const prr_params* params,
                            int stage, int layout, float* r, float* g, float* b, size_t out_len,
                            prr_decode_result* res, prr_error* err) {
    if (!c || !packet || !r) return fail(err, PRR_ERR_INVALID);
    PRR_TRY(c->use_device());
    prr_frame_info f;
    PRR_TRY(prr_frame_info_parse(packet, len, &f, err));
    const size_t n = size_t(f.header.width) * f.header.height;
    if (layout == PRR_PLANAR ? out_len != n : out_len != 3 * n) return fail(err, PRR_ERR_BUFFER);
    if (layout == PRR_PLANAR && (!g || !b)) return fail(err, PRR_ERR_INVALID);
    const size_t ns = size_t(f.coded_width) * f.coded_height;
    PRR_TRY(c->cuda(c->samples.ensure(ns)));
    PRR_TRY(c->cuda(c->planes.ensure(3 * n)));
    prr_decode_result local{};
    prr_decode_result* rr = res ? res : &local;
    PRR_TRY(decode_common(c, packet, len, false, idct, 0, 0, c->samples.p, ns, rr, err));
    prr_params p;
    if (params)
        p = *params;
    else
        params_wb(&f.header, uint32_t(f.header.quant_matrix[0]) * rr->max_qscale, f.header.wb_red,
                  f.header.wb_blue, &p);
    float* dr = c->planes.p;
    float* dg = layout == PRR_PLANAR ? dr + n : nullptr;
    float* db = layout == PRR_PLANAR ? dr + 2 * n : nullptr;
    PRR_TRY(develop_launch(c, &f.header, &p, stage, c->samples.p, layout, dr, dg, db, out_len));
    if (layout == PRR_PLANAR) {
        PRR_TRY(c->cuda(cudaMemcpyAsync(r, dr, n * 4, cudaMemcpyDeviceToHost, c->stream)));
        PRR_TRY(c->cuda(cudaMemcpyAsync(g, dg, n * 4, cudaMemcpyDeviceToHost, c->stream)));
        PRR_TRY(c->cuda(cudaMemcpyAsync(b, db, n * 4, cudaMemcpyDeviceToHost, c->stream)));
    } else {
        PRR_TRY(c->cuda(cudaMemcpyAsync(r, dr, 3 * n * 4, cudaMemcpyDeviceToHost, c->stream)));
    }
    return c->cuda(cudaStreamSynchronize(c->stream));
}

int prr_transform_blocks(prr_ctx* c, int kind, const int16_t* coefs, const int16_t* q, uint16_t* out,
                         size_t n) {
    if (!c || kind < 0 || kind > 3) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return c->cuda(launch_transform_blocks(kind, coefs, q, out, n, c->stream));
}

int prr_decode_components(prr_ctx* c, const uint8_t* packet, const uint32_t* off, const uint32_t* len,
                          size_t n, int log2_blocks, int log2_coefs, int16_t* coefs) {
    if (!c || log2_blocks < 0 || log2_blocks > 4 || (log2_coefs != 6 && log2_coefs != 4 && log2_coefs != 2))
        return PRR_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(packet) & 3) != 0) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return c->cuda(launch_decode_components(packet, off, len, n, log2_blocks, log2_coefs, coefs, c->stream));
}

int prr_div_rn_pairs(prr_ctx* c, const float* a, const float* b, float* q, size_t n) {
    if (!c || (n && (!a || !b || !q))) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return c->cuda(launch_div_rn_pairs(a, b, q, n, c->stream));
}

int prr_sqrt_rn_check(prr_ctx* c, int e_min, int e_max, uint64_t* dev_mismatches) {
    if (!c || !dev_mismatches || e_min < -126 || e_max > 127 || e_min > e_max) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return c->cuda(launch_sqrt_rn_check(e_min, e_max, reinterpret_cast<unsigned long long*>(dev_mismatches),
                                        c->stream));
}

int prr_div_rn_check(prr_ctx* c, uint32_t b_first, uint32_t b_count, uint64_t* dev_mismatches) {
    if (!c || !dev_mismatches || b_first >= (1u << 23) || b_count > (1u << 23) - b_first) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return c->cuda(launch_div_rn_check(b_first, b_count, reinterpret_cast<unsigned long long*>(dev_mismatches),
                                       c->stream));
}

int prr_decode_components_events(prr_ctx* c, const uint8_t* packet, const uint32_t* off, const uint32_t* len,
                                 size_t n, int log2_blocks, int log2_coefs, int staged, uint32_t* lists,
                                 int16_t* coefs, uint32_t* flags) {
    if (!c || log2_blocks < 0 || log2_blocks > 4 || (log2_coefs != 6 && log2_coefs != 4 && log2_coefs != 2))
        return PRR_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(packet) & 3) != 0 || (reinterpret_cast<uintptr_t>(lists) & 15) != 0)
        return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    return c->cuda(launch_decode_components_events(packet, off, len, n, log2_blocks, log2_coefs, staged, lists,
                                                   coefs, flags, c->stream));
}

}  // extern "C"

extern "C" int prr_develop_set_occupancy(prr_ctx* c, uint32_t ctas_per_sm) {
    if (!c || ctas_per_sm > 16) return PRR_ERR_INVALID;
    c->develop_ctas = ctas_per_sm;
    return PRR_OK;
}

extern "C" uint32_t prr_develop_bucket(uint32_t width, uint32_t height) {
    return (ceil_log2_u32(width) << 8) | ceil_log2_u32(height);
}

extern "C" int prr_develop_set_config(prr_ctx* c, uint32_t bucket, const prr_develop_config* cfg) {
    if (!c || !cfg || !develop_shape_supported(cfg->tile_w, cfg->tile_h) || cfg->ctas_per_sm > 16)
        return PRR_ERR_INVALID;
    c->develop_cfgs[bucket] = *cfg;
    return PRR_OK;
}

extern "C" int prr_develop_get_config(prr_ctx* c, uint32_t bucket, prr_develop_config* cfg) {
    if (!c || !cfg) return PRR_ERR_INVALID;
    const auto it = c->develop_cfgs.find(bucket);
    *cfg = it != c->develop_cfgs.end() ? it->second : default_develop_config();
    return PRR_OK;
}

extern "C" int prr_develop_tune(prr_ctx* c, const prr_header* h, const prr_params* params, int stage,
                                const uint16_t* dev_samples, int layout, float* r, float* g, float* b,
                                size_t out_len, uint32_t reps, prr_develop_config* best, float* best_ms) {
    if (!c || !h) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    reps = std::max(reps, 1u);
    static const uint32_t shapes[][2] = {{32, 32}, {32, 16}, {64, 16}};
    // CTAs per SM: as many as fit (0), and caps below that, down to half
    // (a capped develop leaves room to kernels of other streams, and fewer
    // resident CTAs wait less at their barriers).
    std::vector<prr_develop_config> cands;
    for (const auto& sh : shapes) {
        const uint32_t threads = sh[0] * sh[1] / 4;
        const uint32_t fit = std::max(1u, 1024u / threads);  // 64 registers a thread
        for (uint32_t cap = 0; cap <= fit; cap = cap == 0 ? std::max(1u, fit / 2) : cap + 1) {
            if (cap == fit) break;
            prr_develop_config cfg{sh[0], sh[1], cap};
            cands.push_back(cfg);
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = c->cuda(cudaEventCreate(&e0));
    if (rc == PRR_OK) rc = c->cuda(cudaEventCreate(&e1));
    prr_develop_config win = default_develop_config();
    float win_ms = 1e30f;
    for (size_t k = 0; rc == PRR_OK && k < cands.size(); k++) {
        const prr_develop_config& cfg = cands[k];
        const uint32_t saved = c->develop_ctas;
        c->develop_ctas = 0;  // the candidate's own cap
        std::vector<float> ms;
        for (uint32_t i = 0; rc == PRR_OK && i <= reps; i++) {
            rc = c->cuda(cudaEventRecord(e0, c->stream));
            if (rc == PRR_OK) rc = develop_launch(c, h, params, stage, dev_samples, layout, r, g, b, out_len, &cfg);
            if (rc == PRR_OK) rc = c->cuda(cudaEventRecord(e1, c->stream));
            if (rc == PRR_OK) rc = c->cuda(cudaEventSynchronize(e1));
            float t = 0.f;
            if (rc == PRR_OK) rc = c->cuda(cudaEventElapsedTime(&t, e0, e1));
            if (i > 0) ms.push_back(t);  // the first run is untimed
        }
        c->develop_ctas = saved;
        if (rc != PRR_OK) break;
        std::sort(ms.begin(), ms.end());
        const float med = ms[ms.size() / 2];
        if (med < win_ms) {
            win_ms = med;
            win = cfg;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    PRR_TRY(rc);
    c->develop_cfgs[prr_develop_bucket(h->width, h->height)] = win;
    if (best) *best = win;
    if (best_ms) *best_ms = win_ms;
    return PRR_OK;
}
