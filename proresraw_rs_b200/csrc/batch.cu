// batch.cu -- host side of the batched decode (prr_batch_* in prr.h): frame
// parsing and validation, the batch's device buffers, the CUDA graph of
// each shape bucket, the launch shape of each bucket and its autotuner.
//
// A batch runs as: upload of the frame table and the packets, then
// k_batch_tile_index (one CTA per frame: tile offsets, TileOutOfBounds,
// max_qscale, queue reset), k_batch_decode (persistent; entropy chunks of
// all frames, then transform segments of all frames) and the download of
// the per-frame statuses. The last three are captured once per bucket as a
// graph and replayed: their parameters are fixed pointers into the batch
// buffers, and everything that changes from batch to batch is read from the
// uploaded frame table.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <thread>
#include <vector>

#include "../../include/prr.h"
#include "context.h"
#include "kernels.h"

namespace prr {

namespace {

struct Bucket {
    prr_batch_config cfg{};
    bool has_cfg = false;
    cudaGraphExec_t exec = nullptr;
    // The buffers and launch shape the graph was captured with.
    uint64_t gen = 0;
    uint32_t grid_frames = 0, ctas = 0, stage = 0;
};

struct FramePlan {
    size_t job;
    prr_frame_info info;
    uint32_t shift, lc;
    size_t pkt_off;  // bytes into the packet buffer
    size_t words_off;  // tile offsets (ntiles + 1), counts (4 ntiles), skipped (ntiles), in words
    size_t pairs_off;  // words into the list buffer
};

constexpr size_t up64(size_t v) { return (v + 63) & ~size_t(63); }
constexpr size_t up16(size_t v) { return (v + 15) & ~size_t(15); }

uint32_t ceil_log2(uint64_t v) {
    uint32_t k = 0;
    while ((uint64_t(1) << k) < v) k++;
    return k;
}

int fail_job(prr_job& j, int code) {
    std::memset(&j.error, 0, sizeof(j.error));
    j.error.code = code;
    j.status = code;
    return code;
}

}  // namespace

struct BatchState {
    int sms = 0;
    uint64_t gen = 1;  // bumped whenever a device buffer moves: graphs are captured again
    DevBuf<uint8_t> meta;  // BatchHeader, then BatchFrame[]
    DevBuf<BatchQueue> queue;
    DevBuf<uint32_t> flags;
    DevBuf<uint8_t> packets;
    DevBuf<uint32_t> words;
    DevBuf<uint32_t> pairs;
    DevBuf<prr_dev_status> status;
    HostBuf<uint8_t> hmeta;
    HostBuf<uint8_t> hpackets;
    HostBuf<prr_dev_status> hstatus;
    HostBuf<uint32_t> hskipped;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    cudaStream_t cap_stream = nullptr;
    std::map<uint32_t, Bucket> buckets;
    prr_job* jobs = nullptr;
    size_t njobs = 0;
    bool pending = false;
    std::vector<FramePlan> plan;
    float last_ms = 0.f;
    uint32_t wait_limit_us = 0;    // prr_batch_set_wait_limit (0: the 2 s default)
    uint32_t drop_item = NO_TILE;  // prr_batch_drop_chunk_for_test

    // Grow a buffer (by half again at least); a buffer that moves makes the
    // captured graphs stale.
    template <class Buf>
    cudaError_t grow(Buf& b, size_t n) {
        if (n <= b.cap) return cudaSuccess;
        gen++;
        return b.ensure(std::max(n, b.cap + b.cap / 2));
    }
    void release() {
        for (auto& kv : buckets)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        buckets.clear();
        meta.release();
        queue.release();
        flags.release();
        packets.release();
        words.release();
        pairs.release();
        status.release();
        hmeta.release();
        hpackets.release();
        hstatus.release();
        hskipped.release();
        if (ev_start) cudaEventDestroy(ev_start);
        if (ev_stop) cudaEventDestroy(ev_stop);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        ev_start = ev_stop = nullptr;
        cap_stream = nullptr;
    }
};

void batch_state_destroy(BatchState* b) {
    if (!b) return;
    b->release();
    delete b;
}

namespace {

int batch_state(prr_ctx* c, BatchState** out) {
    if (!c->batch) {
        BatchState* b = new BatchState;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = batch_prepare_device();
        if (e == cudaSuccess) e = cudaEventCreate(&b->ev_start);
        if (e == cudaSuccess) e = cudaEventCreate(&b->ev_stop);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = b->queue.ensure(1);
        if (e == cudaSuccess) e = cudaMemset(b->queue.p, 0, sizeof(BatchQueue));
        if (e != cudaSuccess) {
            batch_state_destroy(b);
            return c->cuda(e);
        }
        c->batch = b;
    }
    *out = c->batch;
    return PRR_OK;
}

// Validate the jobs and lay the valid frames out in the batch buffers.
struct Totals {
    size_t packet_bytes = 0, words = 0, pairs = 0;
    uint64_t tiles = 0;
    uint32_t ent_items = 0, seg_items = 0;
};

Totals plan_batch(prr_job* jobs, size_t n, std::vector<FramePlan>& plan) {
    Totals t;
    plan.clear();
    for (size_t i = 0; i < n; i++) {
        prr_job& j = jobs[i];
        std::memset(&j.error, 0, sizeof(j.error));
        j.status = PRR_OK;
        j.result.n_skipped = 0;
        j.result.max_qscale = 0;
        if (!j.packet || !j.dev_out) {
            fail_job(j, PRR_ERR_INVALID);
            continue;
        }
        FramePlan f{};
        f.job = i;
        const int rc = prr_frame_info_parse(j.packet, size_t(j.len), &f.info, &j.error);
        if (rc != PRR_OK) {
            j.status = rc;
            continue;
        }
        j.result.header = f.info.header;
        const uint32_t cw = f.info.coded_width, ch = f.info.coded_height;
        if (j.scale == PRR_SCALE_FULL) {
            if (j.idct != PRR_IDCT_APPLE && j.idct != PRR_IDCT_FFMPEG) {
                fail_job(j, PRR_ERR_INVALID);
                continue;
            }
            if (j.out_len != uint64_t(cw) * ch) {
                fail_job(j, PRR_ERR_BUFFER);
                continue;
            }
        } else {
            if (j.scale < 1 || j.scale > 3 || j.greens < 0 || j.greens > 1) {
                fail_job(j, PRR_ERR_INVALID);
                continue;
            }
            if (j.out_len != 3 * uint64_t(cw >> j.scale) * (ch >> j.scale)) {
                fail_job(j, PRR_ERR_BUFFER);
                continue;
            }
        }
        f.shift = uint32_t(j.scale);
        f.lc = f.shift <= 1 ? 6 : (f.shift == 2 ? 4 : 2);
        const uint32_t ntiles = f.info.ntiles, columns = cw / 16;
        f.pkt_off = t.packet_bytes;
        t.packet_bytes += up16(prr_padded_packet_bytes(size_t(j.len)));
        f.words_off = t.words;
        t.words += up64(ntiles + 1) + up64(4 * size_t(ntiles)) + up64(ntiles);
        f.pairs_off = t.pairs;
        t.pairs += up64((size_t(f.info.tile_rows) * columns * 4) << f.lc);
        t.tiles += ntiles;
        t.seg_items += f.info.tile_rows * ((columns + 15) / 16);
        plan.push_back(f);
    }
    return t;
}

uint32_t bucket_key(size_t nframes, uint64_t tiles) {
    return (ceil_log2(std::max<size_t>(nframes, 1)) << 8) | ceil_log2(std::max<uint64_t>(tiles, 1));
}

prr_batch_config default_config() {
    prr_batch_config c{};
    c.ctas_per_sm = 0;
    c.stage_bytes = 32 * 1024;
    c.use_graph = 1;
    c.streams_per_thread = 2;
    return c;
}

int check_config(const prr_batch_config& c) {
    if (c.stage_bytes == 0 || c.stage_bytes > kBatchMaxStageBytes || (c.stage_bytes & 15) != 0)
        return PRR_ERR_INVALID;
    if (c.streams_per_thread != 0 && c.streams_per_thread != 1 && c.streams_per_thread != 2 &&
        c.streams_per_thread != 4)
        return PRR_ERR_INVALID;
    return PRR_OK;
}

uint32_t streams_per_thread_of(const prr_batch_config& c) { return c.streams_per_thread ? c.streams_per_thread : 2; }

// The jobs' packets into the pinned staging buffer at their planned
// offsets. A large batch is copied by several host threads, each taking
// an equal share of the bytes (a copy from pageable memory runs at a few
// GB/s a thread).
void stage_packets(uint8_t* dst, const prr_job* jobs, const std::vector<FramePlan>& plan, size_t total) {
    const size_t kPerThread = size_t(16) << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nthreads = unsigned(std::min<size_t>({size_t(hw), size_t(16), total / kPerThread + 1}));
    auto copy_range = [&](size_t lo, size_t hi) {
        // Bytes [lo, hi) of the staging buffer: the parts of the frames there.
        for (const FramePlan& f : plan) {
            const size_t a = f.pkt_off, b = f.pkt_off + size_t(jobs[f.job].len);
            const size_t x = std::max(a, lo), y = std::min(b, hi);
            if (x < y) std::memcpy(dst + x, jobs[f.job].packet + (x - a), y - x);
        }
    };
    if (nthreads <= 1) {
        copy_range(0, total);
        return;
    }
    std::vector<std::thread> pool;
    const size_t share = (total + nthreads - 1) / nthreads;
    for (unsigned k = 1; k < nthreads; k++)
        pool.emplace_back(copy_range, std::min(total, k * share), std::min(total, (k + 1) * share));
    copy_range(0, std::min(total, share));
    for (auto& th : pool) th.join();
}

// Enqueue the batch's kernels and the status download (directly, or as the
// bucket's graph).
int enqueue_kernels(prr_ctx* c, BatchState* B, Bucket& bk, const prr_batch_config& cfg, const BatchDesc& desc,
                    uint32_t grid_frames, uint32_t ctas) {
    auto record = [&](cudaStream_t s) -> int {
        PRR_TRY(c->cuda(launch_batch_tile_index(desc, grid_frames, s)));
        PRR_TRY(c->cuda(launch_batch_decode(desc, ctas, s)));
        return c->cuda(cudaMemcpyAsync(B->hstatus.p, B->status.p, grid_frames * sizeof(prr_dev_status),
                                       cudaMemcpyDeviceToHost, s));
    };
    if (!cfg.use_graph) return record(c->stream);
    const bool fresh = bk.exec && bk.gen == B->gen && bk.grid_frames == grid_frames && bk.ctas == ctas &&
                       bk.stage == desc.stage_bytes;
    if (!fresh) {
        if (bk.exec) cudaGraphExecDestroy(bk.exec);
        bk.exec = nullptr;
        PRR_TRY(c->cuda(cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal)));
        const int rc = record(B->cap_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(B->cap_stream, &g);
        if (rc != PRR_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PRR_TRY(c->cuda(e));
        const cudaError_t ei = cudaGraphInstantiate(&bk.exec, g, 0);
        cudaGraphDestroy(g);
        PRR_TRY(c->cuda(ei));
        bk.gen = B->gen;
        bk.grid_frames = grid_frames;
        bk.ctas = ctas;
        bk.stage = desc.stage_bytes;
    }
    // The graph's launches count like direct ones.
    count_launch(2);
    return c->cuda(cudaGraphLaunch(bk.exec, c->stream));
}

// `staged`: the jobs' packets already lie in this pinned host buffer of
// `staged_bytes`, each at a 16-byte aligned offset with its padded length
// inside the buffer; the buffer is uploaded as it is, without the copy into
// the batch's own staging. It must stay unchanged until the batch is waited
// for.
int submit(prr_ctx* c, prr_job* jobs, size_t n, const prr_batch_config* force, const uint8_t* staged = nullptr,
           size_t staged_bytes = 0) {
    if (!c || (!jobs && n > 0)) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    BatchState* B = nullptr;
    PRR_TRY(batch_state(c, &B));
    if (B->pending) return PRR_ERR_INVALID;  // wait for the previous batch first
    Totals t = plan_batch(jobs, n, B->plan);
    const size_t nf = B->plan.size();
    if (staged) {
        for (FramePlan& f : B->plan) {
            const prr_job& j = jobs[f.job];
            const uint8_t* p = j.packet;
            if (p < staged || (p - staged) % 16 != 0 ||
                size_t(p - staged) + up16(prr_padded_packet_bytes(size_t(j.len))) > staged_bytes)
                return PRR_ERR_INVALID;
            f.pkt_off = size_t(p - staged);
        }
        t.packet_bytes = staged_bytes;
    }
    B->jobs = jobs;
    B->njobs = n;
    if (nf == 0) {
        B->pending = true;
        B->last_ms = 0.f;
        return c->cuda(cudaEventRecord(B->ev_stop, c->stream));
    }
    if (t.tiles > 0xFFFFFFFFull / 4 || t.ent_items + uint64_t(t.seg_items) > 0xFFFFFFF0ull) return PRR_ERR_INVALID;
    const uint32_t key = bucket_key(nf, t.tiles);
    Bucket& bk = B->buckets[key];
    const prr_batch_config cfg = force ? *force : (bk.has_cfg ? bk.cfg : default_config());
    PRR_TRY(check_config(cfg));
    // Entropy items of the launch shape: tiles_per_item tiles each.
    const uint32_t spt = streams_per_thread_of(cfg), tiles_per_item = batch_tiles_per_item(spt);
    t.ent_items = 0;
    for (const FramePlan& f : B->plan) t.ent_items += (f.info.ntiles + tiles_per_item - 1) / tiles_per_item;
    if (t.ent_items + uint64_t(t.seg_items) > 0xFFFFFFF0ull) return PRR_ERR_INVALID;
    // Frames rounded up to a power of two: batches of one bucket share the
    // tile-index grid (and so the graph).
    const uint32_t grid_frames = 1u << ceil_log2(nf);
    const size_t meta_bytes = sizeof(BatchHeader) + size_t(grid_frames) * sizeof(BatchFrame);
    PRR_TRY(c->cuda(B->grow(B->meta, meta_bytes)));
    if (B->flags.cap < t.ent_items || B->flags.cap == 0) {
        // Fresh flags hold 0, which no batch's epoch (from 1 on) equals.
        PRR_TRY(c->cuda(B->grow(B->flags, std::max<size_t>(t.ent_items, 1))));
        PRR_TRY(c->cuda(cudaMemsetAsync(B->flags.p, 0, B->flags.cap * sizeof(uint32_t), c->stream)));
    }
    PRR_TRY(c->cuda(B->grow(B->packets, t.packet_bytes)));
    PRR_TRY(c->cuda(B->grow(B->words, t.words)));
    PRR_TRY(c->cuda(B->grow(B->pairs, std::max<size_t>(t.pairs, 64))));
    PRR_TRY(c->cuda(B->grow(B->status, grid_frames)));
    PRR_TRY(c->cuda(B->hmeta.ensure(meta_bytes)));
    if (!staged) PRR_TRY(c->cuda(B->hpackets.ensure(t.packet_bytes)));
    PRR_TRY(c->cuda(B->grow(B->hstatus, grid_frames)));
    int max_per_sm = 0;
    PRR_TRY(c->cuda(batch_max_ctas_per_sm(cfg.stage_bytes, &max_per_sm)));
    if (max_per_sm < 1) return PRR_ERR_INVALID;
    const uint32_t per_sm = cfg.ctas_per_sm == 0 ? uint32_t(max_per_sm)
                                                  : std::min<uint32_t>(cfg.ctas_per_sm, uint32_t(max_per_sm));
    const uint32_t ctas = per_sm * uint32_t(B->sms);

    // Frame table and packets, staged in pinned memory (free: the previous
    // batch was waited for).
    BatchHeader* hh = reinterpret_cast<BatchHeader*>(B->hmeta.p);
    BatchFrame* hf = reinterpret_cast<BatchFrame*>(B->hmeta.p + sizeof(BatchHeader));
    hh->nframes = uint32_t(nf);
    hh->ent_items = t.ent_items;
    hh->seg_items = t.seg_items;
    hh->wait_limit_us = B->wait_limit_us;
    hh->drop_item = B->drop_item;
    hh->streams_per_thread = spt;
    hh->pad[0] = hh->pad[1] = 0;
    uint32_t ent = 0, seg = 0;
    for (size_t i = 0; i < nf; i++) {
        const FramePlan& f = B->plan[i];
        const prr_job& j = jobs[f.job];
        BatchFrame& F = hf[i];
        std::memset(&F, 0, sizeof(F));
        F.d = make_frame_desc(f.info, B->packets.p + f.pkt_off);
        uint32_t* w = B->words.p + f.words_off;
        const uint32_t ntiles = f.info.ntiles;
        F.tile_off = w;
        F.d.counts = w + up64(ntiles + 1);
        F.skipped = F.d.counts + up64(4 * size_t(ntiles));
        F.d.pairs = B->pairs.p + f.pairs_off;
        F.st = B->status.p + i;
        F.out = j.dev_out;
        F.shift = f.shift;
        F.idct = uint32_t(j.idct);
        F.greens = f.shift == 0 ? 1u : uint32_t(j.greens);
        F.lc = f.lc;
        F.ent_begin = ent;
        F.seg_begin = seg;
        ent += (ntiles + tiles_per_item - 1) / tiles_per_item;
        seg += f.info.tile_rows * F.d.segs_per_row;
    }
    if (!staged) stage_packets(B->hpackets.p, jobs, B->plan, t.packet_bytes);
    PRR_TRY(c->cuda(cudaMemcpyAsync(B->meta.p, B->hmeta.p, sizeof(BatchHeader) + nf * sizeof(BatchFrame),
                                    cudaMemcpyHostToDevice, c->stream)));
    PRR_TRY(c->cuda(cudaMemcpyAsync(B->packets.p, staged ? staged : B->hpackets.p, t.packet_bytes,
                                    cudaMemcpyHostToDevice, c->stream)));
    BatchDesc desc{};
    desc.hdr = reinterpret_cast<const BatchHeader*>(B->meta.p);
    desc.frames = reinterpret_cast<const BatchFrame*>(B->meta.p + sizeof(BatchHeader));
    desc.q = B->queue.p;
    desc.flags = B->flags.p;
    desc.stage_bytes = cfg.stage_bytes;
    PRR_TRY(c->cuda(cudaEventRecord(B->ev_start, c->stream)));
    PRR_TRY(enqueue_kernels(c, B, bk, cfg, desc, grid_frames, ctas));
    PRR_TRY(c->cuda(cudaEventRecord(B->ev_stop, c->stream)));
    B->pending = true;
    return PRR_OK;
}

int wait(prr_ctx* c, uint32_t timeout_ms) {
    if (!c) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    BatchState* B = c->batch;
    if (!B || !B->pending) return PRR_ERR_INVALID;
    if (timeout_ms == 0) {
        PRR_TRY(c->cuda(cudaEventSynchronize(B->ev_stop)));
    } else {
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t e = cudaEventQuery(B->ev_stop);
            if (e == cudaSuccess) break;
            if (e != cudaErrorNotReady) return c->cuda(e);
            if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
                return PRR_ERR_TIMEOUT;
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    B->pending = false;
    B->last_ms = 0.f;
    if (!B->plan.empty()) PRR_TRY(c->cuda(cudaEventElapsedTime(&B->last_ms, B->ev_start, B->ev_stop)));
    for (size_t i = 0; i < B->plan.size(); i++) {
        const FramePlan& f = B->plan[i];
        prr_job& j = B->jobs[f.job];
        const prr_dev_status st = B->hstatus.p[i];
        if (st.oob_tile != NO_TILE) {
            fail_job(j, PRR_ERR_TILE_OUT_OF_BOUNDS);
            j.error.index = st.oob_tile;
            continue;
        }
        if (st.error) {
            fail_job(j, PRR_ERR_TIMEOUT);
            continue;
        }
        j.status = PRR_OK;
        j.result.max_qscale = uint8_t(st.max_qscale);
        j.result.n_skipped = st.n_skipped;
        if (st.n_skipped > 0 && j.result.skipped && j.result.skipped_cap > 0) {
            const uint32_t ns = std::min<uint32_t>(st.n_skipped, f.info.ntiles);
            PRR_TRY(c->cuda(B->hskipped.ensure(ns)));
            const uint32_t* src = B->words.p + f.words_off + up64(f.info.ntiles + 1) + up64(4 * size_t(f.info.ntiles));
            PRR_TRY(c->cuda(cudaMemcpyAsync(B->hskipped.p, src, ns * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                            c->stream)));
            PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
            std::sort(B->hskipped.p, B->hskipped.p + ns);
            const size_t m = std::min<size_t>(ns, j.result.skipped_cap);
            for (size_t k = 0; k < m; k++) j.result.skipped[k] = B->hskipped.p[k];
        }
    }
    return PRR_OK;
}

}  // namespace

int batch_submit_staged(prr_ctx* c, prr_job* jobs, size_t n, const uint8_t* staged, size_t staged_bytes) {
    if (!staged) return PRR_ERR_INVALID;
    return submit(c, jobs, n, nullptr, staged, staged_bytes);
}
int batch_wait(prr_ctx* c, uint32_t timeout_ms) { return wait(c, timeout_ms); }
float batch_last_ms(prr_ctx* c) { return c && c->batch ? c->batch->last_ms : 0.f; }
cudaEvent_t batch_start_event(prr_ctx* c) { return c && c->batch ? c->batch->ev_start : nullptr; }
cudaEvent_t batch_stop_event(prr_ctx* c) { return c && c->batch ? c->batch->ev_stop : nullptr; }

}  // namespace prr

using namespace prr;

extern "C" {

int prr_batch_submit(prr_ctx* c, prr_job* jobs, size_t n) { return submit(c, jobs, n, nullptr); }

int prr_batch_wait(prr_ctx* c, uint32_t timeout_ms) { return wait(c, timeout_ms); }

int prr_batch_last_ms(prr_ctx* c, float* ms) {
    if (!c || !ms || !c->batch) return PRR_ERR_INVALID;
    *ms = c->batch->last_ms;
    return PRR_OK;
}

int prr_batch_bucket(prr_ctx* c, const prr_job* jobs, size_t n, uint32_t* bucket) {
    if (!c || !bucket || (!jobs && n > 0)) return PRR_ERR_INVALID;
    size_t nf = 0;
    uint64_t tiles = 0;
    for (size_t i = 0; i < n; i++) {
        prr_frame_info f;
        if (!jobs[i].packet || prr_frame_info_parse(jobs[i].packet, size_t(jobs[i].len), &f, nullptr) != PRR_OK)
            continue;
        nf++;
        tiles += f.ntiles;
    }
    *bucket = bucket_key(nf, tiles);
    return PRR_OK;
}

int prr_batch_set_wait_limit(prr_ctx* c, uint32_t microseconds) {
    if (!c) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    BatchState* B = nullptr;
    PRR_TRY(batch_state(c, &B));
    B->wait_limit_us = microseconds;
    return PRR_OK;
}

int prr_batch_drop_chunk_for_test(prr_ctx* c, uint32_t chunk) {
    if (!c) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    BatchState* B = nullptr;
    PRR_TRY(batch_state(c, &B));
    B->drop_item = chunk;
    return PRR_OK;
}

int prr_batch_set_config(prr_ctx* c, uint32_t bucket, const prr_batch_config* cfg) {
    if (!c || !cfg) return PRR_ERR_INVALID;
    PRR_TRY(check_config(*cfg));
    PRR_TRY(c->use_device());
    BatchState* B = nullptr;
    PRR_TRY(batch_state(c, &B));
    Bucket& bk = B->buckets[bucket];
    bk.cfg = *cfg;
    bk.has_cfg = true;
    return PRR_OK;
}

int prr_batch_get_config(prr_ctx* c, uint32_t bucket, prr_batch_config* cfg) {
    if (!c || !cfg) return PRR_ERR_INVALID;
    *cfg = default_config();
    if (c->batch) {
        auto it = c->batch->buckets.find(bucket);
        if (it != c->batch->buckets.end() && it->second.has_cfg) *cfg = it->second.cfg;
    }
    return PRR_OK;
}

int prr_batch_tune(prr_ctx* c, prr_job* jobs, size_t n, uint32_t reps, prr_batch_config* best, float* best_ms) {
    if (!c || !jobs || n == 0) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    BatchState* B = nullptr;
    PRR_TRY(batch_state(c, &B));
    reps = std::max(reps, 1u);
    uint32_t bucket = 0;
    PRR_TRY(prr_batch_bucket(c, jobs, n, &bucket));
    prr_batch_config win = default_config();
    float win_ms = 1e30f;
    static const uint32_t stages[] = {16 * 1024, 32 * 1024, 48 * 1024, 64 * 1024, 96 * 1024};
    static const uint32_t spts[] = {1, 2, 4};
    for (uint32_t spt : spts)
    for (uint32_t stage : stages) {
        int max_per_sm = 0;
        PRR_TRY(c->cuda(batch_max_ctas_per_sm(stage, &max_per_sm)));
        for (int per_sm = 1; per_sm <= max_per_sm; per_sm++) {
            prr_batch_config cfg{};
            cfg.ctas_per_sm = uint32_t(per_sm);
            cfg.stage_bytes = stage;
            cfg.use_graph = 1;
            cfg.streams_per_thread = spt;
            std::vector<float> ms;
            // One untimed run captures the graph.
            for (uint32_t r = 0; r <= reps; r++) {
                PRR_TRY(submit(c, jobs, n, &cfg));
                PRR_TRY(wait(c, 0));
                if (r > 0) ms.push_back(B->last_ms);
            }
            std::sort(ms.begin(), ms.end());
            const float med = ms[ms.size() / 2];
            if (med < win_ms) {
                win_ms = med;
                win = cfg;
            }
        }
    }
    Bucket& bk = B->buckets[bucket];
    bk.cfg = win;
    bk.has_cfg = true;
    if (best) *best = win;
    if (best_ms) *best_ms = win_ms;
    return PRR_OK;
}

}  // extern "C"
