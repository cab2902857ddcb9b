// clip.cu -- decoding a movie's frames as a pipeline: the step before the
// decode path for a whole clip (src/mov.rs:172-183 feeding
// src/decoder.rs:226-267 frame after frame, as a caller of the crate does).
//
// Frames go in batches to the persistent batch decoder. While the device
// decodes batch k, a pool of host threads reads batch k+2's samples with
// positional reads straight into pinned staging (no second host copy), and
// batch k+1 is already uploaded and queued on the other of two lanes (each a
// context with its own stream, batch state and output buffer), so its
// upload overlaps batch k's kernels and the device never waits for the
// host between batches while the reads keep up.
//
// Buffers: three pinned read slots (batch k's upload may still be in flight
// while k+1 is queued and k+2 is read) and two device output slots (the
// batch handed to the caller and the batch being decoded).

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/prr.h"
#include "context.h"

namespace prr {
int batch_submit_staged(prr_ctx* c, prr_job* jobs, size_t n, const uint8_t* staged, size_t staged_bytes);
int batch_wait(prr_ctx* c, uint32_t timeout_ms);
float batch_last_ms(prr_ctx* c);
cudaEvent_t batch_start_event(prr_ctx* c);
cudaEvent_t batch_stop_event(prr_ctx* c);
int mov_read_fd(int fd, uint64_t offset, uint8_t* buf, size_t len, char* message, size_t message_cap);
int mov_track_fd(const prr_mov_track* t);
}  // namespace prr

namespace {

constexpr int kReadSlots = 3;
constexpr int kLanes = 2;
constexpr uint64_t kNone = ~0ull;

size_t up16(size_t v) { return (v + 15) & ~size_t(15); }
size_t up64(size_t v) { return (v + 63) & ~size_t(63); }

// One batch's samples in pinned memory, filled by the reader threads.
struct ReadSlot {
    HostBuf<uint8_t> buf;
    size_t bytes = 0;
    uint64_t batch = kNone;
    uint64_t first = 0;  // track sample index of the batch's first frame
    uint32_t n = 0;
    std::vector<size_t> off;
    std::vector<int> status;  // PRR_OK or PRR_ERR_MOVIE per frame
    std::vector<std::string> message;
    uint32_t claimed = 0, remaining = 0;  // under the clip's mutex
};

// A range of samples to decode: [first, first + count) in batches of the
// clip's size, numbered from g0 in the clip's sequence of batches (a queued
// range continues the numbering of the one before it).
struct Range {
    uint64_t first = 0, count = 0, nbatches = 0, g0 = 0;
    int32_t scale = 0, idct = 0, greens = 0;
};

// A context (stream + batch state), its output buffer and the jobs of the
// batch it holds.
struct Lane {
    prr_ctx* ctx = nullptr;
    DevBuf<uint16_t> out;
    std::vector<prr_job> jobs;
    std::vector<std::vector<uint64_t>> skipped;
    uint64_t batch = kNone;
    int slot = -1;
    bool pending = false;
};

}  // namespace

struct prr_clip {
    int device = 0;
    int fd = -1;  // the movie file (borrowed)
    uint32_t per_batch = 0;
    std::vector<prr_mov_sample> samples;
    Lane lanes[kLanes];
    ReadSlot slots[kReadSlots];

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int> work;  // read slots with frames left to claim
    bool stop = false;
    std::vector<std::thread> threads;

    // The end of batch g's kernels, recorded on its lane when it is queued
    // (slot g % 3 is recorded again only after batch g is finished): the
    // device time of a batch not overlapping the previous one.
    cudaEvent_t done[kReadSlots] = {};
    // The current range, then the queued one (at most one). Batches are
    // numbered across them: g_next is the next batch handed out; read slot
    // g % 3 and lane g % 2 hold batch g.
    std::deque<Range> ranges;
    uint64_t g_next = 0;
    bool ended = false;  // the current range's end (n = 0) has been handed out
    std::string last_error;

    int fail(int code, const std::string& m) {
        last_error = m;
        return code;
    }
    int cuda(cudaError_t e) {
        if (e == cudaSuccess) return PRR_OK;
        return fail(PRR_ERR_CUDA, cudaGetErrorString(e));
    }

    void reader() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv_work.wait(lk, [&] { return stop || !work.empty(); });
            if (stop) return;
            ReadSlot& r = slots[work.front()];
            if (r.claimed >= r.n) {
                work.pop_front();
                continue;
            }
            const uint32_t i = r.claimed++;
            lk.unlock();
            const prr_mov_sample& s = samples[r.first + i];
            char msg[512] = {0};
            const int rc = prr::mov_read_fd(fd, s.offset, r.buf.p + r.off[i], s.size, msg, sizeof(msg));
            lk.lock();
            r.status[i] = rc == PRR_OK ? PRR_OK : PRR_ERR_MOVIE;
            if (rc != PRR_OK) r.message[i] = msg;
            if (--r.remaining == 0) cv_done.notify_all();
        }
    }

    // The range holding batch g, and g's index in it (null past the ranges).
    const Range* range_of(uint64_t g, uint64_t* k) const {
        for (const Range& R : ranges)
            if (g >= R.g0 && g < R.g0 + R.nbatches) {
                *k = g - R.g0;
                return &R;
            }
        return nullptr;
    }
    bool exists(uint64_t g) const {
        uint64_t k;
        return range_of(g, &k) != nullptr;
    }

    uint32_t batch_frames(const Range& R, uint64_t k) const {
        return uint32_t(std::min<uint64_t>(per_batch, R.count - k * per_batch));
    }

    // Bytes batch k of range R takes in a read slot.
    size_t slot_bytes(const Range& R, uint64_t k) const {
        size_t b = 0;
        const uint64_t f0 = R.first + k * per_batch;
        for (uint32_t i = 0; i < batch_frames(R, k); i++)
            b += up16(prr_padded_packet_bytes(size_t(samples[f0 + i].size)));
        return b;
    }

    // Start the reads of batch g into read slot g % 3, whose previous batch
    // (g - 3) has been handed out and uploaded: the slot grows here if a
    // queued range has larger batches than the slots were sized for.
    int schedule_read(uint64_t g) {
        uint64_t k = 0;
        const Range* R = range_of(g, &k);
        if (!R) return fail(PRR_ERR_INVALID, "clip pipeline out of order");
        ReadSlot& r = slots[g % kReadSlots];
        PRR_TRY(cuda(r.buf.ensure(std::max<size_t>(slot_bytes(*R, k), 16))));
        std::lock_guard<std::mutex> lk(mu);
        r.batch = g;
        r.first = R->first + k * per_batch;
        r.n = batch_frames(*R, k);
        r.off.resize(r.n);
        r.status.assign(r.n, PRR_OK);
        r.message.assign(r.n, std::string());
        size_t o = 0;
        for (uint32_t i = 0; i < r.n; i++) {
            r.off[i] = o;
            o += up16(prr_padded_packet_bytes(size_t(samples[r.first + i].size)));
        }
        r.bytes = o;
        r.claimed = 0;
        r.remaining = r.n;
        work.push_back(int(g % kReadSlots));
        cv_work.notify_all();
        return PRR_OK;
    }

    void wait_read(const ReadSlot& r) {
        std::unique_lock<std::mutex> lk(mu);
        cv_done.wait(lk, [&] { return r.remaining == 0; });
    }

    bool submitted(uint64_t g) const { return lanes[g % kLanes].pending && lanes[g % kLanes].batch == g; }

    // Upload and queue batch k on lane k % 2 once its samples are read.
    int submit(uint64_t k) {
        uint64_t kr = 0;
        const Range* R = range_of(k, &kr);
        Lane& L = lanes[k % kLanes];
        ReadSlot& r = slots[k % kReadSlots];
        if (!R || L.pending || r.batch != k) return fail(PRR_ERR_INVALID, "clip pipeline out of order");
        const int32_t scale = R->scale, idct = R->idct, greens = R->greens;
        wait_read(r);
        L.jobs.assign(r.n, prr_job{});
        L.skipped.resize(r.n);
        // Output offsets from each frame's header (frames of a clip may differ).
        std::vector<size_t> out_off(r.n, 0);
        size_t total = 0;
        for (uint32_t i = 0; i < r.n; i++) {
            prr_job& j = L.jobs[i];
            j.len = samples[r.first + i].size;
            j.scale = scale;
            j.idct = idct;
            j.greens = greens;
            L.skipped[i].clear();
            if (r.status[i] != PRR_OK) continue;  // packet stays NULL: left out of the batch
            j.packet = r.buf.p + r.off[i];
            prr_frame_info info;
            prr_error err;
            if (prr_frame_info_parse(j.packet, size_t(j.len), &info, &err) != PRR_OK) {
                j.out_len = 0;  // the batch reports the parse error
                continue;
            }
            const uint64_t cw = info.coded_width, ch = info.coded_height;
            j.out_len = scale == PRR_SCALE_FULL ? cw * ch : 3 * (cw >> scale) * (ch >> scale);
            out_off[i] = total;
            total += up64(size_t(j.out_len));
            L.skipped[i].resize(info.ntiles);
        }
        PRR_TRY(cuda(L.out.ensure(std::max<size_t>(total, 64))));
        for (uint32_t i = 0; i < r.n; i++) {
            prr_job& j = L.jobs[i];
            // A frame whose header does not parse still needs an output
            // pointer to reach the parse (its status comes from there).
            j.dev_out = L.out.p + out_off[i];
            j.result.skipped = L.skipped[i].empty() ? nullptr : L.skipped[i].data();
            j.result.skipped_cap = L.skipped[i].size();
        }
        const int rc = prr::batch_submit_staged(L.ctx, L.jobs.data(), L.jobs.size(), r.buf.p, r.bytes);
        if (rc != PRR_OK) return fail(rc, L.ctx->last_error.empty() ? "batch submit failed" : L.ctx->last_error);
        PRR_TRY(cuda(cudaEventRecord(done[k % kReadSlots], static_cast<cudaStream_t>(prr_ctx_stream(L.ctx)))));
        L.batch = k;
        L.slot = int(k % kReadSlots);
        L.pending = true;
        return PRR_OK;
    }

    int finish(uint64_t k, prr_clip_batch* out) {
        Lane& L = lanes[k % kLanes];
        if (!L.pending || L.batch != k) return fail(PRR_ERR_INVALID, "clip pipeline out of order");
        const int rc = prr::batch_wait(L.ctx, 0);
        if (rc != PRR_OK) return fail(rc, L.ctx->last_error.empty() ? "batch wait failed" : L.ctx->last_error);
        L.pending = false;
        const ReadSlot& r = slots[L.slot];
        for (uint32_t i = 0; i < r.n; i++) {
            if (r.status[i] != PRR_OK) {
                L.jobs[i].status = PRR_ERR_MOVIE;
                std::memset(&L.jobs[i].error, 0, sizeof(prr_error));
                L.jobs[i].error.code = PRR_ERR_MOVIE;
                last_error = r.message[i];
            }
        }
        out->first = r.first;
        out->n = r.n;
        out->jobs = L.jobs.data();
        out->cuda_stream = prr_ctx_stream(L.ctx);
        out->device_ms = prr::batch_last_ms(L.ctx);
        // Busy time: the batch's kernel interval less the part during which
        // the previous batch (on the other lane) was still running.
        out->busy_ms = out->device_ms;
        if (k > 0 && r.n > 0) {
            float overlap = 0.f;
            if (cudaEventElapsedTime(&overlap, prr::batch_start_event(L.ctx), done[(k - 1) % kReadSlots]) ==
                    cudaSuccess &&
                overlap > 0.f)
                out->busy_ms = std::max(0.f, out->device_ms - overlap);
        }
        return PRR_OK;
    }

    // Wait for every batch in flight and every read (a new range, or the end).
    void drain() {
        for (Lane& L : lanes)
            if (L.pending) {
                prr::batch_wait(L.ctx, 0);
                L.pending = false;
            }
        std::unique_lock<std::mutex> lk(mu);
        cv_done.wait(lk, [&] {
            for (const ReadSlot& r : slots)
                if (r.remaining) return false;
            return true;
        });
        work.clear();
    }
};

namespace {

int check_range(const prr_clip* c, uint64_t first, uint64_t count, int scale) {
    if (first > c->samples.size() || count > c->samples.size() - first) return PRR_ERR_INVALID;
    if (scale != PRR_SCALE_FULL && (scale < 1 || scale > 3)) return PRR_ERR_INVALID;
    return PRR_OK;
}

Range make_range(const prr_clip* c, uint64_t first, uint64_t count, int scale, int idct, int greens,
                 uint64_t g0) {
    Range R;
    R.first = first;
    R.count = count;
    R.nbatches = (count + c->per_batch - 1) / c->per_batch;
    R.g0 = g0;
    R.scale = scale;
    R.idct = idct;
    R.greens = greens;
    return R;
}

}  // namespace

extern "C" {

int prr_clip_create_fd(int device, int fd, const prr_mov_sample* samples, size_t n_samples,
                       uint32_t frames_per_batch, uint32_t reader_threads, prr_clip** out) {
    if (!out || fd < 0 || (!samples && n_samples > 0) || frames_per_batch == 0 || reader_threads == 0 ||
        reader_threads > 256)
        return PRR_ERR_INVALID;
    *out = nullptr;
    auto* c = new prr_clip;
    c->device = device;
    c->fd = fd;
    c->per_batch = frames_per_batch;
    c->samples.assign(samples, samples + n_samples);
    int rc = PRR_OK;
    for (int i = 0; rc == PRR_OK && i < kLanes; i++) rc = prr_ctx_create(device, nullptr, &c->lanes[i].ctx);
    for (int i = 0; rc == PRR_OK && i < kReadSlots; i++)
        if (cudaEventCreate(&c->done[i]) != cudaSuccess) rc = PRR_ERR_CUDA;
    if (rc != PRR_OK) {
        for (Lane& L : c->lanes) prr_ctx_destroy(L.ctx);
        for (cudaEvent_t e : c->done)
            if (e) cudaEventDestroy(e);
        delete c;
        return rc;
    }
    for (uint32_t t = 0; t < reader_threads; t++) c->threads.emplace_back([c] { c->reader(); });
    *out = c;
    return PRR_OK;
}

int prr_clip_create(int device, const prr_mov_track* track, uint32_t frames_per_batch, uint32_t reader_threads,
                    prr_clip** out) {
    if (!out || !track) return PRR_ERR_INVALID;
    prr_mov_info info;
    PRR_TRY(prr_mov_get_info(track, &info));
    std::vector<prr_mov_sample> samples(size_t(info.n_samples));
    PRR_TRY(prr_mov_get_samples(track, 0, samples.size(), samples.data()));
    return prr_clip_create_fd(device, prr::mov_track_fd(track), samples.data(), samples.size(), frames_per_batch,
                              reader_threads, out);
}

void prr_clip_destroy(prr_clip* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    c->drain();
    {
        std::lock_guard<std::mutex> lk(c->mu);
        c->stop = true;
    }
    c->cv_work.notify_all();
    for (auto& t : c->threads) t.join();
    for (Lane& L : c->lanes) {
        L.out.release();
        prr_ctx_destroy(L.ctx);
    }
    for (ReadSlot& r : c->slots) r.buf.release();
    for (cudaEvent_t e : c->done)
        if (e) cudaEventDestroy(e);
    delete c;
}

int prr_clip_start(prr_clip* c, uint64_t first, uint64_t count, int scale, int idct, int greens) {
    if (!c) return PRR_ERR_INVALID;
    PRR_TRY(check_range(c, first, count, scale));
    if (cudaSetDevice(c->device) != cudaSuccess) return PRR_ERR_CUDA;
    c->drain();
    c->ranges.clear();
    c->ranges.push_back(make_range(c, first, count, scale, idct, greens, 0));
    c->g_next = 0;
    c->ended = false;
    for (ReadSlot& r : c->slots) r.batch = kNone;
    for (Lane& L : c->lanes) L.batch = kNone;
    // Every read slot sized for the largest batch of the range up front, so
    // that no pinned buffer is reallocated while batches are in flight.
    const Range& R = c->ranges.front();
    size_t most = 0;
    for (uint64_t k = 0; k < R.nbatches; k++) most = std::max(most, c->slot_bytes(R, k));
    for (ReadSlot& r : c->slots) PRR_TRY(c->cuda(r.buf.ensure(std::max<size_t>(most, 16))));
    return PRR_OK;
}

int prr_clip_queue(prr_clip* c, uint64_t first, uint64_t count, int scale, int idct, int greens) {
    if (!c || c->ranges.empty()) return PRR_ERR_INVALID;
    PRR_TRY(check_range(c, first, count, scale));
    if (c->ended) {
        // The current range is over (its n = 0 handed out): the queued one
        // simply follows it.
        c->ranges.pop_front();
        c->ended = false;
    } else if (c->ranges.size() > 1) {
        return PRR_ERR_INVALID;  // one queued range at a time
    }
    const uint64_t g0 = c->ranges.empty() ? c->g_next : c->ranges.back().g0 + c->ranges.back().nbatches;
    c->ranges.push_back(make_range(c, first, count, scale, idct, greens, g0));
    return PRR_OK;
}

int prr_clip_next(prr_clip* c, prr_clip_batch* out) {
    if (!c || !out || c->ranges.empty()) return PRR_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    if (cudaSetDevice(c->device) != cudaSuccess) return PRR_ERR_CUDA;
    const uint64_t g = c->g_next;
    const Range& R = c->ranges.front();
    if (g >= R.g0 + R.nbatches) {
        // The end of the range: n = 0. A queued range becomes the current
        // one; its first batches may already be read and queued.
        if (c->ranges.size() > 1)
            c->ranges.pop_front();
        else
            c->ended = true;
        return PRR_OK;
    }
    // Batch g and g + 1 read, and g queued, unless an earlier call did so
    // (a range's first batches, or a queued range's, read ahead).
    if (c->slots[g % kReadSlots].batch != g) PRR_TRY(c->schedule_read(g));
    if (c->exists(g + 1) && c->slots[(g + 1) % kReadSlots].batch != g + 1) PRR_TRY(c->schedule_read(g + 1));
    if (!c->submitted(g)) PRR_TRY(c->submit(g));
    // The caller is done with batch g - 1: its lane takes batch g + 1, and
    // its read slot (g + 2's) takes the next reads, into a queued range too.
    if (c->exists(g + 1) && !c->submitted(g + 1)) PRR_TRY(c->submit(g + 1));
    if (c->exists(g + 2) && c->slots[(g + 2) % kReadSlots].batch != g + 2) PRR_TRY(c->schedule_read(g + 2));
    PRR_TRY(c->finish(g, out));
    c->g_next = g + 1;
    return PRR_OK;
}

const char* prr_clip_last_error(const prr_clip* c) { return c ? c->last_error.c_str() : ""; }

}  // extern "C"
