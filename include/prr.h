/*
 * prr.h -- C ABI of the B200 ProRes RAW decode / linearize / develop library
 * (libprr.so, CUDA sm_100a).
 *
 * The entry points mirror the public API of the proresraw_rs crate
 * (src/lib.rs:50-66). Each declaration names the crate item it replaces.
 * Conventions:
 *  - every call returns an int status: 0 = PRR_OK, negative values map 1:1
 *    onto the crate's `Error` variants (src/error.rs:6-63), plus library
 *    statuses (PRR_ERR_BUFFER replaces the crate's panics on wrongly sized
 *    `_into` buffers);
 *  - tiles with an invalid header are not errors: they are skipped, their
 *    sensels written as 0, and listed in frame order (src/decoder.rs:238-245);
 *  - packets are borrowed; device outputs are caller-owned buffers;
 *  - a context binds one device and one CUDA stream; calls on one context
 *    are not thread-safe, calls on different contexts are.
 * Device-resident inputs must be readable for prr_padded_packet_bytes(len)
 * bytes and 4-byte aligned (the stream reader loads aligned 32-bit words).
 */
#ifndef PRR_H
#define PRR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRR_ABI_VERSION 1

enum prr_status {
    PRR_OK = 0,
    /* src/error.rs:6-63, in declaration order */
    PRR_ERR_TRUNCATED = -1,
    PRR_ERR_FRAME_SIZE_MISMATCH = -2,
    PRR_ERR_BAD_QUANT_MATRIX = -3,
    PRR_ERR_BAD_CURVE = -4,
    PRR_ERR_UNEXPECTED_CURVE = -5,
    PRR_ERR_BAD_TAG = -6,
    PRR_ERR_HEADER_TOO_SHORT = -7,
    PRR_ERR_UNSUPPORTED_VERSION = -8,
    PRR_ERR_BAD_DIMENSIONS = -9,
    PRR_ERR_BAD_ALIGNMENT = -10,
    PRR_ERR_TILE_OUT_OF_BOUNDS = -11,
    PRR_ERR_BAD_TILE_HEADER = -12,
    /* library statuses */
    PRR_ERR_BUFFER = -20,  /* an output buffer has the wrong size (the crate panics) */
    PRR_ERR_CUDA = -21,    /* a CUDA call failed; see prr_last_error_string */
    PRR_ERR_TIMEOUT = -22, /* a bounded device loop gave up; the context stays usable */
    PRR_ERR_INVALID = -23, /* an argument is out of range */
    PRR_ERR_NO_MEMORY = -24,
    PRR_ERR_SCRATCH_LIMIT = -25, /* the frame has more tiles than prr_decode_noalloc's fixed scratch holds */
    PRR_ERR_MOVIE = -26,         /* a movie could not be read (mov::Error); the message says why */
};

/* Largest tile count prr_decode_noalloc accepts (8192x4320 at alignment 0
 * has 138,240 tiles). */
#define PRR_NOALLOC_MAX_TILES 262144u

/* Payload of an error: the fields of the matching `Error` variant. */
typedef struct prr_error {
    int32_t code;
    char what[32];       /* Truncated::what */
    uint64_t needed;     /* Truncated::needed */
    uint64_t available;  /* Truncated::available */
    uint32_t declared;   /* FrameSizeMismatch::declared */
    uint64_t actual;     /* FrameSizeMismatch::actual */
    uint64_t index;      /* BadQuantMatrix::index; TileOutOfBounds::tile; BadTileHeader::tile */
    uint32_t value;      /* BadQuantMatrix::value; UnsupportedVersion; BadAlignment; HeaderTooShort */
    uint16_t width, height; /* BadDimensions */
    uint16_t curve[8];   /* BadCurve */
    uint8_t tag[4];      /* BadTag */
} prr_error;

/* FrameHeader, src/header.rs:112-146. */
typedef struct prr_header {
    uint8_t version;
    uint8_t vendor[4];
    uint8_t bayer_pattern; /* header code: 0 RGGB, 1 GRBG, 2 GBRG, 3 BGGR */
    uint16_t width, height;
    uint8_t crop[4]; /* left, right, top, bottom */
    uint16_t white_level;
    uint16_t wb_cct;
    uint16_t flags;
    uint8_t alignment;
    uint8_t pad0;
    float wb_red, wb_blue;
    float color_matrix[9]; /* row-major camera RGB -> XYZ */
    float gain;
    uint8_t quant_matrix[64];
    uint16_t curve[8];
} prr_header;

/* Header plus tile grid: the host half of parse_frame (src/decoder.rs:76-123). */
typedef struct prr_frame_info {
    prr_header header;
    uint64_t packet_len;
    uint64_t table_offset; /* byte offset of the tile size table */
    uint32_t ntiles, tiles_per_row, tile_rows;
    uint32_t coded_width, coded_height;
    uint32_t pad0;
} prr_frame_info;

/* DemosaicParams, src/demosaic.rs:57-74. */
typedef struct prr_params {
    int32_t cfa_phase;
    int32_t black;
    float one_over_range;
    float noise[3];
    float clip[2];
    float black_over_range;
    float wb[2];
} prr_params;

/* Results of a synchronous decode: Frame / RgbFrame metadata
 * (src/decoder.rs:132-145, src/reduced.rs:76-94). */
typedef struct prr_decode_result {
    prr_header header;
    uint64_t n_skipped;   /* number of skipped tiles */
    uint64_t* skipped;    /* caller array, frame order, first skipped_cap entries */
    uint64_t skipped_cap;
    uint8_t max_qscale;
    uint8_t pad[7];
} prr_decode_result;

/* Status written on the device by the asynchronous decode entry points. */
typedef struct prr_dev_status {
    uint32_t oob_tile;   /* first tile whose size-table entry reaches past the packet, or 0xFFFFFFFF */
    uint32_t n_skipped;  /* tiles skipped for an invalid header */
    uint32_t max_qscale; /* ParsedFrame::max_qscale */
    uint32_t error;      /* nonzero when a bounded device loop gave up */
} prr_dev_status;

enum prr_idct { PRR_IDCT_APPLE = 0, PRR_IDCT_FFMPEG = 1 };             /* src/idct.rs:20-26 */
enum prr_scale { PRR_SCALE_HALF = 1, PRR_SCALE_QUARTER = 2, PRR_SCALE_EIGHTH = 3 }; /* src/reduced.rs:25-32, value = log2 factor */
enum prr_greens { PRR_GREENS_FIRST = 0, PRR_GREENS_AVERAGE = 1 };      /* src/reduced.rs:65-72 */
enum prr_stage { PRR_STAGE_DEMOSAICED = 0, PRR_STAGE_WHITE_BALANCED = 1, PRR_STAGE_REC2020 = 2 }; /* src/demosaic.rs:112-123 */
enum prr_exposure { PRR_EXPOSURE_NORMALIZED = 0, PRR_EXPOSURE_REFLECTION = 1 }; /* src/demosaic.rs:127-133 */
enum prr_layout { PRR_INTERLEAVED = 0, PRR_PLANAR = 1 };

typedef struct prr_ctx prr_ctx;

/* --- context ------------------------------------------------------------------ */
/* One device and one CUDA stream (NULL: the context creates its own
 * non-blocking stream; pass cudaStreamLegacy, (void*)0x1, to run on the
 * legacy default stream). */
int prr_ctx_create(int device, void* cuda_stream, prr_ctx** out);
void prr_ctx_destroy(prr_ctx* ctx);
/* The stream the context enqueues on (a cudaStream_t). */
void* prr_ctx_stream(prr_ctx* ctx);
/* Wait for all work enqueued on the context's stream. */
int prr_sync(prr_ctx* ctx);
const char* prr_status_string(int status);
/* Text of the last CUDA error seen by the context (or "" ). */
const char* prr_last_error_string(prr_ctx* ctx);
/* Bytes a device packet buffer must provide for a packet of `len` bytes. */
size_t prr_padded_packet_bytes(size_t len);
/* Counter of kernel launches made through this library (all contexts). */
uint64_t prr_kernel_launches(void);

/* --- host-side parsing -------------------------------------------------------- */
/* header_len, src/decoder.rs:58-73 */
int prr_header_len(const uint8_t* packet, size_t len, size_t* out, prr_error* err);
/* parse_header, src/decoder.rs:45-53 */
int prr_parse_header(const uint8_t* packet, size_t len, prr_header* out, prr_error* err);
/* parse_frame, src/decoder.rs:76-123, host half: prefix, header and size
 * table bounds; the per-tile walk (offsets, TileOutOfBounds, max_qscale)
 * runs on the device during decode. */
int prr_frame_info_parse(const uint8_t* packet, size_t len, prr_frame_info* out, prr_error* err);
/* parse_frame, src/decoder.rs:76-123, complete on the host: also walks the
 * size table for TileOutOfBounds and max_qscale (frame_quantizer,
 * src/demosaic.rs:50-52). */
int prr_parse_frame(const uint8_t* packet, size_t len, prr_frame_info* out, uint8_t* max_qscale,
                    prr_error* err);

/* --- decode (synchronous; packet in host memory) ----------------------------- */
/* decode_frame / decode_frame_with, src/decoder.rs:221-267. `dev_samples`
 * is a device buffer of coded_width * coded_height u16 (Frame::samples). */
int prr_decode(prr_ctx* ctx, const uint8_t* packet, size_t len, int idct, uint16_t* dev_samples,
               size_t samples_len, prr_decode_result* res, prr_error* err);
/* decode_frame_reduced / _with, src/reduced.rs:142-201. `dev_rgb` holds
 * 3 * (coded_width >> s) * (coded_height >> s) u16 (RgbFrame::samples). */
int prr_decode_reduced(prr_ctx* ctx, const uint8_t* packet, size_t len, int scale, int greens,
                       uint16_t* dev_rgb, size_t rgb_len, prr_decode_result* res, prr_error* err);

/* --- decode (asynchronous; packet resident on the device) -------------------- */
/* Device scratch bytes the asynchronous decodes need for a frame. */
size_t prr_decode_scratch_bytes(const prr_frame_info* info);
/* Enqueue the decode of `info` (from prr_frame_info_parse) whose bytes are
 * at `dev_packet`; writes code values (mode full) or linear RGB (reduced),
 * a prr_dev_status and the skipped tile indices (unordered, up to ntiles)
 * to device memory. No synchronization, no allocation: suitable for CUDA
 * graph capture. `dev_scratch` holds prr_decode_scratch_bytes(info) bytes. */
int prr_decode_async(prr_ctx* ctx, const prr_frame_info* info, const uint8_t* dev_packet, int idct,
                     uint16_t* dev_samples, prr_dev_status* dev_status, uint32_t* dev_skipped,
                     void* dev_scratch, size_t scratch_bytes);
int prr_decode_reduced_async(prr_ctx* ctx, const prr_frame_info* info, const uint8_t* dev_packet,
                             int scale, int greens, uint16_t* dev_rgb, prr_dev_status* dev_status,
                             uint32_t* dev_skipped, void* dev_scratch, size_t scratch_bytes);

/* A full-resolution decode that allocates no memory at all, for callers
 * that may not allocate device memory while they decode: plug-ins whose
 * host application owns the device memory and passes in only the input and
 * output buffers, and real-time loops in which a cudaMalloc would stall the
 * device or could fail because another allocator has reserved it. No
 * counterpart in the reference crate.
 * The caller passes the packet (device, padded as for prr_decode_async),
 * the code-value output, the status and the skipped-tile list; the one
 * piece of scratch, the tile-offset table, is a fixed array of
 * PRR_NOALLOC_MAX_TILES + 1 words inside the library, held by every device
 * that loads the library until the process exits. Frames with more tiles
 * return PRR_ERR_SCRATCH_LIMIT. The first call on a device looks the array
 * up (with `device` made current) and should come before any stream
 * capture on that device; the address is kept for the life of the process
 * and is not valid after a cudaDeviceReset. All calls share the array:
 * calls whose work overlaps on the GPU (other streams, other threads) race;
 * serialize them on one stream. `cuda_stream` is a cudaStream_t (NULL:
 * legacy default). `device` is an ordinal below 64 (else PRR_ERR_INVALID);
 * the calling thread's current device is the same on return as on entry. */
int prr_decode_noalloc(int device, void* cuda_stream, const prr_frame_info* info,
                       const uint8_t* dev_packet, int idct, uint16_t* dev_samples,
                       prr_dev_status* dev_status, uint32_t* dev_skipped);

/* --- batched decode ----------------------------------------------------------- */
/* Many frames at once -- any mix of sizes, bitstream versions, Bayer
 * patterns, qscales and tile alignments, at full resolution or reduced --
 * decoded by one persistent kernel that drains a device queue of work items
 * from all frames (after one tile-offset pass per frame). No counterpart in
 * the crate: each job is decode_frame_with (src/decoder.rs:226-267) or
 * decode_frame_reduced_with (src/reduced.rs:147-201) with the same output,
 * skipped-tile list and errors. */
#define PRR_SCALE_FULL 0
typedef struct prr_job {
    const uint8_t* packet;   /* host memory; read during prr_batch_submit */
    uint64_t len;
    int32_t scale;           /* PRR_SCALE_FULL or a prr_scale */
    int32_t idct;            /* full resolution: a prr_idct */
    int32_t greens;          /* reduced: a prr_greens */
    int32_t status;          /* result: PRR_OK or this frame's error */
    uint16_t* dev_out;       /* device: coded_width * coded_height u16 (full) or
                                3 * (coded_width >> s) * (coded_height >> s) u16 (reduced) */
    uint64_t out_len;
    prr_decode_result result; /* header, max_qscale, skipped tiles (caller array) */
    prr_error error;
} prr_job;

/* Launch shape of the batch kernel, per bucket of batches. */
typedef struct prr_batch_config {
    uint32_t ctas_per_sm;  /* persistent CTAs per SM; 0: as many as fit */
    uint32_t stage_bytes;  /* packet bytes an entropy item stages in shared memory:
                              a multiple of 16, at most 98304 */
    uint32_t use_graph;    /* replay a CUDA graph captured for the bucket */
    uint32_t streams_per_thread; /* component streams each of a CTA's 256 threads decodes in an
                                    entropy item: 1, 2 or 4 (items of 64, 128 or 256 tiles);
                                    0: 2 */
} prr_batch_config;

/* Parse the jobs' packets, upload them and enqueue the batch on the
 * context's stream. Jobs whose packet fails to parse or whose arguments are
 * wrong get their status now and are left out; the others are decoded.
 * Returns an error only for the call itself (bad context, CUDA failure).
 * `jobs` must stay valid until prr_batch_wait returns. */
int prr_batch_submit(prr_ctx* ctx, prr_job* jobs, size_t n);
/* Wait for the submitted batch (timeout_ms 0: no limit; PRR_ERR_TIMEOUT if
 * it has not finished, and the batch stays pending) and fill each job's
 * status, result and error. */
int prr_batch_wait(prr_ctx* ctx, uint32_t timeout_ms);
/* Device time of the last batch's kernels, in milliseconds. */
int prr_batch_last_ms(prr_ctx* ctx, float* ms);
/* The shape bucket of a batch: ceil(log2) of its frame count and of its
 * tile count. */
int prr_batch_bucket(prr_ctx* ctx, const prr_job* jobs, size_t n, uint32_t* bucket);
/* The autotuner: decodes the batch `reps` times under each candidate launch
 * shape (stage bytes x CTAs per SM), keeps the fastest as the config of the
 * batch's bucket and returns it with its median device time. The jobs'
 * results are those of the last run. */
int prr_batch_tune(prr_ctx* ctx, prr_job* jobs, size_t n, uint32_t reps, prr_batch_config* best,
                   float* best_ms);
/* Set or read the config of a bucket (unset buckets use the default). */
int prr_batch_set_config(prr_ctx* ctx, uint32_t bucket, const prr_batch_config* cfg);
/* The batch kernel's transform segments wait for the entropy chunks of
 * their tiles through flags in device memory; each wait gives up after
 * this many microseconds (0: the default of 2 s), the segment is left
 * unwritten and its frame's job reports PRR_ERR_TIMEOUT while the other
 * frames of the batch and the context stay usable. Applies to the batches
 * submitted after the call. No counterpart in the crate: its one device
 * wait is the map of a download buffer (src/gpu.rs:1231-1278). */
int prr_batch_set_wait_limit(prr_ctx* ctx, uint32_t microseconds);
/* Test hook for that limit: from the next batch on, entropy chunk `chunk`
 * (counted over the batch's frames in job order, 128 tiles a chunk) is
 * claimed and abandoned, as a CTA that died would leave it, so its flag is
 * never set. 0xFFFFFFFF turns it off. */
int prr_batch_drop_chunk_for_test(prr_ctx* ctx, uint32_t chunk);
int prr_batch_get_config(prr_ctx* ctx, uint32_t bucket, prr_batch_config* cfg);

/* --- linearize ---------------------------------------------------------------- */
/* Frame::linearize_into, src/decoder.rs:197-216: coded code values (device)
 * -> width*height linear values (device). Asynchronous. */
int prr_linearize(prr_ctx* ctx, const prr_header* header, const uint16_t* dev_samples,
                  uint16_t* dev_out, size_t out_len);

/* --- develop ------------------------------------------------------------------ */
/* DemosaicParams::new, src/demosaic.rs:80-82 */
int prr_params_new(const prr_header* header, uint32_t quantizer, prr_params* out);
/* DemosaicParams::with_white_balance, src/demosaic.rs:86-106 */
int prr_params_with_white_balance(const prr_header* header, uint32_t quantizer, float red,
                                  float blue, prr_params* out);
/* output_matrix, src/demosaic.rs:138-153 */
int prr_output_matrix(const prr_header* header, int exposure, float m[9]);
/* develop_into / develop_planar_into, src/demosaic.rs:223-261, on device
 * buffers. Interleaved: `r` holds 3*w*h floats (g, b unused). Planar: r, g,
 * b hold w*h floats each. Asynchronous. */
int prr_develop(prr_ctx* ctx, const prr_header* header, const prr_params* params, int stage,
                const uint16_t* dev_samples, int layout, float* r, float* g, float* b,
                size_t out_len);

/* --- learned develop ---------------------------------------------------------- */
/* A small convolutional network on the tensor cores (bf16 products, f32
 * accumulation) offered beside the plain develop: input the half-resolution
 * Bayer quads (colour differences against the quad's mean green, green level,
 * gradients and Laplacian) plus a noise channel from the plain develop's
 * noise model,
 * six 3x3 conv layers of 32 channels with ReLU, a 3x3 head of 12 channels
 * shuffled to full-resolution RGB on top of each quad's own colour. No
 * counterpart in the crate. Parameters are f32, layer by layer (weights
 * [cout][cin][9], bias [cout]; cin 16 then 32, cout 32 then 16 for the
 * head), prr_sg_param_count() of them. */
size_t prr_sg_param_count(void);

typedef struct prr_sg_model {
    const float* dev_params; /* device, prr_sg_param_count() floats */
    float noise_lo, noise_hi; /* range of the noise channel the network was trained on */
} prr_sg_model;

/* develop_into / develop_planar_into (src/demosaic.rs:223-261) by the
 * network, for the white-balanced and Rec.2020 stages (Demosaiced: white
 * balance 1). A 32x32 tile in which any quad's noise channel leaves
 * [noise_lo, noise_hi] is developed by the plain kernel instead (the
 * per-tile fallback); `fallback_tiles` (nullable; when given the call waits
 * for the device) receives how many. Buffers as for prr_develop. */
int prr_develop_learned(prr_ctx* ctx, const prr_header* header, const prr_params* params, int stage,
                        const uint16_t* dev_samples, const prr_sg_model* model, int layout, float* r,
                        float* g, float* b, size_t out_len, uint32_t* fallback_tiles);

/* Diagnostic: the network input and quad colours prr_develop_learned packs
 * from a decoded frame (stage as there), into host buffers: in16
 * [16][hq][wq] (the bf16 channels widened to f32) and base3 [3][hq][wq]
 * (red, mean green, blue), hq x wq = the frame's quads, network frame (the
 * picture mirrored so that red sits top left). Waits for the device. */
int prr_sg_pack(prr_ctx* ctx, const prr_header* header, const prr_params* params, int stage,
                const uint16_t* dev_samples, float* in16, float* base3);

/* Training on the device with the library's own forward (tensor cores) and
 * backward (f32) kernels and Adam. Frames are added decoded; their plain
 * white-balanced develop is the target. A step trains on `batch` crops of
 * crop x crop pixels (frame index, x, y; x and y even, the crop inside the
 * frame) with 8 quads of context around each. */
typedef struct prr_sg_trainer prr_sg_trainer;
int prr_sg_trainer_create(prr_ctx* ctx, uint32_t batch, uint32_t crop, prr_sg_trainer** out);
void prr_sg_trainer_destroy(prr_sg_trainer* t);
int prr_sg_trainer_add_frame(prr_sg_trainer* t, const prr_header* header, const prr_params* params,
                             const uint16_t* dev_samples, uint32_t* index);
/* The noise-channel range over the frames added so far. */
int prr_sg_trainer_noise_range(prr_sg_trainer* t, float* lo, float* hi);
/* Host parameters in (Adam state reset) or out. */
int prr_sg_trainer_set_params(prr_sg_trainer* t, const float* host_params);
int prr_sg_trainer_get_params(prr_sg_trainer* t, float* host_params);
/* The trainer's device parameters (for prr_develop_learned). */
const float* prr_sg_trainer_device_params(prr_sg_trainer* t);
/* One Adam step (beta 0.9 / 0.999); `crops` holds 3 * batch values; `loss`
 * (nullable; when given the call waits) receives the batch's mean squared
 * error before the step. */
int prr_sg_trainer_step(prr_sg_trainer* t, const uint32_t* crops, float lr, float* loss);
/* Forward, loss and parameter gradient of one explicit image: in16 [16][hq][wq],
 * base3 [3][hq][wq], target3 [3][2hq][2wq] planar f32, host memory. For
 * checking the device gradients. */
int prr_sg_gradients(prr_ctx* ctx, const float* in16, const float* base3, const float* target3, uint32_t hq,
                     uint32_t wq, const float* params, float* head_out, float* dparams, double* loss);

/* Cap prr_develop at `ctas_per_sm` CTAs per SM (0: as many as fit, the
 * default), so that kernels of another stream -- the next frame's decode --
 * find room on every SM while this context's develop runs. */
int prr_develop_set_occupancy(prr_ctx* ctx, uint32_t ctas_per_sm);

/* Launch shape of the develop kernel, per bucket of frame sizes: the
 * output tile (32x32, the default; 32x16; 64x16) and the CTAs per SM (0: as
 * many as fit). Every shape gives the same output bit for bit. The
 * crate's analogous knob is GpuDeveloper::set_band_rows
 * (src/gpu/develop.rs:44,281); a tile shape replaces its band height. */
typedef struct prr_develop_config {
    uint32_t tile_w, tile_h;
    uint32_t ctas_per_sm;
} prr_develop_config;
/* The bucket of a frame size: (ceil log2 width) << 8 | ceil log2 height. */
uint32_t prr_develop_bucket(uint32_t width, uint32_t height);
/* Use `cfg` for the frames of `bucket` (PRR_ERR_INVALID for a shape not
 * listed above). prr_develop_set_occupancy, when nonzero, still caps the
 * CTAs per SM. */
int prr_develop_set_config(prr_ctx* ctx, uint32_t bucket, const prr_develop_config* cfg);
/* The config of `bucket` (the default when none was set or tuned). */
int prr_develop_get_config(prr_ctx* ctx, uint32_t bucket, prr_develop_config* cfg);
/* Autotuner: develop this frame (arguments as prr_develop; the outputs are
 * written) with every candidate shape, `reps` timed runs each after an
 * untimed one, and keep the fastest (median device time) as the config of
 * the frame's bucket. Synchronous. */
int prr_develop_tune(prr_ctx* ctx, const prr_header* header, const prr_params* params, int stage,
                     const uint16_t* dev_samples, int layout, float* r, float* g, float* b,
                     size_t out_len, uint32_t reps, prr_develop_config* best, float* best_ms);

/* --- host-buffer conveniences (synchronous) ----------------------------------- */
/* decode_frame_with + develop_planar_into / develop_into with host input and
 * host outputs: uploads the packet, decodes and develops on the device and
 * copies the result back. params NULL: DemosaicParams::new(header,
 * Frame::quantizer). */
int prr_decode_develop_host(prr_ctx* ctx, const uint8_t* packet, size_t len, int idct,
                            const prr_params* params, int stage, int layout, float* r, float* g,
                            float* b, size_t out_len, prr_decode_result* res, prr_error* err);

/* --- movie sample tables (src/mov.rs) ------------------------------------------ */
/* The first enabled video track of a QuickTime / ISO movie: the samples it
 * presents (after the first non-empty edit), its rate and the movie's text
 * metadata. Host code; only the `moov` atom is read into memory. A track
 * keeps the file open for prr_mov_read_at (positional reads, safe from any
 * number of threads at once). */
typedef struct prr_mov_track prr_mov_track;

/* The sample description's fourcc filter, `accept: fn(&[u8; 4]) -> bool`
 * (src/mov.rs:173). Non-zero accepts. */
typedef int (*prr_mov_accept_fn)(const uint8_t fourcc[4], void* user);

/* mov::Sample (src/mov.rs:91-98). */
typedef struct prr_mov_sample {
    uint64_t offset; /* byte offset of the sample in the file */
    uint32_t size;   /* the sample's length in bytes */
    uint32_t pad;
} prr_mov_sample;

/* mov::Track without its vectors (src/mov.rs:100-124). orientation is the
 * EXIF value 1..8 (Orientation::exif, src/mov.rs:150-157). */
typedef struct prr_mov_info {
    uint8_t fourcc[4];
    uint32_t fps_num, fps_den;
    uint8_t variable_durations;
    uint8_t orientation;
    uint8_t has_creation_time;
    uint8_t reserved;
    uint64_t creation_time; /* seconds since 1904-01-01 UTC (mvhd), when has_creation_time */
    uint64_t n_samples;
    uint32_t n_warnings;
    uint32_t n_metadata;
} prr_mov_info;

/* mov::read_video_track (src/mov.rs:172-177) on the file at path. accept
 * NULL: is_prores_raw_fourcc (src/lib.rs:72-75). On failure returns
 * PRR_ERR_MOVIE with the crate's message in msg (truncated to msg_cap). */
int prr_mov_open(const char* path, prr_mov_accept_fn accept, void* user, prr_mov_track** out, char* msg,
                 size_t msg_cap);
void prr_mov_close(prr_mov_track* track);
int prr_mov_get_info(const prr_mov_track* track, prr_mov_info* info);
/* Track::samples[first .. first + count]. */
int prr_mov_get_samples(const prr_mov_track* track, size_t first, size_t count, prr_mov_sample* out);
/* Track::warnings[i]; NULL past the end. Owned by the track. */
const char* prr_mov_warning(const prr_mov_track* track, size_t i);
/* Track::metadata[i] as UTF-8 key and value, owned by the track. */
int prr_mov_metadata(const prr_mov_track* track, size_t i, const char** key, const char** value);
/* mov::read_at (src/mov.rs:179-183): len bytes at offset of the track's file. */
int prr_mov_read_at(const prr_mov_track* track, uint64_t offset, uint8_t* buf, size_t len, char* msg,
                    size_t msg_cap);

/* --- clip pipeline: a movie's frames through the batch decoder --------------- */
/* The frames of a movie track decoded batch by batch, the host's reads and
 * uploads overlapping the device's decode. No single counterpart in the
 * crate: each frame is mov::read_at (src/mov.rs:179-183) then
 * decode_frame_with / decode_frame_reduced_with (src/decoder.rs:226-267,
 * src/reduced.rs:147-201), with their outputs and errors. While the device
 * decodes batch k, batch k+1 is uploaded and queued on a second stream and
 * reader threads read batch k+2's samples straight into pinned memory. */
typedef struct prr_clip prr_clip;
typedef struct prr_clip_batch {
    uint64_t first;    /* track sample index of the batch's first frame */
    uint32_t n;        /* frames in the batch; 0 past the end of the range */
    float device_ms;   /* device time of the batch's kernels */
    float busy_ms;     /* the part of device_ms after the previous batch's kernels
                          ended: summed over a range, the device's busy time */
    uint32_t pad;
    prr_job* jobs;     /* n jobs, owned by the clip: each frame's status, result
                          (header, max_qscale, skipped tiles), error and device
                          output (dev_out, out_len); PRR_ERR_MOVIE when its
                          sample could not be read (prr_clip_last_error) */
    void* cuda_stream; /* the cudaStream_t the batch was decoded on */
} prr_clip_batch;

/* A pipeline over `track` (which must stay open): frames_per_batch frames a
 * batch, reader_threads host threads for the reads. */
int prr_clip_create(int device, const prr_mov_track* track, uint32_t frames_per_batch, uint32_t reader_threads,
                    prr_clip** out);
/* The same over a caller's own sample table (mov::Track::samples) and open
 * file descriptor (the movie's File, which must stay open), for callers
 * with their own movie reader. */
int prr_clip_create_fd(int device, int fd, const prr_mov_sample* samples, size_t n_samples,
                       uint32_t frames_per_batch, uint32_t reader_threads, prr_clip** out);
void prr_clip_destroy(prr_clip* clip);
/* Begin decoding samples [first, first + count) at `scale` (PRR_SCALE_FULL
 * with `idct`, or a prr_scale with `greens`); ends any range in progress. */
int prr_clip_start(prr_clip* clip, uint64_t first, uint64_t count, int scale, int idct, int greens);
/* The range to decode after the current one, same arguments as
 * prr_clip_start: once the current range's reads near their end, the
 * pipeline reads and uploads the queued range's first batches, so that its
 * first batch does not wait for its reads. prr_clip_next hands out the
 * current range's end (n = 0), then the queued range's batches. One range
 * queued at a time (PRR_ERR_INVALID for a second, or before any start);
 * prr_clip_start drops a queued range. No counterpart in the crate. */
int prr_clip_queue(prr_clip* clip, uint64_t first, uint64_t count, int scale, int idct, int greens);
/* The next decoded batch, in order (n = 0 at the end). Its outputs stay valid
 * until the next call; work reading them must be enqueued on cuda_stream,
 * which orders it before the buffers are reused, or be complete by then.
 * An error status ends the range (start again). */
int prr_clip_next(prr_clip* clip, prr_clip_batch* out);
/* The message of the last failed read or call. */
const char* prr_clip_last_error(const prr_clip* clip);

/* --- DNG export (examples/prr2dng) --------------------------------------------- */
/* Lossless JPEG tiles of a 16-bit CFA image (DNG compression 7): the tile x
 * tile squares of the image, row by row, each cut as dng::tile does
 * (examples/prr2dng/dng.rs:115-127: sensels past the right or bottom edge
 * repeat the nearest edge sensel of the same colour) and coded as
 * lj92::encode(tile, tile, tile, 2) does (examples/prr2dng/lj92.rs:14-69),
 * byte for byte. tile: even, 2..256 (DNG files use 256); width and height
 * at least 2; the image's rows are `stride` samples apart. */
uint64_t prr_lj92_tile_bound(uint32_t tile); /* worst-case bytes of one tile's stream */
/* Asynchronous: tile i's stream at dev_out + dev_offsets[i] (device array
 * of ntiles + 1 entries, the last the total). out_cap must hold ntiles x
 * prr_lj92_tile_bound(tile) bytes (PRR_ERR_BUFFER otherwise). */
int prr_lj92_encode(prr_ctx* ctx, const uint16_t* dev_image, uint32_t width, uint32_t height, uint64_t stride,
                    uint32_t tile, uint8_t* dev_out, uint64_t out_cap, uint64_t* dev_offsets);
/* The same into host memory (synchronous): offsets[ntiles + 1] and *total
 * are always set; PRR_ERR_BUFFER when cap < *total. */
int prr_lj92_encode_host(prr_ctx* ctx, const uint16_t* dev_image, uint32_t width, uint32_t height, uint64_t stride,
                         uint32_t tile, uint8_t* out, size_t cap, uint64_t* offsets, size_t* total);

/* ClipInfo (examples/prr2dng/dng.rs:46-57) and the writer's text. */
typedef struct prr_dng_clip {
    const char* make;      /* NULL: absent */
    const char* model;     /* NULL: absent */
    const char* date_time; /* "YYYY:MM:DD HH:MM:SS" (prr_dng_date_time); NULL: absent */
    const char* software;  /* tag 305; NULL: "proresraw_rs prr2dng 0.1.0" */
    uint32_t fps_num, fps_den; /* fps_den 0: no FrameRate */
    uint8_t orientation;   /* EXIF 1..8 (mov Orientation); 0 counts as 1 */
    uint8_t pad[7];
} prr_dng_clip;
enum prr_dng_samples { PRR_DNG_CODE_VALUES = 0, PRR_DNG_LINEAR = 1 };      /* dng::Samples */
enum prr_dng_compression { PRR_DNG_UNCOMPRESSED = 0, PRR_DNG_LJ92 = 1 };  /* dng::Compression */
typedef struct prr_dng_file prr_dng_file;

/* dng::write (examples/prr2dng/dng.rs:77-111) of a decoded frame on the
 * device (dev_samples: the decoder's code values over the coded size).
 * Linear samples are linearized on the device; LJ92 tiles of 256 are
 * encoded on the device; the TIFF container is written on the host. */
int prr_dng_write(prr_ctx* ctx, const prr_header* header, const uint16_t* dev_samples, int samples,
                  int compression, const prr_dng_clip* clip, prr_dng_file** out);
/* The same into a caller's buffer (pinned memory takes the copy from the
 * device fastest): *len is always set to the file's size; PRR_ERR_BUFFER
 * when out is NULL or cap < *len (nothing written). */
int prr_dng_write_into(prr_ctx* ctx, const prr_header* header, const uint16_t* dev_samples, int samples,
                       int compression, const prr_dng_clip* clip, uint8_t* out, size_t cap, size_t* len);
/* The container alone (host): `nchunks` chunks of `data` at offsets[0 ..
 * nchunks] -- one strip of the visible samples (little-endian u16,
 * uncompressed) or the frame's 256-square LJ92 tiles in order. */
int prr_dng_assemble(const prr_header* header, const prr_dng_clip* clip, int samples, int compression,
                     const uint8_t* data, const uint64_t* offsets, size_t nchunks, prr_dng_file** out);
const uint8_t* prr_dng_data(const prr_dng_file* file, size_t* len);
void prr_dng_free(prr_dng_file* file);

/* DngColour (examples/prr2dng/colour.rs:58-120): the colour tags of a header. */
typedef struct prr_dng_colour {
    double temperature;        /* kelvin */
    double color_matrix[9];    /* ColorMatrix1, row-major */
    double forward_matrix[9];  /* ForwardMatrix1 */
    double as_shot_neutral[3];
    double baseline_exposure;  /* stops */
    uint16_t illuminant;       /* CalibrationIlluminant1 (EXIF light source) */
    uint8_t pad[6];
} prr_dng_colour;
int prr_dng_colour_of(const prr_header* header, prr_dng_colour* out);
/* Value::srational / Value::rational (examples/prr2dng/tiff.rs:62-98). */
int prr_dng_srational(double v, int32_t* num, int32_t* den);
int prr_dng_rational(double v, uint32_t* num, uint32_t* den);
/* quicktime_date_time (examples/prr2dng/dng.rs:211-232): UTC text of seconds
 * since 1904, 19 characters and a NUL; PRR_ERR_BUFFER past the year 9999,
 * whose text would be longer. */
int prr_dng_date_time(uint64_t seconds, char out[20]);

/* --- diagnostics -------------------------------------------------------------- */
/* The device inverse transforms on raw blocks (idct.rs): kind 0 Apple 8x8,
 * 1 FFmpeg 8x8, 2 Apple 4x4 (16 coefficients per block), 3 Apple 2x2 (4).
 * q always holds 64 entries per block. Device buffers; asynchronous. */
int prr_transform_blocks(prr_ctx* ctx, int kind, const int16_t* dev_coefs, const int16_t* dev_q,
                         uint16_t* dev_out, size_t nblocks);
/* decode_component_reduced (src/coefficients.rs:37-146) on the device for
 * n streams of one packet: stream i at byte dev offset off[i] (alignment =
 * off[i] & 3) of length len[i], writing (64 or 16 or 4) << log2_blocks
 * coefficients per stream (not dequantized). off/len are device arrays. */
int prr_decode_components(prr_ctx* ctx, const uint8_t* dev_packet, const uint32_t* dev_off,
                          const uint32_t* dev_len, size_t n, int log2_blocks, int log2_coefs,
                          int16_t* dev_coefs);
/* The develop's paired division (fastdiv.cuh in the library's sources):
 * q[i] = a[i] / b[i] rounded to nearest, two a thread as the develop runs
 * it. It equals IEEE division for |a|, |b| in [2^-100, 2^100] and quotients
 * in [2^-120, 2^120] (outside that range the develop does not use it).
 * Device arrays; asynchronous. No counterpart in the crate. */
int prr_div_rn_pairs(prr_ctx* ctx, const float* dev_a, const float* dev_b, float* dev_q, size_t n);
/* Adds to *dev_mismatches (a device u64) the number of pairs (a, b), a over
 * every significand in [1, 2), b over the significands [b_first, b_first +
 * b_count) of [1, 2) (of 2^23), whose paired quotient differs from IEEE
 * division, plus each b whose paired reciprocal does not scale exactly
 * over the exponents [-100, 100]. b_first = 0, b_count = 2^23 checks all
 * 2^46 pairs. Asynchronous. No counterpart in the crate. */
int prr_div_rn_check(prr_ctx* ctx, uint32_t b_first, uint32_t b_count, uint64_t* dev_mismatches);
/* The develop's paired square root: adds to *dev_mismatches the number of
 * floats with exponent in [e_min, e_max] (every significand) whose paired
 * square root differs from IEEE sqrt. It equals IEEE sqrt on [2^-60, 2^60],
 * the range the develop uses it in. Asynchronous. No counterpart in the
 * crate. */
int prr_sqrt_rn_check(prr_ctx* ctx, int e_min, int e_max, uint64_t* dev_mismatches);
/* The same streams through the frame decode's entropy decoder (the one the
 * full and reduced frame decodes and the batch decode run; the decoder
 * above is the one inside the fused transform kernels): each stream's
 * (position, value) list goes to dev_lists (n << (log2_blocks +
 * log2_coefs) u32, 16-byte aligned), is replayed in order into dev_coefs
 * as above, and dev_flags[i] = list entries | 1 << 30 when the symbol
 * budget ran out | 1 << 31 when a zero run wrapped back over stored
 * positions (then entries past the list's capacity are dropped and the
 * frame decode decodes the stream again). `staged` != 0: streams are read
 * from a shared-memory copy of the CTA's span when it fits 32 KB, as in
 * the frame decode. Same stream semantics as src/coefficients.rs:37-146. */
int prr_decode_components_events(prr_ctx* ctx, const uint8_t* dev_packet, const uint32_t* dev_off,
                                 const uint32_t* dev_len, size_t n, int log2_blocks, int log2_coefs,
                                 int staged, uint32_t* dev_lists, int16_t* dev_coefs, uint32_t* dev_flags);

#ifdef __cplusplus
}
#endif
#endif
