/*
 * prores_b200.h -- C ABI of the B200 ProRes (SMPTE RDD 36) slice pipeline.
 *
 * The entry points replace the rivet-prores crate's public codec API
 * (imported as `prores`): Decoder::{new, with_bit_depth, with_threads,
 * decode} (src/decode.rs:28-104), Encoder::{new, encode} with Config and
 * Profile (src/encode.rs:31-287), and the Error kinds (src/error.rs:6-21).
 * Plain pointers and sizes only; no CUDA or torch types cross this boundary.
 *
 * Frame layout (src/frame.rs:172-266): one u16 buffer holding Y', then Cb,
 * then Cr, each tightly packed (stride == width); 4:2:2 chroma planes are
 * ceil(width/2) wide. Alpha, when present, is a separate width*height plane.
 * Samples carry their value in the low bit_depth bits.
 *
 * Threading: a context may be used from several threads at once; each call
 * takes its own device workspace and stream. Output never depends on the
 * batch composition, the thread count or the launch shape.
 */
#ifndef PRORES_B200_H
#define PRORES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. 1-3 are the crate's Error::{Invalid, Unsupported, Config}
 * (src/error.rs:6-21) and come back for exactly the inputs the crate refuses;
 * 4 and 5 are new: a CUDA failure, and a device wait that ran out. */
#define PRORES_OK 0
#define PRORES_INVALID 1
#define PRORES_UNSUPPORTED 2
#define PRORES_CONFIG 3
#define PRORES_DEVICE 4
#define PRORES_TIMEOUT 5

/* chroma_format codes (src/frame.rs:25-40) */
#define PRORES_CHROMA_422 2
#define PRORES_CHROMA_444 3

/* Profile (src/encode.rs:30-44), lowest rate first. */
#define PRORES_PROFILE_PROXY 0
#define PRORES_PROFILE_LT 1
#define PRORES_PROFILE_STANDARD 2
#define PRORES_PROFILE_HQ 3
#define PRORES_PROFILE_4444 4
#define PRORES_PROFILE_4444XQ 5

/* alpha_channel_type (src/header.rs:10-40) */
#define PRORES_ALPHA_NONE 0
#define PRORES_ALPHA_8 1
#define PRORES_ALPHA_16 2

typedef struct prores_ctx prores_ctx;

/* A picture (src/frame.rs:179-203). For decode into caller memory, set
 * data/alpha to buffers of data_len/alpha_len samples (prores_probe gives
 * the sizes); with data == NULL the library allocates and
 * prores_frame_free releases. */
typedef struct prores_frame {
    uint32_t width, height, bit_depth;
    int32_t chroma;    /* PRORES_CHROMA_422 or PRORES_CHROMA_444 */
    int32_t interlace; /* 0 progressive, 1 top field first, 2 bottom field first */
    uint8_t aspect_ratio, frame_rate_code, color_primaries, transfer_characteristic,
        matrix_coefficients, reserved_[3]; /* Metadata (src/frame.rs:84-96) */
    uint16_t *data;
    size_t data_len; /* samples in data */
    uint16_t *alpha; /* NULL: no alpha plane */
    size_t alpha_len;
} prores_frame;

/* Config (src/encode.rs:135-174). Defaults (Config::new): log2_slice_mbs 3,
 * alpha PRORES_ALPHA_16, no matrices, target_frame_bytes -1 (the profile's),
 * encoder_identifier "rivt", threads 0. prores_config_default fills them. */
typedef struct prores_config {
    int32_t profile;
    uint32_t log2_slice_mbs;
    int32_t alpha;
    int32_t has_luma_matrix, has_chroma_matrix;
    uint8_t luma_matrix[64], chroma_matrix[64]; /* raster order, weights 2-63 */
    int64_t target_frame_bytes;                 /* < 0: Profile::target_frame_bytes */
    uint8_t encoder_identifier[4];
    uint32_t threads; /* accepted and ignored: the output does not depend on it */
} prores_config;

/* One byte buffer (a ProRes frame: the bytes of one MOV sample). */
typedef struct prores_buf {
    const uint8_t *data;
    size_t len;
} prores_buf;

/* The parsed frame header (FrameHeader, src/header.rs:43-72). */
typedef struct prores_frame_header {
    uint32_t frame_size;
    uint16_t header_size;
    uint8_t bitstream_version;
    uint8_t encoder_identifier[4];
    uint8_t reserved_;
    uint16_t width, height;
    int32_t chroma, interlace, alpha; /* alpha: PRORES_ALPHA_* */
    uint8_t aspect_ratio, frame_rate_code, color_primaries, transfer_characteristic,
        matrix_coefficients, reserved2_[3];
    int32_t has_luma_matrix, has_chroma_matrix;
    uint8_t luma_matrix[64], chroma_matrix[64]; /* raster order */
} prores_frame_header;

/* ---- context ---------------------------------------------------------- */

/* A context on CUDA device `device`; NULL on failure (no device, or not
 * sm_100). Replaces constructing Decoder/Encoder values: the crate's are
 * stateless settings holders, this one owns device workspaces. A finished
 * call's workspace stays with the context, buffers and all, for the next
 * call; idle ones keep at most a quarter of the device's memory, and are
 * all freed when a call's allocation would otherwise fail. */
prores_ctx *prores_create(int device);
void prores_destroy(prores_ctx *ctx);

/* Bound, in ms, on every wait of the host for the device in calls made on
 * ctx from now on (0: no bound; default 60000). A call whose wait runs out
 * returns PRORES_TIMEOUT and leaves its device work running: a job stays
 * valid (its fetch can be called again), and a one-shot call's device
 * buffers are reused only after that work has finished. No reference
 * counterpart: the crate never waits on a device; this keeps its promise
 * that every failure comes back as an error (src/error.rs:3-5) when a
 * device stops making progress. */
int prores_set_timeout(prores_ctx *ctx, uint32_t ms);
uint32_t prores_get_timeout(prores_ctx *ctx);

/* Message of the last failing call made on this thread, formatted like the
 * crate's Error Display ("invalid ProRes data: ..."). */
const char *prores_last_error(void);

/* Message of frame i of the last batch call (decode or encode, including a
 * job's fetch) made on this thread; "" when that frame succeeded. */
const char *prores_batch_error(int i);

/* ---- decode (Decoder::decode, src/decode.rs:61-104) ------------------- */

/* Parses the frame header (FrameHeader::parse, src/header.rs:82-170) and the
 * plausibility check (src/decode.rs:113-128) without decoding: fills
 * width/height/bit_depth/chroma/interlace/metadata, data_len and alpha_len.
 * out_bit_depth 0 is the natural depth (10 for 4:2:2, 12 for 4:4:4); else
 * 8-16 (Decoder::with_bit_depth, src/decode.rs:37-47). */
int prores_probe(const uint8_t *data, size_t len, uint32_t out_bit_depth, prores_frame *info);

/* FrameHeader::parse (src/header.rs:82-170): host only, no device needed. */
int prores_parse_frame_header(const uint8_t *data, size_t len, prores_frame_header *out);

/* Decodes one frame. Bytes after frame_size are ignored. */
int prores_decode(prores_ctx *ctx, const uint8_t *data, size_t len, uint32_t out_bit_depth,
                  prores_frame *out);

/* Decodes n frames of any sizes and formats in one batched launch. status[i]
 * gets each frame's code (the message of the first failing one is kept for
 * prores_last_error); the call returns PRORES_OK unless a device error hit
 * the whole batch. */
int prores_decode_batch(prores_ctx *ctx, const prores_buf *in, int n, uint32_t out_bit_depth,
                        prores_frame *out, int *status);

void prores_frame_free(prores_frame *f);

/* ---- encode (Encoder::encode, src/encode.rs:223-287) ------------------ */

void prores_config_default(prores_config *cfg, int32_t profile);

/* Profile::target_frame_bytes (src/encode.rs:112-117). */
size_t prores_target_frame_bytes(int32_t profile, uint32_t width, uint32_t height);

/* Encodes one frame into a library-allocated packet (prores_buffer_free). */
int prores_encode(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, uint8_t **out,
                  size_t *out_len);

/* Encodes n frames (each with its own config) in one batched launch; out[i]
 * gets a library-allocated packet (prores_buffer_free each data). */
int prores_encode_batch(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n,
                        prores_buf *out, int *status);

void prores_buffer_free(void *p);

/* ---- one batch over several devices ------------------------------------ */

/* The frame-to-device split the *_multi calls use: part[i] in [0, parts)
 * for frame i of width[i] x height[i]. Largest frames first, each to the
 * part with the fewest macroblocks so far (ties to the lower part). No
 * reference counterpart: the crate leaves frame-level parallelism to its
 * caller (src/decode.rs:15-17, src/pool.rs:3-8); this is that caller's
 * split, done once for every user. Host only, no device needed. */
int prores_shard_frames(const uint32_t *width, const uint32_t *height, int n, int parts, int *part);

/* prores_decode_batch over several devices: ctxs[0..n_ctx) are contexts
 * (normally one per GPU). The frames are split by prores_shard_frames on
 * their headers' sizes, each context decodes its share in one batched call
 * on a host thread of its own, and out[i], status[i] and
 * prores_batch_error(i) come back in input order as from one call. The
 * devices exchange nothing: frames are independent. */
int prores_decode_batch_multi(prores_ctx *const *ctxs, int n_ctx, const prores_buf *in, int n,
                              uint32_t out_bit_depth, prores_frame *out, int *status);

/* prores_encode_batch over several devices, split and gathered the same
 * way; out[i] are library-allocated packets (prores_buffer_free). */
int prores_encode_batch_multi(prores_ctx *const *ctxs, int n_ctx, const prores_config *cfg, const prores_frame *in,
                              int n, prores_buf *out, int *status);

/* ---- frames found in a MOV, frames in device memory -------------------- */

/* Where one frame lies in a buffer. */
typedef struct prores_span {
    size_t offset;
    size_t len;
} prores_span;

/* The crate's scan for whole frames in a MOV file (or a prefix of one)
 * without parsing the container (tests/sample.rs:20-38,
 * examples/prores_bench.rs:103-121): at each byte position i from 4, "icpf"
 * with a big-endian frame_size >= 28 at i - 4 that ends inside the data is a
 * frame, and the scan resumes at its end. Writes up to cap spans and returns
 * how many frames there are (which may exceed cap). */
size_t prores_scan_frames(const uint8_t *data, size_t len, prores_span *frames, size_t cap);

/* The same scan over data in device memory (d_data, len bytes): a kernel
 * finds every "icpf" at once and the host resolves them in order by the
 * same rule, so the spans equal prores_scan_frames's. *count gets the number
 * of frames; up to cap spans are written. `stream` (a cudaStream_t, or NULL)
 * orders the scan after the caller's writes of d_data. No reference
 * counterpart for device memory. */
int prores_scan_frames_device(prores_ctx *ctx, const uint8_t *d_data, size_t len, prores_span *frames, size_t cap,
                              size_t *count, void *stream);

/* prores_probe for n frames that lie in device memory (d_data, data_len
 * bytes; frames[i] inside it): only the frame headers are read back.
 * status[i] and prores_batch_error(i) as in prores_decode_batch. */
int prores_probe_device(prores_ctx *ctx, const uint8_t *d_data, size_t data_len, const prores_span *frames, int n,
                        uint32_t out_bit_depth, prores_frame *info, int *status);

/* Decoder::decode (src/decode.rs:61-104) for n frames that lie in device
 * memory, into the caller's device buffers: out[i].data (data_len samples,
 * Y'‖Cb‖Cr as in prores_frame) and out[i].alpha (alpha_len samples, for a
 * frame with alpha) are device pointers, sized as prores_probe_device
 * says. Only the header bytes planning needs are read back to the host; the
 * bitstreams are copied device to device and the planes written in place.
 * The work runs on `stream` (a cudaStream_t, or NULL for the library's own)
 * and the call returns when it is done; the metadata fields of out[i] and
 * status[i] are filled as in prores_decode_batch. PRORES_CONFIG when a span
 * lies outside data_len or an output buffer is too small. */
int prores_decode_device(prores_ctx *ctx, const uint8_t *d_data, size_t data_len, const prores_span *frames, int n,
                         uint32_t out_bit_depth, prores_frame *out, int *status, void *stream);

/* Encoder::encode (src/encode.rs:223-287) for n frames whose planes (and
 * alpha) lie in device memory: in[i].data and in[i].alpha are device
 * pointers, everything else as in prores_encode_batch, whose packets (host,
 * library-allocated) and statuses this returns. The planes are copied
 * device to device; the work runs on `stream` (a cudaStream_t, or NULL)
 * and the call returns when it is done. */
int prores_encode_device(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n, prores_buf *out,
                         int *status, void *stream);

/* ---- decode without device allocation --------------------------------- */

/* Size of the fixed device array prores_decode_noalloc keeps its scratch in.
 * A frame fits when 4 bytes per coefficient position (512 positions per
 * 4:2:2 macroblock, 768 per 4:4:4 one), its frame_size bytes and 64 bytes
 * per slice, plus 53 KiB, come to no more than this: every 1920x1080 frame
 * whose packet is under about 40 MB (4:4:4) or 50 MB (4:2:2); UHD frames
 * do not fit. */
#define PRORES_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Decodes one frame, like prores_decode, without allocating any device
 * memory. It has no counterpart in the reference crate. It is for callers
 * that cannot allocate while they decode: a real-time playback thread (a
 * cudaMalloc can stall it, and cudaFree waits for the whole device), or a
 * host application whose device memory all comes from its own pool
 * allocator, which an allocation outside the pool would break. The caller
 * passes the frame's bytes in host memory and device buffers for the output
 * (d_planes: Y'‖Cb‖Cr, planes_len samples; d_alpha: the alpha plane, NULL
 * for a frame without alpha; prores_probe gives both sizes). The decoder's
 * scratch lives in one static device array of PRORES_NOALLOC_SCRATCH_BYTES
 * that every GPU which loads it holds until the process exits; a frame that
 * needs more (see PRORES_NOALLOC_SCRATCH_BYTES) is refused with PRORES_CONFIG. No
 * context is needed: the first call on a device sets that device up (the
 * array's address, the kernels' settings, the decoder's tables), so make that
 * first call before any stream capture. Every call shares the one array; the
 * call resets what must start at zero and returns after `stream` (a
 * cudaStream_t, or NULL) has finished, and calls whose work overlaps on the
 * GPU (from several threads or streams at once) race and must not be made. */
int prores_decode_noalloc(int device, const uint8_t *data, size_t len, uint32_t out_bit_depth,
                          uint16_t *d_planes, size_t planes_len, uint16_t *d_alpha, size_t alpha_len,
                          void *stream);

/* ---- resident jobs (batching and serving) ----------------------------- */

/* A decode job keeps a batch's bitstreams and planes resident in device
 * memory so that the batch can be decoded again without host traffic (and,
 * with use_graph, as one CUDA-graph launch). `stream` is a cudaStream_t
 * given as void* (NULL: the job's own stream). */
typedef struct prores_decode_job prores_decode_job;
int prores_decode_job_create(prores_ctx *ctx, const prores_buf *in, int n, uint32_t out_bit_depth,
                             prores_decode_job **job);
/* Enqueues the device work only (kernels over the resident bitstreams into
 * the resident planes); returns without waiting. */
int prores_decode_job_launch(prores_decode_job *job, void *stream, int use_graph);
/* Copies new bitstreams of the same sizes in (host to device) on `stream`. */
int prores_decode_job_upload(prores_decode_job *job, const prores_buf *in, int n, void *stream);
/* Waits for `stream`, copies the planes out and sets status[i]. */
int prores_decode_job_fetch(prores_decode_job *job, void *stream, prores_frame *out, int *status);
/* Device pointer of frame i's planes (Y'‖Cb‖Cr) and alpha in the job. */
int prores_decode_job_planes(prores_decode_job *job, int i, uint16_t **data, uint16_t **alpha);
void prores_decode_job_destroy(prores_decode_job *job);

typedef struct prores_encode_job prores_encode_job;
int prores_encode_job_create(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n,
                             prores_encode_job **job);
int prores_encode_job_launch(prores_encode_job *job, void *stream, int use_graph);
int prores_encode_job_upload(prores_encode_job *job, const prores_frame *in, int n, void *stream);
/* Waits for `stream`; out[i].data points into job-owned pinned host memory
 * (so it can feed a decode upload without a staging copy), valid
 * until the next fetch or destroy. */
int prores_encode_job_fetch(prores_encode_job *job, void *stream, prores_buf *out, int *status);
void prores_encode_job_destroy(prores_encode_job *job);

/* Per-kernel device time of the last launch of a job that was created with
 * profiling on (PRORES_PROFILE_KERNELS=1 in the environment): names[i] and
 * ms[i] for up to cap kernels; returns the count. */
int prores_job_kernel_times(const void *job, int is_encode, const char **names, float *ms, int cap);

/* Launch shapes and host pipeline depth. No reference counterpart: the
 * crate's only knob of this kind is Config/Decoder `threads`
 * (src/encode.rs:155-158, src/decode.rs:48-56), which likewise never changes
 * an output. None of these changes any decoded sample or encoded byte;
 * rivet_prores_b200.autotune times them on the device at hand. */
typedef struct prores_tuning {
    /* Rate-control costing runs a lane per slice component when the batch
     * has at least this many components per SM, else a warp per component. */
    int32_t cost_lane_items_per_sm;
    /* Entropy decoder: warps per block (1-16), resident blocks per SM (0 =
     * as many as fit), and slice components a lane takes per grab of the
     * shared work counter (1, 2 or 4). */
    int32_t entropy_warps_per_block;
    int32_t entropy_blocks_per_sm;
    int32_t entropy_components_per_lane;
    /* Batches a caller keeps in flight when it streams host buffers through
     * jobs (1-64): stored for the caller, read by no kernel. */
    int32_t staging_depth;
    /* Decoder: 1 runs the per-slice decode as one kernel (entropy decoding
     * into shared memory, then the IDCT and stores, per group of slices);
     * 0 as two (entropy decoding into lists in device memory, then the
     * IDCT). decode_slot_positions (512-65536): coefficient positions one
     * CTA of the fused kernel holds, which sets how many slices it takes
     * at once; decode_slot_bytes (1 or 2): the bytes each takes there (a
     * value the type cannot hold goes through device memory). */
    int32_t decode_fused;
    int32_t decode_slot_positions;
    int32_t decode_slot_bytes;
} prores_tuning;

void prores_tuning_default(prores_tuning *t);
/* Applies to the launches that follow on ctx; a job's CUDA graph keeps the
 * shapes it was captured with. PRORES_CONFIG for a value out of range. */
int prores_set_tuning(prores_ctx *ctx, const prores_tuning *t);
int prores_get_tuning(prores_ctx *ctx, prores_tuning *t);

#ifdef __cplusplus
}
#endif
#endif
