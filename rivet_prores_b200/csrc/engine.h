// engine.h -- host side of the library: contexts, device workspaces, batch
// plans and CUDA-graph capture around the decode and encode kernels.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/prores_b200.h"
#include "device_types.h"
#include "host_headers.h"

namespace prores {

// A device allocation that only grows.
// A device buffer that grows on demand. It is allocated stream-ordered on
// its workspace's stream (set when the workspace is made), and the growth
// waits for that stream only: cudaFree and cudaMalloc would wait for the
// whole device, which stalls every other thread's batch.
struct Context;

struct DeviceBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaStream_t stream = nullptr;
    uint32_t wait_ms = 0;  // bound on the wait for a growth (0: none)
    // The context whose idle workspaces are freed when a growth finds the
    // device out of memory (then the growth is tried once more).
    Context *owner = nullptr;
    cudaError_t reserve(size_t bytes);
    template <class T>
    T *as() const {
        return static_cast<T *>(p);
    }
    ~DeviceBuf();
};

struct PinnedBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t bytes);
    ~PinnedBuf();
};

// Copies between the device and host memory that may be pageable. Page-
// locked memory is copied straight (asynchronously); pageable memory goes
// through a ring of pinned chunks, because a CUDA copy to or from pageable
// memory returns only when it is done and holds up other host threads' CUDA
// calls meanwhile. Chunks read back are copied out by finish().
struct Stager {
    static constexpr int kSlots = 4;
    static constexpr size_t kChunk = 8u << 20;
    PinnedBuf buf;
    cudaEvent_t ev[kSlots] = {};
    uint32_t wait_ms = 0;  // bound on each wait for a chunk (0: none)
    struct Pending {
        uint8_t *dst = nullptr;  // host destination of a chunk read back
        size_t len = 0;
    } pend[kSlots];
    uint64_t issued = 0;
    ~Stager();
    cudaError_t h2d(void *dst, const void *src, size_t len, cudaStream_t s);
    cudaError_t d2h(void *dst, const void *src, size_t len, cudaStream_t s);
    // Waits for the chunks still read back and copies them out.
    cudaError_t finish();
    // Forgets chunks read back for a call that gave up: their host
    // destinations belong to that call's caller.
    void forget();

  private:
    cudaError_t slot(int &i);  // the next slot, free for the host
};

bool is_page_locked(const void *p);

// The library's default bound on a host wait for the device, in ms.
constexpr uint32_t kDefaultWaitMs = 60000;

// Waits until event `e` has completed, polling, for at most `limit_ms` (0:
// no bound). cudaErrorNotReady when the bound ran out first; the event's
// work is then still in flight.
cudaError_t wait_event(cudaEvent_t e, uint32_t limit_ms);
// Waits for everything enqueued on `s` so far the same way. PRORES_TIMEOUT
// when the bound runs out (the work is left running), PRORES_DEVICE on a
// CUDA failure.
Status wait_stream(cudaStream_t s, uint32_t limit_ms, const char *what);

// Per-call device state: a stream and the buffers a batch needs.
struct Workspace {
    int device = 0;
    uint32_t wait_ms = kDefaultWaitMs;  // the context's bound when the workspace was taken
    cudaStream_t stream = nullptr;
    DeviceBuf bits, frames, pics, slices, slot_status, pic_status, coef, coef_count, planes, alpha, weights, counter;
    // encode
    DeviceBuf enc_in, enc_alpha_in, enc_coef, enc_cost, enc_pic_state, enc_out, enc_slice_out, enc_alpha_bits,
        enc_alpha_bytes, enc_frame_out;
    PinnedBuf host_stage;
    // Points every DeviceBuf at the workspace's stream and at `owner`.
    void bind_stream(Context *owner);
    // Device bytes its buffers hold.
    size_t device_bytes() const;
    // Statuses and sizes read back each call. Pinned, because a copy into
    // pageable memory returns only when done and keeps other host threads'
    // CUDA calls waiting meanwhile.
    PinnedBuf host_small;
    Stager stager;
    ~Workspace();
};

struct KernelTimes {
    bool enabled = false;
    std::vector<cudaEvent_t> events;
    std::vector<const char *> names;
    std::vector<float> ms;
};

// Launch shapes and pipeline depth (prores_tuning); none changes any output.
struct Tuning {
    int cost_lane_items_per_sm = 640;  // the autotuner's choice on a B200: lanes from 8 UHD frames up
    int entropy_warps_per_block = 8;
    int entropy_blocks_per_sm = 0;
    int entropy_components_per_lane = 1;
    int staging_depth = 4;
    int decode_fused = 0;               // one kernel for the per-slice decode (else entropy, then IDCT)
    int decode_slot_positions = 65536;  // coefficient positions a CTA of the fused decode holds
    int decode_slot_bytes = 1;          // bytes a coefficient takes there (1: int8, 2: int16)
};

struct Context {
    int device = 0;
    int sm_count = 0;
    DeviceTables tables{};
    std::mutex m;
    // Read by every plan, under the mutex: a launch takes the shapes of the
    // moment; a CUDA graph keeps those it was captured with.
    Tuning tuning;
    EntropyShape entropy{8, 0};
    // Bound on every host wait for the device (prores_set_timeout).
    uint32_t wait_ms = kDefaultWaitMs;
    Tuning current_tuning();
    EntropyShape current_entropy();
    // Idle workspaces, kept with their buffers for the next call; at most
    // keep_free_bytes of device memory stays in them (the largest go first).
    std::vector<std::unique_ptr<Workspace>> free_ws;
    size_t keep_free_bytes = 0;
    // Frees idle workspaces, the largest first, until they hold at most
    // `keep` device bytes.
    void trim(size_t keep);
    // Workspaces whose stream still had work when a wait ran out or their
    // call gave up: reused once that work is done, never before.
    struct Retired {
        std::unique_ptr<Workspace> ws;
        cudaGraphExec_t graph = nullptr;  // destroyed with it
    };
    std::vector<Retired> retired;
    std::unique_ptr<Workspace> acquire();
    void release(std::unique_ptr<Workspace> ws);
    // Returns `ws` to the pool if its stream is idle, else keeps it (and
    // `graph`) aside until it is.
    void release_or_retire(std::unique_ptr<Workspace> ws, cudaGraphExec_t graph = nullptr);
    // Gives a job's workspace the context's current wait bound.
    void refresh(Workspace &ws);
    ~Context();
};

Status cuda_status(cudaError_t e, const char *what);

// ---- decode

struct DecodeFrame {
    Status err;  // a frame-header failure: nothing of the frame is decoded
    FrameHeader hdr;
    uint32_t depth = 0;
    uint32_t first_pic = 0, n_pics = 0;  // pictures handed to the device
    Status late;                         // a picture-level failure after those pictures
    size_t bits_off = 0;
    size_t plane_off = 0, samples = 0, alpha_off = 0, alpha_samples = 0;
    int desc = -1;  // FrameDesc index
};

struct DecodePlan {
    std::vector<DecodeFrame> frames;
    std::vector<FrameDesc> fdesc;
    std::vector<PicDesc> pdesc;
    std::vector<uint8_t> weights;
    size_t bits_total = 0, planes_total = 0, alpha_total = 0, coef_total = 0;
    uint32_t n_slices = 0;
    struct Copy {
        const uint8_t *src;
        size_t dst, len;
    };
    std::vector<Copy> copies;
    bool device_bits = false;  // the frames lie in device memory: copies are device to device
};

// Where plan_decode reads the frames' header bytes: read(i, pos, len) gives
// a host pointer to bytes [pos, pos + len) of frame i, or null when they are
// not at hand. Without it, the frames themselves are host memory.
using FrameBytes = std::function<const uint8_t *(int frame, size_t pos, size_t len)>;
// The bytes of the frame header that planning reads (8 + 20 + two 64-byte
// matrices, rounded up).
constexpr size_t kFrameHeadBytes = 160;
Status plan_decode(const prores_buf *in, int n, uint32_t out_depth, DecodePlan &plan,
                   const FrameBytes *bytes = nullptr);
Status upload_decode(Context &ctx, Workspace &ws, const DecodePlan &plan, cudaStream_t s);
Status upload_decode_bits(Workspace &ws, const DecodePlan &plan, const prores_buf *in, cudaStream_t s);
DecodeLaunch decode_launch_params(Context &ctx, Workspace &ws, const DecodePlan &plan);
// The fused decode's group: slices a CTA takes at once, and the coefficient
// positions it holds for them, for CTAs of at most `slot_positions`.
void fused_group(const DecodePlan &plan, uint32_t slot_positions, uint32_t &group, uint32_t &positions);
Status enqueue_decode(Context &ctx, Workspace &ws, const DecodePlan &plan, cudaStream_t s, KernelTimes *kt);
Status fetch_decode(Workspace &ws, const DecodePlan &plan, cudaStream_t s, prores_frame *out, int *status,
                    Status *first_err, bool device_out = false);

// ---- encode

struct EncodePlan;
struct EncodePlanDeleter {
    void operator()(EncodePlan *p) const;
};
using EncodePlanPtr = std::unique_ptr<EncodePlan, EncodePlanDeleter>;
Status plan_encode(const prores_config *cfg, const prores_frame *in, int n, EncodePlanPtr &plan);
Status upload_encode(Context &ctx, Workspace &ws, EncodePlan &plan, const prores_frame *in, cudaStream_t s,
                     bool descriptors, bool device_frames = false);
Status enqueue_encode(Context &ctx, Workspace &ws, EncodePlan &plan, cudaStream_t s, KernelTimes *kt);
// Waits for the encode and stages the packets in the workspace's pinned
// buffer; out[i] points into it until the workspace's next fetch.
Status fetch_encode(Context &ctx, Workspace &ws, EncodePlan &plan, cudaStream_t s, std::vector<prores_buf> &out,
                    int *status, Status *first_err);

void set_last_error(const Status &s);
// The same with messages already displayed (taken from another thread's).
void set_last_error_text(const std::string &text);
void set_batch_error_texts(const std::vector<std::string> &texts);
// prores_probe's work: the frame header, checked, as sizes and metadata.
Status probe_frame(const uint8_t *data, size_t len, uint32_t out_bit_depth, prores_frame *info);
// Per-frame messages of the last batch call on this thread.
void set_batch_errors(const std::vector<Status> &errs);
Status record_kernel(KernelTimes *kt, const char *name, cudaStream_t s);

}  // namespace prores

struct prores_ctx {
    prores::Context impl;
};

struct prores_decode_job {
    prores_ctx *ctx = nullptr;
    std::unique_ptr<prores::Workspace> ws;
    prores::DecodePlan plan;
    cudaGraphExec_t graph = nullptr;
    prores::KernelTimes kt;
};

struct prores_encode_job {
    prores_ctx *ctx = nullptr;
    std::unique_ptr<prores::Workspace> ws;
    prores::EncodePlanPtr plan;
    std::vector<prores_buf> packets;  // into the workspace's pinned staging buffer
    prores::KernelTimes kt;
};
