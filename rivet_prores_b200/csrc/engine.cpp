// engine.cpp -- contexts, workspaces and the decode side of the batch engine.
//
// A batch of frames becomes one flat list of frames, pictures and slices:
// the host parses each frame's header and picture headers (src/header.rs),
// lays the frames' bytes end to end in one device buffer, and the kernels do
// everything per slice. Errors keep the crate's precedence: a frame-header
// failure first; then, picture by picture, a picture-header or slice-table
// failure, a slice that runs past picture_size, and the first failing slice
// component in picture order (src/decode.rs:85-104, :188-290).

#include "engine.h"

#include <sched.h>
#include <time.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "codec_tables.h"

namespace prores {

cudaError_t configure_decode_kernels();
cudaError_t configure_encode_kernels();

static thread_local std::string g_last_error;

static thread_local std::vector<std::string> g_batch_errors;

void set_last_error(const Status &s) { g_last_error = display(s); }

void set_last_error_text(const std::string &text) { g_last_error = text; }

void set_batch_error_texts(const std::vector<std::string> &texts) { g_batch_errors = texts; }

void set_batch_errors(const std::vector<Status> &errs) {
    g_batch_errors.assign(errs.size(), std::string());
    for (size_t i = 0; i < errs.size(); i++)
        if (errs[i]) g_batch_errors[i] = display(errs[i]);
}

Status cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return Status();
    // Only the bounded waits below report "not ready" up to here.
    if (e == cudaErrorNotReady)
        return make_status(PRORES_TIMEOUT, strf("%s: the device did not finish within the wait limit", what));
    return make_status(PRORES_DEVICE, strf("%s: %s", what, cudaGetErrorString(e)));
}

cudaError_t wait_event(cudaEvent_t e, uint32_t limit_ms) {
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(e);
        if (q != cudaErrorNotReady) return q;
        const double us = std::chrono::duration<double, std::micro>(clock::now() - t0).count();
        if (limit_ms && us >= 1000.0 * limit_ms) return cudaErrorNotReady;
        // Short waits (most of them) are polled; a long one sleeps between
        // polls, a little longer the longer it has waited.
        if (us < 2000.0) {
            sched_yield();
        } else {
            const long ns = us < 20000.0 ? 20000L : 100000L;
            timespec ts{0, ns};
            nanosleep(&ts, nullptr);
        }
    }
}

Status wait_stream(cudaStream_t s, uint32_t limit_ms, const char *what) {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (r != cudaSuccess) return cuda_status(r, what);
    r = cudaEventRecord(e, s);
    if (r == cudaSuccess) r = wait_event(e, limit_ms);
    cudaEventDestroy(e);
    return cuda_status(r, what);
}

#define PR_CUDA(expr, what)                                   \
    do {                                                      \
        Status st_ = cuda_status((expr), what);               \
        if (st_) return st_;                                  \
    } while (0)

// Capacity for `bytes`: at least half as much again as asked and a whole
// number of MiB, so that a workspace serving batches of changing sizes
// settles after a few growths (each reallocation waits for the device).
static size_t grown(size_t bytes, size_t cap) {
    size_t want = bytes + bytes / 2 + 4096;
    if (want < cap + cap / 2) want = cap + cap / 2;
    return (want + (1u << 20) - 1) & ~(size_t)((1u << 20) - 1);
}

cudaError_t DeviceBuf::reserve(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = grown(bytes, cap);
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocAsync(&p, want, stream);
    if (e == cudaErrorMemoryAllocation && owner) {
        // Idle workspaces may hold what this growth needs.
        cudaGetLastError();
        owner->trim(0);
        e = cudaMallocAsync(&p, want, stream);
    }
    // Usable from any stream once the workspace's stream has passed it.
    if (e == cudaSuccess) {
        cudaEvent_t ev;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) {
            e = cudaEventRecord(ev, stream);
            if (e == cudaSuccess) e = wait_event(ev, wait_ms);
            cudaEventDestroy(ev);
        }
        if (e == cudaErrorNotReady) return e;  // the allocation stands; the caller's workspace is retired
    }
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    cap = want;
    return cudaSuccess;
}

DeviceBuf::~DeviceBuf() {
    if (p) cudaFree(p);
}

cudaError_t PinnedBuf::reserve(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = grown(bytes, cap);
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    cap = want;
    return cudaSuccess;
}

PinnedBuf::~PinnedBuf() {
    if (p) cudaFreeHost(p);
}

bool is_page_locked(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

Stager::~Stager() {
    for (auto e : ev)
        if (e) cudaEventDestroy(e);
}

cudaError_t Stager::slot(int &i) {
    if (!buf.p) {
        cudaError_t e = buf.reserve(kSlots * kChunk);
        if (e != cudaSuccess) return e;
        for (auto &x : ev)
            if ((e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    i = (int)(issued % kSlots);
    if (issued >= (uint64_t)kSlots) {
        cudaError_t e = wait_event(ev[i], wait_ms);
        if (e != cudaSuccess) return e;
        if (pend[i].dst) memcpy(pend[i].dst, static_cast<uint8_t *>(buf.p) + (size_t)i * kChunk, pend[i].len);
    }
    pend[i] = Pending{};
    return cudaSuccess;
}

cudaError_t Stager::h2d(void *dst, const void *src, size_t len, cudaStream_t s) {
    if (!len) return cudaSuccess;
    if (is_page_locked(src)) return cudaMemcpyAsync(dst, src, len, cudaMemcpyHostToDevice, s);
    for (size_t off = 0; off < len; off += kChunk) {
        const size_t n = len - off < kChunk ? len - off : kChunk;
        int i;
        cudaError_t e = slot(i);
        if (e != cudaSuccess) return e;
        uint8_t *chunk = static_cast<uint8_t *>(buf.p) + (size_t)i * kChunk;
        memcpy(chunk, static_cast<const uint8_t *>(src) + off, n);
        if ((e = cudaMemcpyAsync(static_cast<uint8_t *>(dst) + off, chunk, n, cudaMemcpyHostToDevice, s)) !=
                cudaSuccess ||
            (e = cudaEventRecord(ev[i], s)) != cudaSuccess)
            return e;
        issued++;
    }
    return cudaSuccess;
}

cudaError_t Stager::d2h(void *dst, const void *src, size_t len, cudaStream_t s) {
    if (!len) return cudaSuccess;
    if (is_page_locked(dst)) return cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToHost, s);
    for (size_t off = 0; off < len; off += kChunk) {
        const size_t n = len - off < kChunk ? len - off : kChunk;
        int i;
        cudaError_t e = slot(i);
        if (e != cudaSuccess) return e;
        uint8_t *chunk = static_cast<uint8_t *>(buf.p) + (size_t)i * kChunk;
        if ((e = cudaMemcpyAsync(chunk, static_cast<const uint8_t *>(src) + off, n, cudaMemcpyDeviceToHost, s)) !=
                cudaSuccess ||
            (e = cudaEventRecord(ev[i], s)) != cudaSuccess)
            return e;
        pend[i] = Pending{static_cast<uint8_t *>(dst) + off, n};
        issued++;
    }
    return cudaSuccess;
}

void Stager::forget() {
    for (auto &p : pend) p = Pending{};
}

cudaError_t Stager::finish() {
    const uint64_t first = issued > (uint64_t)kSlots ? issued - kSlots : 0;
    for (uint64_t k = first; k < issued; k++) {
        const int i = (int)(k % kSlots);
        if (!pend[i].dst) continue;
        cudaError_t e = wait_event(ev[i], wait_ms);
        if (e != cudaSuccess) return e;
        memcpy(pend[i].dst, static_cast<uint8_t *>(buf.p) + (size_t)i * kChunk, pend[i].len);
        pend[i] = Pending{};
    }
    return cudaSuccess;
}

void Workspace::bind_stream(Context *owner) {
    for (DeviceBuf *b : {&bits, &frames, &pics, &slices, &slot_status, &pic_status, &coef, &coef_count, &planes,
                         &alpha, &weights, &counter, &enc_in, &enc_alpha_in, &enc_coef, &enc_cost, &enc_pic_state,
                         &enc_out, &enc_slice_out, &enc_alpha_bits, &enc_alpha_bytes, &enc_frame_out}) {
        b->stream = stream;
        b->wait_ms = wait_ms;
        b->owner = owner;
    }
}

size_t Workspace::device_bytes() const {
    size_t n = 0;
    for (const DeviceBuf *b : {&bits, &frames, &pics, &slices, &slot_status, &pic_status, &coef, &coef_count, &planes,
                               &alpha, &weights, &counter, &enc_in, &enc_alpha_in, &enc_coef, &enc_cost,
                               &enc_pic_state, &enc_out, &enc_slice_out, &enc_alpha_bits, &enc_alpha_bytes,
                               &enc_frame_out})
        n += b->cap;
    return n;
}

Workspace::~Workspace() {
    if (stream) cudaStreamDestroy(stream);
}

std::unique_ptr<Workspace> Context::acquire() {
    uint32_t limit;
    {
        std::lock_guard<std::mutex> g(m);
        limit = wait_ms;
        // Retired workspaces whose work has finished go back to the pool.
        for (size_t i = 0; i < retired.size();) {
            if (cudaStreamQuery(retired[i].ws->stream) == cudaSuccess) {
                if (retired[i].graph) cudaGraphExecDestroy(retired[i].graph);
                free_ws.push_back(std::move(retired[i].ws));
                retired.erase(retired.begin() + (long)i);
            } else {
                cudaGetLastError();
                i++;
            }
        }
        if (!free_ws.empty()) {
            auto ws = std::move(free_ws.back());
            free_ws.pop_back();
            ws->wait_ms = ws->stager.wait_ms = limit;
            ws->bind_stream(this);
            return ws;
        }
    }
    auto ws = std::make_unique<Workspace>();
    ws->device = device;
    ws->wait_ms = ws->stager.wait_ms = limit;
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    ws->bind_stream(this);
    return ws;
}

void Context::release(std::unique_ptr<Workspace> ws) {
    if (!ws) return;
    ws->stager.forget();
    size_t held = 0;
    {
        std::lock_guard<std::mutex> g(m);
        free_ws.push_back(std::move(ws));
        for (const auto &w : free_ws) held += w->device_bytes();
    }
    if (held > keep_free_bytes) trim(keep_free_bytes);
}

void Context::trim(size_t keep) {
    std::vector<std::unique_ptr<Workspace>> drop;
    {
        std::lock_guard<std::mutex> g(m);
        std::sort(free_ws.begin(), free_ws.end(),
                  [](const std::unique_ptr<Workspace> &a, const std::unique_ptr<Workspace> &b) {
                      return a->device_bytes() < b->device_bytes();
                  });
        size_t held = 0;
        for (const auto &w : free_ws) held += w->device_bytes();
        while (held > keep && !free_ws.empty()) {
            held -= free_ws.back()->device_bytes();
            drop.push_back(std::move(free_ws.back()));
            free_ws.pop_back();
        }
    }
    // Freed outside the lock: each cudaFree waits for the device.
    cudaSetDevice(device);
    drop.clear();
}

void Context::refresh(Workspace &ws) {
    uint32_t limit;
    {
        std::lock_guard<std::mutex> g(m);
        limit = wait_ms;
    }
    ws.wait_ms = ws.stager.wait_ms = limit;
    ws.bind_stream(this);
}

void Context::release_or_retire(std::unique_ptr<Workspace> ws, cudaGraphExec_t graph) {
    if (!ws) return;
    const cudaError_t q = cudaStreamQuery(ws->stream);
    if (q == cudaSuccess) {
        if (graph) cudaGraphExecDestroy(graph);
        release(std::move(ws));
        return;
    }
    cudaGetLastError();
    ws->stager.forget();
    std::lock_guard<std::mutex> g(m);
    retired.push_back(Retired{std::move(ws), graph});
}

Tuning Context::current_tuning() {
    std::lock_guard<std::mutex> g(m);
    return tuning;
}

EntropyShape Context::current_entropy() {
    std::lock_guard<std::mutex> g(m);
    return entropy;
}

Context::~Context() {
    cudaSetDevice(device);
    free_ws.clear();
    for (auto &r : retired) {
        cudaStreamSynchronize(r.ws->stream);
        if (r.graph) cudaGraphExecDestroy(r.graph);
    }
    retired.clear();
    if (tables.run_books) cudaFree(tables.run_books);
    if (tables.level_books) cudaFree(tables.level_books);
    if (tables.basis) cudaFree(tables.basis);
}

Status record_kernel(KernelTimes *kt, const char *name, cudaStream_t s) {
    if (!kt || !kt->enabled) return Status();
    cudaEvent_t e;
    PR_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    PR_CUDA(cudaEventRecord(e, s), "cudaEventRecord");
    kt->events.push_back(e);
    kt->names.push_back(name);
    return Status();
}

// ------------------------------------------------------------------ decode

static const char *device_message(int code) {
    switch (code) {
    case DE_PAST_END: return "a codeword runs past the end of its data";
    case DE_PREFIX: return "a variable-length code's prefix is too long";
    case DE_RANGE: return "a variable-length code's value is out of range";
    case DE_DC_OVERFLOW: return "a DC coefficient overflows";
    case DE_RUN_PAST_END: return "a run passes the end of the coefficient array";
    case DE_ALPHA_RUN: return "an alpha run passes the end of the slice";
    case DE_SLICE_SHORT: return "a slice is shorter than its header";
    case DE_COMP_SIZES: return "slice component sizes exceed the slice";
    }
    return "unknown slice failure";
}

static Status slot_status(int code, int aux) {
    if (code == DE_SLICE_HDR_SIZE) return make_status(PRORES_INVALID, strf("slice_header_size %d is out of range", aux));
    if (code == DE_QINDEX) return make_status(PRORES_INVALID, strf("quantization_index %d is reserved", aux));
    return make_status(PRORES_INVALID, device_message(code));
}

static uint32_t add_weights(std::vector<uint8_t> &w, const FrameHeader &h) {
    uint8_t set[128];
    h.luma_weights(set);
    h.chroma_weights(set + 64);
    for (size_t i = 0; i + 128 <= w.size(); i += 128)
        if (memcmp(&w[i], set, 128) == 0) return (uint32_t)(i / 128);
    w.insert(w.end(), set, set + 128);
    return (uint32_t)(w.size() / 128 - 1);
}

Status plan_decode(const prores_buf *in, int n, uint32_t out_depth, DecodePlan &plan, const FrameBytes *bytes) {
    plan = DecodePlan();
    plan.device_bits = bytes != nullptr;
    const auto read = [&](int i, size_t pos, size_t len) -> const uint8_t * {
        return bytes ? (*bytes)(i, pos, len) : in[i].data + pos;
    };
    plan.frames.resize(n);
    size_t bits_pos = 0;
    const uint8_t *prev_end = nullptr;
    for (int i = 0; i < n; i++) {
        DecodeFrame &f = plan.frames[i];
        // The frame's bytes go after the previous frame's; host-adjacent
        // buffers go over in one copy.
        f.bits_off = bits_pos;
        if (in[i].len) {
            if (!plan.copies.empty() && prev_end == in[i].data)
                plan.copies.back().len += in[i].len;
            else
                plan.copies.push_back({in[i].data, bits_pos, in[i].len});
            prev_end = in[i].data + in[i].len;
            bits_pos += in[i].len;
        }
        if (out_depth != 0 && (out_depth < 8 || out_depth > 16)) {
            f.err = make_status(PRORES_CONFIG, strf("output bit depth %u is outside 8\xe2\x80\x93" "16", out_depth));
            continue;
        }
        const uint8_t *head = read(i, 0, std::min(in[i].len, kFrameHeadBytes));
        if (!head) {
            f.err = make_status(PRORES_DEVICE, "the frame header was not fetched");
            continue;
        }
        if ((f.err = parse_frame_header(head, in[i].len, &f.hdr))) continue;
        if ((f.err = check_plausible_size(f.hdr))) continue;
        const FrameHeader &h = f.hdr;
        f.depth = out_depth ? out_depth : (h.chroma == PRORES_CHROMA_422 ? 10u : 12u);
        FrameDesc fd{};
        size_t off[3];
        f.samples = frame_layout(h.width, h.height, h.chroma, off, fd.plane_w);
        f.plane_off = plan.planes_total;
        plan.planes_total += f.samples;
        for (int c = 0; c < 3; c++) fd.plane_off[c] = f.plane_off + off[c];
        if (h.alpha) {
            f.alpha_samples = (size_t)h.width * h.height;
            f.alpha_off = plan.alpha_total;
            plan.alpha_total += f.alpha_samples;
        }
        fd.alpha_off = f.alpha_off;
        fd.width = h.width;
        fd.height = h.height;
        fd.chroma = (uint32_t)h.chroma;
        fd.alpha_bits = h.alpha_bits();
        fd.bit_depth = f.depth;
        fd.weights = add_weights(plan.weights, h);
        if (fd.alpha_bits) {
            fd.rescale_m = rescale_multiplier(fd.alpha_bits, f.depth);
            fd.rescale_identity = fd.alpha_bits == f.depth;
        }
        // §7.5.1: s = floor(v 2^b / 512 + 2^(b-1) + 1/2) in [0, 2^b - 1].
        fd.out_scale = (float)(1u << f.depth) / 512.0f;
        fd.out_bias = (float)(1u << (f.depth - 1)) + 0.5f;
        fd.out_max = (float)((1u << f.depth) - 1);
        f.desc = (int)plan.fdesc.size();
        plan.fdesc.push_back(fd);

        // Pictures: headers and slice tables are checked here; what fails is
        // reported after the pictures before it are decoded.
        const uint32_t cpm = h.chroma == PRORES_CHROMA_422 ? 2u : 4u;
        const uint32_t width_in_mb = (h.width + 15u) / 16u;
        size_t pos = 8 + (size_t)h.header_size;
        const size_t flen = h.frame_size;
        f.first_pic = (uint32_t)plan.pdesc.size();
        for (uint32_t index = 0; index < h.picture_count(); index++) {
            if (pos > flen) {
                f.late = make_status(PRORES_INVALID, "a picture starts past the end of the frame");
                break;
            }
            PictureHeader ph;
            const uint8_t *pic = read(i, pos, std::min(flen - pos, (size_t)kPictureHeaderSize));
            if (!pic) {
                f.late = make_status(PRORES_DEVICE, "a picture header was not fetched");
                break;
            }
            if ((f.late = parse_picture_header(pic, flen - pos, &ph))) break;
            const uint32_t height = h.picture_height(index);
            const uint32_t height_in_mb = (height + 15u) / 16u;
            const uint32_t spr = slices_per_row(width_in_mb, ph.log2_slice_mbs);
            const uint64_t n_slices = (uint64_t)spr * height_in_mb;
            if ((uint64_t)ph.header_size + 2 * n_slices > ph.picture_size) {
                f.late = make_status(PRORES_INVALID, "the slice table runs past picture_size");
                break;
            }
            PicDesc p{};
            p.off = f.bits_off + pos;
            p.coef_base = plan.coef_total;
            p.header_size = ph.header_size;
            p.picture_size = ph.picture_size;
            p.n_slices = (uint32_t)n_slices;
            p.slices_per_row = spr;
            p.width_in_mb = width_in_mb;
            p.height_in_mb = height_in_mb;
            p.log2_slice_mbs = ph.log2_slice_mbs;
            p.slice_base = plan.n_slices;
            p.frame = (uint32_t)f.desc;
            p.height = height;
            h.picture_rows(index, &p.first_row, &p.row_step);
            p.interlaced_scan = h.interlace != 0;
            plan.pdesc.push_back(p);
            plan.n_slices += (uint32_t)n_slices;
            plan.coef_total += (size_t)width_in_mb * height_in_mb * 64u * (4u + 2u * cpm);
            f.n_pics++;
            pos += ph.picture_size;
        }
    }
    plan.bits_total = bits_pos;
    return Status();
}

Status upload_decode_bits(Workspace &ws, const DecodePlan &plan, const prores_buf *in, cudaStream_t s) {
    (void)in;
    for (const auto &c : plan.copies)
        PR_CUDA(plan.device_bits ? cudaMemcpyAsync(ws.bits.as<uint8_t>() + c.dst, c.src, c.len,
                                                   cudaMemcpyDeviceToDevice, s)
                                 : ws.stager.h2d(ws.bits.as<uint8_t>() + c.dst, c.src, c.len, s),
                "bitstream upload");
    return Status();
}

Status upload_decode(Context &ctx, Workspace &ws, const DecodePlan &plan, cudaStream_t s) {
    (void)ctx;
    // 64 bytes of zero padding after the bitstreams: the readers fetch the
    // aligned word after the one they are in.
    PR_CUDA(ws.bits.reserve(plan.bits_total + 64), "cudaMalloc bitstream");
    PR_CUDA(cudaMemsetAsync(ws.bits.as<uint8_t>() + plan.bits_total, 0, 64, s), "memset");
    PR_CUDA(ws.frames.reserve(sizeof(FrameDesc) * (plan.fdesc.size() + 1)), "cudaMalloc");
    PR_CUDA(ws.pics.reserve(sizeof(PicDesc) * (plan.pdesc.size() + 1)), "cudaMalloc");
    PR_CUDA(ws.slices.reserve(sizeof(SliceDesc) * (plan.n_slices + 1)), "cudaMalloc");
    PR_CUDA(ws.slot_status.reserve(sizeof(int2) * 4 * ((size_t)plan.n_slices + 1)), "cudaMalloc");
    PR_CUDA(ws.pic_status.reserve(sizeof(PicStatus) * (plan.pdesc.size() + 1)), "cudaMalloc");
    PR_CUDA(ws.planes.reserve(2 * (plan.planes_total + 8)), "cudaMalloc planes");
    PR_CUDA(ws.alpha.reserve(2 * (plan.alpha_total + 8)), "cudaMalloc alpha");
    PR_CUDA(ws.weights.reserve(plan.weights.size() + 128), "cudaMalloc");
    PR_CUDA(ws.counter.reserve(64), "cudaMalloc");
    PR_CUDA(ws.coef.reserve(8 * (plan.coef_total + 64)), "cudaMalloc coefficient lists");
    PR_CUDA(ws.coef_count.reserve(4 * 3 * ((size_t)plan.n_slices + 1)), "cudaMalloc");
    if (!plan.fdesc.empty())
        PR_CUDA(ws.stager.h2d(ws.frames.p, plan.fdesc.data(), sizeof(FrameDesc) * plan.fdesc.size(), s),
                "upload");
    if (!plan.pdesc.empty())
        PR_CUDA(ws.stager.h2d(ws.pics.p, plan.pdesc.data(), sizeof(PicDesc) * plan.pdesc.size(), s),
                "upload");
    if (!plan.weights.empty())
        PR_CUDA(ws.stager.h2d(ws.weights.p, plan.weights.data(), plan.weights.size(), s),
                "upload");
    // The descriptor vectors are pageable: the stager copies them into
    // pinned chunks before returning, so the plan may change afterwards.
    return Status();
}

void fused_group(const DecodePlan &plan, uint32_t slot_positions, uint32_t &group, uint32_t &positions) {
    // The most coefficient positions any slice of the batch has: 64 per
    // block, 4 + 2 chroma blocks per macroblock, up to 2^log2_slice_mbs
    // macroblocks (no more than the picture is wide).
    uint32_t most = 64u * 8u;
    for (const PicDesc &p : plan.pdesc) {
        const uint32_t cpm = plan.fdesc[p.frame].chroma == PRORES_CHROMA_422 ? 2u : 4u;
        const uint32_t mbs = std::min(1u << p.log2_slice_mbs, p.width_in_mb);
        most = std::max(most, 64u * (4u + 2u * cpm) * mbs);
    }
    group = std::max(1u, std::min(kDecodeMaxGroup, slot_positions / most));
    positions = group * most;
}

DecodeLaunch decode_launch_params(Context &ctx, Workspace &ws, const DecodePlan &plan) {
    DecodeLaunch d{};
    d.bits = ws.bits.as<uint8_t>();
    d.bits_len = plan.bits_total;
    d.frames = ws.frames.as<FrameDesc>();
    d.pics = ws.pics.as<PicDesc>();
    d.slices = ws.slices.as<SliceDesc>();
    d.slot_status = ws.slot_status.as<int2>();
    d.pic_status = ws.pic_status.as<PicStatus>();
    d.coef = ws.coef.as<uint64_t>();
    d.coef_count = ws.coef_count.as<uint32_t>();
    d.planes = ws.planes.as<uint16_t>();
    d.alpha = ws.alpha.as<uint16_t>();
    d.weights = ws.weights.as<uint8_t>();
    d.work_counter = ws.counter.as<unsigned int>();
    d.n_frames = (uint32_t)plan.fdesc.size();
    d.n_pics = (uint32_t)plan.pdesc.size();
    d.n_slices = plan.n_slices;
    const Tuning t = ctx.current_tuning();
    d.entropy_per_lane = (uint32_t)t.entropy_components_per_lane;
    fused_group(plan, (uint32_t)t.decode_slot_positions, d.group, d.group_positions);
    d.slot_bytes = (uint32_t)t.decode_slot_bytes;
    d.tables = ctx.tables;
    return d;
}

Status enqueue_decode(Context &ctx, Workspace &ws, const DecodePlan &plan, cudaStream_t s, KernelTimes *kt) {
    const DecodeLaunch d = decode_launch_params(ctx, ws, plan);
    PR_CUDA(cudaMemsetAsync(d.work_counter, 0, sizeof(unsigned int), s), "memset");
    Status st;
    if ((st = record_kernel(kt, "start", s))) return st;
    PR_CUDA(launch_locate(d, s), "k_locate");
    if ((st = record_kernel(kt, "k_locate", s))) return st;
    if (ctx.current_tuning().decode_fused) {
        PR_CUDA(launch_decode(d, decode_grid(ctx.device, d.group, d.group_positions, d.slot_bytes), s), "k_decode");
        if ((st = record_kernel(kt, "k_decode", s))) return st;
    } else {
        PR_CUDA(launch_entropy(d, ctx.current_entropy(), s), "k_entropy");
        if ((st = record_kernel(kt, "k_entropy", s))) return st;
        PR_CUDA(launch_idct(d, s), "k_idct");
        if ((st = record_kernel(kt, "k_idct", s))) return st;
    }
    PR_CUDA(launch_status(d, s), "k_status");
    if ((st = record_kernel(kt, "k_status", s))) return st;
    return Status();
}

Status fetch_decode(Workspace &ws, const DecodePlan &plan, cudaStream_t s, prores_frame *out, int *status,
                    Status *first_err, bool device_out) {
    const size_t n_pics = plan.pdesc.size();
    PR_CUDA(ws.host_small.reserve(sizeof(PicStatus) * (n_pics + 1)), "cudaMallocHost");
    PicStatus *ps_host = static_cast<PicStatus *>(ws.host_small.p);
    if (n_pics)
        PR_CUDA(cudaMemcpyAsync(ps_host, ws.pic_status.p, sizeof(PicStatus) * n_pics, cudaMemcpyDeviceToHost, s),
                "status download");
    // Planes straight into the caller's buffers (one copy per run of
    // host-adjacent frames).
    struct Run {
        uint16_t *dst;
        size_t src, len;
        bool alpha;
    };
    std::vector<Run> runs;
    const int n = (int)plan.frames.size();
    for (int i = 0; i < n && !device_out; i++) {
        const DecodeFrame &f = plan.frames[i];
        prores_frame &o = out[i];
        if (f.err) continue;
        if (!o.data) {
            o.data = static_cast<uint16_t *>(malloc(2 * (f.samples ? f.samples : 1)));
            o.data_len = f.samples;
            if (f.alpha_samples) {
                o.alpha = static_cast<uint16_t *>(malloc(2 * f.alpha_samples));
                o.alpha_len = f.alpha_samples;
            } else {
                o.alpha = nullptr;
                o.alpha_len = 0;
            }
            if (!o.data || (f.alpha_samples && !o.alpha)) return make_status(PRORES_DEVICE, "host allocation failed");
        } else if (o.data_len < f.samples || (f.alpha_samples && (!o.alpha || o.alpha_len < f.alpha_samples))) {
            return make_status(PRORES_CONFIG, "an output buffer is smaller than its frame");
        }
        const auto add = [&](uint16_t *dst, size_t src, size_t len, bool alpha) {
            if (!len) return;
            if (!runs.empty() && runs.back().alpha == alpha && runs.back().dst + runs.back().len == dst &&
                runs.back().src + runs.back().len == src)
                runs.back().len += len;
            else
                runs.push_back({dst, src, len, alpha});
        };
        add(o.data, f.plane_off, f.samples, false);
        if (f.alpha_samples) add(o.alpha, f.alpha_off, f.alpha_samples, true);
    }
    for (const Run &r : runs) {
        const uint16_t *src = (r.alpha ? ws.alpha.as<uint16_t>() : ws.planes.as<uint16_t>()) + r.src;
        PR_CUDA(ws.stager.d2h(r.dst, src, 2 * r.len, s), "plane download");
    }
    {
        Status w = wait_stream(s, ws.wait_ms, "decode");
        if (w) return w;
    }
    PR_CUDA(ws.stager.finish(), "plane download");
    std::vector<Status> errs(n);
    for (int i = 0; i < n; i++) {
        const DecodeFrame &f = plan.frames[i];
        prores_frame &o = out[i];
        Status st = f.err;
        if (!st) {
            const FrameHeader &h = f.hdr;
            o.width = h.width;
            o.height = h.height;
            o.bit_depth = f.depth;
            o.chroma = h.chroma;
            o.interlace = h.interlace;
            o.aspect_ratio = h.aspect_ratio;
            o.frame_rate_code = h.frame_rate_code;
            o.color_primaries = h.color_primaries;
            o.transfer_characteristic = h.transfer_characteristic;
            o.matrix_coefficients = h.matrix_coefficients;
            for (uint32_t p = 0; p < f.n_pics && !st; p++) {
                const PicStatus &q = ps_host[f.first_pic + p];
                if (q.locate_slice >= 0)
                    st = make_status(PRORES_INVALID, "a slice runs past picture_size");
                else if (q.slot >= 0)
                    st = slot_status(q.code, q.aux);
            }
            if (!st && f.late) st = f.late;
        }
        status[i] = st.code;
        errs[i] = st;
        if (st && first_err && !*first_err) *first_err = st;
    }
    set_batch_errors(errs);
    return Status();
}

}  // namespace prores

// ====================================================================== C ABI

using namespace prores;

static int fail(const Status &s) {
    set_last_error(s);
    return s.code;
}

static int fail_or_ok(const Status &s) { return s ? fail(s) : PRORES_OK; }

static Status make_tables(Context &c) {
    std::vector<uint16_t> run6(kBookTableWords), level6(kBookTableWords);
    build_book_tables(run6.data(), level6.data());
    PR_CUDA(cudaMalloc(&c.tables.run_books, run6.size() * 2), "cudaMalloc");
    PR_CUDA(cudaMalloc(&c.tables.level_books, level6.size() * 2), "cudaMalloc");
    PR_CUDA(cudaMemcpy(c.tables.run_books, run6.data(), run6.size() * 2, cudaMemcpyHostToDevice), "upload");
    PR_CUDA(cudaMemcpy(c.tables.level_books, level6.data(), level6.size() * 2, cudaMemcpyHostToDevice), "upload");
    float basis[64];
    dct_basis(basis);
    PR_CUDA(cudaMalloc(&c.tables.basis, sizeof basis), "cudaMalloc");
    PR_CUDA(cudaMemcpy(c.tables.basis, basis, sizeof basis, cudaMemcpyHostToDevice), "upload");
    return Status();
}

static bool profiling_requested() {
    const char *v = getenv("PRORES_PROFILE_KERNELS");
    return v && v[0] && v[0] != '0';
}

namespace prores {

Status probe_frame(const uint8_t *data, size_t len, uint32_t out_bit_depth, prores_frame *info) {
    if (out_bit_depth != 0 && (out_bit_depth < 8 || out_bit_depth > 16))
        return (make_status(PRORES_CONFIG, strf("output bit depth %u is outside 8\xe2\x80\x93" "16", out_bit_depth)));
    FrameHeader h;
    Status st = parse_frame_header(data, len, &h);
    if (!st) st = check_plausible_size(h);
    if (st) return st;
    memset(info, 0, sizeof *info);
    info->width = h.width;
    info->height = h.height;
    info->bit_depth = out_bit_depth ? out_bit_depth : (h.chroma == PRORES_CHROMA_422 ? 10u : 12u);
    info->chroma = h.chroma;
    info->interlace = h.interlace;
    info->aspect_ratio = h.aspect_ratio;
    info->frame_rate_code = h.frame_rate_code;
    info->color_primaries = h.color_primaries;
    info->transfer_characteristic = h.transfer_characteristic;
    info->matrix_coefficients = h.matrix_coefficients;
    size_t off[3];
    uint32_t w[3];
    info->data_len = frame_layout(h.width, h.height, h.chroma, off, w);
    info->alpha_len = h.alpha ? (size_t)h.width * h.height : 0;
    return Status();
}

}  // namespace prores

extern "C" {

prores_ctx *prores_create(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        fail(make_status(PRORES_DEVICE, "no such CUDA device"));
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        fail(make_status(PRORES_DEVICE, "this library is built for sm_100 (B200) devices"));
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        fail(make_status(PRORES_DEVICE, "cudaSetDevice failed"));
        return nullptr;
    }
    auto *ctx = new prores_ctx();
    ctx->impl.device = device;
    ctx->impl.sm_count = prop.multiProcessorCount;
    Status st = make_tables(ctx->impl);
    if (!st) st = cuda_status(configure_decode_kernels(), "configure decode kernels");
    if (!st) st = cuda_status(configure_encode_kernels(), "configure encode kernels");
    if (st) {
        fail(st);
        delete ctx;
        return nullptr;
    }
    // Workspace buffers are allocated stream-ordered from the device's
    // default pool; keep up to 8 GiB of freed memory in it for the next
    // growth instead of handing it back at every synchronisation.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = 8ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    // Idle workspaces keep their buffers for the next call, up to a quarter
    // of the device's memory; past that the largest are freed.
    ctx->impl.keep_free_bytes = prop.totalGlobalMem / 4;
    ctx->impl.entropy = EntropyShape{ctx->impl.tuning.entropy_warps_per_block,
                                     entropy_grid(device, ctx->impl.tuning.entropy_warps_per_block,
                                                  ctx->impl.tuning.entropy_blocks_per_sm)};
    return ctx;
}

void prores_tuning_default(prores_tuning *t) {
    if (!t) return;
    const Tuning d;
    t->cost_lane_items_per_sm = d.cost_lane_items_per_sm;
    t->entropy_warps_per_block = d.entropy_warps_per_block;
    t->entropy_blocks_per_sm = d.entropy_blocks_per_sm;
    t->entropy_components_per_lane = d.entropy_components_per_lane;
    t->staging_depth = d.staging_depth;
    t->decode_fused = d.decode_fused;
    t->decode_slot_positions = d.decode_slot_positions;
    t->decode_slot_bytes = d.decode_slot_bytes;
}

int prores_set_tuning(prores_ctx *ctx, const prores_tuning *t) {
    if (!ctx || !t) return fail(make_status(PRORES_CONFIG, "no context or tuning"));
    if (t->cost_lane_items_per_sm < 0 || t->entropy_warps_per_block < 1 || t->entropy_warps_per_block > 16 ||
        t->entropy_blocks_per_sm < 0 || t->entropy_blocks_per_sm > 32 ||
        !(t->entropy_components_per_lane == 1 || t->entropy_components_per_lane == 2 ||
          t->entropy_components_per_lane == 4) ||
        t->staging_depth < 1 || t->staging_depth > 64 || t->decode_fused < 0 || t->decode_fused > 1 ||
        t->decode_slot_positions < 512 || t->decode_slot_positions > 65536 ||
        (t->decode_slot_bytes != 1 && t->decode_slot_bytes != 2))
        return fail(make_status(PRORES_CONFIG, "tuning value out of range"));
    cudaSetDevice(ctx->impl.device);
    const int grid = entropy_grid(ctx->impl.device, t->entropy_warps_per_block, t->entropy_blocks_per_sm);
    std::lock_guard<std::mutex> g(ctx->impl.m);
    ctx->impl.tuning = Tuning{t->cost_lane_items_per_sm, t->entropy_warps_per_block, t->entropy_blocks_per_sm,
                              t->entropy_components_per_lane, t->staging_depth, t->decode_fused,
                              t->decode_slot_positions, t->decode_slot_bytes};
    ctx->impl.entropy = EntropyShape{t->entropy_warps_per_block, grid};
    return PRORES_OK;
}

int prores_get_tuning(prores_ctx *ctx, prores_tuning *t) {
    if (!ctx || !t) return fail(make_status(PRORES_CONFIG, "no context or tuning"));
    const Tuning c = ctx->impl.current_tuning();
    t->cost_lane_items_per_sm = c.cost_lane_items_per_sm;
    t->entropy_warps_per_block = c.entropy_warps_per_block;
    t->entropy_blocks_per_sm = c.entropy_blocks_per_sm;
    t->entropy_components_per_lane = c.entropy_components_per_lane;
    t->staging_depth = c.staging_depth;
    t->decode_fused = c.decode_fused;
    t->decode_slot_positions = c.decode_slot_positions;
    t->decode_slot_bytes = c.decode_slot_bytes;
    return PRORES_OK;
}

int prores_set_timeout(prores_ctx *ctx, uint32_t ms) {
    if (!ctx) return fail(make_status(PRORES_CONFIG, "no context"));
    std::lock_guard<std::mutex> g(ctx->impl.m);
    ctx->impl.wait_ms = ms;
    return PRORES_OK;
}

uint32_t prores_get_timeout(prores_ctx *ctx) {
    if (!ctx) return 0;
    std::lock_guard<std::mutex> g(ctx->impl.m);
    return ctx->impl.wait_ms;
}

void prores_destroy(prores_ctx *ctx) { delete ctx; }

const char *prores_last_error(void) { return g_last_error.c_str(); }

const char *prores_batch_error(int i) {
    if (i < 0 || (size_t)i >= g_batch_errors.size()) return "";
    return g_batch_errors[i].c_str();
}

int prores_probe(const uint8_t *data, size_t len, uint32_t out_bit_depth, prores_frame *info) {
    return fail_or_ok(probe_frame(data, len, out_bit_depth, info));
}

int prores_parse_frame_header(const uint8_t *data, size_t len, prores_frame_header *out) {
    FrameHeader h;
    Status st = parse_frame_header(data, len, &h);
    if (st) return fail(st);
    memset(out, 0, sizeof *out);
    out->frame_size = h.frame_size;
    out->header_size = h.header_size;
    out->bitstream_version = h.bitstream_version;
    memcpy(out->encoder_identifier, h.encoder_identifier, 4);
    out->width = h.width;
    out->height = h.height;
    out->chroma = h.chroma;
    out->interlace = h.interlace;
    out->alpha = h.alpha;
    out->aspect_ratio = h.aspect_ratio;
    out->frame_rate_code = h.frame_rate_code;
    out->color_primaries = h.color_primaries;
    out->transfer_characteristic = h.transfer_characteristic;
    out->matrix_coefficients = h.matrix_coefficients;
    out->has_luma_matrix = h.has_luma;
    out->has_chroma_matrix = h.has_chroma;
    memcpy(out->luma_matrix, h.luma_matrix, 64);
    memcpy(out->chroma_matrix, h.chroma_matrix, 64);
    return PRORES_OK;
}

int prores_decode_batch(prores_ctx *ctx, const prores_buf *in, int n, uint32_t out_bit_depth, prores_frame *out,
                        int *status) {
    if (!ctx || n < 0) return fail(make_status(PRORES_CONFIG, "no context"));
    cudaSetDevice(ctx->impl.device);
    DecodePlan plan;
    Status st = plan_decode(in, n, out_bit_depth, plan);
    if (st) return fail(st);
    auto ws = ctx->impl.acquire();
    if (!ws) return fail(make_status(PRORES_DEVICE, "no stream"));
    cudaStream_t s = ws->stream;
    st = upload_decode(ctx->impl, *ws, plan, s);
    if (!st) st = upload_decode_bits(*ws, plan, in, s);
    if (!st) st = enqueue_decode(ctx->impl, *ws, plan, s, nullptr);
    Status first;
    if (!st) st = fetch_decode(*ws, plan, s, out, status, &first);
    if (st) {
        ctx->impl.release_or_retire(std::move(ws));
        return fail(st);
    }
    ctx->impl.release(std::move(ws));
    if (first) set_last_error(first);
    return PRORES_OK;
}

int prores_decode(prores_ctx *ctx, const uint8_t *data, size_t len, uint32_t out_bit_depth, prores_frame *out) {
    prores_buf b{data, len};
    int status = PRORES_OK;
    int r = prores_decode_batch(ctx, &b, 1, out_bit_depth, out, &status);
    if (r != PRORES_OK) return r;
    return status;
}

void prores_frame_free(prores_frame *f) {
    if (!f) return;
    free(f->data);
    free(f->alpha);
    f->data = nullptr;
    f->alpha = nullptr;
    f->data_len = f->alpha_len = 0;
}

void prores_buffer_free(void *p) { free(p); }

size_t prores_target_frame_bytes(int32_t profile, uint32_t width, uint32_t height) {
    if (profile < 0 || profile > 5) return 0;
    return target_frame_bytes(profile, width, height);
}

void prores_config_default(prores_config *cfg, int32_t profile) {
    memset(cfg, 0, sizeof *cfg);
    cfg->profile = profile;
    cfg->log2_slice_mbs = 3;
    cfg->alpha = PRORES_ALPHA_16;
    cfg->target_frame_bytes = -1;
    memcpy(cfg->encoder_identifier, "rivt", 4);
}

// ---- resident decode jobs

int prores_decode_job_create(prores_ctx *ctx, const prores_buf *in, int n, uint32_t out_bit_depth,
                             prores_decode_job **job) {
    if (!ctx || n < 0) return fail(make_status(PRORES_CONFIG, "no context"));
    cudaSetDevice(ctx->impl.device);
    auto *j = new prores_decode_job();
    j->ctx = ctx;
    j->kt.enabled = profiling_requested();
    Status st = plan_decode(in, n, out_bit_depth, j->plan);
    if (!st) {
        j->ws = ctx->impl.acquire();
        if (!j->ws) st = make_status(PRORES_DEVICE, "no stream");
    }
    if (!st) st = upload_decode(ctx->impl, *j->ws, j->plan, j->ws->stream);
    if (!st) st = upload_decode_bits(*j->ws, j->plan, in, j->ws->stream);
    if (!st) st = wait_stream(j->ws->stream, j->ws->wait_ms, "upload");
    if (st) {
        prores_decode_job_destroy(j);
        return fail(st);
    }
    *job = j;
    return PRORES_OK;
}

int prores_decode_job_upload(prores_decode_job *job, const prores_buf *in, int n, void *stream) {
    if ((size_t)n != job->plan.frames.size()) return fail(make_status(PRORES_CONFIG, "a job's batch size is fixed"));
    cudaSetDevice(job->ctx->impl.device);
    job->ctx->impl.refresh(*job->ws);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : job->ws->stream;
    size_t pos = 0;
    for (int i = 0; i < n; i++) {
        if (in[i].len != (i + 1 < n ? job->plan.frames[i + 1].bits_off : job->plan.bits_total) - job->plan.frames[i].bits_off)
            return fail(make_status(PRORES_CONFIG, "a job's frame sizes are fixed"));
        (void)pos;
    }
    // Same sizes, same places: one copy per host-adjacent run.
    const uint8_t *prev_end = nullptr;
    size_t run_dst = 0, run_len = 0;
    const uint8_t *run_src = nullptr;
    for (int i = 0; i < n; i++) {
        if (!in[i].len) continue;
        if (run_src && prev_end == in[i].data) {
            run_len += in[i].len;
        } else {
            if (run_src) {
                Status st = cuda_status(job->ws->stager.h2d(job->ws->bits.as<uint8_t>() + run_dst, run_src, run_len, s),
                                        "bitstream upload");
                if (st) return fail(st);
            }
            run_src = in[i].data;
            run_dst = job->plan.frames[i].bits_off;
            run_len = in[i].len;
        }
        prev_end = in[i].data + in[i].len;
    }
    if (run_src) {
        Status st = cuda_status(
            job->ws->stager.h2d(job->ws->bits.as<uint8_t>() + run_dst, run_src, run_len, s),
            "bitstream upload");
        if (st) return fail(st);
    }
    return PRORES_OK;
}

int prores_decode_job_launch(prores_decode_job *job, void *stream, int use_graph) {
    Context &c = job->ctx->impl;
    cudaSetDevice(c.device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : job->ws->stream;
    if (use_graph) {
        if (!job->graph) {
            cudaGraph_t g;
            cudaStream_t cap = job->ws->stream;
            Status st = cuda_status(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "capture");
            if (!st) {
                st = enqueue_decode(c, *job->ws, job->plan, cap, nullptr);
                cudaError_t e = cudaStreamEndCapture(cap, &g);
                if (!st) st = cuda_status(e, "capture");
            }
            if (!st) {
                st = cuda_status(cudaGraphInstantiate(&job->graph, g, 0), "graph instantiate");
                cudaGraphDestroy(g);
            }
            if (st) return fail(st);
        }
        return fail_or_ok(cuda_status(cudaGraphLaunch(job->graph, s), "graph launch"));
    }
    for (auto e : job->kt.events) cudaEventDestroy(e);
    job->kt.events.clear();
    job->kt.names.clear();
    Status st = enqueue_decode(c, *job->ws, job->plan, s, &job->kt);
    if (st) return fail(st);
    return PRORES_OK;
}

int prores_decode_job_fetch(prores_decode_job *job, void *stream, prores_frame *out, int *status) {
    cudaSetDevice(job->ctx->impl.device);
    job->ctx->impl.refresh(*job->ws);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : job->ws->stream;
    Status first;
    Status st = fetch_decode(*job->ws, job->plan, s, out, status, &first);
    if (st) return fail(st);
    if (first) set_last_error(first);
    return PRORES_OK;
}

int prores_decode_job_planes(prores_decode_job *job, int i, uint16_t **data, uint16_t **alpha) {
    if (i < 0 || (size_t)i >= job->plan.frames.size()) return fail(make_status(PRORES_CONFIG, "no such frame"));
    const DecodeFrame &f = job->plan.frames[i];
    *data = job->ws->planes.as<uint16_t>() + f.plane_off;
    *alpha = f.alpha_samples ? job->ws->alpha.as<uint16_t>() + f.alpha_off : nullptr;
    return PRORES_OK;
}

int prores_job_kernel_times(const void *job, int is_encode, const char **names, float *ms, int cap) {
    const KernelTimes &kt = is_encode ? static_cast<const prores_encode_job *>(job)->kt
                                      : static_cast<const prores_decode_job *>(job)->kt;
    if (!kt.enabled || kt.events.size() < 2) return 0;
    const uint32_t limit = is_encode ? static_cast<const prores_encode_job *>(job)->ws->wait_ms
                                     : static_cast<const prores_decode_job *>(job)->ws->wait_ms;
    {
        Status st = cuda_status(wait_event(kt.events.back(), limit), "kernel times");
        if (st) return fail(st);
    }
    int n = 0;
    for (size_t i = 1; i < kt.events.size() && n < cap; i++, n++) {
        float t = 0;
        cudaEventElapsedTime(&t, kt.events[i - 1], kt.events[i]);
        names[n] = kt.names[i];
        ms[n] = t;
    }
    return n;
}

void prores_decode_job_destroy(prores_decode_job *job) {
    if (!job) return;
    cudaSetDevice(job->ctx->impl.device);
    for (auto e : job->kt.events) cudaEventDestroy(e);
    if (job->ws) {
        // Its work may still run (a fetch that timed out): the workspace and
        // graph are then kept until it is done.
        job->ctx->impl.release_or_retire(std::move(job->ws), job->graph);
    } else if (job->graph) {
        cudaGraphExecDestroy(job->graph);
    }
    delete job;
}

}  // extern "C"
