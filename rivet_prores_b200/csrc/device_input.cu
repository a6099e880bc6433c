// Frames that arrive as a MOV (or a run of MOV samples) and frames that
// already lie in device memory.
//
// The crate finds whole frames in a file without parsing the container
// (tests/sample.rs:20-38, examples/prores_bench.rs:103-121): at each byte
// position i from 4, the four bytes "icpf" with a big-endian frame_size of
// at least 28 at i - 4 that ends inside the data are a frame, and the scan
// resumes where that frame ends; anything else moves on by one byte.
// prores_scan_frames restates that walk on the host. On the device a kernel
// finds every "icpf" at once (all candidates, whatever frame they fall in),
// and the host resolves them in position order with the same rule, which
// gives the same frames: a candidate inside an accepted frame is exactly one
// the sequential walk never reaches.
//
// prores_decode_device then decodes such frames where they lie: the host
// fetches only the header bytes it plans with (the frame header, then each
// picture header), the bitstreams are copied device to device into the
// workspace's padded buffer, and the kernels write the planes straight into
// the caller's device buffers.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "engine.h"

#define PR_CUDA(expr, what)                     \
    do {                                        \
        Status st_ = cuda_status((expr), what); \
        if (st_) return st_;                    \
    } while (0)

namespace prores {
namespace {

constexpr int kScanThreads = 256;
constexpr uint32_t kScanSpan = 16;  // positions a thread checks

__device__ __forceinline__ uint8_t byte_at(const uint8_t *data, uint64_t i) { return __ldg(data + i); }

// Every position i (4 <= i, i + 4 <= len) where "icpf" starts, with the
// big-endian word before it, appended in no particular order.
__global__ void __launch_bounds__(kScanThreads) k_scan_icpf(const uint8_t *data, uint64_t len, uint64_t *pos,
                                                            uint32_t *size, unsigned int *count, uint32_t cap) {
    const uint64_t t = (uint64_t)blockIdx.x * kScanThreads + threadIdx.x;
    const uint64_t lo = max((uint64_t)4, t * kScanSpan);
    const uint64_t hi = min(t * kScanSpan + kScanSpan, len >= 3 ? len - 3 : 0);  // i + 4 <= len
    for (uint64_t i = lo; i < hi; i++) {
        if (byte_at(data, i) != 'i' || byte_at(data, i + 1) != 'c' || byte_at(data, i + 2) != 'p' ||
            byte_at(data, i + 3) != 'f')
            continue;
        const uint32_t sz = ((uint32_t)byte_at(data, i - 4) << 24) | ((uint32_t)byte_at(data, i - 3) << 16) |
                            ((uint32_t)byte_at(data, i - 2) << 8) | (uint32_t)byte_at(data, i - 1);
        const unsigned int k = atomicAdd(count, 1u);
        if (k < cap) {
            pos[k] = i;
            size[k] = sz;
        }
    }
}

// The crate's acceptance rule for the "icpf" at i with frame_size `size`.
bool accepted(uint64_t i, uint64_t size, uint64_t len) { return size >= 28 && i - 4 + size <= len; }

size_t resolve(std::vector<std::pair<uint64_t, uint32_t>> &cand, uint64_t len, prores_span *out, size_t cap) {
    std::sort(cand.begin(), cand.end());
    size_t n = 0;
    uint64_t next = 4;  // the sequential walk's position
    for (const auto &c : cand) {
        if (c.first < next || !accepted(c.first, c.second, len)) continue;
        if (n < cap) out[n] = prores_span{(size_t)(c.first - 4), (size_t)c.second};
        n++;
        next = c.first - 4 + c.second;
    }
    return n;
}

int fail_status(const Status &s) {
    set_last_error(s);
    return s.code;
}

Status check_spans(const prores_span *frames, int n, size_t data_len) {
    for (int i = 0; i < n; i++)
        if (frames[i].offset > data_len || frames[i].len > data_len - frames[i].offset)
            return make_status(PRORES_CONFIG, strf("frame %d lies outside the %zu bytes given", i, data_len));
    return Status();
}

// The header regions plan_decode reads, fetched from device memory in three
// rounds (frame headers; first picture headers; second picture headers of
// interlaced frames), each one small copy per frame into pinned memory.
struct DeviceHeads {
    std::vector<std::vector<uint8_t>> head;
    std::vector<std::map<size_t, std::vector<uint8_t>>> pics;

    Status fetch(Workspace &ws, const uint8_t *d_data, const prores_span *frames, int n, cudaStream_t s) {
        head.assign(n, {});
        pics.assign(n, {});
        std::vector<size_t> want(n);
        for (int i = 0; i < n; i++) want[i] = std::min(frames[i].len, kFrameHeadBytes);
        Status st = round(ws, d_data, frames, n, s, [&](int i, size_t &pos, size_t &len) {
            pos = 0;
            len = want[i];
            return true;
        }, [&](int i, const uint8_t *p, size_t len) { head[i].assign(p, p + len); });
        if (st) return st;
        // Where each picture header is, as plan_decode walks to it.
        std::vector<FrameHeader> hdr(n);
        std::vector<int> ok(n, 0);
        for (int i = 0; i < n; i++)
            ok[i] = !parse_frame_header(head[i].data(), frames[i].len, &hdr[i]) && !check_plausible_size(hdr[i]);
        std::vector<size_t> pos(n, 0);
        for (int i = 0; i < n; i++) pos[i] = ok[i] ? 8 + (size_t)hdr[i].header_size : 0;
        for (uint32_t index = 0; index < 2; index++) {
            st = round(ws, d_data, frames, n, s, [&](int i, size_t &p, size_t &len) {
                if (!ok[i] || index >= hdr[i].picture_count() || pos[i] > hdr[i].frame_size) return false;
                p = pos[i];
                len = std::min((size_t)hdr[i].frame_size - pos[i], kPictureHeaderSize);
                return true;
            }, [&](int i, const uint8_t *p, size_t len) { pics[i][pos[i]].assign(p, p + len); });
            if (st) return st;
            for (int i = 0; i < n; i++) {
                auto it = pics[i].find(pos[i]);
                if (!ok[i] || it == pics[i].end()) {
                    ok[i] = 0;
                    continue;
                }
                PictureHeader ph;
                if (parse_picture_header(it->second.data(), hdr[i].frame_size - pos[i], &ph)) {
                    ok[i] = 0;
                    continue;
                }
                pos[i] += ph.picture_size;
            }
        }
        return Status();
    }

    const uint8_t *bytes(int i, size_t pos, size_t len) const {
        static const uint8_t none = 0;
        if (len == 0) return &none;
        if (pos == 0) return len <= head[i].size() ? head[i].data() : nullptr;
        auto it = pics[i].find(pos);
        return it != pics[i].end() && len <= it->second.size() ? it->second.data() : nullptr;
    }

  private:
    template <class Which, class Keep>
    Status round(Workspace &ws, const uint8_t *d_data, const prores_span *frames, int n, cudaStream_t s, Which which,
                 Keep keep) {
        std::vector<size_t> at(n, SIZE_MAX), len(n, 0);
        size_t total = 0;
        for (int i = 0; i < n; i++) {
            size_t p, l;
            if (!which(i, p, l)) continue;
            at[i] = total;
            len[i] = l;
            total += (l + 15) & ~(size_t)15;
            (void)p;
        }
        if (!total) return Status();
        PR_CUDA(ws.host_small.reserve(total), "cudaMallocHost");
        uint8_t *host = static_cast<uint8_t *>(ws.host_small.p);
        for (int i = 0; i < n; i++) {
            size_t p, l;
            if (at[i] == SIZE_MAX || !which(i, p, l) || !l) continue;
            PR_CUDA(cudaMemcpyAsync(host + at[i], d_data + frames[i].offset + p, l, cudaMemcpyDeviceToHost, s),
                    "header fetch");
        }
        {
            Status w = wait_stream(s, ws.wait_ms, "header fetch");
            if (w) return w;
        }
        for (int i = 0; i < n; i++)
            if (at[i] != SIZE_MAX) keep(i, host + at[i], len[i]);
        return Status();
    }
};

}  // namespace
}  // namespace prores

using namespace prores;

extern "C" {

size_t prores_scan_frames(const uint8_t *data, size_t len, prores_span *frames, size_t cap) {
    size_t n = 0;
    size_t i = 4;
    while (data && i + 4 <= len) {
        if (memcmp(data + i, "icpf", 4) == 0) {
            const uint64_t size = ((uint64_t)data[i - 4] << 24) | ((uint64_t)data[i - 3] << 16) |
                                  ((uint64_t)data[i - 2] << 8) | (uint64_t)data[i - 1];
            if (accepted(i, size, len)) {
                if (n < cap) frames[n] = prores_span{i - 4, (size_t)size};
                n++;
                i += size - 4;
                continue;
            }
        }
        i++;
    }
    return n;
}

int prores_scan_frames_device(prores_ctx *ctx, const uint8_t *d_data, size_t len, prores_span *frames, size_t cap,
                              size_t *count, void *stream) {
    if (!ctx || (!d_data && len) || !count) return fail_status(make_status(PRORES_CONFIG, "no context or data"));
    cudaSetDevice(ctx->impl.device);
    auto ws = ctx->impl.acquire();
    if (!ws) return fail_status(make_status(PRORES_DEVICE, "no stream"));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    Status st;
    uint32_t room = 1u << 16;
    std::vector<std::pair<uint64_t, uint32_t>> cand;
    for (int attempt = 0; attempt < 2 && !st; attempt++) {
        // Candidate positions, their words, and the counter.
        st = cuda_status(ws->slices.reserve((size_t)room * 12 + 64), "cudaMalloc");
        if (st) break;
        uint64_t *pos = ws->slices.as<uint64_t>();
        uint32_t *size = reinterpret_cast<uint32_t *>(pos + room);
        unsigned int *counter = reinterpret_cast<unsigned int *>(size + room);
        st = cuda_status(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s), "memset");
        const uint64_t threads = len / kScanSpan + 1;
        const uint64_t blocks = (threads + kScanThreads - 1) / kScanThreads;
        if (!st && len >= 8) {
            k_scan_icpf<<<(unsigned int)blocks, kScanThreads, 0, s>>>(d_data, len, pos, size, counter, room);
            st = cuda_status(cudaGetLastError(), "k_scan_icpf");
        }
        if (!st) st = cuda_status(ws->host_small.reserve((size_t)room * 12 + 64), "cudaMallocHost");
        if (st) break;
        uint8_t *host = static_cast<uint8_t *>(ws->host_small.p);
        unsigned int found = 0;
        st = cuda_status(cudaMemcpyAsync(host, counter, sizeof found, cudaMemcpyDeviceToHost, s), "scan");
        if (!st) st = wait_stream(s, ws->wait_ms, "scan");
        if (st) break;
        memcpy(&found, host, sizeof found);
        if (found > room) {  // more candidates than room: once more with room for all
            room = found;
            continue;
        }
        if (found) {
            st = cuda_status(cudaMemcpyAsync(host, pos, 8ull * found, cudaMemcpyDeviceToHost, s), "scan");
            if (!st)
                st = cuda_status(cudaMemcpyAsync(host + 8ull * found, size, 4ull * found, cudaMemcpyDeviceToHost, s),
                                 "scan");
            if (!st) st = wait_stream(s, ws->wait_ms, "scan");
            if (st) break;
            cand.resize(found);
            for (unsigned int k = 0; k < found; k++) {
                memcpy(&cand[k].first, host + 8ull * k, 8);
                memcpy(&cand[k].second, host + 8ull * found + 4ull * k, 4);
            }
        }
        *count = resolve(cand, len, frames, cap);
        break;
    }
    ctx->impl.release_or_retire(std::move(ws));
    return st ? fail_status(st) : PRORES_OK;
}

int prores_probe_device(prores_ctx *ctx, const uint8_t *d_data, size_t data_len, const prores_span *frames, int n,
                        uint32_t out_bit_depth, prores_frame *info, int *status) {
    if (!ctx || n < 0 || (n && (!frames || !info || !status)))
        return fail_status(make_status(PRORES_CONFIG, "no context or frames"));
    Status st = check_spans(frames, n, data_len);
    if (st) return fail_status(st);
    cudaSetDevice(ctx->impl.device);
    auto ws = ctx->impl.acquire();
    if (!ws) return fail_status(make_status(PRORES_DEVICE, "no stream"));
    DeviceHeads heads;
    st = heads.fetch(*ws, d_data, frames, n, ws->stream);
    ctx->impl.release_or_retire(std::move(ws));
    if (st) return fail_status(st);
    std::vector<Status> errs(n);
    for (int i = 0; i < n; i++) {
        static const uint8_t none = 0;
        const uint8_t *h = heads.head[i].empty() ? &none : heads.head[i].data();
        errs[i] = probe_frame(h, frames[i].len, out_bit_depth, &info[i]);  // reads the frame header only
        status[i] = errs[i].code;
    }
    set_batch_errors(errs);
    return PRORES_OK;
}

int prores_decode_device(prores_ctx *ctx, const uint8_t *d_data, size_t data_len, const prores_span *frames, int n,
                         uint32_t out_bit_depth, prores_frame *out, int *status, void *stream) {
    if (!ctx || n < 0 || (n && (!frames || !out || !status)))
        return fail_status(make_status(PRORES_CONFIG, "no context or frames"));
    Status st = check_spans(frames, n, data_len);
    if (st) return fail_status(st);
    cudaSetDevice(ctx->impl.device);
    auto ws = ctx->impl.acquire();
    if (!ws) return fail_status(make_status(PRORES_DEVICE, "no stream"));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    DeviceHeads heads;
    st = heads.fetch(*ws, d_data, frames, n, s);
    DecodePlan plan;
    std::vector<prores_buf> bufs(n);
    for (int i = 0; i < n; i++) bufs[i] = prores_buf{d_data + frames[i].offset, frames[i].len};
    const FrameBytes read = [&](int i, size_t pos, size_t len) { return heads.bytes(i, pos, len); };
    if (!st) st = plan_decode(bufs.data(), n, out_bit_depth, plan, &read);
    // The planes go straight into the caller's device buffers.
    for (int i = 0; i < n && !st; i++) {
        const DecodeFrame &f = plan.frames[i];
        if (f.err || f.desc < 0) continue;
        prores_frame &o = out[i];
        if (!o.data || o.data_len < f.samples || (f.alpha_samples && (!o.alpha || o.alpha_len < f.alpha_samples)))
            st = make_status(PRORES_CONFIG, "an output buffer is smaller than its frame");
        FrameDesc &fd = plan.fdesc[f.desc];
        fd.out_planes = o.data;
        fd.out_alpha = f.alpha_samples ? o.alpha : nullptr;
    }
    plan.planes_total = 0;  // nothing lands in the workspace's plane buffers
    plan.alpha_total = 0;
    if (!st) st = upload_decode(ctx->impl, *ws, plan, s);
    if (!st) st = upload_decode_bits(*ws, plan, bufs.data(), s);
    if (!st) st = enqueue_decode(ctx->impl, *ws, plan, s, nullptr);
    Status first;
    if (!st) st = fetch_decode(*ws, plan, s, out, status, &first, true);
    if (st) {
        ctx->impl.release_or_retire(std::move(ws));
        return fail_status(st);
    }
    ctx->impl.release(std::move(ws));
    if (first) set_last_error(first);
    return PRORES_OK;
}

}  // extern "C"
