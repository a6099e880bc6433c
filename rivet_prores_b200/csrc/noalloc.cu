// noalloc.cu -- frame decode that allocates no device memory.
//
// Some callers cannot allocate device memory while they decode: real-time
// playback threads, where cudaMalloc can stall and cudaFree waits for the
// whole device; and host applications whose device memory belongs to their
// own pool allocator, so that any allocation outside it breaks their
// accounting or fails outright. prores_decode_noalloc serves them. The
// caller passes the frame's bytes and device buffers for the planes; all
// the decoder's scratch (its tables, the frame and slice descriptors, a
// copy of the bitstream, the statuses, and room for the rare coefficient
// too wide for the kernel's 16-bit shared-memory slots) lives in one
// static device array of PRORES_NOALLOC_SCRATCH_BYTES, which every GPU that
// loads this part of the library holds until the process exits.
//
// The kernels are the ones every other decode runs (decode.cu: the slice
// table scan, the fused per-slice decode, the status reduction); only where
// their scratch lives differs.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/prores_b200.h"
#include "codec_tables.h"
#include "device_types.h"
#include "engine.h"
#include "host_headers.h"

namespace prores {

cudaError_t configure_decode_kernels();

namespace {

static __device__ __align__(256) unsigned char g_scratch[PRORES_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr size_t kTablesBytes = 2 * 2 * kBookTableWords;  // the run and level prefix tables (a row per codebook)
static_assert(kTablesBytes % 256 == 0, "the descriptors after the tables stay 256-byte aligned");
constexpr size_t kDescBytes = 4 << 10;     // frame and picture descriptors, statuses, weights, counter

struct DeviceSetup {
    bool done = false;
    unsigned char *base = nullptr;  // device address of g_scratch on this device
};

std::mutex g_lock;
DeviceSetup g_setup[kMaxDevices];

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Once per device, with the device current: the array's device address,
// the kernels' configuration, and the constant tables copied into the
// array's first bytes.
Status setup(int device, DeviceSetup **out) {
    std::lock_guard<std::mutex> g(g_lock);
    DeviceSetup &d = g_setup[device];
    if (!d.done) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress of the no-allocation scratch");
        e = configure_decode_kernels();
        if (e != cudaSuccess) return cuda_status(e, "configure decode kernels");
        static uint16_t run[kBookTableWords], level[kBookTableWords];
        build_book_tables(run, level);
        unsigned char *base = static_cast<unsigned char *>(ptr);
        if ((e = cudaMemcpy(base, run, sizeof run, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(base + sizeof run, level, sizeof level, cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_status(e, "upload of the decode tables");
        d.base = base;
        d.done = true;
    }
    *out = &d;
    return Status();
}

const char *slot_message(int code) {
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

int finish(const Status &s) {
    if (s) set_last_error(s);
    return s.code;
}

}  // namespace

}  // namespace prores

using namespace prores;

extern "C" int prores_decode_noalloc(int device, const uint8_t *data, size_t len, uint32_t out_bit_depth,
                                     uint16_t *d_planes, size_t planes_len, uint16_t *d_alpha, size_t alpha_len,
                                     void *stream) {
    if (device < 0 || device >= kMaxDevices) return finish(make_status(PRORES_DEVICE, "no such CUDA device"));
    int previous = 0;
    cudaGetDevice(&previous);
    if (cudaSetDevice(device) != cudaSuccess) return finish(make_status(PRORES_DEVICE, "no such CUDA device"));
    struct Restore {
        int dev;
        ~Restore() { cudaSetDevice(dev); }
    } restore{previous};
    DeviceSetup *dev = nullptr;
    Status st = setup(device, &dev);
    if (st) return finish(st);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // The frame's headers, on the host (src/header.rs, src/decode.rs:61-128).
    if (out_bit_depth != 0 && (out_bit_depth < 8 || out_bit_depth > 16))
        return finish(
            make_status(PRORES_CONFIG, strf("output bit depth %u is outside 8\xe2\x80\x93" "16", out_bit_depth)));
    FrameHeader h;
    if ((st = parse_frame_header(data, len, &h))) return finish(st);
    if ((st = check_plausible_size(h))) return finish(st);
    const uint32_t depth = out_bit_depth ? out_bit_depth : (h.chroma == PRORES_CHROMA_422 ? 10u : 12u);
    FrameDesc fd{};
    size_t off[3];
    const size_t samples = frame_layout(h.width, h.height, h.chroma, off, fd.plane_w);
    const size_t alpha_samples = h.alpha ? (size_t)h.width * h.height : 0;
    if (!d_planes || planes_len < samples || (alpha_samples && (!d_alpha || alpha_len < alpha_samples)))
        return finish(make_status(PRORES_CONFIG, "an output buffer is smaller than its frame"));
    for (int c = 0; c < 3; c++) fd.plane_off[c] = off[c];
    fd.width = h.width;
    fd.height = h.height;
    fd.chroma = (uint32_t)h.chroma;
    fd.alpha_bits = h.alpha_bits();
    fd.bit_depth = depth;
    fd.weights = 0;
    if (fd.alpha_bits) {
        fd.rescale_m = rescale_multiplier(fd.alpha_bits, depth);
        fd.rescale_identity = fd.alpha_bits == depth;
    }
    fd.out_scale = (float)(1u << depth) / 512.0f;
    fd.out_bias = (float)(1u << (depth - 1)) + 0.5f;
    fd.out_max = (float)((1u << depth) - 1);
    uint8_t weights[128];
    h.luma_weights(weights);
    h.chroma_weights(weights + 64);

    // Pictures: a failure found here comes after the pictures before it.
    PicDesc pics[2]{};
    uint32_t n_pics = 0, n_slices = 0;
    uint64_t coef_total = 0;
    uint32_t most = 64u * 8u;  // the most coefficient positions of any slice
    Status late;
    const uint32_t cpm = h.chroma == PRORES_CHROMA_422 ? 2u : 4u;
    const uint32_t width_in_mb = (h.width + 15u) / 16u;
    size_t pos = 8 + (size_t)h.header_size;
    for (uint32_t index = 0; index < h.picture_count(); index++) {
        if (pos > h.frame_size) {
            late = make_status(PRORES_INVALID, "a picture starts past the end of the frame");
            break;
        }
        PictureHeader ph;
        if ((late = parse_picture_header(data + pos, h.frame_size - pos, &ph))) break;
        const uint32_t height = h.picture_height(index);
        const uint32_t height_in_mb = (height + 15u) / 16u;
        const uint32_t spr = slices_per_row(width_in_mb, ph.log2_slice_mbs);
        const uint64_t ns = (uint64_t)spr * height_in_mb;
        if ((uint64_t)ph.header_size + 2 * ns > ph.picture_size) {
            late = make_status(PRORES_INVALID, "the slice table runs past picture_size");
            break;
        }
        PicDesc &p = pics[n_pics];
        p.off = pos;
        p.coef_base = coef_total;
        p.header_size = ph.header_size;
        p.picture_size = ph.picture_size;
        p.n_slices = (uint32_t)ns;
        p.slices_per_row = spr;
        p.width_in_mb = width_in_mb;
        p.height_in_mb = height_in_mb;
        p.log2_slice_mbs = ph.log2_slice_mbs;
        p.slice_base = n_slices;
        p.frame = 0;
        p.height = height;
        h.picture_rows(index, &p.first_row, &p.row_step);
        p.interlaced_scan = h.interlace != 0;
        n_slices += (uint32_t)ns;
        coef_total += (uint64_t)width_in_mb * height_in_mb * 64u * (4u + 2u * cpm);
        most = std::max(most, 64u * (4u + 2u * cpm) * std::min(1u << ph.log2_slice_mbs, width_in_mb));
        n_pics++;
        pos += ph.picture_size;
    }

    // Where everything goes in the array, and whether it fits.
    const size_t o_desc = kTablesBytes;
    const size_t o_slices = o_desc + kDescBytes;
    const size_t o_slots = o_slices + align256(sizeof(SliceDesc) * ((size_t)n_slices + 1));
    const size_t o_bits = o_slots + align256(sizeof(int2) * 4 * ((size_t)n_slices + 1));
    const size_t o_wide = o_bits + align256((size_t)h.frame_size + 64);
    const size_t need = o_wide + 4 * (size_t)coef_total;
    if (need > PRORES_NOALLOC_SCRATCH_BYTES)
        return finish(make_status(
            PRORES_CONFIG, strf("a %u\xc3\x97%u frame needs %zu bytes of decoder scratch; prores_decode_noalloc has "
                                "%u (4 bytes a coefficient position, the frame's bytes and 64 a slice)",
                                h.width, h.height, need, (unsigned)PRORES_NOALLOC_SCRATCH_BYTES)));

    unsigned char *base = dev->base;
    FrameDesc *d_frame = reinterpret_cast<FrameDesc *>(base + o_desc);
    PicDesc *d_pics = reinterpret_cast<PicDesc *>(base + o_desc + 256);
    PicStatus *d_status = reinterpret_cast<PicStatus *>(base + o_desc + 1024);
    uint8_t *d_weights = base + o_desc + 2048;
    unsigned int *d_counter = reinterpret_cast<unsigned int *>(base + o_desc + 3072);
    uint8_t *d_bits = base + o_bits;
    // What must start at zero: the work counter and the bitstream's padding.
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_frame, &fd, sizeof fd, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (n_pics && (e = cudaMemcpyAsync(d_pics, pics, sizeof(PicDesc) * n_pics, cudaMemcpyHostToDevice, s)) !=
                       cudaSuccess) ||
        (e = cudaMemcpyAsync(d_weights, weights, sizeof weights, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_bits, data, h.frame_size, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(d_bits + h.frame_size, 0, 64, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), s)) != cudaSuccess)
        return finish(cuda_status(e, "upload"));

    DecodeLaunch d{};
    d.bits = d_bits;
    d.bits_len = h.frame_size;
    d.frames = d_frame;
    d.pics = d_pics;
    d.slices = reinterpret_cast<SliceDesc *>(base + o_slices);
    d.slot_status = reinterpret_cast<int2 *>(base + o_slots);
    d.pic_status = d_status;
    d.coef = reinterpret_cast<uint64_t *>(base + o_wide);  // values past 16 bits, at their positions
    d.coef_count = nullptr;
    d.planes = d_planes;
    d.alpha = d_alpha;
    d.weights = d_weights;
    d.work_counter = d_counter;
    d.n_frames = 1;
    d.n_pics = n_pics;
    d.n_slices = n_slices;
    d.entropy_per_lane = 1;
    d.group = std::max(1u, std::min(kDecodeMaxGroup, 16384u / most));
    d.group_positions = d.group * most;
    d.slot_bytes = 2;
    d.tables.run_books = reinterpret_cast<uint16_t *>(base);
    d.tables.level_books = reinterpret_cast<uint16_t *>(base + 2 * kBookTableWords);
    if ((e = launch_locate(d, s)) != cudaSuccess ||
        (e = launch_decode(d, decode_grid(device, d.group, d.group_positions, d.slot_bytes), s)) != cudaSuccess ||
        (e = launch_status(d, s)) != cudaSuccess)
        return finish(cuda_status(e, "decode launch"));
    PicStatus ps[2]{};
    if (n_pics && (e = cudaMemcpyAsync(ps, d_status, sizeof(PicStatus) * n_pics, cudaMemcpyDeviceToHost, s)) !=
                      cudaSuccess)
        return finish(cuda_status(e, "status download"));
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return finish(cuda_status(e, "decode"));

    // The first failure in picture order (src/decode.rs:85-104, :288-289).
    for (uint32_t p = 0; p < n_pics; p++) {
        if (ps[p].locate_slice >= 0) return finish(make_status(PRORES_INVALID, "a slice runs past picture_size"));
        if (ps[p].slot >= 0) {
            if (ps[p].code == DE_SLICE_HDR_SIZE)
                return finish(make_status(PRORES_INVALID, strf("slice_header_size %d is out of range", ps[p].aux)));
            if (ps[p].code == DE_QINDEX)
                return finish(make_status(PRORES_INVALID, strf("quantization_index %d is reserved", ps[p].aux)));
            return finish(make_status(PRORES_INVALID, slot_message(ps[p].code)));
        }
    }
    return finish(late);
}
