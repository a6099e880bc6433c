// encode_engine.cpp -- the encode side of the batch engine.
//
// The host checks the configuration and the frames (src/encode.rs:176-192,
// :223-244; src/frame.rs:299-340), writes each frame header
// (src/header.rs:174-199), works out the target and each picture's share
// (src/encode.rs:265-272) and lists every slice of the batch; the device does
// the rest: transform, rate control, layout and packing. Frames land in
// regions of one output buffer sized for their target plus the worst alpha;
// a frame that outgrows its region (possible only when even quantiser 224
// misses the target) is laid out again in a larger one.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "codec_tables.h"
#include "encode_types.h"
#include "engine.h"

namespace prores {

#define PR_CUDA(expr, what)                     \
    do {                                        \
        Status st_ = cuda_status((expr), what); \
        if (st_) return st_;                    \
    } while (0)

struct EncodeFrame {
    Status err;
    FrameHeader hdr;
    std::vector<uint8_t> header;
    size_t target = 0;
    size_t samples = 0, alpha_samples = 0;
    int desc = -1;
};

struct EncodePlan {
    std::vector<EncodeFrame> frames;
    std::vector<EncFrameDesc> fdesc;
    std::vector<EncPicDesc> pdesc;
    std::vector<EncSliceDesc> sdesc;
    std::vector<float> quant;
    std::vector<uint8_t> quant_keys;  // 129 bytes per set: weights and scan
    std::vector<uint8_t> headers;
    size_t in_total = 0, alpha_total = 0, coef_total = 0, out_total = 0;
    uint32_t n_slices = 0;
    bool any_alpha = false;
    std::vector<uint64_t> frame_size;
    std::vector<uint32_t> frame_status;
    cudaGraphExec_t graph = nullptr;
    ~EncodePlan() {
        if (graph) cudaGraphExecDestroy(graph);
    }
};

void EncodePlanDeleter::operator()(EncodePlan *p) const { delete p; }

static const char *kProfileName[6] = {"Proxy", "Lt", "Standard", "Hq", "P4444", "P4444Xq"};
static const char *chroma_name(int c) { return c == PRORES_CHROMA_422 ? "Yuv422" : "Yuv444"; }

// src/encode.rs:176-192 and :223-244, src/frame.rs:299-340.
static Status validate(const prores_config &cfg, const prores_frame &f, int *alpha) {
    if (cfg.profile < 0 || cfg.profile > 5) return make_status(PRORES_CONFIG, strf("profile %d is not 0-5", cfg.profile));
    if (cfg.log2_slice_mbs > 3)
        return make_status(PRORES_CONFIG, strf("log2_slice_mbs %u is outside 0\xe2\x80\x93" "3", cfg.log2_slice_mbs));
    for (int m = 0; m < 2; m++) {
        if (!(m == 0 ? cfg.has_luma_matrix : cfg.has_chroma_matrix)) continue;
        const uint8_t *w = m == 0 ? cfg.luma_matrix : cfg.chroma_matrix;
        for (int i = 0; i < 64; i++)
            if (w[i] < 2 || w[i] > 63) return make_status(PRORES_CONFIG, "quantisation weights must be 2\xe2\x80\x93" "63");
    }
    if (f.chroma != PRORES_CHROMA_422 && f.chroma != PRORES_CHROMA_444)
        return make_status(PRORES_CONFIG, strf("chroma code %d is not 4:2:2 (2) or 4:4:4 (3)", f.chroma));
    if (f.interlace < 0 || f.interlace > 2)
        return make_status(PRORES_CONFIG, strf("interlace code %d is not 0-2", f.interlace));
    if (f.width == 0 || f.height == 0 || f.width > 65535 || f.height > 65535)
        return make_status(PRORES_CONFIG, strf("a frame of %u\xc3\x97%u cannot be coded", f.width, f.height));
    if (f.bit_depth < 8 || f.bit_depth > 16)
        return make_status(PRORES_CONFIG, strf("bit depth %u is outside 8\xe2\x80\x93" "16", f.bit_depth));
    size_t off[3];
    uint32_t w[3];
    frame_layout(f.width, f.height, f.chroma, off, w);
    for (int i = 0; i < 3; i++)
        if (!f.data || off[i] + (size_t)w[i] * f.height > f.data_len)
            return make_status(PRORES_CONFIG, strf("plane %d runs past the end of the frame's data", i));
    if (f.alpha && f.alpha_len != (size_t)f.width * f.height)
        return make_status(PRORES_CONFIG, strf("the alpha plane has %zu samples, not %u\xc3\x97%u", f.alpha_len, f.width,
                                               f.height));
    const int pchroma = cfg.profile >= 4 ? PRORES_CHROMA_444 : PRORES_CHROMA_422;
    if (f.chroma != pchroma)
        return make_status(PRORES_CONFIG, strf("%s codes %s, and the frame is %s", kProfileName[cfg.profile],
                                               chroma_name(pchroma), chroma_name(f.chroma)));
    *alpha = PRORES_ALPHA_NONE;
    if (f.alpha) {
        if (pchroma == PRORES_CHROMA_422)
            return make_status(PRORES_CONFIG, strf("%s carries no alpha channel", kProfileName[cfg.profile]));
        if (cfg.alpha < 0 || cfg.alpha > 2) return make_status(PRORES_CONFIG, strf("alpha type %d is not 0-2", cfg.alpha));
        *alpha = cfg.alpha;
    }
    return Status();
}

// A lower bound on the |F| that quantise to a non-zero AC level at inverse
// weight inv. A level is non-zero when fl(fl(|F| inv) + 0.42f) >= 1, which
// needs the exact sum fl(|F| inv) + 0.42f to reach 1 - 2^-25 (the midpoint
// below 1), and so |F| inv >= (1 - 2^-25 - 0.42f)(1 - 2^-24). The bound takes
// a margin of 2^-22 and is rounded down, so every non-zero lies at or above
// it; the kernels re-quantise each candidate exactly.
static float nonzero_bound(float inv) {
    const double y0 = 1.0 - std::ldexp(1.0, -25) - (double)0.42f;
    const double t = y0 * (1.0 - std::ldexp(1.0, -22)) / (double)inv;
    float b = (float)t;
    if ((double)b > t) b = std::nextafter(b, 0.0f);
    return b;
}

// Per quantization_index, kQuantStride floats (the layout is given beside
// kQuantStride): inv[scan[k]] = 8 / (W[k] qScale) in single precision for
// luma and chroma (src/encode.rs:303-329), the non-zero bound of each, and
// the least bound over each chunk of 32 scanned coefficients.
static uint32_t add_quant(EncodePlan &plan, const FrameHeader &h) {
    uint8_t key[129];
    h.luma_weights(key);
    h.chroma_weights(key + 64);
    key[128] = h.interlace != 0;
    for (size_t i = 0; i + 129 <= plan.quant_keys.size(); i += 129)
        if (memcmp(&plan.quant_keys[i], key, 129) == 0) return (uint32_t)(i / 129);
    plan.quant_keys.insert(plan.quant_keys.end(), key, key + 129);
    const uint8_t *scan = h.interlace ? kInterlacedScan : kProgressiveScan;
    const size_t base = plan.quant.size();
    plan.quant.resize(base + 225 * kQuantStride);
    for (uint32_t qi = 0; qi <= 224; qi++) {
        const uint32_t q = qscale(qi < 1 ? 1 : qi);
        float *t = &plan.quant[base + qi * kQuantStride];
        for (int k = 0; k < 64; k++) {
            t[scan[k]] = 8.0f / (float)((uint32_t)key[k] * q);
            t[64 + scan[k]] = 8.0f / (float)((uint32_t)key[64 + k] * q);
        }
        for (int k = 0; k < 128; k++) t[128 + k] = nonzero_bound(t[k]);
        for (uint32_t g = 0; g < 2; g++) {
            const float *bound = t + 128 + 64 * g;
            for (uint32_t n = 2; n <= 16; n *= 2) {
                float *chunk = t + 256 + 60 * g + (2 * n - 4);
                for (uint32_t j = 0; j < 2 * n; j++) {
                    float m = bound[32 * j / n];
                    for (uint32_t k = 32 * j / n; k < 32 * (j + 1) / n; k++) m = std::min(m, bound[k]);
                    chunk[j] = m;
                }
            }
        }
    }
    return (uint32_t)(plan.quant_keys.size() / 129 - 1);
}

Status plan_encode(const prores_config *cfg, const prores_frame *in, int n, EncodePlanPtr &out) {
    EncodePlanPtr plan(new EncodePlan());
    plan->frames.resize(n);
    for (int i = 0; i < n; i++) {
        EncodeFrame &ef = plan->frames[i];
        const prores_config &c = cfg[i];
        const prores_frame &f = in[i];
        int alpha = 0;
        if ((ef.err = validate(c, f, &alpha))) continue;
        FrameHeader &h = ef.hdr;
        h.bitstream_version = (f.chroma == PRORES_CHROMA_422 && alpha == PRORES_ALPHA_NONE) ? 0 : 1;
        memcpy(h.encoder_identifier, c.encoder_identifier, 4);
        h.width = (uint16_t)f.width;
        h.height = (uint16_t)f.height;
        h.chroma = f.chroma;
        h.interlace = f.interlace;
        h.aspect_ratio = f.aspect_ratio;
        h.frame_rate_code = f.frame_rate_code;
        h.color_primaries = f.color_primaries;
        h.transfer_characteristic = f.transfer_characteristic;
        h.matrix_coefficients = f.matrix_coefficients;
        h.alpha = alpha;
        h.has_luma = c.has_luma_matrix != 0;
        h.has_chroma = c.has_chroma_matrix != 0;
        memcpy(h.luma_matrix, c.luma_matrix, 64);
        memcpy(h.chroma_matrix, c.chroma_matrix, 64);
        write_frame_header(h, ef.header);
        ef.target = c.target_frame_bytes >= 0 ? (size_t)c.target_frame_bytes
                                              : target_frame_bytes(c.profile, f.width, f.height);
        const size_t pictures = h.picture_count();
        const size_t hl = ef.header.size();
        const size_t per_picture = (ef.target > hl ? ef.target - hl : 0) / pictures;

        EncFrameDesc fd{};
        size_t off[3];
        ef.samples = frame_layout(f.width, f.height, f.chroma, off, fd.plane_w);
        for (int p = 0; p < 3; p++) fd.in_off[p] = plan->in_total + off[p];
        plan->in_total += ef.samples;
        if (alpha) {
            ef.alpha_samples = (size_t)f.width * f.height;
            fd.alpha_in_off = plan->alpha_total;
            plan->alpha_total += ef.alpha_samples;
            plan->any_alpha = true;
        }
        fd.width = f.width;
        fd.height = f.height;
        fd.chroma = (uint32_t)f.chroma;
        fd.bit_depth = f.bit_depth;
        fd.alpha_bits = h.alpha_bits();
        if (fd.alpha_bits) {
            fd.rescale_m = rescale_multiplier(f.bit_depth, fd.alpha_bits);
            fd.rescale_identity = f.bit_depth == fd.alpha_bits;
        }
        fd.in_scale = 512.0f / (float)(1u << f.bit_depth);
        fd.header_len = (uint32_t)hl;
        fd.header_slot = (uint32_t)(plan->headers.size() / kHeaderSlot);
        plan->headers.resize(plan->headers.size() + kHeaderSlot, 0);
        memcpy(&plan->headers[(size_t)fd.header_slot * kHeaderSlot], ef.header.data(), hl);
        fd.first_pic = (uint32_t)plan->pdesc.size();
        fd.n_pics = (uint32_t)pictures;

        const uint32_t cpm = f.chroma == PRORES_CHROMA_422 ? 2u : 4u;
        const uint32_t width_in_mb = (f.width + 15u) / 16u;
        const std::vector<uint32_t> widths = slice_widths(width_in_mb, c.log2_slice_mbs);
        const uint32_t quant = add_quant(*plan, h);
        size_t slices_in_frame = 0, mbs_in_frame = 0;
        for (uint32_t index = 0; index < pictures; index++) {
            EncPicDesc p{};
            p.height = h.picture_height(index);
            h.picture_rows(index, &p.first_row, &p.row_step);
            p.width_in_mb = width_in_mb;
            p.height_in_mb = (p.height + 15u) / 16u;
            p.slices_per_row = (uint32_t)widths.size();
            p.n_slices = p.slices_per_row * p.height_in_mb;
            p.log2_slice_mbs = c.log2_slice_mbs;
            p.slice_base = plan->n_slices;
            p.coef_base = plan->coef_total;
            p.budget_in = per_picture;
            p.frame = (uint32_t)plan->fdesc.size();
            p.quant = quant;
            p.header_bytes = alpha ? 8u : 6u;
            p.interlaced_scan = h.interlace != 0;
            const uint32_t pic_index = (uint32_t)plan->pdesc.size();
            for (uint32_t my = 0; my < p.height_in_mb; my++) {
                uint32_t mx = 0;
                for (uint32_t w : widths) {
                    EncSliceDesc s{};
                    s.coef = plan->coef_total + ((uint64_t)my * width_in_mb + mx) * 64u * (4u + 2u * cpm);
                    s.pic = pic_index;
                    s.mb_x = (uint16_t)mx;
                    s.mb_y = (uint16_t)my;
                    s.mbs = w;
                    plan->sdesc.push_back(s);
                    mx += w;
                }
            }
            plan->coef_total += (uint64_t)width_in_mb * p.height_in_mb * 64u * (4u + 2u * cpm);
            plan->n_slices += p.n_slices;
            slices_in_frame += p.n_slices;
            mbs_in_frame += (size_t)width_in_mb * p.height_in_mb;
            plan->pdesc.push_back(p);
        }
        // Region: the target (which the frame meets whenever quantiser 224
        // fits), the worst lossless alpha (18 bits a value), headers.
        const size_t worst_alpha = alpha ? mbs_in_frame * 576 + slices_in_frame : 0;
        size_t cap = std::max(ef.target, hl + pictures * 8 + 2 * slices_in_frame) + worst_alpha + 1024;
        cap = (cap + 255) & ~(size_t)255;
        fd.out_base = plan->out_total;
        fd.out_cap = cap;
        plan->out_total += cap;
        ef.desc = (int)plan->fdesc.size();
        plan->fdesc.push_back(fd);
    }
    plan->frame_size.assign(plan->fdesc.size(), 0);
    plan->frame_status.assign(plan->fdesc.size(), 0);
    out = std::move(plan);
    return Status();
}

static EncodeLaunch encode_params(Context &ctx, Workspace &ws, const EncodePlan &plan) {
    EncodeLaunch e{};
    char *base = ws.enc_cost.as<char>();
    const size_t ns = plan.n_slices + 1;
    e.in = ws.enc_in.as<uint16_t>();
    e.alpha_in = ws.enc_alpha_in.as<uint16_t>();
    e.frames = ws.frames.as<EncFrameDesc>();
    e.pics = ws.pics.as<EncPicDesc>();
    e.slices = ws.slices.as<EncSliceDesc>();
    e.state = ws.enc_pic_state.as<EncPicState>();
    e.coef = ws.enc_coef.as<float>();
    e.coef_max = e.coef + plan.coef_total + 64;
    e.quant = ws.weights.as<float>();
    e.basis = ctx.tables.basis;
    // The per-slice tables share one allocation.
    size_t o = 0;
    e.alpha_bytes = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * ns;
    e.probe_comp = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * 3 * ns * kProbeSteps;
    e.win_comp = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * 3 * ns * kWindow;
    e.final_comp = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * 3 * ns;
    e.final_qi = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * ns;
    o = (o + 15) & ~(size_t)15;
    e.slice_off = reinterpret_cast<uint64_t *>(base + o);
    o += 8 * ns;
    e.share_prep = reinterpret_cast<SharePrep *>(base + o);
    o += sizeof(SharePrep) * ns;
    e.share_steps = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * ns;
    e.deep_count = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * ns;
    o = (o + 15) & ~(size_t)15;
    e.deep = reinterpret_cast<uint2 *>(base + o);
    o += sizeof(uint2) * kDeepLevels * ns;
    e.win_list = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * ns;
    e.win_count = reinterpret_cast<uint32_t *>(base + o);
    o += 4 * kWindow;
    e.cost_taken = reinterpret_cast<uint32_t *>(base + o);
    e.out = ws.enc_out.as<uint32_t>();
    e.headers = ws.enc_frame_out.as<uint8_t>();
    e.frame_status = ws.enc_alpha_bits.as<uint32_t>();
    e.frame_size = ws.enc_alpha_bytes.as<uint64_t>();
    e.n_frames = (uint32_t)plan.fdesc.size();
    e.n_pics = (uint32_t)plan.pdesc.size();
    e.n_slices = plan.n_slices;
    e.any_alpha = plan.any_alpha;
    e.sm_count = ctx.sm_count;
    e.lane_items_per_sm = ctx.current_tuning().cost_lane_items_per_sm;
    return e;
}

static size_t cost_bytes(const EncodePlan &plan) {
    const size_t ns = plan.n_slices + 1;
    return 4 * ns * (1 + 3 * kProbeSteps + 3 * kWindow + 3 + 1) + 8 * ns + sizeof(SharePrep) * ns + 4 * ns + 4 * ns +
           4 * ns + sizeof(uint2) * kDeepLevels * ns + 4 * kWindow + 4 * kProbeSteps + 256;
}

static Status upload_frames(Workspace &ws, const EncodePlan &plan, const prores_frame *in, cudaStream_t s,
                            bool device_frames) {
    // One copy per host-adjacent run of planes.
    struct Run {
        const uint8_t *src;
        size_t dst, len;
    };
    std::vector<Run> planes, alpha;
    const auto add = [](std::vector<Run> &v, const void *src, size_t dst, size_t len) {
        const uint8_t *p = static_cast<const uint8_t *>(src);
        if (!v.empty() && v.back().src + v.back().len == p && v.back().dst + v.back().len == dst)
            v.back().len += len;
        else
            v.push_back({p, dst, len});
    };
    for (size_t i = 0; i < plan.frames.size(); i++) {
        const EncodeFrame &ef = plan.frames[i];
        if (ef.err) continue;
        const EncFrameDesc &fd = plan.fdesc[ef.desc];
        add(planes, in[i].data, 2 * fd.in_off[0], 2 * ef.samples);
        if (ef.alpha_samples) add(alpha, in[i].alpha, 2 * fd.alpha_in_off, 2 * ef.alpha_samples);
    }
    // Frames in device memory are copied device to device.
    const auto copy = [&](uint8_t *dst, const uint8_t *src, size_t len) {
        return device_frames ? cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToDevice, s)
                             : ws.stager.h2d(dst, src, len, s);
    };
    for (const Run &r : planes)
        PR_CUDA(copy(ws.enc_in.as<uint8_t>() + r.dst, r.src, r.len), "frame upload");
    for (const Run &r : alpha)
        PR_CUDA(copy(ws.enc_alpha_in.as<uint8_t>() + r.dst, r.src, r.len),
                "alpha upload");
    return Status();
}

Status upload_encode(Context &ctx, Workspace &ws, EncodePlan &plan, const prores_frame *in, cudaStream_t s,
                     bool descriptors, bool device_frames) {
    (void)ctx;
    if (descriptors) {
        PR_CUDA(ws.enc_in.reserve(2 * (plan.in_total + 8)), "cudaMalloc frames");
        PR_CUDA(ws.enc_alpha_in.reserve(2 * (plan.alpha_total + 8)), "cudaMalloc alpha");
        PR_CUDA(ws.frames.reserve(sizeof(EncFrameDesc) * (plan.fdesc.size() + 1)), "cudaMalloc");
        PR_CUDA(ws.pics.reserve(sizeof(EncPicDesc) * (plan.pdesc.size() + 1)), "cudaMalloc");
        PR_CUDA(ws.slices.reserve(sizeof(EncSliceDesc) * (plan.n_slices + 1)), "cudaMalloc");
        PR_CUDA(ws.enc_pic_state.reserve(sizeof(EncPicState) * (plan.pdesc.size() + 1)), "cudaMalloc");
        // The coefficients, then (64 floats on) one chunk maximum per 32.
        PR_CUDA(ws.enc_coef.reserve(4 * (plan.coef_total + plan.coef_total / 32 + 128)), "cudaMalloc coefficients");
        PR_CUDA(ws.weights.reserve(4 * (plan.quant.size() + 64)), "cudaMalloc");
        PR_CUDA(ws.enc_cost.reserve(cost_bytes(plan)), "cudaMalloc");
        PR_CUDA(ws.enc_out.reserve(plan.out_total + 64), "cudaMalloc output");
        PR_CUDA(ws.enc_frame_out.reserve(plan.headers.size() + 64), "cudaMalloc");
        PR_CUDA(ws.enc_alpha_bits.reserve(4 * (plan.fdesc.size() + 1)), "cudaMalloc");
        PR_CUDA(ws.enc_alpha_bytes.reserve(8 * (plan.fdesc.size() + 1)), "cudaMalloc");
        if (!plan.fdesc.empty())
            PR_CUDA(ws.stager.h2d(ws.frames.p, plan.fdesc.data(), sizeof(EncFrameDesc) * plan.fdesc.size(), s),
                    "upload");
        if (!plan.pdesc.empty())
            PR_CUDA(ws.stager.h2d(ws.pics.p, plan.pdesc.data(), sizeof(EncPicDesc) * plan.pdesc.size(), s),
                    "upload");
        if (!plan.sdesc.empty())
            PR_CUDA(ws.stager.h2d(ws.slices.p, plan.sdesc.data(), sizeof(EncSliceDesc) * plan.sdesc.size(), s),
                    "upload");
        if (!plan.quant.empty())
            PR_CUDA(ws.stager.h2d(ws.weights.p, plan.quant.data(), 4 * plan.quant.size(), s),
                    "upload");
        if (!plan.headers.empty())
            PR_CUDA(ws.stager.h2d(ws.enc_frame_out.p, plan.headers.data(), plan.headers.size(), s),
                    "upload");
    }
    return upload_frames(ws, plan, in, s, device_frames);
}

static Status enqueue_tail(Context &ctx, Workspace &ws, EncodePlan &plan, cudaStream_t s, KernelTimes *kt) {
    const EncodeLaunch e = encode_params(ctx, ws, plan);
    Status st;
    PR_CUDA(cudaMemsetAsync(ws.enc_out.p, 0, plan.out_total + 64, s), "memset output");
    PR_CUDA(launch_layout(e, s), "k_layout");
    if ((st = record_kernel(kt, "k_layout", s))) return st;
    PR_CUDA(launch_pack(e, s), "k_pack");
    if ((st = record_kernel(kt, "k_pack", s))) return st;
    return Status();
}

Status enqueue_encode(Context &ctx, Workspace &ws, EncodePlan &plan, cudaStream_t s, KernelTimes *kt) {
    const EncodeLaunch e = encode_params(ctx, ws, plan);
    Status st;
    if ((st = record_kernel(kt, "start", s))) return st;
    PR_CUDA(launch_fdct(e, s), "k_fdct");
    if ((st = record_kernel(kt, "k_fdct", s))) return st;
    PR_CUDA(launch_alpha_size(e, s), "k_alpha_size");
    if ((st = record_kernel(kt, "k_alpha_size", s))) return st;
    PR_CUDA(launch_rc_init(e, s), "k_rc_init");
    for (int step = 0; step < kProbeSteps; step++) {
        PR_CUDA(launch_cost(e, step, s), "k_cost");
        if ((st = record_kernel(kt, "k_cost", s))) return st;
        PR_CUDA(launch_rc_step(e, step, s), "k_rc_step");
        if ((st = record_kernel(kt, "k_rc_step", s))) return st;
    }
    for (int level = 0; level < kWindow; level++) {
        PR_CUDA(launch_cost_window(e, level, s), "k_cost_window");
        if ((st = record_kernel(kt, "k_cost_window", s))) return st;
    }
    PR_CUDA(launch_cost_deep(e, s), "k_cost_deep");
    if ((st = record_kernel(kt, "k_cost_deep", s))) return st;
    PR_CUDA(launch_shareout(e, s), "k_shareout");
    if ((st = record_kernel(kt, "k_shareout", s))) return st;
    return enqueue_tail(ctx, ws, plan, s, kt);
}

Status fetch_encode(Context &ctx, Workspace &ws, EncodePlan &plan, cudaStream_t s, std::vector<prores_buf> &out,
                    int *status, Status *first_err) {
    const size_t nf = plan.fdesc.size();
    for (int attempt = 0; attempt < 2; attempt++) {
        // Through pinned memory: a copy into pageable memory would hold up
        // other host threads' CUDA calls until the encode is done.
        PR_CUDA(ws.host_small.reserve(12 * (nf + 1)), "cudaMallocHost");
        uint64_t *sizes = static_cast<uint64_t *>(ws.host_small.p);
        uint32_t *flags = reinterpret_cast<uint32_t *>(sizes + nf);
        if (nf) {
            PR_CUDA(cudaMemcpyAsync(sizes, ws.enc_alpha_bytes.p, 8 * nf, cudaMemcpyDeviceToHost, s), "size download");
            PR_CUDA(cudaMemcpyAsync(flags, ws.enc_alpha_bits.p, 4 * nf, cudaMemcpyDeviceToHost, s), "size download");
        }
        {
            Status w = wait_stream(s, ws.wait_ms, "encode");
            if (w) return w;
        }
        std::copy(sizes, sizes + nf, plan.frame_size.begin());
        std::copy(flags, flags + nf, plan.frame_status.begin());
        bool over = false;
        for (size_t f = 0; f < nf; f++) over = over || plan.frame_status[f];
        if (!over) break;
        if (attempt == 1) return make_status(PRORES_DEVICE, "a frame outgrew its output region twice");
        // Lay the frames out again with regions that hold what they came to.
        size_t total = 0;
        for (size_t f = 0; f < nf; f++) {
            EncFrameDesc &fd = plan.fdesc[f];
            if (plan.frame_status[f]) fd.out_cap = (plan.frame_size[f] + 1024 + 255) & ~(size_t)255;
            fd.out_base = total;
            total += fd.out_cap;
        }
        plan.out_total = total;
        PR_CUDA(ws.enc_out.reserve(plan.out_total + 64), "cudaMalloc output");
        PR_CUDA(ws.stager.h2d(ws.frames.p, plan.fdesc.data(), sizeof(EncFrameDesc) * nf, s),
                "upload");
        if (plan.graph) {
            cudaGraphExecDestroy(plan.graph);
            plan.graph = nullptr;
        }
        Status st = enqueue_tail(ctx, ws, plan, s, nullptr);
        if (st) return st;
    }
    size_t total = 0;
    for (size_t f = 0; f < nf; f++) total += plan.frame_size[f];
    PR_CUDA(ws.host_stage.reserve(total + 64), "cudaMallocHost");
    size_t pos = 0;
    for (size_t f = 0; f < nf; f++) {
        PR_CUDA(cudaMemcpyAsync(static_cast<uint8_t *>(ws.host_stage.p) + pos,
                                ws.enc_out.as<uint8_t>() + plan.fdesc[f].out_base, plan.frame_size[f],
                                cudaMemcpyDeviceToHost, s),
                "packet download");
        pos += plan.frame_size[f];
    }
    {
        Status w = wait_stream(s, ws.wait_ms, "encode");
        if (w) return w;
    }
    out.assign(plan.frames.size(), prores_buf{nullptr, 0});
    pos = 0;
    std::vector<Status> errs(plan.frames.size());
    for (size_t i = 0; i < plan.frames.size(); i++) {
        const EncodeFrame &ef = plan.frames[i];
        status[i] = ef.err.code;
        errs[i] = ef.err;
        if (ef.err) {
            if (first_err && !*first_err) *first_err = ef.err;
            continue;
        }
        const size_t n = plan.frame_size[ef.desc];
        out[i].data = static_cast<uint8_t *>(ws.host_stage.p) + pos;
        out[i].len = n;
        pos += n;
    }
    set_batch_errors(errs);
    return Status();
}

}  // namespace prores

// ====================================================================== C ABI

using namespace prores;


static int efail(const Status &s) {
    set_last_error(s);
    return s.code;
}

static bool profiling_on() {
    const char *v = getenv("PRORES_PROFILE_KERNELS");
    return v && v[0] && v[0] != '0';
}

extern "C" {

static int encode_batch(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n, prores_buf *out,
                        int *status, bool device_frames, void *stream) {
    if (!ctx || n < 0) return efail(make_status(PRORES_CONFIG, "no context"));
    cudaSetDevice(ctx->impl.device);
    EncodePlanPtr plan;
    Status st = plan_encode(cfg, in, n, plan);
    if (st) return efail(st);
    auto ws = ctx->impl.acquire();
    if (!ws) return efail(make_status(PRORES_DEVICE, "no stream"));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    st = upload_encode(ctx->impl, *ws, *plan, in, s, true, device_frames);
    if (!st) st = enqueue_encode(ctx->impl, *ws, *plan, s, nullptr);
    std::vector<prores_buf> packets;
    Status first;
    if (!st) st = fetch_encode(ctx->impl, *ws, *plan, s, packets, status, &first);
    if (st) {
        ctx->impl.release_or_retire(std::move(ws));
        return efail(st);
    }
    // The packets lie in the workspace's staging buffer: copied out before
    // the workspace goes back to the pool.
    for (int i = 0; i < n; i++) {
        out[i].data = nullptr;
        out[i].len = 0;
    }
    for (int i = 0; i < n; i++) {
        if (status[i] != PRORES_OK) continue;
        uint8_t *p = static_cast<uint8_t *>(malloc(packets[i].len ? packets[i].len : 1));
        if (!p) {
            for (int j = 0; j < i; j++) free(const_cast<uint8_t *>(out[j].data));
            for (int j = 0; j < i; j++) out[j] = prores_buf{nullptr, 0};
            ctx->impl.release(std::move(ws));
            return efail(make_status(PRORES_DEVICE, "host allocation failed"));
        }
        memcpy(p, packets[i].data, packets[i].len);
        out[i].data = p;
        out[i].len = packets[i].len;
    }
    ctx->impl.release(std::move(ws));
    if (first) set_last_error(first);
    return PRORES_OK;
}

int prores_encode_batch(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n, prores_buf *out,
                        int *status) {
    return encode_batch(ctx, cfg, in, n, out, status, false, nullptr);
}

int prores_encode_device(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n, prores_buf *out,
                         int *status, void *stream) {
    return encode_batch(ctx, cfg, in, n, out, status, true, stream);
}

int prores_encode(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, uint8_t **out, size_t *out_len) {
    prores_buf b{nullptr, 0};
    int status = PRORES_OK;
    int r = prores_encode_batch(ctx, cfg, in, 1, &b, &status);
    if (r != PRORES_OK) return r;
    *out = const_cast<uint8_t *>(b.data);
    *out_len = b.len;
    return status;
}

int prores_encode_job_create(prores_ctx *ctx, const prores_config *cfg, const prores_frame *in, int n,
                             prores_encode_job **job) {
    if (!ctx || n < 0) return efail(make_status(PRORES_CONFIG, "no context"));
    cudaSetDevice(ctx->impl.device);
    auto *j = new prores_encode_job();
    j->ctx = ctx;
    j->kt.enabled = profiling_on();
    Status st = plan_encode(cfg, in, n, j->plan);
    if (!st) {
        j->ws = ctx->impl.acquire();
        if (!j->ws) st = make_status(PRORES_DEVICE, "no stream");
    }
    if (!st) st = upload_encode(ctx->impl, *j->ws, *j->plan, in, j->ws->stream, true, false);
    if (!st) st = wait_stream(j->ws->stream, j->ws->wait_ms, "upload");
    if (st) {
        prores_encode_job_destroy(j);
        return efail(st);
    }
    *job = j;
    return PRORES_OK;
}

int prores_encode_job_upload(prores_encode_job *job, const prores_frame *in, int n, void *stream) {
    if ((size_t)n != job->plan->frames.size()) return efail(make_status(PRORES_CONFIG, "a job's batch size is fixed"));
    for (int i = 0; i < n; i++) {
        const EncodeFrame &ef = job->plan->frames[i];
        if (ef.err) continue;
        if (in[i].width != ef.hdr.width || in[i].height != ef.hdr.height || in[i].chroma != ef.hdr.chroma ||
            (in[i].alpha != nullptr) != (ef.alpha_samples != 0) || in[i].data_len < ef.samples)
            return efail(make_status(PRORES_CONFIG, "a job's frame formats are fixed"));
    }
    cudaSetDevice(job->ctx->impl.device);
    job->ctx->impl.refresh(*job->ws);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : job->ws->stream;
    Status st = upload_encode(job->ctx->impl, *job->ws, *job->plan, in, s, false, false);
    return st ? efail(st) : PRORES_OK;
}

int prores_encode_job_launch(prores_encode_job *job, void *stream, int use_graph) {
    Context &c = job->ctx->impl;
    cudaSetDevice(c.device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : job->ws->stream;
    if (use_graph) {
        if (!job->plan->graph) {
            cudaGraph_t g;
            cudaStream_t cap = job->ws->stream;
            Status st = cuda_status(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "capture");
            if (!st) {
                st = enqueue_encode(c, *job->ws, *job->plan, cap, nullptr);
                cudaError_t e = cudaStreamEndCapture(cap, &g);
                if (!st) st = cuda_status(e, "capture");
            }
            if (!st) {
                st = cuda_status(cudaGraphInstantiate(&job->plan->graph, g, 0), "graph instantiate");
                cudaGraphDestroy(g);
            }
            if (st) return efail(st);
        }
        Status st = cuda_status(cudaGraphLaunch(job->plan->graph, s), "graph launch");
        return st ? efail(st) : PRORES_OK;
    }
    for (auto e : job->kt.events) cudaEventDestroy(e);
    job->kt.events.clear();
    job->kt.names.clear();
    Status st = enqueue_encode(c, *job->ws, *job->plan, s, &job->kt);
    return st ? efail(st) : PRORES_OK;
}

int prores_encode_job_fetch(prores_encode_job *job, void *stream, prores_buf *out, int *status) {
    cudaSetDevice(job->ctx->impl.device);
    job->ctx->impl.refresh(*job->ws);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : job->ws->stream;
    Status first;
    Status st = fetch_encode(job->ctx->impl, *job->ws, *job->plan, s, job->packets, status, &first);
    if (st) return efail(st);
    for (size_t i = 0; i < job->packets.size(); i++) out[i] = job->packets[i];
    if (first) set_last_error(first);
    return PRORES_OK;
}

void prores_encode_job_destroy(prores_encode_job *job) {
    if (!job) return;
    cudaSetDevice(job->ctx->impl.device);
    for (auto e : job->kt.events) cudaEventDestroy(e);
    if (job->ws) {
        // Its work may still run (a fetch that timed out): the workspace and
        // graph are then kept until it is done.
        cudaGraphExec_t graph = job->plan ? job->plan->graph : nullptr;
        if (job->plan) job->plan->graph = nullptr;
        job->plan.reset();
        job->ctx->impl.release_or_retire(std::move(job->ws), graph);
    }
    delete job;
}

}  // extern "C"
