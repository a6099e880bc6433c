// encode_types.h -- descriptors and launch parameters of the encode kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace prores {

// Bisection steps after the probe at 224: the interval [1, 224] halves
// (rounding up) to one value in 8 steps (src/encode.rs:700-713).
constexpr int kProbeSteps = 9;
// Finer quantisers costed before the share-out (the first for every slice,
// the next ones for the slices that could reach them); the share-out costs
// anything else it needs itself.
constexpr int kWindow = 4;
// Finer quantisers past the window costed ahead of the share-out for a
// slice that could reach them (the same prefetch rule, level after level):
// at most this many per slice; the share-out costs any further one itself.
constexpr int kDeepLevels = 128;
// Bytes per frame-header template: 8 + a frame_header() of at most 148.
constexpr uint32_t kHeaderSlot = 160;

struct EncFrameDesc {
    uint64_t in_off[3];     // sample offsets of Y', Cb, Cr in the input plane buffer
    uint64_t alpha_in_off;  // sample offset of the alpha plane in the input alpha buffer
    uint64_t out_base;      // byte offset of the frame's region in the output buffer (4-aligned)
    uint64_t out_cap;       // bytes available there
    uint64_t rescale_m;     // input depth -> coded alpha bits (src/encode.rs:850-852)
    uint32_t width, height;
    uint32_t plane_w[3];
    uint32_t chroma;      // 2 or 3
    uint32_t bit_depth;   // input depth, 8-16
    uint32_t alpha_bits;  // coded alpha: 0, 8 or 16
    uint32_t rescale_identity;
    uint32_t header_len;  // frame_size + 'icpf' + frame_header() bytes
    uint32_t header_slot; // index of the frame's header template (kHeaderSlot bytes each)
    uint32_t first_pic, n_pics;
    float in_scale;  // 512 / 2^b (src/encode.rs:524-525)
};

struct EncPicDesc {
    uint64_t coef_base;  // first f32 coefficient of the picture
    uint64_t budget_in;  // the picture's share of the target (src/encode.rs:272)
    uint32_t slice_base, n_slices, slices_per_row, width_in_mb, height_in_mb;
    uint32_t log2_slice_mbs;
    uint32_t frame;
    uint32_t height, first_row, row_step;
    uint32_t quant;         // index of the picture's quantiser table set
    uint32_t header_bytes;  // slice header: 6, or 8 with alpha
    uint32_t interlaced_scan;
};

struct EncSliceDesc {
    uint64_t coef;  // first coefficient (scanned order, Y' then Cb then Cr)
    uint32_t pic;
    uint16_t mb_x, mb_y;
    uint32_t mbs;
};

// Rate-control state of one picture (src/encode.rs:685-794).
struct EncPicState {
    uint64_t budget;     // bytes for the slices
    uint64_t pic_size;   // picture_size once coded
    uint64_t pic_off;    // byte offset of the picture in its frame
    uint64_t hi_total;   // the slices' bytes at `hi`
    int32_t lo, hi;      // bisection interval
    int32_t probe_qi;    // quantiser of the pass in flight (0: none)
    int32_t hi_probe;    // the probe step whose sizes are at `hi`
    int32_t lo_probe;    // the failed probe step at lo - 1, or -1
    int32_t fits_at_all;
    int32_t uniform;
    uint8_t step_qi[12];  // the quantiser each probe step costed (0: none)
};

// A window entry that was not costed (the share-out costs it if needed).
constexpr uint32_t kNotCosted = 0xFFFFFFFFu;

// A slice's share-out inputs: its size at the uniform quantiser, and per
// window level (bit j of `known` when costed) the smallest D that lets it
// step there (~0 when the size does not fit) and the size over the base.
struct SharePrep {
    uint64_t thr[kWindow];
    int32_t delta[kWindow];
    uint32_t base;
    uint32_t known;
    // For the levels past the window (deep_count of them, in `deep`): the
    // slice header and alpha bytes, the macroblocks from the slice to the
    // end of the picture, and log2 of the slice's macroblocks.
    uint32_t hba, rem, shift, deep_count;
};

// Per quantiser set and quantization_index, kQuantStride floats:
//   [0, 128)    8 / (W qScale) at the scanned positions, luma then chroma;
//   [128, 256)  the least |F| that can quantise to a non-zero AC level at each;
//   [256, 376)  per component group (luma, chroma: 60 each) the least of
//               those bounds over each 32-coefficient chunk of a component
//               of n blocks, n = 2, 4, 8, 16 (2n chunks each, at 2n - 4).
// For n = 32 a chunk is one scanned position, whose bound is in [128, 256).
constexpr uint32_t kQuantStride = 384;

struct EncodeLaunch {
    const uint16_t *in;        // input planes
    const uint16_t *alpha_in;  // input alpha planes
    const EncFrameDesc *frames;
    const EncPicDesc *pics;
    const EncSliceDesc *slices;
    EncPicState *state;
    float *coef;           // transformed slices, scanned order
    float *coef_max;       // [coef / 32] the largest |F| of each 32 scanned coefficients (a chunk)
    const float *quant;    // [set][225 qi][kQuantStride], see quant_base
    const float *basis;    // T[x][u]
    uint32_t *alpha_bytes; // per slice
    uint32_t *probe_comp;  // [kProbeSteps][slice][3] component bytes
    uint32_t *win_comp;    // [kWindow][slice][3]
    uint32_t *win_list;    // [slice] the slices costed at the current window level
    uint32_t *win_count;   // [kWindow] list lengths
    uint32_t *cost_taken;  // [kProbeSteps] items the warps of each probe's k_cost have taken
    uint32_t *final_comp;  // [slice][3]
    uint32_t *final_qi;    // [slice]
    uint64_t *slice_off;   // [slice] byte offset of the slice in its frame
    SharePrep *share_prep; // [slice]
    uint32_t *share_steps; // [slice] finer steps taken (top bit: sizes already in final_comp)
    uint2 *deep;           // [slice][kDeepLevels] component bytes past the window: x = Y' | Cb << 16,
                           //   y = Cr | fits << 16 (sizes saturate at 65535, which never fits)
    uint32_t *deep_count;  // [slice] levels in deep
    uint32_t *out;         // output buffer (zeroed before packing), big-endian bit order
    const uint8_t *headers;  // frame header templates
    uint32_t *frame_status;  // per frame: 0, or 1 when the frame outgrew its region
    uint64_t *frame_size;    // per frame
    uint32_t n_frames, n_pics, n_slices;
    int any_alpha;
    int sm_count;
    int lane_items_per_sm;  // a lane per slice component when 3 n_slices >= this x sm_count
};

cudaError_t launch_fdct(const EncodeLaunch &e, cudaStream_t s);
cudaError_t launch_alpha_size(const EncodeLaunch &e, cudaStream_t s);
cudaError_t launch_rc_init(const EncodeLaunch &e, cudaStream_t s);
cudaError_t launch_cost(const EncodeLaunch &e, int step, cudaStream_t s);
cudaError_t launch_rc_step(const EncodeLaunch &e, int step, cudaStream_t s);
cudaError_t launch_cost_window(const EncodeLaunch &e, int level, cudaStream_t s);
cudaError_t launch_cost_deep(const EncodeLaunch &e, cudaStream_t s);
cudaError_t launch_shareout(const EncodeLaunch &e, cudaStream_t s);
cudaError_t launch_layout(const EncodeLaunch &e, cudaStream_t s);
cudaError_t launch_pack(const EncodeLaunch &e, cudaStream_t s);

}  // namespace prores
