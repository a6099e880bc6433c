// device_types.h -- descriptors the host engine builds for the kernels, and
// the kernels' launch wrappers. One flattened list of frames, pictures and
// slices covers a whole batch of frames of any size, format and slice width.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace prores {

// Where a frame's planes live in the batch's sample buffers and how samples
// are produced (RDD 36 §7.5).
struct FrameDesc {
    uint64_t plane_off[3];  // sample offsets of Y', Cb, Cr in the plane buffer
    uint64_t alpha_off;     // sample offset of the alpha plane in the alpha buffer
    uint64_t rescale_m;     // alpha: round((2^out - 1) a / (2^in - 1)) = (a m + 2^39) >> 40
    uint32_t width, height;
    uint32_t plane_w[3];
    uint32_t chroma;      // 2 (4:2:2) or 3 (4:4:4)
    uint32_t alpha_bits;  // 0, 8 or 16
    uint32_t bit_depth;   // output (decode) or input (encode) sample depth
    uint32_t weights;     // index of this frame's (luma, chroma) weight pair
    uint32_t rescale_identity;
    float out_scale, out_bias, out_max;  // §7.5.1: floor(v scale + bias) in [0, max]
    // When set (decoding into caller device memory): the frame's packed
    // planes Y'‖Cb‖Cr (same layout as in the plane buffer) and its alpha
    // plane go here instead of the workspace's buffers.
    uint16_t *out_planes;
    uint16_t *out_alpha;
};

// One picture (a frame, or one field of an interlaced frame).
struct PicDesc {
    uint64_t off;        // byte offset of picture_header() in the bitstream buffer
    uint64_t coef_base;  // first coefficient of the picture in the scratch
    uint32_t header_size, picture_size;
    uint32_t n_slices, slices_per_row, width_in_mb, height_in_mb;
    uint32_t log2_slice_mbs;
    uint32_t slice_base;  // index of the picture's first slice in the batch
    uint32_t frame;
    uint32_t height, first_row, row_step;  // picture rows and where they land in the frame
    uint32_t interlaced_scan;
};

// One slice, located (filled on the device from the slice table).
struct SliceDesc {
    uint64_t off;   // byte offset of the slice in the bitstream buffer
    uint64_t coef;  // first entry of the slice's coefficient lists (Y', Cb, Cr regions)
    uint32_t size;  // bytes
    uint32_t pic;
    uint16_t mb_x, mb_y;
    uint32_t mbs;
};

// Device-side failures, one per (slice, component) slot; the host names
// them with the crate's messages.
enum DevErr : int32_t {
    DE_OK = 0,
    DE_PAST_END = 1,        // a codeword runs past the end of its data
    DE_PREFIX = 2,          // a variable-length code's prefix is too long
    DE_RANGE = 3,           // a variable-length code's value is out of range
    DE_DC_OVERFLOW = 4,     // a DC coefficient overflows
    DE_RUN_PAST_END = 5,    // a run passes the end of the coefficient array
    DE_ALPHA_RUN = 6,       // an alpha run passes the end of the slice
    DE_SLICE_SHORT = 7,     // a slice is shorter than its header
    DE_SLICE_HDR_SIZE = 8,  // slice_header_size {aux} is out of range
    DE_QINDEX = 9,          // quantization_index {aux} is reserved
    DE_COMP_SIZES = 10,     // slice component sizes exceed the slice
};

// First failing slot of a picture, reduced on the device.
struct PicStatus {
    int32_t locate_slice;  // first slice that runs past picture_size, or -1
    int32_t slot;          // first failing (slice * 4 + component), or -1
    int32_t code, aux;
};

// Constant tables the kernels read (built once per device).
struct DeviceTables {
    uint16_t *run_books;     // 6 x 512 packed prefix entries: a row per distinct run codebook (Table 10)
    uint16_t *level_books;   // 6 x 512: a row per distinct level codebook (Table 11)
    float *basis;            // T[x][u] at 8x + u, as the crate computes it
};

struct DecodeLaunch {
    const uint8_t *bits;  // bitstream buffer (64 bytes of zero padding after the end)
    uint64_t bits_len;
    const FrameDesc *frames;
    const PicDesc *pics;
    SliceDesc *slices;
    int2 *slot_status;  // 4 per slice
    PicStatus *pic_status;
    // 8 bytes per coefficient position of every slice component. The
    // two-kernel decode keeps each component's coefficient list there: 32-bit
    // entries (scanned position << 21 | 21-bit value; larger values at the
    // region's back, see CoefList in decode.cu) in position order, with
    // coef_count[3 s + c] entries. The fused decode keeps only values that do
    // not fit 16 bits there, as int32 at their position (see SlotOut).
    uint64_t *coef;
    uint32_t *coef_count;
    uint16_t *planes;
    uint16_t *alpha;
    const uint8_t *weights;  // [set][2][64] raster weights
    unsigned int *work_counter;
    uint32_t n_frames, n_pics, n_slices;
    uint32_t entropy_per_lane;  // slice components a lane decodes per grab of the work counter
    // Fused decode: slices a CTA takes at once, and the coefficient
    // positions its shared memory holds for them (group x the most any
    // slice of the batch has).
    uint32_t group, group_positions;
    uint32_t slot_bytes;  // 1 or 2: bytes a coefficient takes in shared memory (int8_t or int16_t)
    DeviceTables tables;
};

// Launch shapes of the entropy decoder: none changes any output.
struct EntropyShape {
    int warps_per_block;  // 1-16
    int grid;             // resident blocks in all
};

// Kernel launch wrappers (decode.cu). Each returns the launch's error.
cudaError_t launch_locate(const DecodeLaunch &d, cudaStream_t s);
cudaError_t launch_entropy(const DecodeLaunch &d, const EntropyShape &shape, cudaStream_t s);
cudaError_t launch_idct(const DecodeLaunch &d, cudaStream_t s);
cudaError_t launch_status(const DecodeLaunch &d, cudaStream_t s);
// The fused decode (k_decode): `grid` CTAs (0: as many as fit on the device).
cudaError_t launch_decode(const DecodeLaunch &d, int grid, cudaStream_t s);
// Dynamic shared memory k_decode takes for a group of `group` slices holding
// `group_positions` coefficient positions in all, `slot_bytes` each.
size_t decode_smem_bytes(uint32_t group, uint32_t group_positions, uint32_t slot_bytes);
// The most CTAs of k_decode resident on `device` at that shared memory.
int decode_grid(int device, uint32_t group, uint32_t group_positions, uint32_t slot_bytes);
constexpr uint32_t kDecodeMaxGroup = 32;
// The grid that keeps blocks_per_sm blocks of warps_per_block warps
// resident on every SM (0: as many as fit).
int entropy_grid(int device, int warps_per_block, int blocks_per_sm);

}  // namespace prores
