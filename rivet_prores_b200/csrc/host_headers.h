// host_headers.h -- the container-facing headers, parsed on the host: the
// frame header (RDD 36 §5.1.1, the crate's src/header.rs:82-170), the
// picture header (§5.2.1, :269-290), the slice layout (:308-320), field
// geometry (:212-255), the decoder's size guard (src/decode.rs:113-128) and
// the encoder's target size (src/encode.rs:112-131). Messages are the
// crate's, so callers see the same errors.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/prores_b200.h"

namespace prores {

struct Status {
    int code = PRORES_OK;
    std::string msg;
    explicit operator bool() const { return code != PRORES_OK; }
};
Status make_status(int code, std::string msg);
std::string strf(const char *f, ...);
// The crate's Display strings (src/error.rs:9-20).
std::string display(const Status &s);

struct FrameHeader {
    uint32_t frame_size = 0;
    uint16_t header_size = 0;
    uint8_t bitstream_version = 0;
    uint8_t encoder_identifier[4] = {0, 0, 0, 0};
    uint16_t width = 0, height = 0;
    int chroma = PRORES_CHROMA_422;
    int interlace = 0;
    uint8_t aspect_ratio = 0, frame_rate_code = 0, color_primaries = 2, transfer_characteristic = 2,
            matrix_coefficients = 2;
    int alpha = PRORES_ALPHA_NONE;
    bool has_luma = false, has_chroma = false;
    uint8_t luma_matrix[64] = {}, chroma_matrix[64] = {};

    uint32_t alpha_bits() const { return alpha == PRORES_ALPHA_8 ? 8u : alpha == PRORES_ALPHA_16 ? 16u : 0u; }
    void luma_weights(uint8_t w[64]) const;
    void chroma_weights(uint8_t w[64]) const;
    uint32_t picture_count() const { return interlace == 0 ? 1u : 2u; }
    bool is_top_field(uint32_t index) const { return (interlace == 1) == (index == 0); }
    uint32_t picture_height(uint32_t index) const;
    void picture_rows(uint32_t index, uint32_t *first_row, uint32_t *step) const;
};

constexpr size_t kFrameHeaderFixed = 20;
constexpr size_t kPictureHeaderSize = 8;

Status parse_frame_header(const uint8_t *data, size_t len, FrameHeader *out);
void write_frame_header(const FrameHeader &h, std::vector<uint8_t> &out);

struct PictureHeader {
    uint32_t header_size = 0, picture_size = 0, log2_slice_mbs = 0;
};
Status parse_picture_header(const uint8_t *data, size_t len, PictureHeader *out);

// Slices per row of macroblocks and the slice widths (full slices from the
// left, then halving).
uint32_t slices_per_row(uint32_t width_in_mb, uint32_t log2_slice_mbs);
std::vector<uint32_t> slice_widths(uint32_t width_in_mb, uint32_t log2_slice_mbs);

Status check_plausible_size(const FrameHeader &h);

// Plane offsets/widths of a packed Y'‖Cb‖Cr frame; returns total samples.
size_t frame_layout(uint32_t width, uint32_t height, int chroma, size_t off[3], uint32_t w[3]);

size_t target_frame_bytes(int profile, uint32_t width, uint32_t height);

// round((2^out - 1) a / (2^in - 1)) as (a m + 2^39) >> 40 (src/decode.rs:446-469).
uint64_t rescale_multiplier(uint32_t bits_in, uint32_t bits_out);

}  // namespace prores
