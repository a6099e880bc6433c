// host_headers.cpp -- see host_headers.h.

#include "host_headers.h"

#include <cstdarg>
#include <cstdio>

namespace prores {

Status make_status(int code, std::string msg) {
    Status s;
    s.code = code;
    s.msg = std::move(msg);
    return s;
}

std::string strf(const char *f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

std::string display(const Status &s) {
    switch (s.code) {
    case PRORES_INVALID: return "invalid ProRes data: " + s.msg;
    case PRORES_UNSUPPORTED: return "unsupported ProRes feature: " + s.msg;
    case PRORES_CONFIG: return "invalid ProRes configuration: " + s.msg;
    case PRORES_DEVICE: return "CUDA device error: " + s.msg;
    case PRORES_TIMEOUT: return "device wait timed out: " + s.msg;
    }
    return s.msg;
}

static inline uint16_t be16(const uint8_t *p) { return (uint16_t)((p[0] << 8) | p[1]); }
static inline uint32_t be32(const uint8_t *p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

void FrameHeader::luma_weights(uint8_t w[64]) const {
    // §7.3: all weights 4 unless a matrix is loaded.
    for (int i = 0; i < 64; i++) w[i] = has_luma ? luma_matrix[i] : 4;
}

void FrameHeader::chroma_weights(uint8_t w[64]) const {
    if (has_chroma)
        memcpy(w, chroma_matrix, 64);
    else
        luma_weights(w);
}

uint32_t FrameHeader::picture_height(uint32_t index) const {
    // §6.2: the top field has the extra row of an odd frame.
    if (interlace == 0) return height;
    return is_top_field(index) ? (height + 1u) / 2u : height / 2u;
}

void FrameHeader::picture_rows(uint32_t index, uint32_t *first_row, uint32_t *step) const {
    // §7.5.3: top field on even frame rows, bottom on odd ones.
    if (interlace == 0) {
        *first_row = 0;
        *step = 1;
    } else {
        *first_row = is_top_field(index) ? 0u : 1u;
        *step = 2;
    }
}

Status parse_frame_header(const uint8_t *data, size_t len, FrameHeader *out) {
    if (len < 8 + kFrameHeaderFixed)
        return make_status(PRORES_INVALID, strf("%zu bytes is too short for a ProRes frame header", len));
    const uint32_t frame_size = be32(data);
    if (memcmp(data + 4, "icpf", 4) != 0) return make_status(PRORES_INVALID, "no 'icpf' frame identifier");
    if ((size_t)frame_size > len)
        return make_status(PRORES_INVALID, strf("frame_size %u exceeds the %zu bytes given", frame_size, len));
    if ((size_t)frame_size < 8 + kFrameHeaderFixed)
        return make_status(PRORES_INVALID, "frame_size leaves no room for the frame header");
    const uint8_t *h = data + 8;
    const uint16_t header_size = be16(h);
    if (header_size < kFrameHeaderFixed || (size_t)header_size > (size_t)frame_size - 8)
        return make_status(PRORES_INVALID, strf("frame_header_size %u is out of range", header_size));
    FrameHeader f;
    f.frame_size = frame_size;
    f.header_size = header_size;
    f.bitstream_version = h[3];
    // §6.4: a decoder refuses versions it does not know.
    if (f.bitstream_version > 1)
        return make_status(PRORES_UNSUPPORTED, strf("bitstream_version %u", f.bitstream_version));
    memcpy(f.encoder_identifier, h + 4, 4);
    f.width = be16(h + 8);
    f.height = be16(h + 10);
    if (f.width == 0 || f.height == 0)
        return make_status(PRORES_INVALID, strf("a %u\xc3\x97%u frame", f.width, f.height));
    const int cf = h[12] >> 6;
    if (cf != PRORES_CHROMA_422 && cf != PRORES_CHROMA_444)
        return make_status(PRORES_INVALID, strf("chroma_format %d is reserved", cf));
    f.chroma = cf;
    const int im = (h[12] >> 2) & 3;
    if (im == 3) return make_status(PRORES_INVALID, "interlace_mode 3 is reserved");
    f.interlace = im;
    f.aspect_ratio = h[13] >> 4;
    f.frame_rate_code = h[13] & 15;
    f.color_primaries = h[14];
    f.transfer_characteristic = h[15];
    f.matrix_coefficients = h[16];
    const int at = h[17] & 15;
    if (at > 2) return make_status(PRORES_INVALID, strf("alpha_channel_type %d is reserved", at));
    f.alpha = at;
    size_t pos = kFrameHeaderFixed;
    const bool load_luma = (h[19] & 2) != 0, load_chroma = (h[19] & 1) != 0;
    if (load_luma) {
        if (pos + 64 > header_size)
            return make_status(PRORES_INVALID, "a quantisation matrix runs past frame_header_size");
        memcpy(f.luma_matrix, h + pos, 64);
        f.has_luma = true;
        pos += 64;
    }
    if (load_chroma) {
        if (pos + 64 > header_size)
            return make_status(PRORES_INVALID, "a quantisation matrix runs past frame_header_size");
        memcpy(f.chroma_matrix, h + pos, 64);
        f.has_chroma = true;
    }
    *out = f;
    return Status();
}

void write_frame_header(const FrameHeader &h, std::vector<uint8_t> &out) {
    const size_t size = kFrameHeaderFixed + 64 * ((size_t)h.has_luma + (size_t)h.has_chroma);
    const uint8_t fixed[28] = {0, 0, 0, 0, 'i', 'c', 'p', 'f', (uint8_t)(size >> 8), (uint8_t)size, 0,
                               h.bitstream_version, h.encoder_identifier[0], h.encoder_identifier[1],
                               h.encoder_identifier[2], h.encoder_identifier[3], (uint8_t)(h.width >> 8),
                               (uint8_t)h.width, (uint8_t)(h.height >> 8), (uint8_t)h.height,
                               (uint8_t)((h.chroma << 6) | (h.interlace << 2)),
                               (uint8_t)((h.aspect_ratio << 4) | (h.frame_rate_code & 15)), h.color_primaries,
                               h.transfer_characteristic, h.matrix_coefficients, (uint8_t)h.alpha, 0,
                               (uint8_t)(((int)h.has_luma << 1) | (int)h.has_chroma)};
    out.insert(out.end(), fixed, fixed + 28);
    if (h.has_luma) out.insert(out.end(), h.luma_matrix, h.luma_matrix + 64);
    if (h.has_chroma) out.insert(out.end(), h.chroma_matrix, h.chroma_matrix + 64);
}

Status parse_picture_header(const uint8_t *data, size_t len, PictureHeader *out) {
    if (len < kPictureHeaderSize)
        return make_status(PRORES_INVALID, "a picture header runs past the end of the frame");
    const uint32_t header_size = data[0] >> 3;
    const uint32_t picture_size = be32(data + 1);
    if (header_size < kPictureHeaderSize || header_size > len)
        return make_status(PRORES_INVALID, strf("picture_header_size %u is out of range", header_size));
    if (picture_size < header_size || picture_size > len)
        return make_status(PRORES_INVALID, strf("picture_size %u is out of range", picture_size));
    out->header_size = header_size;
    out->picture_size = picture_size;
    out->log2_slice_mbs = (data[7] >> 4) & 3u;
    return Status();
}

uint32_t slices_per_row(uint32_t width_in_mb, uint32_t log2_slice_mbs) {
    const uint32_t s = 1u << log2_slice_mbs;
    return (width_in_mb >> log2_slice_mbs) + (uint32_t)__builtin_popcount(width_in_mb & (s - 1u));
}

std::vector<uint32_t> slice_widths(uint32_t width_in_mb, uint32_t log2_slice_mbs) {
    std::vector<uint32_t> v;
    uint32_t size = 1u << log2_slice_mbs, left = width_in_mb;
    for (; left > 0; size >>= 1)
        for (; left >= size; left -= size) v.push_back(size);
    return v;
}

Status check_plausible_size(const FrameHeader &h) {
    // Each slice needs 11 bytes at least (table entry, 6-byte header, a byte
    // per colour component); a picture has a slice per 8 macroblocks at least.
    const uint64_t width_in_mb = (h.width + 15u) / 16u;
    uint64_t need = 8 + (uint64_t)h.header_size;
    for (uint32_t i = 0; i < h.picture_count(); i++) {
        const uint64_t slices = (uint64_t)slices_per_row((uint32_t)width_in_mb, 3) * ((h.picture_height(i) + 15u) / 16u);
        need += kPictureHeaderSize + 11 * slices;
    }
    if ((uint64_t)h.frame_size < need)
        return make_status(PRORES_INVALID,
                           strf("frame_size %u is too small for a %u\xc3\x97%u frame (at least %llu bytes)",
                                h.frame_size, h.width, h.height, (unsigned long long)need));
    return Status();
}

size_t frame_layout(uint32_t width, uint32_t height, int chroma, size_t off[3], uint32_t w[3]) {
    const uint32_t cw = chroma == PRORES_CHROMA_422 ? (width + 1u) / 2u : width;
    w[0] = width;
    w[1] = w[2] = cw;
    off[0] = 0;
    off[1] = (size_t)width * height;
    off[2] = off[1] + (size_t)cw * height;
    return off[2] + (size_t)cw * height;
}

static uint64_t macroblocks(uint32_t w, uint32_t h) { return (uint64_t)((w + 15u) / 16u) * ((h + 15u) / 16u); }

static size_t default_headers(uint32_t w, uint32_t h) {
    // frame header without matrices, a picture header, and per slice a
    // table entry and a 6-byte slice header (8-macroblock slices).
    const size_t slices = (size_t)slices_per_row((w + 15u) / 16u, 3) * ((h + 15u) / 16u);
    return 8 + kFrameHeaderFixed + kPictureHeaderSize + 8 * slices;
}

size_t target_frame_bytes(int profile, uint32_t width, uint32_t height) {
    // Apple's rate for 1920x1080 at 29.97 frames/s, as bytes per macroblock
    // of coded data, times the frame's macroblocks, plus its headers.
    static const double kRate[6] = {45e6, 102e6, 147e6, 220e6, 330e6, 500e6};
    const double per_frame = kRate[profile] * 1001.0 / 30000.0 / 8.0;
    const double per_mb = (per_frame - (double)default_headers(1920, 1080)) / (double)macroblocks(1920, 1080);
    return (size_t)(per_mb * (double)macroblocks(width, height)) + default_headers(width, height);
}

uint64_t rescale_multiplier(uint32_t bits_in, uint32_t bits_out) {
    const uint64_t max_in = (1ull << bits_in) - 1, max_out = (1ull << bits_out) - 1;
    return ((max_out << 40) + max_in - 1) / max_in;
}

}  // namespace prores
