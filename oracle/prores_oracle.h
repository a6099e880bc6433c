/*
 * prores_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of the rivet-prores crate's RDD 36 slice pipeline
 * (decode, and encode with rate control), used as the checker for the
 * CUDA implementation. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; the product library never links or calls it.
 *
 * The crate is Rust and cannot be compiled here (no cargo/rustc), so parity
 * between this restatement and the crate is pinned by the crate's own
 * known-answer tests and published figures (codewords, hand-built frames,
 * target sizes, round-trip byte counts); see tests/test_oracle_pins.py.
 */
#ifndef PRORES_ORACLE_H
#define PRORES_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error kinds, as the crate's Error enum (src/error.rs:6-21). */
enum { ORA_OK = 0, ORA_INVALID = 1, ORA_UNSUPPORTED = 2, ORA_CONFIG = 3 };

/* A picture: planar u16 Y'‖Cb‖Cr, tightly packed, plus optional alpha
 * (src/frame.rs:180-203). chroma is the header code: 2 = 4:2:2, 3 = 4:4:4. */
typedef struct {
    uint32_t width, height, bit_depth;
    int32_t chroma;
    int32_t interlace; /* 0 progressive, 1 top field first, 2 bottom first */
    uint8_t aspect_ratio, frame_rate_code, color_primaries,
        transfer_characteristic, matrix_coefficients, pad_[3];
    uint16_t *data;
    size_t data_len; /* samples */
    uint16_t *alpha; /* NULL: no alpha */
    size_t alpha_len;
} ora_frame;

/* Encoder configuration (src/encode.rs:135-174). */
typedef struct {
    int32_t profile; /* 0 Proxy, 1 LT, 2 422, 3 HQ, 4 4444, 5 4444 XQ */
    uint32_t log2_slice_mbs;
    int32_t alpha; /* 0 none, 1 8-bit, 2 16-bit */
    int32_t has_luma_matrix, has_chroma_matrix;
    uint8_t luma_matrix[64], chroma_matrix[64];
    int64_t target_frame_bytes; /* < 0: the profile's default */
    uint8_t encoder_identifier[4];
    uint32_t threads; /* 0: one per CPU */
} ora_config;

/* ---- whole-frame codec ---- */

/* Decodes one frame. On success *out holds malloc'd planes (free with
 * ora_frame_free). Returns an ORA_* kind; msg gets the error text. */
int ora_decode(const uint8_t *data, size_t len, uint32_t out_bit_depth /*0 natural*/,
               uint32_t threads, ora_frame *out, char *msg, size_t msg_cap);
void ora_frame_free(ora_frame *f);

/* Encodes one frame into a malloc'd packet (free with ora_free). */
int ora_encode(const ora_config *cfg, const ora_frame *in, uint8_t **out, size_t *out_len,
               char *msg, size_t msg_cap);
void ora_free(void *p);

/* Rate control detail: the per-slice quantisation indices the encoder chose
 * for picture `picture` of the last ora_encode on this thread. */
size_t ora_last_qindices(int picture, uint8_t *out, size_t cap);

size_t ora_target_frame_bytes(int profile, uint32_t width, uint32_t height);

/* ---- building blocks exposed for known-answer tests ---- */

size_t ora_slice_sizes(uint32_t width_in_mb, uint32_t log2_slice_mbs, uint32_t *out, size_t cap);
/* Codebook ids: 0..3 DC (Table 9), 4..19 run (Table 10), 20..28 level
 * (Table 11), 29 first DC (EG5). Writes the codeword as '0'/'1' chars. */
int ora_codeword(int book, uint32_t n, char *bits, size_t cap);
uint32_t ora_codeword_len(int book, uint32_t n);
/* Reads one symbol from `bits` bytes with the crate's BitReader semantics;
 * returns kind, *value and *consumed bits. */
int ora_codebook_read(int book, const uint8_t *data, size_t len, uint32_t *value, uint32_t *consumed);
int ora_alpha_run_code(uint32_t run, char *bits, size_t cap);
int ora_alpha_diff_code(int32_t diff, uint32_t bits, char *out, size_t cap);
uint16_t ora_rescale(uint32_t bits_in, uint32_t bits_out, uint16_t a);
uint32_t ora_qscale(uint32_t qindex);
void ora_scans(uint8_t progressive[64], uint8_t interlaced[64]);
void ora_basis(float basis[64]);

/* Block kernels (src/dsp/scalar.rs). */
void ora_idct_put(const int32_t coef[64], const float scale[64], uint32_t bit_depth, uint16_t out[64]);
void ora_fdct_load(const uint16_t pix[64], float scale, float out[64]);
/* Whether the dsp kernels (IDCT, FDCT, quantise) run their AVX2 forms (the
 * default) or the scalar ones; both give the same results. */
void ora_set_simd(int on);
void ora_quantise(const float *f, size_t n, const float inv[64], float ac_rounding, int32_t *out,
                  uint64_t *mask);

/* Entropy coding of one component (scanned order, n_blocks blocks). */
size_t ora_encode_coefficients(const int32_t *scanned, size_t n_blocks, uint8_t *out, size_t cap,
                               size_t *bits);
int ora_decode_coefficients(const uint8_t *data, size_t len, size_t n_blocks, int32_t *scanned,
                            char *msg, size_t msg_cap);
size_t ora_encode_alpha(const uint16_t *values, size_t n, uint32_t bits, uint8_t *out, size_t cap);
int ora_decode_alpha(const uint8_t *data, size_t len, uint32_t bits, size_t count, size_t needed,
                     uint16_t *out, size_t *got);

/* ---- test pictures ---- */

/* tests/common/mod.rs:26-80 (gradients, rectangles, stripes, grain). */
void ora_test_frame(uint32_t width, uint32_t height, int32_t chroma, uint32_t bit_depth,
                    int32_t grain, uint32_t seed, uint16_t *data);

#ifdef __cplusplus
}
#endif
#endif
