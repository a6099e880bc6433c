// codec_tables.h -- RDD 36 constants shared by host and device code: the
// variable-length codebooks (Tables 9-11, §7.1.1.1), the scans (Figures 4
// and 5) and Table 15's qScale, with the codeword arithmetic the entropy
// kernels use. The tables must be RDD 36's, so they match the crate's
// src/vlc.rs:28-68 and src/tables.rs:6-38 entry for entry.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define PR_HD __host__ __device__ __forceinline__
#else
#define PR_HD inline
#endif

namespace prores {

// A codebook as RICE_EXP_COMBO_CODE(lastRiceQ q, kRice r, kExp e); an
// exp-Golomb code of order k is the combination (0, k, k + 1) (the note at
// the end of RDD 36 §7.1.1.1), and `eg` records which form the table names.
struct Codebook {
    uint8_t eg, q, r, e;
};

#define PR_EG(k) Codebook{1, 0, (uint8_t)(k), (uint8_t)((k) + 1)}
#define PR_CB(q, r, e) Codebook{0, (uint8_t)(q), (uint8_t)(r), (uint8_t)(e)}

static constexpr Codebook kFirstDcBook = PR_EG(5);

// Longest accepted zero prefix and largest accepted symbol: a bound that
// keeps every read inside a 64-bit window (the crate's src/vlc.rs:19-26).
static constexpr uint32_t kMaxPrefix = 32;
static constexpr uint32_t kMaxSymbol = 1u << 30;

// Figure 4 and Figure 5: scan[8 v + u] is the scanned index of the
// coefficient at row v, column u.
static constexpr uint8_t kProgressiveScan[64] = {
    0,  1,  4,  5,  16, 17, 21, 22, 2,  3,  6,  7,  18, 20, 23, 28, 8,  9,  12, 13, 19, 24,
    27, 29, 10, 11, 14, 15, 25, 26, 30, 31, 32, 33, 37, 38, 45, 46, 53, 54, 34, 36, 39, 44,
    47, 52, 55, 60, 35, 40, 43, 48, 51, 56, 59, 61, 41, 42, 49, 50, 57, 58, 62, 63};
static constexpr uint8_t kInterlacedScan[64] = {
    0,  2,  8,  10, 32, 34, 35, 41, 1,  3,  9,  11, 33, 36, 40, 42, 4,  6,  12, 14, 37, 39,
    43, 49, 5,  7,  13, 15, 38, 44, 48, 50, 16, 18, 19, 25, 45, 47, 51, 57, 17, 20, 24, 26,
    46, 52, 56, 58, 21, 23, 27, 30, 53, 55, 59, 62, 22, 28, 29, 31, 54, 60, 61, 63};

// Table 15.
PR_HD uint32_t qscale(uint32_t q) { return q <= 128 ? q : 128 + 4 * (q - 128); }

PR_HD uint32_t clz64(uint64_t v) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)__clzll((long long)v);
#else
    return v ? (uint32_t)__builtin_clzll(v) : 64u;
#endif
}
PR_HD uint32_t bit_len64(uint64_t v) { return 64u - clz64(v); }

// Length of an exp-Golomb codeword of order k for n: (q zeros) then n + 2^k
// in q + k + 1 bits, q = floor(log2(n + 2^k)) - k.
PR_HD uint32_t eg_len(uint64_t n, uint32_t k) { return 2u * bit_len64(n + (1ull << k)) - k - 1u; }

// Length in bits of the codeword for symbol n.
PR_HD uint32_t cb_len(Codebook cb, uint32_t n32) {
    uint64_t n = n32;
    if (cb.eg) return eg_len(n, cb.r);
    uint64_t threshold = (uint64_t)(cb.q + 1) << cb.r;
    if (n < threshold) return (uint32_t)(n >> cb.r) + 1u + cb.r;
    return cb.q + 1u + eg_len(n - threshold, cb.e);
}

// The codeword for symbol n as its significant bits (the leading zeros are
// implied by the length): Rice part `1` + r bits, or the exp-Golomb value
// n - threshold + 2^e after q + 1 zeros.
PR_HD uint64_t cb_bits(Codebook cb, uint32_t n32) {
    uint64_t n = n32;
    uint64_t threshold = (uint64_t)(cb.q + 1) << cb.r;
    if (n < threshold) return (1ull << cb.r) | (n & ((1ull << cb.r) - 1));
    return n - threshold + (1ull << cb.e);
}

// §7.1.1.2: 0, -1, 1, -2, 2, ... -> 0, 1, 2, 3, 4, ...
PR_HD uint32_t signed_to_symbol(int32_t n) {
    return n >= 0 ? 2u * (uint32_t)n : 2u * (0u - (uint32_t)n) - 1u;
}
PR_HD int32_t symbol_to_signed(uint32_t s) {
    return (s & 1u) == 0 ? (int32_t)(s >> 1) : -(int32_t)((s + 1u) >> 1);
}

// Table 9: the DC difference's codebook by |previousDCDiff| (3 and above
// share the last entry).
PR_HD Codebook dc_book(int32_t prev_diff) {
    const uint32_t a = prev_diff < 0 ? 0u - (uint32_t)prev_diff : (uint32_t)prev_diff;
    if (a == 0) return PR_EG(0);
    if (a == 1) return PR_EG(1);
    if (a == 2) return PR_CB(1, 2, 3);
    return PR_EG(3);
}
// Table 10: the run's codebook by previousRun (15 and above share the last).
PR_HD Codebook run_book(uint32_t prev_run) {
    if (prev_run <= 1) return PR_CB(2, 0, 1);
    if (prev_run <= 3) return PR_CB(1, 0, 1);
    if (prev_run == 4) return PR_EG(0);
    if (prev_run <= 8) return PR_CB(1, 1, 2);
    if (prev_run <= 14) return PR_EG(1);
    return PR_EG(2);
}
// Table 11: abs_level_minus_1's codebook by previousLevelSymbol (8 and above
// share the last).
PR_HD Codebook level_book(uint32_t prev) {
    if (prev == 0) return PR_CB(2, 0, 2);
    if (prev == 1) return PR_CB(1, 0, 1);
    if (prev == 2) return PR_CB(2, 0, 1);
    if (prev == 3) return PR_EG(0);
    if (prev <= 7) return PR_EG(1);
    return PR_EG(2);
}

// T[x][u] = C(u)/2 cos((2x+1) u pi / 16), computed in double and rounded
// once to single precision (the crate's src/dct.rs:11-25). Host only.
inline void dct_basis(float out[64]) {
    for (int x = 0; x < 8; x++)
        for (int u = 0; u < 8; u++) {
            const double cu = u == 0 ? 0.70710678118654752440 : 1.0;
            const double a = (double)((2 * x + 1) * u) * 3.14159265358979323846 / 16.0;
            out[8 * x + u] = (float)(cu / 2.0 * cos(a));
        }
}

// Prefix tables for the decoder, one row per distinct codebook: Table 10's
// run codebooks for previousRun 0-1, 2-3, 4, 5-8, 9-14, 15+ (rows 0-5) and
// Table 11's level codebooks for previousLevelSymbol 0, 1, 2, 3, 4-7, 8+
// (rows 0-5). For every kBookBits-bit window prefix an entry holds the
// codeword it starts with when that is kBookBits bits or fewer and its
// symbol is below 64: its length (4 bits), its symbol (6 bits) and the row
// the next code of the same kind is read with, the row of the context this
// symbol makes (3 bits); 0 otherwise (the decoder then reads the codeword
// by arithmetic). Eleven bits hold all but about 0.1 % of the run and level
// codewords of UHD 422 HQ frames (nine bits left about 1 %).
static constexpr uint32_t kBookBits = 11;
static constexpr uint32_t kBookEntries = 1u << kBookBits;
static constexpr uint32_t kBookTableWords = 6 * kBookEntries;

PR_HD uint32_t run_book_row(uint32_t prev_run) {
    return (uint32_t)(0x5444444333321100ull >> (4u * (prev_run < 15u ? prev_run : 15u))) & 15u;
}
PR_HD uint32_t level_book_row(uint32_t prev_level) {
    return (uint32_t)(0x544443210ull >> (4u * (prev_level < 8u ? prev_level : 8u))) & 15u;
}

inline void build_book_tables(uint16_t *run, uint16_t *level) {
    static const uint32_t run_ctx[6] = {0, 2, 4, 5, 9, 15};
    static const uint32_t level_ctx[6] = {0, 1, 2, 3, 4, 8};
    for (int kind = 0; kind < 2; kind++) {
        uint16_t *out = kind == 0 ? run : level;
        for (uint32_t row = 0; row < 6; row++) {
            const Codebook cb = kind == 0 ? run_book(run_ctx[row]) : level_book(level_ctx[row]);
            uint16_t *r = out + row * kBookEntries;
            for (uint32_t i = 0; i < kBookEntries; i++) r[i] = 0;
            for (uint32_t n = 0; n < 64; n++) {
                const uint32_t len = cb_len(cb, n);
                if (len > kBookBits) continue;
                const uint32_t next = kind == 0 ? run_book_row(n) : level_book_row(n);
                const uint32_t first = (uint32_t)cb_bits(cb, n) << (kBookBits - len);
                for (uint32_t p = 0; p < (1u << (kBookBits - len)); p++)
                    r[first + p] = (uint16_t)(len | (n << 4) | (next << 10));
            }
        }
    }
}

}  // namespace prores
