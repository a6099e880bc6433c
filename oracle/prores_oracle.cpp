// prores_oracle.cpp -- TEST INFRASTRUCTURE ONLY: a CPU restatement of the
// rivet-prores crate (SMPTE RDD 36 decode and encode) used as the checker
// of the CUDA implementation and as the timed CPU baseline. The product
// library never links or calls this file.
//
// Every function cites the crate file:line it restates. Build with
// -ffp-contract=off and without fast-math: the crate's single-precision
// arithmetic is a multiply then an add, never fused (src/dsp/mod.rs:11-20),
// and the decoded pictures depend on that order.

#include "prores_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <immintrin.h>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------- errors
// src/error.rs:6-42: three kinds, each with a message.
struct Error {
    int kind = ORA_OK;
    std::string msg;
    explicit operator bool() const { return kind != ORA_OK; }
};

std::string fmt(const char *f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}
Error invalid(std::string m) { return {ORA_INVALID, std::move(m)}; }
Error unsupported(std::string m) { return {ORA_UNSUPPORTED, std::move(m)}; }
Error config(std::string m) { return {ORA_CONFIG, std::move(m)}; }

// Entropy-level failures are counted in a code and named once at the top;
// the messages are the crate's (src/bits.rs:67,87,90; src/vlc.rs:227;
// src/decode.rs:496,514,531,590).
enum Fail {
    F_OK = 0,
    F_PAST_END,
    F_PREFIX,
    F_RANGE,
    F_DC_OVERFLOW,
    F_RUN_PAST_END,
    F_ALPHA_RUN,
};
const char *fail_message(int f) {
    switch (f) {
    case F_PAST_END: return "a codeword runs past the end of its data";
    case F_PREFIX: return "a variable-length code's prefix is too long";
    case F_RANGE: return "a variable-length code's value is out of range";
    case F_DC_OVERFLOW: return "a DC coefficient overflows";
    case F_RUN_PAST_END: return "a run passes the end of the coefficient array";
    case F_ALPHA_RUN: return "an alpha run passes the end of the slice";
    }
    return "";
}

inline uint32_t clz64(uint64_t v) { return v ? (uint32_t)__builtin_clzll(v) : 64u; }
inline uint32_t bit_len(uint64_t v) { return 64u - clz64(v); }
inline uint64_t be64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
    return v;
}
inline uint16_t be16(const uint8_t *p) { return (uint16_t)((p[0] << 8) | p[1]); }
inline uint32_t be32(const uint8_t *p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

// ---------------------------------------------------------------- bits
// src/bits.rs:10-102: MSB-first reader over one component's bytes.
struct BitReader {
    const uint8_t *data;
    size_t len;
    size_t pos = 0;  // bits
    BitReader(const uint8_t *d, size_t n) : data(d), len(n) {}
    size_t remaining() const { return len * 8 - pos; }
    // :30-40, zero past the end.
    uint64_t peek64() const {
        size_t byte = pos >> 3;
        uint8_t buf[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (byte + 8 <= len)
            memcpy(buf, data + byte, 8);
        else if (byte < len)
            memcpy(buf, data + byte, len - byte);
        return be64(buf) << (pos & 7);
    }
    // :46-50
    bool peek_fast(uint64_t *w) const {
        size_t byte = pos >> 3;
        if (byte + 8 > len) return false;
        *w = be64(data + byte) << (pos & 7);
        return true;
    }
    void skip(uint32_t n) { pos += n; }
    // :61-72
    int read(uint32_t n, uint64_t *v) {
        if (n == 0) {
            *v = 0;
            return F_OK;
        }
        if ((size_t)n > remaining()) return F_PAST_END;
        *v = peek64() >> (64 - n);
        pos += n;
        return F_OK;
    }
    int read_bit(uint32_t *b) {
        uint64_t v;
        int f = read(1, &v);
        *b = (uint32_t)v;
        return f;
    }
    // :84-94
    int leading_zeros(uint32_t max, uint32_t *out) {
        uint32_t lz = clz64(peek64());
        if (lz > max) return F_PREFIX;
        if ((size_t)lz >= remaining()) return F_PAST_END;
        pos += lz;
        *out = lz;
        return F_OK;
    }
    // :98-101
    bool end_of_data() const {
        size_t r = remaining();
        return r <= 31 && (r == 0 || (peek64() >> (64 - r)) == 0);
    }
};

// src/bits.rs:106-134: a sink that counts bits.
struct BitCounter {
    size_t n = 0;
    void put(uint64_t, uint32_t bits) { n += bits; }
    size_t bits() const { return n; }
    void align() {
        size_t r = n % 8;
        if (r) put(0, 8 - (uint32_t)r);
    }
};

// src/bits.rs:138-202: MSB-first writer, 64-bit accumulator.
struct BitWriter {
    std::vector<uint8_t> *out;
    size_t start;
    uint64_t acc = 0;
    uint32_t nacc = 0;
    explicit BitWriter(std::vector<uint8_t> *o) : out(o), start(o->size()) {}
    void put(uint64_t v, uint32_t n) {
        v &= (n >= 64) ? ~0ull : ((1ull << n) - 1);
        uint32_t free_bits = 64 - nacc;
        if (n < free_bits) {
            acc = (acc << n) | v;
            nacc += n;
        } else {
            uint32_t rest = n - free_bits;
            uint64_t full = (acc << free_bits) | (v >> rest);
            for (int i = 7; i >= 0; i--) out->push_back((uint8_t)(full >> (8 * i)));
            acc = v & ((1ull << rest) - 1);
            nacc = rest;
        }
    }
    size_t bits() const { return (out->size() - start) * 8 + nacc; }
    void align() {
        size_t r = bits() % 8;
        if (r) put(0, 8 - (uint32_t)r);
    }
    size_t finish() {
        align();
        if (nacc > 0) {
            uint64_t b = acc << (64 - nacc);
            for (uint32_t i = 0; i < nacc / 8; i++) out->push_back((uint8_t)(b >> (56 - 8 * i)));
            acc = 0;
            nacc = 0;
        }
        return out->size() - start;
    }
};

// ---------------------------------------------------------------- vlc
// src/vlc.rs:9-83: ExpGolomb(k) and Combo(lastRiceQ, kRice, kExp).
struct Codebook {
    bool eg;
    uint32_t q, r, e;  // for eg: q=0, r=k, e=k+1 (the combination form)
};
constexpr Codebook EG(uint32_t k) { return {true, 0, k, k + 1}; }
constexpr Codebook CB(uint32_t q, uint32_t r, uint32_t e) { return {false, q, r, e}; }

constexpr uint32_t MAX_PREFIX = 32;        // src/vlc.rs:23
constexpr uint32_t MAX_SYMBOL = 1u << 30;  // src/vlc.rs:26

const Codebook DC_CODEBOOKS[4] = {EG(0), EG(1), CB(1, 2, 3), EG(3)};  // Table 9
const Codebook RUN_CODEBOOKS[16] = {CB(2, 0, 1), CB(2, 0, 1), CB(1, 0, 1), CB(1, 0, 1),
                                    EG(0),       CB(1, 1, 2), CB(1, 1, 2), CB(1, 1, 2),
                                    CB(1, 1, 2), EG(1),       EG(1),       EG(1),
                                    EG(1),       EG(1),       EG(1),       EG(2)};  // Table 10
const Codebook LEVEL_CODEBOOKS[9] = {CB(2, 0, 2), CB(1, 0, 1), CB(2, 0, 1), EG(0), EG(1),
                                     EG(1),       EG(1),       EG(1),       EG(2)};  // Table 11
constexpr Codebook FIRST_DC_CODEBOOK = EG(5);  // src/vlc.rs:68

inline Codebook dc_codebook(int32_t prev_diff) {
    uint32_t a = prev_diff < 0 ? 0u - (uint32_t)prev_diff : (uint32_t)prev_diff;
    return DC_CODEBOOKS[std::min(a, 3u)];
}
inline Codebook run_codebook(uint32_t prev_run) { return RUN_CODEBOOKS[std::min(prev_run, 15u)]; }
inline Codebook level_codebook(uint32_t prev) { return LEVEL_CODEBOOKS[std::min(prev, 8u)]; }

// src/vlc.rs:94-104
template <class S>
void put_exp_golomb(S &s, uint64_t n, uint32_t k) {
    uint64_t v = n + (1ull << k);
    uint32_t len = bit_len(v);
    uint32_t q = len - k - 1;
    if (len + q <= 57) {
        s.put(v, len + q);
    } else {
        s.put(0, q);
        s.put(v, len);
    }
}

// src/vlc.rs:109-126
template <class S>
void cb_put(Codebook cb, S &s, uint32_t n32) {
    uint64_t n = n32;
    if (cb.eg) {
        put_exp_golomb(s, n, cb.r);
        return;
    }
    uint64_t threshold = (uint64_t)(cb.q + 1) << cb.r;
    if (n < threshold) {
        uint32_t q = (uint32_t)(n >> cb.r);
        uint64_t rem = n & ((1ull << cb.r) - 1);
        s.put((1ull << cb.r) | rem, q + 1 + cb.r);
    } else {
        s.put(0, cb.q + 1);
        put_exp_golomb(s, n - threshold, cb.e);
    }
}

// src/vlc.rs:131-151: the codeword as (bits, len) when it is 57 bits or shorter.
bool cb_code(Codebook cb, uint32_t n32, uint64_t *bits, uint32_t *len) {
    uint64_t n = n32;
    uint64_t threshold = (uint64_t)(cb.q + 1) << cb.r;
    if (n < threshold) {
        uint32_t q = (uint32_t)(n >> cb.r);
        *bits = (1ull << cb.r) | (n & ((1ull << cb.r) - 1));
        *len = q + 1 + cb.r;
        return true;
    }
    uint64_t v = n - threshold + (1ull << cb.e);
    uint32_t b = bit_len(v);
    uint32_t l = cb.q + 1 + 2 * b - cb.e - 1;
    if (l > 57) return false;
    *bits = v;
    *len = l;
    return true;
}

// src/vlc.rs:155-172
inline uint32_t eg_len(uint64_t n, uint32_t k) {
    uint32_t len = bit_len(n + (1ull << k));
    return 2 * len - k - 1;
}
inline uint32_t cb_len(Codebook cb, uint32_t n32) {
    uint64_t n = n32;
    if (cb.eg) return eg_len(n, cb.r);
    uint64_t threshold = (uint64_t)(cb.q + 1) << cb.r;
    if (n < threshold) return (uint32_t)(n >> cb.r) + 1 + cb.r;
    return cb.q + 1 + eg_len(n - threshold, cb.e);
}

// src/vlc.rs:180-204: decode from a window whose first 57 bits are real.
bool cb_peek(Codebook cb, uint64_t w, uint32_t *sym, uint32_t *len) {
    uint32_t last_q = cb.q, k_rice = cb.r, k_exp = cb.e;
    uint32_t q = clz64(w);
    if (q <= last_q) {
        uint32_t l = q + 1 + k_rice;
        uint64_t v = (w >> (64 - l)) & ((1ull << k_rice) - 1);
        *sym = (uint32_t)(((uint64_t)q << k_rice) | v);
        *len = l;
        return true;
    }
    if (q > MAX_PREFIX) return false;
    uint32_t tail = q - (last_q + 1) + k_exp + 1;
    uint32_t l = q + tail;
    if (l > 57) return false;
    uint64_t v = (w << q) >> (64 - tail);
    uint64_t n = v - (1ull << k_exp) + ((uint64_t)(last_q + 1) << k_rice);
    if (n > MAX_SYMBOL) return false;
    *sym = (uint32_t)n;
    *len = l;
    return true;
}

// src/vlc.rs:207-230
int cb_read(Codebook cb, BitReader &r, uint32_t *out) {
    uint32_t q;
    int f = r.leading_zeros(MAX_PREFIX, &q);
    if (f) return f;
    uint32_t q_exp, k_exp;
    uint64_t offset;
    if (cb.eg) {
        q_exp = q;
        k_exp = cb.r;
        offset = 0;
    } else {
        if (q <= cb.q) {
            uint64_t v;
            f = r.read(1 + cb.r, &v);
            if (f) return f;
            v &= (1ull << cb.r) - 1;
            *out = (uint32_t)(((uint64_t)q << cb.r) | v);
            return F_OK;
        }
        q_exp = q - (cb.q + 1);
        k_exp = cb.e;
        offset = (uint64_t)(cb.q + 1) << cb.r;
    }
    uint64_t v;
    f = r.read(q_exp + k_exp + 1, &v);
    if (f) return f;
    uint64_t n = v - (1ull << k_exp) + offset;
    if (n > MAX_SYMBOL) return F_RANGE;
    *out = (uint32_t)n;
    return F_OK;
}

// src/vlc.rs:235-251
inline uint32_t signed_to_symbol(int32_t n) {
    return n >= 0 ? 2u * (uint32_t)n : 2u * (0u - (uint32_t)n) - 1u;
}
inline int32_t symbol_to_signed(uint32_t s) {
    return (s & 1) == 0 ? (int32_t)(s >> 1) : -(int32_t)((s + 1) / 2);
}

// src/vlc.rs:254-299: alpha runs (Table 12) and differences (13, 14).
template <class S>
void put_alpha_run(S &s, uint32_t run) {
    if (run == 1)
        s.put(1, 1);
    else if (run <= 16)
        s.put(run - 1, 5);
    else
        s.put(run - 1, 16);
}
int read_alpha_run(BitReader &r, uint32_t *run) {
    uint32_t b;
    int f = r.read_bit(&b);
    if (f) return f;
    if (b == 1) {
        *run = 1;
        return F_OK;
    }
    uint64_t v;
    if ((f = r.read(4, &v))) return f;
    if (v != 0) {
        *run = (uint32_t)v + 1;
        return F_OK;
    }
    if ((f = r.read(11, &v))) return f;
    *run = (uint32_t)v + 1;
    return F_OK;
}
template <class S>
void put_alpha_difference(S &s, int32_t diff, uint32_t bits) {
    uint32_t mag_bits = bits == 8 ? 3 : 6, max = bits == 8 ? 8 : 64;
    uint32_t a = diff < 0 ? 0u - (uint32_t)diff : (uint32_t)diff;
    if (a >= 1 && a <= max) {
        uint64_t code = ((uint64_t)(a - 1) << 1) | (uint64_t)(diff < 0);
        s.put(code, 1 + mag_bits + 1);
    } else {
        uint32_t m = (uint32_t)diff & ((1u << bits) - 1);
        s.put((1ull << bits) | m, 1 + bits);
    }
}
int read_alpha_difference(BitReader &r, uint32_t bits, int32_t *diff) {
    uint32_t mag_bits = bits == 8 ? 3 : 6;
    uint32_t b;
    int f = r.read_bit(&b);
    if (f) return f;
    uint64_t v;
    if (b == 1) {
        if ((f = r.read(bits, &v))) return f;
        *diff = (int32_t)v;
        return F_OK;
    }
    if ((f = r.read(mag_bits, &v))) return f;
    int32_t a = (int32_t)v + 1;
    uint32_t neg;
    if ((f = r.read_bit(&neg))) return f;
    *diff = neg ? -a : a;
    return F_OK;
}

// src/vlc.rs:303-366: 9-bit prefix tables for run and level decoding.
constexpr uint32_t DECODE_BITS = 9;
struct DecodeTables {
    uint16_t run[16][1 << DECODE_BITS];
    uint16_t level[9][1 << DECODE_BITS];
    DecodeTables() {
        fill(RUN_CODEBOOKS, 16, &run[0][0]);
        fill(LEVEL_CODEBOOKS, 9, &level[0][0]);
    }
    static void fill(const Codebook *books, int n_books, uint16_t *t) {
        for (int c = 0; c < n_books; c++) {
            uint16_t *row = t + c * (1 << DECODE_BITS);
            for (int i = 0; i < (1 << DECODE_BITS); i++) row[i] = 0;
            for (uint32_t n = 0;; n++) {
                uint32_t len = cb_len(books[c], n);
                if (len <= DECODE_BITS) {
                    uint64_t bits = 0;
                    uint32_t l = 0;
                    cb_code(books[c], n, &bits, &l);
                    uint32_t first = (uint32_t)bits << (DECODE_BITS - len);
                    for (uint32_t p = 0; p < (1u << (DECODE_BITS - len)); p++)
                        row[first + p] = (uint16_t)((n << 5) | len);
                } else if (n > (1u << DECODE_BITS)) {
                    break;
                }
            }
        }
    }
};
const DecodeTables &tables() {
    static DecodeTables t;
    return t;
}
inline bool peek_run(uint32_t prev_run, uint64_t w, uint32_t *sym, uint32_t *len) {
    uint32_t c = std::min(prev_run, 15u);
    uint16_t e = tables().run[c][w >> (64 - DECODE_BITS)];
    if (e) {
        *sym = e >> 5;
        *len = e & 31;
        return true;
    }
    return cb_peek(RUN_CODEBOOKS[c], w, sym, len);
}
inline bool peek_level(uint32_t prev, uint64_t w, uint32_t *sym, uint32_t *len) {
    uint32_t c = std::min(prev, 8u);
    uint16_t e = tables().level[c][w >> (64 - DECODE_BITS)];
    if (e) {
        *sym = e >> 5;
        *len = e & 31;
        return true;
    }
    return cb_peek(LEVEL_CODEBOOKS[c], w, sym, len);
}

// ---------------------------------------------------------------- tables
// src/tables.rs:6-38 (RDD 36 Figures 4 and 5, Table 15).
const uint8_t PROGRESSIVE_SCAN[64] = {
    0,  1,  4,  5,  16, 17, 21, 22, 2,  3,  6,  7,  18, 20, 23, 28, 8,  9,  12, 13, 19, 24,
    27, 29, 10, 11, 14, 15, 25, 26, 30, 31, 32, 33, 37, 38, 45, 46, 53, 54, 34, 36, 39, 44,
    47, 52, 55, 60, 35, 40, 43, 48, 51, 56, 59, 61, 41, 42, 49, 50, 57, 58, 62, 63};
const uint8_t INTERLACED_SCAN[64] = {
    0,  2,  8,  10, 32, 34, 35, 41, 1,  3,  9,  11, 33, 36, 40, 42, 4,  6,  12, 14, 37, 39,
    43, 49, 5,  7,  13, 15, 38, 44, 48, 50, 16, 18, 19, 25, 45, 47, 51, 57, 17, 20, 24, 26,
    46, 52, 56, 58, 21, 23, 27, 30, 53, 55, 59, 62, 22, 28, 29, 31, 54, 60, 61, 63};
inline uint32_t qscale(uint32_t q) { return q <= 128 ? q : 128 + 4 * (q - 128); }

// ---------------------------------------------------------------- dct
// src/dct.rs:11-25: T[x][u] = C(u)/2 cos((2x+1)u pi/16), computed in f64.
struct Basis {
    float t[64];
    Basis() {
        for (int x = 0; x < 8; x++)
            for (int u = 0; u < 8; u++) {
                double c = u == 0 ? M_SQRT1_2 : 1.0;
                double a = (double)((2 * x + 1) * u) * M_PI / 16.0;
                t[8 * x + u] = (float)(c / 2.0 * cos(a));
            }
    }
};
const Basis &basis() {
    static Basis b;
    return b;
}

// src/dct.rs:36-66
void idct(const float coef[64], float out[64]) {
    const float *t = basis().t;
    float tmp[64] = {0};
    for (int v = 0; v < 8; v++) {
        const float *row = coef + 8 * v;
        bool zero = true;
        for (int u = 0; u < 8; u++) zero = zero && row[u] == 0.0f;
        if (zero) continue;
        for (int x = 0; x < 8; x++) {
            const float *b = t + 8 * x;
            float s = 0.0f;
            for (int u = 0; u < 8; u++) s += row[u] * b[u];
            tmp[8 * v + x] = s;
        }
    }
    for (int i = 0; i < 64; i++) out[i] = 0.0f;
    for (int y = 0; y < 8; y++) {
        const float *b = t + 8 * y;
        for (int v = 0; v < 8; v++) {
            float w = b[v];
            for (int x = 0; x < 8; x++) out[8 * y + x] += w * tmp[8 * v + x];
        }
    }
}

// src/dct.rs:70-93
void fdct(const float pix[64], float out[64]) {
    const float *t = basis().t;
    float tmp[64] = {0};
    for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
            float p = pix[8 * y + x];
            for (int u = 0; u < 8; u++) tmp[8 * y + u] += p * t[8 * x + u];
        }
    for (int i = 0; i < 64; i++) out[i] = 0.0f;
    for (int y = 0; y < 8; y++)
        for (int v = 0; v < 8; v++) {
            float w = t[8 * y + v];
            for (int u = 0; u < 8; u++) out[8 * v + u] += w * tmp[8 * y + u];
        }
}

// src/dsp/mod.rs:315-329
struct Output {
    float scale, bias, max;
    explicit Output(uint32_t bit_depth)
        : scale((float)(1u << bit_depth) / 512.0f),
          bias((float)(1u << (bit_depth - 1)) + 0.5f),
          max((float)((1u << bit_depth) - 1)) {}
};

// Rust's saturating float-to-int casts.
inline int32_t sat_i32(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x < -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
inline uint16_t sat_u16(float x) {
    if (x != x || x <= 0.0f) return 0;
    if (x >= 65535.0f) return 65535;
    return (uint16_t)x;
}

// src/dsp/scalar.rs:8-12
void idct_put_scalar(const int32_t coef[64], const float scale[64], Output o, uint16_t out[64]) {
    float f[64], v[64];
    for (int k = 0; k < 64; k++) f[k] = (float)coef[k] * scale[k];
    idct(f, v);
    for (int k = 0; k < 64; k++) {
        float s = floorf(v[k] * o.scale + o.bias);
        s = s < 0.0f ? 0.0f : (s > o.max ? o.max : s);
        out[k] = sat_u16(s);
    }
}

// src/dsp/scalar.rs:14-17
void fdct_load_scalar(const uint16_t pix[64], float scale, float out[64]) {
    float p[64];
    for (int k = 0; k < 64; k++) p[k] = (float)pix[k] * scale - 256.0f;
    fdct(p, out);
}

// src/dsp/scalar.rs:19-39
void quantise_scalar(const float *f, size_t n, const float inv[64], float ac_rounding, int32_t *out,
                     uint64_t *mask) {
    for (size_t i = 0; i < n; i++) mask[i] = 0;
    for (size_t s = 0; s < 64; s++) {
        float r = s == 0 ? 0.5f : ac_rounding;
        float iv = inv[s];
        for (size_t b = 0; b < n; b++) {
            size_t i = n * s + b;
            float x = f[i] * iv;
            int32_t m = sat_i32(floorf(fabsf(x) + r));
            int32_t q = x < 0.0f ? -m : m;
            out[i] = q;
            mask[i / 64] |= (uint64_t)(q != 0) << (i % 64);
        }
    }
}

// ---------------------------------------------------------------- dsp, AVX2
// The crate dispatches its dsp kernels to SIMD forms that give the scalar
// forms' results bit for bit (src/dsp/mod.rs:1-20, :102-178). These are
// this oracle's own 8-wide forms of the three scalar kernels above: every
// lane does the scalar kernel's multiplies and adds in the same order, one
// rounding each (-ffp-contract=off keeps the intrinsics unfused), so each
// output equals the scalar one. They make the timed CPU baseline closer to
// the crate's speed; `ora_set_simd(0)` runs the scalar forms instead, and
// the tests check that both give the same bytes and samples.
std::atomic<bool> g_simd{true};

// The basis transposed, tt[8 u + x] = t[8 x + u]: the row of products a
// coefficient u contributes to the eight outputs x.
struct BasisT {
    alignas(32) float tt[64];
    BasisT() {
        const float *t = basis().t;
        for (int x = 0; x < 8; x++)
            for (int u = 0; u < 8; u++) tt[8 * u + x] = t[8 * x + u];
    }
};
const BasisT &basis_t() {
    static BasisT b;
    return b;
}

// idct_put_scalar, eight outputs at a time.
void idct_put_avx2(const int32_t coef[64], const float scale[64], Output o, uint16_t out[64]) {
    const float *t = basis().t, *tt = basis_t().tt;
    alignas(32) float f[64];
    for (int v = 0; v < 8; v++)
        _mm256_store_ps(f + 8 * v, _mm256_mul_ps(_mm256_cvtepi32_ps(_mm256_loadu_si256(
                                                      reinterpret_cast<const __m256i *>(coef + 8 * v))),
                                                  _mm256_loadu_ps(scale + 8 * v)));
    // Rows: tmp[v][x] = 0 + row[0] T[x][0] + ... + row[7] T[x][7]; an
    // all-zero row (-0 counts as zero) stays zero.
    const __m256 zero = _mm256_setzero_ps();
    __m256 tmp[8];
    for (int v = 0; v < 8; v++) {
        const __m256 row = _mm256_load_ps(f + 8 * v);
        tmp[v] = zero;
        if (_mm256_movemask_ps(_mm256_cmp_ps(row, zero, _CMP_EQ_OQ)) == 0xFF) continue;
        __m256 acc = zero;
        for (int u = 0; u < 8; u++)
            acc = _mm256_add_ps(acc, _mm256_mul_ps(_mm256_broadcast_ss(f + 8 * v + u), _mm256_load_ps(tt + 8 * u)));
        tmp[v] = acc;
    }
    // Columns: out[y][x] = 0 + T[y][0] tmp[0][x] + ... + T[y][7] tmp[7][x],
    // then floor(v scale + bias) clamped to [0, max].
    const __m256 sc = _mm256_set1_ps(o.scale), bias = _mm256_set1_ps(o.bias), mx = _mm256_set1_ps(o.max);
    for (int y = 0; y < 8; y++) {
        __m256 acc = zero;
        for (int v = 0; v < 8; v++) acc = _mm256_add_ps(acc, _mm256_mul_ps(_mm256_broadcast_ss(t + 8 * y + v), tmp[v]));
        __m256 s = _mm256_round_ps(_mm256_add_ps(_mm256_mul_ps(acc, sc), bias),
                                   _MM_FROUND_TO_NEG_INF | _MM_FROUND_NO_EXC);
        // max(s, 0) first: a NaN (which finite inputs cannot give) becomes 0,
        // as in the scalar form.
        s = _mm256_min_ps(_mm256_max_ps(s, zero), mx);
        const __m256i w = _mm256_cvttps_epi32(s);
        _mm_storeu_si128(reinterpret_cast<__m128i *>(out + 8 * y),
                         _mm_packus_epi32(_mm256_castsi256_si128(w), _mm256_extracti128_si256(w, 1)));
    }
}

// fdct_load_scalar, eight outputs at a time.
void fdct_load_avx2(const uint16_t pix[64], float scale, float out[64]) {
    const float *t = basis().t;
    const __m256 zero = _mm256_setzero_ps(), sc = _mm256_set1_ps(scale), off = _mm256_set1_ps(256.0f);
    alignas(32) float p[64];
    for (int y = 0; y < 8; y++) {
        const __m256i px = _mm256_cvtepu16_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i *>(pix + 8 * y)));
        _mm256_store_ps(p + 8 * y, _mm256_sub_ps(_mm256_mul_ps(_mm256_cvtepi32_ps(px), sc), off));
    }
    // Rows: tmp[y][u] = 0 + p[y][0] T[0][u] + ... + p[y][7] T[7][u].
    __m256 tmp[8];
    for (int y = 0; y < 8; y++) {
        __m256 acc = zero;
        for (int x = 0; x < 8; x++)
            acc = _mm256_add_ps(acc, _mm256_mul_ps(_mm256_broadcast_ss(p + 8 * y + x), _mm256_loadu_ps(t + 8 * x)));
        tmp[y] = acc;
    }
    // Columns: out[v][u] = 0 + T[0][v] tmp[0][u] + ... + T[7][v] tmp[7][u].
    for (int v = 0; v < 8; v++) {
        __m256 acc = zero;
        for (int y = 0; y < 8; y++) acc = _mm256_add_ps(acc, _mm256_mul_ps(_mm256_broadcast_ss(t + 8 * y + v), tmp[y]));
        _mm256_storeu_ps(out + 8 * v, acc);
    }
}

// quantise_scalar, eight blocks of a scanned position at a time (n, the
// component's block count, a multiple of 8; smaller components take the
// scalar form).
void quantise_avx2(const float *f, size_t n, const float inv[64], float ac_rounding, int32_t *out, uint64_t *mask) {
    if (n % 8 != 0) return quantise_scalar(f, n, inv, ac_rounding, out, mask);
    for (size_t i = 0; i < n; i++) mask[i] = 0;
    const __m256 zero = _mm256_setzero_ps(), sign = _mm256_set1_ps(-0.0f), big = _mm256_set1_ps(2147483648.0f);
    const __m256i imax = _mm256_set1_epi32(INT32_MAX), izero = _mm256_setzero_si256();
    for (size_t s = 0; s < 64; s++) {
        const __m256 r = _mm256_set1_ps(s == 0 ? 0.5f : ac_rounding), iv = _mm256_set1_ps(inv[s]);
        for (size_t b = 0; b < n; b += 8) {
            const size_t i = n * s + b;
            const __m256 x = _mm256_mul_ps(_mm256_loadu_ps(f + i), iv);
            const __m256 fl = _mm256_round_ps(_mm256_add_ps(_mm256_andnot_ps(sign, x), r),
                                              _MM_FROUND_TO_NEG_INF | _MM_FROUND_NO_EXC);
            // Rust's saturating cast: NaN to 0, 2^31 and up to INT32_MAX.
            __m256i m = _mm256_cvttps_epi32(fl);
            m = _mm256_blendv_epi8(m, imax, _mm256_castps_si256(_mm256_cmp_ps(fl, big, _CMP_GE_OQ)));
            m = _mm256_blendv_epi8(m, izero, _mm256_castps_si256(_mm256_cmp_ps(fl, fl, _CMP_UNORD_Q)));
            const __m256i q = _mm256_blendv_epi8(m, _mm256_sub_epi32(izero, m),
                                                 _mm256_castps_si256(_mm256_cmp_ps(x, zero, _CMP_LT_OQ)));
            _mm256_storeu_si256(reinterpret_cast<__m256i *>(out + i), q);
            const __m256i is_zero = _mm256_cmpeq_epi32(q, izero);
            const uint32_t nz = ~(uint32_t)_mm256_movemask_ps(_mm256_castsi256_ps(is_zero)) & 0xFFu;
            mask[i / 64] |= (uint64_t)nz << (i % 64);
        }
    }
}

void idct_put(const int32_t coef[64], const float scale[64], Output o, uint16_t out[64]) {
    g_simd.load(std::memory_order_relaxed) ? idct_put_avx2(coef, scale, o, out) : idct_put_scalar(coef, scale, o, out);
}
void fdct_load(const uint16_t pix[64], float scale, float out[64]) {
    g_simd.load(std::memory_order_relaxed) ? fdct_load_avx2(pix, scale, out) : fdct_load_scalar(pix, scale, out);
}
void quantise(const float *f, size_t n, const float inv[64], float ac_rounding, int32_t *out, uint64_t *mask) {
    if (g_simd.load(std::memory_order_relaxed))
        quantise_avx2(f, n, inv, ac_rounding, out, mask);
    else
        quantise_scalar(f, n, inv, ac_rounding, out, mask);
}

// ---------------------------------------------------------------- pool
// src/pool.rs: a process-wide pool; callers take part; tasks claimed from
// an atomic counter, one at a time (Large) or in chunks of 1-8 (Small).
unsigned parallelism() {
    static unsigned n = std::max(1u, std::thread::hardware_concurrency());
    return n;
}
unsigned resolve(unsigned threads) { return threads == 0 ? parallelism() : threads; }

struct Job {
    const std::function<void(size_t)> *f;
    size_t tasks, chunk;
    std::atomic<size_t> next{0};
    size_t max_helpers;
    std::mutex m;
    std::condition_variable cv;
    size_t joined = 0, left = 0;
    void work() {
        for (;;) {
            size_t first = next.fetch_add(chunk, std::memory_order_relaxed);
            if (first >= tasks) return;
            size_t end = std::min(first + chunk, tasks);
            for (size_t i = first; i < end; i++) (*f)(i);
        }
    }
};

struct Pool {
    std::mutex m;
    std::condition_variable cv;
    std::vector<std::shared_ptr<Job>> queue;
    Pool() {
        for (unsigned i = 0; i + 1 < parallelism(); i++) std::thread([this] { worker(); }).detach();
    }
    void worker() {
        for (;;) {
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> lk(m);
                for (;;) {
                    for (auto &j : queue) {
                        std::lock_guard<std::mutex> g(j->m);
                        if (j->joined < j->max_helpers &&
                            j->next.load(std::memory_order_relaxed) < j->tasks) {
                            j->joined++;
                            job = j;
                            break;
                        }
                    }
                    if (job) break;
                    cv.wait(lk);
                }
            }
            job->work();
            std::lock_guard<std::mutex> g(job->m);
            job->left++;
            job->cv.notify_all();
        }
    }
};
Pool &pool() {
    static Pool *p = new Pool();
    return *p;
}

enum TaskSize { LARGE, SMALL };
// src/pool.rs:164-209
void pool_run(unsigned threads, size_t tasks, TaskSize size, const std::function<void(size_t)> &f) {
    size_t helpers = std::min<size_t>(resolve(threads), tasks);
    helpers = helpers > 0 ? helpers - 1 : 0;
    if (helpers == 0) {
        for (size_t i = 0; i < tasks; i++) f(i);
        return;
    }
    Pool &p = pool();
    auto job = std::make_shared<Job>();
    job->f = &f;
    job->tasks = tasks;
    job->chunk = size == LARGE ? 1 : std::min<size_t>(8, std::max<size_t>(1, tasks / (4 * (helpers + 1))));
    job->max_helpers = helpers;
    {
        std::lock_guard<std::mutex> g(p.m);
        p.queue.push_back(job);
    }
    p.cv.notify_all();
    job->work();
    {
        std::lock_guard<std::mutex> g(p.m);
        p.queue.erase(std::remove(p.queue.begin(), p.queue.end(), job), p.queue.end());
    }
    std::unique_lock<std::mutex> lk(job->m);
    job->cv.wait(lk, [&] { return job->left >= job->joined; });
}

// ---------------------------------------------------------------- header
// src/header.rs:44-72 and src/frame.rs:84-96.
struct FrameHeader {
    uint32_t frame_size = 0;
    uint16_t header_size = 0;
    uint8_t bitstream_version = 0;
    uint8_t encoder_identifier[4] = {0, 0, 0, 0};
    uint16_t width = 0, height = 0;
    int chroma = 2;     // 2 or 3
    int interlace = 0;  // 0, 1, 2
    uint8_t aspect_ratio = 0, frame_rate_code = 0, color_primaries = 2, transfer_characteristic = 2,
            matrix_coefficients = 2;
    int alpha = 0;  // 0 none, 1 8-bit, 2 16-bit
    bool has_luma = false, has_chroma = false;
    uint8_t luma_matrix[64], chroma_matrix[64];

    uint32_t alpha_bits() const { return alpha == 1 ? 8 : alpha == 2 ? 16 : 0; }
    // :202-210
    void luma_weights(uint8_t w[64]) const {
        for (int i = 0; i < 64; i++) w[i] = has_luma ? luma_matrix[i] : 4;
    }
    void chroma_weights(uint8_t w[64]) const {
        if (has_chroma)
            memcpy(w, chroma_matrix, 64);
        else
            luma_weights(w);
    }
    // :213-255
    size_t picture_count() const { return interlace == 0 ? 1 : 2; }
    bool is_top_field(size_t index) const { return (interlace == 1) == (index == 0); }
    uint32_t picture_height(size_t index) const {
        uint32_t v = height;
        if (interlace == 0) return v;
        return is_top_field(index) ? (v + 1) / 2 : v / 2;
    }
    void picture_rows(size_t index, size_t *first_row, size_t *step) const {
        if (interlace == 0) {
            *first_row = 0;
            *step = 1;
        } else if (is_top_field(index)) {
            *first_row = 0;
            *step = 2;
        } else {
            *first_row = 1;
            *step = 2;
        }
    }
};

constexpr size_t FRAME_HEADER_FIXED = 20;   // src/header.rs:75
constexpr size_t PICTURE_HEADER_SIZE = 8;  // src/header.rs:258

// src/header.rs:82-170
Error parse_frame_header(const uint8_t *data, size_t len, FrameHeader *out) {
    if (len < 8 + FRAME_HEADER_FIXED)
        return invalid(fmt("%zu bytes is too short for a ProRes frame header", len));
    uint32_t frame_size = be32(data);
    if (memcmp(data + 4, "icpf", 4) != 0) return invalid("no 'icpf' frame identifier");
    if ((size_t)frame_size > len)
        return invalid(fmt("frame_size %u exceeds the %zu bytes given", frame_size, len));
    if ((size_t)frame_size < 8 + FRAME_HEADER_FIXED)
        return invalid("frame_size leaves no room for the frame header");
    const uint8_t *h = data + 8;
    size_t hlen = frame_size - 8;
    uint16_t header_size = be16(h);
    if ((size_t)header_size < FRAME_HEADER_FIXED || (size_t)header_size > hlen)
        return invalid(fmt("frame_header_size %u is out of range", header_size));
    hlen = header_size;
    FrameHeader f;
    f.frame_size = frame_size;
    f.header_size = header_size;
    f.bitstream_version = h[3];
    if (f.bitstream_version > 1) return unsupported(fmt("bitstream_version %u", f.bitstream_version));
    memcpy(f.encoder_identifier, h + 4, 4);
    f.width = be16(h + 8);
    f.height = be16(h + 10);
    if (f.width == 0 || f.height == 0) return invalid(fmt("a %u\xc3\x97%u frame", f.width, f.height));
    int cf = h[12] >> 6;
    if (cf != 2 && cf != 3) return invalid(fmt("chroma_format %d is reserved", cf));
    f.chroma = cf;
    int im = (h[12] >> 2) & 3;
    if (im == 3) return invalid("interlace_mode 3 is reserved");
    f.interlace = im;
    f.aspect_ratio = h[13] >> 4;
    f.frame_rate_code = h[13] & 15;
    f.color_primaries = h[14];
    f.transfer_characteristic = h[15];
    f.matrix_coefficients = h[16];
    int at = h[17] & 15;
    if (at > 2) return invalid(fmt("alpha_channel_type %d is reserved", at));
    f.alpha = at;
    bool load_luma = (h[19] & 2) != 0, load_chroma = (h[19] & 1) != 0;
    size_t pos = FRAME_HEADER_FIXED;
    if (load_luma) {
        if (pos + 64 > hlen) return invalid("a quantisation matrix runs past frame_header_size");
        memcpy(f.luma_matrix, h + pos, 64);
        f.has_luma = true;
        pos += 64;
    }
    if (load_chroma) {
        if (pos + 64 > hlen) return invalid("a quantisation matrix runs past frame_header_size");
        memcpy(f.chroma_matrix, h + pos, 64);
        f.has_chroma = true;
        pos += 64;
    }
    *out = f;
    return {};
}

// src/header.rs:174-199
void write_frame_header(const FrameHeader &h, std::vector<uint8_t> &out) {
    size_t size = FRAME_HEADER_FIXED + 64 * ((size_t)h.has_luma + (size_t)h.has_chroma);
    const uint8_t zero4[4] = {0, 0, 0, 0};
    out.insert(out.end(), zero4, zero4 + 4);
    out.insert(out.end(), {'i', 'c', 'p', 'f'});
    out.push_back((uint8_t)(size >> 8));
    out.push_back((uint8_t)size);
    out.push_back(0);
    out.push_back(h.bitstream_version);
    out.insert(out.end(), h.encoder_identifier, h.encoder_identifier + 4);
    out.push_back((uint8_t)(h.width >> 8));
    out.push_back((uint8_t)h.width);
    out.push_back((uint8_t)(h.height >> 8));
    out.push_back((uint8_t)h.height);
    out.push_back((uint8_t)((h.chroma << 6) | (h.interlace << 2)));
    out.push_back((uint8_t)((h.aspect_ratio << 4) | (h.frame_rate_code & 15)));
    out.push_back(h.color_primaries);
    out.push_back(h.transfer_characteristic);
    out.push_back(h.matrix_coefficients);
    out.push_back((uint8_t)h.alpha);
    out.push_back(0);
    out.push_back((uint8_t)(((int)h.has_luma << 1) | (int)h.has_chroma));
    if (h.has_luma) out.insert(out.end(), h.luma_matrix, h.luma_matrix + 64);
    if (h.has_chroma) out.insert(out.end(), h.chroma_matrix, h.chroma_matrix + 64);
}

struct PictureHeader {
    size_t header_size, picture_size;
    uint32_t log2_slice_mbs;
};

// src/header.rs:269-290
Error parse_picture_header(const uint8_t *data, size_t len, PictureHeader *out) {
    if (len < PICTURE_HEADER_SIZE) return invalid("a picture header runs past the end of the frame");
    size_t header_size = data[0] >> 3;
    size_t picture_size = be32(data + 1);
    if (header_size < PICTURE_HEADER_SIZE || header_size > len)
        return invalid(fmt("picture_header_size %zu is out of range", header_size));
    if (picture_size < header_size || picture_size > len)
        return invalid(fmt("picture_size %zu is out of range", picture_size));
    *out = {header_size, picture_size, (uint32_t)((data[7] >> 4) & 3)};
    return {};
}

// src/header.rs:292-304
void write_picture_header(std::vector<uint8_t> &out, uint32_t picture_size, size_t slice_count,
                          uint32_t log2_slice_mbs) {
    out.push_back((uint8_t)(PICTURE_HEADER_SIZE << 3));
    for (int i = 3; i >= 0; i--) out.push_back((uint8_t)(picture_size >> (8 * i)));
    uint16_t n = slice_count <= 65535 ? (uint16_t)slice_count : 0;
    out.push_back((uint8_t)(n >> 8));
    out.push_back((uint8_t)n);
    out.push_back((uint8_t)((log2_slice_mbs & 3) << 4));
}

// src/header.rs:308-320
std::vector<uint32_t> slice_sizes(uint32_t width_in_mb, uint32_t log2_slice_mbs) {
    std::vector<uint32_t> sizes;
    uint32_t size = 1u << log2_slice_mbs;
    uint32_t remaining = width_in_mb;
    while (remaining > 0) {
        while (remaining >= size) {
            sizes.push_back(size);
            remaining -= size;
        }
        size /= 2;
    }
    return sizes;
}

// ---------------------------------------------------------------- frame
// src/frame.rs:247-266: Y' then Cb then Cr, chroma ceil(w/2) wide for 4:2:2.
struct Plane {
    size_t offset;
    uint32_t width, height;
    size_t len() const { return (size_t)width * height; }
};
void frame_layout(uint32_t w, uint32_t h, int chroma, Plane p[3]) {
    uint32_t cw = chroma == 2 ? (w + 1) / 2 : w;
    p[0] = {0, w, h};
    p[1] = {p[0].len(), cw, h};
    p[2] = {p[1].offset + p[1].len(), cw, h};
}
const char *chroma_name(int c) { return c == 2 ? "Yuv422" : "Yuv444"; }

// src/frame.rs:299-340
Error validate_frame(const ora_frame *f) {
    if (f->chroma != 2 && f->chroma != 3) return config(fmt("chroma code %d is not 4:2:2 (2) or 4:4:4 (3)", f->chroma));
    if (f->interlace < 0 || f->interlace > 2) return config(fmt("interlace code %d is not 0-2", f->interlace));
    if (f->width == 0 || f->height == 0 || f->width > 65535 || f->height > 65535)
        return config(fmt("a frame of %u\xc3\x97%u cannot be coded", f->width, f->height));
    if (f->bit_depth < 8 || f->bit_depth > 16)
        return config(fmt("bit depth %u is outside 8\xe2\x80\x93" "16", f->bit_depth));
    Plane p[3];
    frame_layout(f->width, f->height, f->chroma, p);
    for (int i = 0; i < 3; i++)
        if (p[i].offset + p[i].len() > f->data_len)
            return config(fmt("plane %d runs past the end of the frame's data", i));
    if (f->alpha && f->alpha_len != (size_t)f->width * f->height)
        return config(fmt("the alpha plane has %zu samples, not %u\xc3\x97%u", f->alpha_len, f->width,
                          f->height));
    return {};
}

// ---------------------------------------------------------------- decode
// src/decode.rs:446-469: round((2^out - 1) a / (2^in - 1)) by a multiply.
struct Rescale {
    uint64_t m;
    bool identity;
    Rescale(uint32_t bits_in, uint32_t bits_out) {
        uint64_t max_in = (1ull << bits_in) - 1, max_out = (1ull << bits_out) - 1;
        m = ((max_out << 40) + max_in - 1) / max_in;
        identity = bits_in == bits_out;
    }
    uint16_t apply(uint16_t a) const {
        return identity ? a : (uint16_t)(((uint64_t)a * m + (1ull << 39)) >> 40);
    }
};

// src/decode.rs:484-540 (the fast path of :507-523 gives what the plain
// path gives; both are kept, as in the crate).
template <class Put>
int decode_scanned(const uint8_t *data, size_t len, size_t n_blocks, Put put) {
    BitReader r(data, len);
    uint32_t sym;
    int f = cb_read(FIRST_DC_CODEBOOK, r, &sym);
    if (f) return f;
    int32_t first = symbol_to_signed(sym);
    put(0, first);
    int32_t prev_dc = first, prev_diff = 3;
    for (size_t i = 1; i < n_blocks; i++) {
        if ((f = cb_read(dc_codebook(prev_diff), r, &sym))) return f;
        int32_t n = symbol_to_signed(sym);
        int32_t diff = prev_diff < 0 ? -n : n;
        int64_t s = (int64_t)prev_dc + diff;
        if (s > INT32_MAX || s < INT32_MIN) return F_DC_OVERFLOW;
        prev_dc = (int32_t)s;
        put(i, prev_dc);
        prev_diff = diff;
    }
    size_t total = n_blocks * 64, n = n_blocks;
    uint32_t prev_run = 4, prev_level = 1;
    for (;;) {
        uint64_t w;
        uint32_t run, l1, lvl, l2;
        if (r.peek_fast(&w) && peek_run(prev_run, w, &run, &l1) &&
            peek_level(prev_level, w << l1, &lvl, &l2) && l1 + l2 < 57) {
            n += run;
            if (n >= total) return F_RUN_PAST_END;
            int32_t level = (int32_t)lvl + 1;
            bool negative = ((w << (l1 + l2)) >> 63) == 1;
            r.skip(l1 + l2 + 1);
            put(n, negative ? -level : level);
            n += 1;
            prev_run = run;
            prev_level = lvl;
            continue;
        }
        if (r.end_of_data()) break;
        if ((f = cb_read(run_codebook(prev_run), r, &run))) return f;
        prev_run = run;
        n += run;
        if (n >= total) return F_RUN_PAST_END;
        if ((f = cb_read(level_codebook(prev_level), r, &lvl))) return f;
        prev_level = lvl;
        int32_t level = (int32_t)lvl + 1;
        uint32_t sign;
        if ((f = r.read_bit(&sign))) return f;
        put(n, sign == 1 ? -level : level);
        n += 1;
    }
    return F_OK;
}

// src/decode.rs:554-566
int decode_coefficients_raster(const uint8_t *data, size_t len, size_t n_blocks,
                               const uint8_t unscan[64], int32_t *out) {
    uint32_t shift = (uint32_t)__builtin_ctzll(n_blocks);
    size_t mask = n_blocks - 1;
    return decode_scanned(data, len, n_blocks, [&](size_t n, int32_t v) {
        out[((n & mask) << 6) | unscan[n >> shift]] = v;
    });
}

// src/decode.rs:570-595
int decode_alpha(const uint8_t *data, size_t len, uint32_t bits, size_t count, size_t needed,
                 std::vector<uint16_t> &out) {
    BitReader r(data, len);
    int32_t mask = (int32_t)((1u << bits) - 1);
    out.clear();
    int32_t prev = -1;
    while (out.size() < count) {
        if (out.size() >= needed && r.end_of_data()) break;
        int32_t diff;
        int f = read_alpha_difference(r, bits, &diff);
        if (f) return f;
        int32_t alpha = (int32_t)((uint32_t)prev + (uint32_t)diff) & mask;
        prev = alpha;
        uint32_t run;
        if ((f = read_alpha_run(r, &run))) return f;
        if (out.size() + run > count) return F_ALPHA_RUN;
        out.insert(out.end(), run, (uint16_t)alpha);
    }
    return F_OK;
}

// src/decode.rs:395-413: top-left sample of block b of macroblock m.
void block_position(int plane, int chroma, uint32_t mb_x, size_t mb_y, size_t m, size_t b, size_t *bx,
                    size_t *by) {
    size_t x = mb_x + m, y0 = 16 * mb_y;
    if (plane == 0) {
        *bx = 16 * x + 8 * (b & 1);
        *by = y0 + 8 * (b >> 1);
    } else if (chroma == 2) {
        *bx = 8 * x;
        *by = y0 + 8 * b;
    } else {
        *bx = 16 * x + 8 * (b >> 1);
        *by = y0 + 8 * (b & 1);
    }
}

struct DecodeContext {
    const FrameHeader *hdr;
    uint8_t luma_w[64], chroma_w[64], unscan[64];
    uint32_t bit_depth;
    Output out;
    Plane planes[3];
    uint16_t *data;
    uint16_t *alpha;
    DecodeContext(const FrameHeader *h, uint32_t depth) : hdr(h), bit_depth(depth), out(depth) {
        h->luma_weights(luma_w);
        h->chroma_weights(chroma_w);
        const uint8_t *scan = h->interlace == 0 ? PROGRESSIVE_SCAN : INTERLACED_SCAN;
        for (int k = 0; k < 64; k++) unscan[scan[k]] = (uint8_t)k;
    }
};

struct Placement {
    size_t height, first_row, row_step;
};

// src/decode.rs:418-438, in frame coordinates (the band split of :223-266
// only makes rows disjoint for the threads).
void put_block(DecodeContext &ctx, int plane, size_t bx, size_t by, const uint16_t v[64],
               const Placement &pl) {
    size_t pw = ctx.planes[plane].width;
    if (bx >= pw) return;
    size_t cols = std::min<size_t>(pw - bx, 8);
    size_t rows = pl.height > by ? std::min<size_t>(pl.height - by, 8) : 0;
    uint16_t *base = ctx.data + ctx.planes[plane].offset;
    for (size_t y = 0; y < rows; y++) {
        size_t row = pl.first_row + pl.row_step * (by + y);
        memcpy(base + row * pw + bx, v + 8 * y, cols * 2);
    }
}

// src/decode.rs:292-391
Error decode_slice(DecodeContext &ctx, uint32_t mb_x, uint32_t mbs, const uint8_t *s, size_t slen,
                   size_t mb_y, size_t height_in_mb, const Placement &pl, std::vector<int32_t> &coeffs,
                   std::vector<uint16_t> &alpha_vals) {
    const FrameHeader &hdr = *ctx.hdr;
    bool has_alpha = hdr.alpha != 0;
    size_t min_header = has_alpha ? 8 : 6;
    if (slen < min_header) return invalid("a slice is shorter than its header");
    size_t header_size = s[0] >> 3;
    if (header_size < min_header || header_size > slen)
        return invalid(fmt("slice_header_size %zu is out of range", header_size));
    uint32_t qindex = s[1];
    if (qindex < 1 || qindex > 224) return invalid(fmt("quantization_index %u is reserved", qindex));
    uint32_t q = qscale(qindex);
    size_t y_size = be16(s + 2), cb_size = be16(s + 4);
    size_t body = slen - header_size;
    size_t cr_size;
    if (has_alpha) {
        cr_size = be16(s + 6);
    } else {
        if (y_size + cb_size > body) return invalid("slice component sizes exceed the slice");
        cr_size = body - (y_size + cb_size);
    }
    if (y_size + cb_size + cr_size > body) return invalid("slice component sizes exceed the slice");
    const uint8_t *comp_data[3] = {s + header_size, s + header_size + y_size,
                                   s + header_size + y_size + cb_size};
    size_t comp_len[3] = {y_size, cb_size, cr_size};
    const uint8_t *alpha_data = s + header_size + y_size + cb_size + cr_size;
    size_t alpha_len = slen - (header_size + y_size + cb_size + cr_size);

    size_t chroma_per_mb = hdr.chroma == 2 ? 2 : 4;
    for (int plane = 0; plane < 3; plane++) {
        size_t per_mb = plane == 0 ? 4 : chroma_per_mb;
        const uint8_t *weights = plane == 0 ? ctx.luma_w : ctx.chroma_w;
        size_t n_blocks = per_mb * mbs;
        coeffs.assign(n_blocks * 64, 0);
        int f = decode_coefficients_raster(comp_data[plane], comp_len[plane], n_blocks, ctx.unscan,
                                           coeffs.data());
        if (f) return invalid(fail_message(f));
        float scale[64];
        for (int k = 0; k < 64; k++) scale[k] = (float)(weights[k] * q) / 8.0f;
        for (size_t blk = 0; blk < n_blocks; blk++) {
            uint16_t v[64];
            idct_put(coeffs.data() + 64 * blk, scale, ctx.out, v);
            size_t bx, by;
            block_position(plane, hdr.chroma, mb_x, mb_y, blk / per_mb, blk % per_mb, &bx, &by);
            put_block(ctx, plane, bx, by, v, pl);
        }
    }
    if (has_alpha) {
        size_t rows = mb_y + 1 < height_in_mb ? 16 : pl.height - 16 * (height_in_mb - 1);
        size_t cols = 16 * (size_t)mbs;
        int f = decode_alpha(alpha_data, alpha_len, hdr.alpha_bits(), cols * 16, cols * rows, alpha_vals);
        if (f) return invalid(fail_message(f));
        Rescale convert(hdr.alpha_bits(), ctx.bit_depth);
        size_t width = ctx.planes[0].width;
        size_t x0 = 16 * (size_t)mb_x;
        size_t n = std::min(cols, width > x0 ? width - x0 : 0);
        for (size_t r = 0; r < rows; r++) {
            size_t row = pl.first_row + pl.row_step * (16 * mb_y + r);
            uint16_t *o = ctx.alpha + row * width + x0;
            for (size_t i = 0; i < n; i++) o[i] = convert.apply(alpha_vals[cols * r + i]);
        }
    }
    return {};
}

// src/decode.rs:188-290
Error decode_picture(DecodeContext &ctx, size_t index, const PictureHeader &ph, const uint8_t *pic,
                     unsigned threads) {
    const FrameHeader &hdr = *ctx.hdr;
    uint32_t width_in_mb = (hdr.width + 15) / 16;
    uint32_t height = hdr.picture_height(index);
    size_t height_in_mb = (height + 15) / 16;
    std::vector<uint32_t> sizes = slice_sizes(width_in_mb, ph.log2_slice_mbs);
    size_t n_slices = sizes.size() * height_in_mb;
    if (ph.header_size + 2 * n_slices > ph.picture_size)
        return invalid("the slice table runs past picture_size");
    const uint8_t *table = pic + ph.header_size;
    Placement pl;
    pl.height = height;
    ctx.hdr->picture_rows(index, &pl.first_row, &pl.row_step);
    std::vector<size_t> offs(n_slices), lens(n_slices);
    size_t pos = ph.header_size + 2 * n_slices;
    for (size_t k = 0; k < n_slices; k++) {
        size_t size = be16(table + 2 * k);
        if (pos + size > ph.picture_size) return invalid("a slice runs past picture_size");
        offs[k] = pos;
        lens[k] = size;
        pos += size;
    }
    size_t row_slices = sizes.size();
    std::vector<Error> results(height_in_mb);
    pool_run(threads, height_in_mb, LARGE, [&](size_t i) {
        std::vector<int32_t> coeffs;
        std::vector<uint16_t> alpha_vals;
        uint32_t mb_x = 0;
        for (size_t j = 0; j < row_slices; j++) {
            size_t k = i * row_slices + j;
            Error e = decode_slice(ctx, mb_x, sizes[j], pic + offs[k], lens[k], i, height_in_mb, pl, coeffs,
                                   alpha_vals);
            if (e) {
                results[i] = e;
                return;
            }
            mb_x += sizes[j];
        }
    });
    for (auto &e : results)
        if (e) return e;
    return {};
}

// src/decode.rs:113-128
Error check_plausible_size(const FrameHeader &hdr) {
    uint64_t width_in_mb = (hdr.width + 15) / 16;
    uint64_t need = 8 + (uint64_t)hdr.header_size;
    for (size_t index = 0; index < hdr.picture_count(); index++) {
        uint64_t slices = (uint64_t)slice_sizes((uint32_t)width_in_mb, 3).size() *
                          ((hdr.picture_height(index) + 15) / 16);
        need += PICTURE_HEADER_SIZE + 11 * slices;
    }
    if ((uint64_t)hdr.frame_size < need)
        return invalid(fmt("frame_size %u is too small for a %u\xc3\x97%u frame (at least %llu bytes)",
                           hdr.frame_size, hdr.width, hdr.height, (unsigned long long)need));
    return {};
}

// src/decode.rs:61-104
Error decode_frame(const uint8_t *data, size_t len, uint32_t out_depth, unsigned threads, ora_frame *out) {
    if (out_depth != 0 && (out_depth < 8 || out_depth > 16))
        return config(fmt("output bit depth %u is outside 8\xe2\x80\x93" "16", out_depth));
    FrameHeader hdr;
    Error e = parse_frame_header(data, len, &hdr);
    if (e) return e;
    if ((e = check_plausible_size(hdr))) return e;
    uint32_t depth = out_depth ? out_depth : (hdr.chroma == 2 ? 10 : 12);
    DecodeContext ctx(&hdr, depth);
    frame_layout(hdr.width, hdr.height, hdr.chroma, ctx.planes);
    size_t total = ctx.planes[2].offset + ctx.planes[2].len();
    out->width = hdr.width;
    out->height = hdr.height;
    out->bit_depth = depth;
    out->chroma = hdr.chroma;
    out->interlace = hdr.interlace;
    out->aspect_ratio = hdr.aspect_ratio;
    out->frame_rate_code = hdr.frame_rate_code;
    out->color_primaries = hdr.color_primaries;
    out->transfer_characteristic = hdr.transfer_characteristic;
    out->matrix_coefficients = hdr.matrix_coefficients;
    out->data = (uint16_t *)calloc(total, 2);
    out->data_len = total;
    out->alpha = nullptr;
    out->alpha_len = 0;
    if (hdr.alpha) {
        out->alpha_len = (size_t)hdr.width * hdr.height;
        out->alpha = (uint16_t *)calloc(out->alpha_len, 2);
    }
    ctx.data = out->data;
    ctx.alpha = out->alpha;
    size_t flen = hdr.frame_size;
    size_t pos = 8 + hdr.header_size;
    for (size_t index = 0; index < hdr.picture_count(); index++) {
        if (pos > flen) return invalid("a picture starts past the end of the frame");
        PictureHeader ph{0, 0, 0};
        if ((e = parse_picture_header(data + pos, flen - pos, &ph))) return e;
        if ((e = decode_picture(ctx, index, ph, data + pos, threads))) return e;
        pos += ph.picture_size;
    }
    return {};
}

// ---------------------------------------------------------------- encode
// src/encode.rs:31-131
const uint64_t REFERENCE_BITRATE[6] = {45000000, 102000000, 147000000, 220000000, 330000000, 500000000};
const char *PROFILE_NAME[6] = {"Proxy", "Lt", "Standard", "Hq", "P4444", "P4444Xq"};
inline int profile_chroma(int p) { return p >= 4 ? 3 : 2; }
uint64_t macroblocks(uint32_t w, uint32_t h) { return (uint64_t)((w + 15) / 16) * ((h + 15) / 16); }
size_t default_headers(uint32_t w, uint32_t h) {
    size_t slices = slice_sizes((w + 15) / 16, 3).size() * (size_t)((h + 15) / 16);
    return 8 + FRAME_HEADER_FIXED + PICTURE_HEADER_SIZE + (2 + 6) * slices;
}
size_t target_frame_bytes(int profile, uint32_t w, uint32_t h) {
    double per_frame = (double)REFERENCE_BITRATE[profile] * 1001.0 / 30000.0 / 8.0;
    double per_mb = (per_frame - (double)default_headers(1920, 1080)) / (double)macroblocks(1920, 1080);
    double v = per_mb * (double)macroblocks(w, h);
    return (size_t)v + default_headers(w, h);
}

constexpr float AC_ROUNDING = 0.42f;  // src/encode.rs:204

// src/encode.rs:303-329
struct Quantisers {
    std::vector<float> inv;  // [qi][plane>0][64]
    Quantisers(const uint8_t luma[64], const uint8_t chroma[64], const uint8_t scan[64]) : inv(225 * 2 * 64) {
        for (uint32_t qi = 0; qi <= 224; qi++) {
            uint32_t q = qscale(qi < 1 ? 1 : qi);
            for (int k = 0; k < 64; k++) {
                inv[(qi * 2 + 0) * 64 + scan[k]] = 8.0f / (float)(luma[k] * q);
                inv[(qi * 2 + 1) * 64 + scan[k]] = 8.0f / (float)(chroma[k] * q);
            }
        }
    }
    const float *get(uint32_t qi, int plane) const { return &inv[(qi * 2 + (plane > 0)) * 64]; }
};

struct Quantised {
    std::vector<int32_t> values;
    std::vector<uint64_t> mask;
    void quantise_(const float *f, size_t len, const float inv[64]) {
        size_t n = len / 64;
        values.resize(64 * n);
        mask.resize(n);
        quantise(f, n, inv, AC_ROUNDING, values.data(), mask.data());
    }
};

// src/encode.rs:366-378
template <class F>
void for_each_set_bit(const std::vector<uint64_t> &mask, size_t from, F f) {
    for (size_t w = from / 64; w < mask.size(); w++) {
        uint64_t bits = w == from / 64 ? mask[w] & (~0ull << (from % 64)) : mask[w];
        while (bits) {
            f(64 * w + (size_t)__builtin_ctzll(bits));
            bits &= bits - 1;
        }
    }
}

// src/encode.rs:383-395
template <class F>
void dc_symbols(const int32_t *scanned, size_t n_blocks, F f) {
    int32_t first = scanned[0];
    f(FIRST_DC_CODEBOOK, signed_to_symbol(first));
    int32_t prev_dc = first, prev_diff = 3;
    for (size_t i = 1; i < n_blocks; i++) {
        int32_t dc = scanned[i];
        int32_t diff = (int32_t)((uint32_t)dc - (uint32_t)prev_dc);
        int32_t n = prev_diff < 0 ? -diff : diff;
        f(dc_codebook(prev_diff), signed_to_symbol(n));
        prev_diff = diff;
        prev_dc = dc;
    }
}

// src/encode.rs:398-409
size_t coefficient_bits(const Quantised &q, size_t n_blocks) {
    uint32_t bits = 0;
    dc_symbols(q.values.data(), n_blocks, [&](Codebook cb, uint32_t n) { bits += cb_len(cb, n); });
    uint32_t prev_run = 4, prev_level = 1;
    size_t pos = n_blocks;
    for_each_set_bit(q.mask, n_blocks, [&](size_t i) {
        uint32_t run = (uint32_t)(i - pos);
        int32_t v = q.values[i];
        uint32_t level = (v < 0 ? 0u - (uint32_t)v : (uint32_t)v) - 1;
        bits += cb_len(run_codebook(prev_run), run) + cb_len(level_codebook(prev_level), level) + 1;
        prev_run = run;
        prev_level = level;
        pos = i + 1;
    });
    return bits;
}

// src/encode.rs:413-437
template <class S>
void encode_coefficients_masked(S &s, const Quantised &q, size_t n_blocks) {
    dc_symbols(q.values.data(), n_blocks, [&](Codebook cb, uint32_t n) { cb_put(cb, s, n); });
    uint32_t prev_run = 4, prev_level = 1;
    size_t pos = n_blocks;
    for_each_set_bit(q.mask, n_blocks, [&](size_t i) {
        uint32_t run = (uint32_t)(i - pos);
        int32_t c = q.values[i];
        uint32_t level = (c < 0 ? 0u - (uint32_t)c : (uint32_t)c) - 1;
        uint64_t rb, lb;
        uint32_t rl, ll;
        if (cb_code(run_codebook(prev_run), run, &rb, &rl) &&
            cb_code(level_codebook(prev_level), level, &lb, &ll) && rl + ll < 57) {
            s.put((((rb << ll) | lb) << 1) | (uint64_t)(c < 0), rl + ll + 1);
        } else {
            cb_put(run_codebook(prev_run), s, run);
            cb_put(level_codebook(prev_level), s, level);
            s.put((uint64_t)(c < 0), 1);
        }
        prev_run = run;
        prev_level = level;
        pos = i + 1;
    });
    s.align();
}

// src/encode.rs:457-470
template <class S>
void encode_alpha(S &s, const uint16_t *values, size_t len, uint32_t bits) {
    int32_t prev = -1;
    size_t i = 0;
    while (i < len) {
        uint16_t a = values[i];
        size_t end = std::min(i + 2048, len);
        size_t run = 1;
        while (i + run < end && values[i + run] == a) run++;
        put_alpha_difference(s, (int32_t)a - prev, bits);
        put_alpha_run(s, (uint32_t)run);
        prev = a;
        i += run;
    }
    s.align();
}

struct SliceBlocks {
    uint32_t mbs;
    const float *comps[3];
    size_t comp_len[3];
    std::vector<uint8_t> alpha;
};

struct PictureLayout {
    const ora_frame *frame;
    const FrameHeader *hdr;
    Plane planes[3];
    size_t height, first_row, step;
    const uint8_t *scan;

    // src/encode.rs:488-505: edge-replicated 8x8 gather.
    void block(int plane, size_t bx, size_t by, uint16_t pix[64]) const {
        const Plane &p = planes[plane];
        const uint16_t *src = frame->data + p.offset;
        size_t w = p.width;
        for (size_t y = 0; y < 8; y++) {
            size_t row = first_row + step * std::min(by + y, height - 1);
            const uint16_t *line = src + row * w;
            for (size_t x = 0; x < 8; x++) pix[8 * y + x] = line[std::min(bx + x, w - 1)];
        }
    }
    size_t slice_len(uint32_t mbs) const {
        size_t cpm = frame->chroma == 2 ? 2 : 4;
        return 64 * (4 + 2 * cpm) * (size_t)mbs;
    }
    // src/encode.rs:518-555
    std::vector<uint8_t> transform(uint32_t mb_x, uint32_t mbs, size_t mb_y, float *out) const;
};

// src/encode.rs:838-868
std::vector<uint8_t> slice_alpha(const ora_frame *frame, const uint16_t *alpha, uint32_t bits, uint32_t mb_x,
                                 uint32_t mbs, size_t mb_y, size_t height, size_t first_row, size_t step) {
    size_t width = frame->width;
    uint16_t max_in = (uint16_t)(0xFFFFu >> (16 - frame->bit_depth));
    Rescale convert(frame->bit_depth, bits);
    size_t cols = 16 * (size_t)mbs, x0 = 16 * (size_t)mb_x;
    std::vector<uint16_t> values;
    values.reserve(cols * 16);
    for (size_t r = 0; r < 16; r++) {
        size_t row = first_row + step * std::min(16 * mb_y + r, height - 1);
        for (size_t n = 0; n < cols; n++) {
            uint16_t a = alpha[row * width + std::min(x0 + n, width - 1)];
            values.push_back(convert.apply(std::min(a, max_in)));
        }
    }
    std::vector<uint8_t> out;
    BitWriter w(&out);
    encode_alpha(w, values.data(), values.size(), bits);
    w.finish();
    return out;
}

std::vector<uint8_t> PictureLayout::transform(uint32_t mb_x, uint32_t mbs, size_t mb_y, float *out) const {
    size_t cpm = frame->chroma == 2 ? 2 : 4;
    float scale = 512.0f / (float)(1u << frame->bit_depth);
    float *rest = out;
    for (int plane = 0; plane < 3; plane++) {
        size_t per_mb = plane == 0 ? 4 : cpm;
        size_t n = per_mb * mbs;
        for (size_t blk = 0; blk < n; blk++) {
            size_t bx, by;
            block_position(plane, frame->chroma, mb_x, mb_y, blk / per_mb, blk % per_mb, &bx, &by);
            uint16_t pix[64];
            block(plane, bx, by, pix);
            float f[64];
            fdct_load(pix, scale, f);
            for (int k = 0; k < 64; k++) rest[n * scan[k] + blk] = f[k];
        }
        rest += 64 * n;
    }
    if (frame->alpha && hdr->alpha != 0)
        return slice_alpha(frame, frame->alpha, hdr->alpha_bits(), mb_x, mbs, mb_y, height, first_row, step);
    return {};
}

thread_local std::vector<std::vector<uint8_t>> g_last_qindices;

// src/encode.rs:657-830
void code_picture(const FrameHeader &hdr, const std::vector<SliceBlocks> &slices, const uint8_t scan[64],
                  uint32_t log2_slice_mbs, size_t budget_in, unsigned threads, std::vector<uint8_t> &out) {
    size_t header_bytes = hdr.alpha != 0 ? 8 : 6;
    uint8_t lw[64], cw[64];
    hdr.luma_weights(lw);
    hdr.chroma_weights(cw);
    Quantisers quantisers(lw, cw, scan);
    struct Size {
        size_t n;
        bool fits;
    };
    auto slice_size = [&](const SliceBlocks &s, uint32_t qi) -> Size {
        thread_local Quantised q;
        size_t comp[3];
        for (int plane = 0; plane < 3; plane++) {
            q.quantise_(s.comps[plane], s.comp_len[plane], quantisers.get(qi, plane));
            comp[plane] = (coefficient_bits(q, s.comp_len[plane] / 64) + 7) / 8;
        }
        size_t total = header_bytes + comp[0] + comp[1] + comp[2] + s.alpha.size();
        return {total, total <= 65535 && comp[0] <= 65535 && comp[1] <= 65535 && comp[2] <= 65535};
    };
    size_t ns = slices.size();
    auto sizes_at = [&](uint32_t qi) {
        std::vector<Size> v(ns);
        pool_run(threads, ns, SMALL, [&](size_t i) { v[i] = slice_size(slices[i], qi); });
        return v;
    };
    size_t overhead = PICTURE_HEADER_SIZE + 2 * ns;
    size_t alpha_bytes = 0;
    for (auto &s : slices) alpha_bytes += s.alpha.size();
    size_t budget = budget_in + alpha_bytes;
    budget = budget > overhead ? budget - overhead : 0;
    std::vector<std::vector<Size>> probed(225);
    std::vector<bool> have(225, false);
    auto totals = [&](uint32_t qi) {
        std::vector<Size> v = sizes_at(qi);
        bool all = true;
        size_t sum = 0;
        for (auto &s : v) {
            all = all && s.fits;
            sum += s.n;
        }
        probed[qi] = std::move(v);
        have[qi] = true;
        return all && sum <= budget;
    };
    uint32_t lo = 1, hi = 224;
    bool fits_at_all = totals(224);
    if (fits_at_all) {
        while (lo < hi) {
            uint32_t mid = lo + (hi - lo) / 2;
            if (totals(mid))
                hi = mid;
            else
                lo = mid + 1;
        }
    }
    uint32_t uniform = hi;
    std::vector<size_t> used(ns);
    for (size_t i = 0; i < ns; i++) used[i] = probed[uniform][i].n;
    std::vector<uint8_t> qindices(ns, (uint8_t)uniform);
    if (uniform > 1 && fits_at_all) {
        // The crate computes sizes at the next few finer quantisers in
        // parallel first (:732-768) only to save time; what the share-out
        // reads is the size of a slice at a quantiser, whoever computes it.
        std::vector<std::vector<Size>> finer;
        std::vector<std::vector<bool>> finer_have;
        uint64_t slack0 = budget;
        size_t used_sum = 0;
        for (auto u : used) used_sum += u;
        slack0 -= used_sum;
        std::vector<uint64_t> mbs_from(ns + 1, 0);
        for (size_t i = ns; i-- > 0;) mbs_from[i] = mbs_from[i + 1] + slices[i].mbs;
        auto most = [&](size_t i) { return used[i] + (size_t)(slack0 * slices[i].mbs / mbs_from[i]); };
        const size_t WINDOW = 3;
        for (size_t j = 0; j < std::min<size_t>(uniform - 1, WINDOW); j++) {
            uint32_t qi = uniform - 1 - (uint32_t)j;
            if (j == 0 && have[qi]) {
                finer.push_back(probed[qi]);
                finer_have.push_back(std::vector<bool>(ns, true));
                continue;
            }
            std::vector<size_t> cand;
            for (size_t i = 0; i < ns; i++) {
                bool wanted = j == 0 || (finer_have[j - 1][i] && finer[j - 1][i].fits &&
                                         finer[j - 1][i].n <= most(i));
                if (wanted) cand.push_back(i);
            }
            if (cand.empty()) break;
            std::vector<Size> row(ns);
            std::vector<bool> rh(ns, false);
            pool_run(threads, cand.size(), SMALL, [&](size_t c) { row[cand[c]] = slice_size(slices[cand[c]], qi); });
            for (auto i : cand) rh[i] = true;
            finer.push_back(std::move(row));
            finer_have.push_back(std::move(rh));
        }
        size_t remaining_budget = budget, remaining_base = used_sum;
        uint64_t remaining_mbs = 0;
        for (auto &s : slices) remaining_mbs += s.mbs;
        for (size_t i = 0; i < ns; i++) {
            size_t base = used[i];
            uint64_t slack = remaining_budget - remaining_base;
            size_t allowed = base + (size_t)(slack * slices[i].mbs / remaining_mbs);
            uint32_t qi = uniform;
            while (qi > 1) {
                size_t step = uniform - qi;
                Size sz;
                if (step < finer.size() && finer_have[step][i])
                    sz = finer[step][i];
                else
                    sz = slice_size(slices[i], qi - 1);
                if (!(sz.fits && sz.n <= allowed)) break;
                qi -= 1;
                used[i] = sz.n;
            }
            qindices[i] = (uint8_t)qi;
            remaining_budget -= used[i];
            remaining_base -= base;
            remaining_mbs -= slices[i].mbs;
        }
    }
    g_last_qindices.push_back(qindices);

    // :797-819: code every slice.
    std::vector<std::vector<uint8_t>> coded(ns);
    pool_run(threads, ns, SMALL, [&](size_t i) {
        const SliceBlocks &s = slices[i];
        uint32_t qi = qindices[i];
        std::vector<uint8_t> &bytes = coded[i];
        bytes.reserve(used[i]);
        bytes.push_back((uint8_t)(header_bytes << 3));
        bytes.push_back((uint8_t)qi);
        bytes.resize(header_bytes, 0);
        size_t comp_sizes[3];
        thread_local Quantised q;
        for (int plane = 0; plane < 3; plane++) {
            q.quantise_(s.comps[plane], s.comp_len[plane], quantisers.get(qi, plane));
            BitWriter bw(&bytes);
            encode_coefficients_masked(bw, q, s.comp_len[plane] / 64);
            comp_sizes[plane] = bw.finish();
        }
        bytes[2] = (uint8_t)(comp_sizes[0] >> 8);
        bytes[3] = (uint8_t)comp_sizes[0];
        bytes[4] = (uint8_t)(comp_sizes[1] >> 8);
        bytes[5] = (uint8_t)comp_sizes[1];
        if (header_bytes == 8) {
            bytes[6] = (uint8_t)(comp_sizes[2] >> 8);
            bytes[7] = (uint8_t)comp_sizes[2];
        }
        bytes.insert(bytes.end(), s.alpha.begin(), s.alpha.end());
    });
    size_t pic_start = out.size();
    write_picture_header(out, 0, ns, log2_slice_mbs);
    for (auto &s : coded) {
        uint16_t n = (uint16_t)s.size();
        out.push_back((uint8_t)(n >> 8));
        out.push_back((uint8_t)n);
    }
    for (auto &s : coded) out.insert(out.end(), s.begin(), s.end());
    uint32_t picture_size = (uint32_t)(out.size() - pic_start);
    for (int i = 0; i < 4; i++) out[pic_start + 1 + i] = (uint8_t)(picture_size >> (24 - 8 * i));
}

// src/encode.rs:567-653
void encode_picture(const FrameHeader &hdr, size_t index, const ora_frame *frame, uint32_t log2, size_t budget,
                    unsigned threads, std::vector<uint8_t> &out) {
    uint32_t width_in_mb = (frame->width + 15) / 16;
    size_t height = hdr.picture_height(index);
    size_t height_in_mb = (height + 15) / 16;
    PictureLayout layout;
    layout.frame = frame;
    layout.hdr = &hdr;
    frame_layout(frame->width, frame->height, frame->chroma, layout.planes);
    layout.height = height;
    hdr.picture_rows(index, &layout.first_row, &layout.step);
    layout.scan = hdr.interlace == 0 ? PROGRESSIVE_SCAN : INTERLACED_SCAN;
    std::vector<uint32_t> sizes = slice_sizes(width_in_mb, log2);
    struct Place {
        uint32_t mb_x, mbs;
        size_t mb_y;
    };
    std::vector<Place> places;
    for (size_t mb_y = 0; mb_y < height_in_mb; mb_y++) {
        uint32_t mb_x = 0;
        for (auto mbs : sizes) {
            places.push_back({mb_x, mbs, mb_y});
            mb_x += mbs;
        }
    }
    std::vector<size_t> starts(places.size() + 1, 0);
    for (size_t i = 0; i < places.size(); i++) starts[i + 1] = starts[i] + layout.slice_len(places[i].mbs);
    std::vector<float> coefficients(starts.back());
    std::vector<std::vector<uint8_t>> alphas(places.size());
    pool_run(threads, places.size(), SMALL, [&](size_t i) {
        alphas[i] = layout.transform(places[i].mb_x, places[i].mbs, places[i].mb_y, coefficients.data() + starts[i]);
    });
    std::vector<SliceBlocks> slices(places.size());
    for (size_t i = 0; i < places.size(); i++) {
        SliceBlocks &s = slices[i];
        s.mbs = places[i].mbs;
        size_t luma = 64 * 4 * (size_t)s.mbs;
        size_t chroma = (layout.slice_len(s.mbs) - luma) / 2;
        const float *c = coefficients.data() + starts[i];
        s.comps[0] = c;
        s.comp_len[0] = luma;
        s.comps[1] = c + luma;
        s.comp_len[1] = chroma;
        s.comps[2] = c + luma + chroma;
        s.comp_len[2] = chroma;
        s.alpha = std::move(alphas[i]);
    }
    code_picture(hdr, slices, layout.scan, log2, budget, threads, out);
}

// src/encode.rs:176-192, :223-287
Error encode_frame(const ora_config *cfg, const ora_frame *frame, std::vector<uint8_t> &out) {
    if (cfg->log2_slice_mbs > 3) return config(fmt("log2_slice_mbs %u is outside 0\xe2\x80\x93" "3", cfg->log2_slice_mbs));
    for (int m = 0; m < 2; m++) {
        if (!(m == 0 ? cfg->has_luma_matrix : cfg->has_chroma_matrix)) continue;
        const uint8_t *w = m == 0 ? cfg->luma_matrix : cfg->chroma_matrix;
        for (int i = 0; i < 64; i++)
            if (w[i] < 2 || w[i] > 63) return config("quantisation weights must be 2\xe2\x80\x93" "63");
    }
    Error e = validate_frame(frame);
    if (e) return e;
    int pchroma = profile_chroma(cfg->profile);
    if (frame->chroma != pchroma)
        return config(fmt("%s codes %s, and the frame is %s", PROFILE_NAME[cfg->profile], chroma_name(pchroma),
                          chroma_name(frame->chroma)));
    int alpha = 0;
    if (frame->alpha) {
        if (pchroma == 2) return config(fmt("%s carries no alpha channel", PROFILE_NAME[cfg->profile]));
        alpha = cfg->alpha;
    }
    FrameHeader hdr;
    hdr.bitstream_version = (frame->chroma == 2 && alpha == 0) ? 0 : 1;
    memcpy(hdr.encoder_identifier, cfg->encoder_identifier, 4);
    hdr.width = (uint16_t)frame->width;
    hdr.height = (uint16_t)frame->height;
    hdr.chroma = frame->chroma;
    hdr.interlace = frame->interlace;
    hdr.aspect_ratio = frame->aspect_ratio;
    hdr.frame_rate_code = frame->frame_rate_code;
    hdr.color_primaries = frame->color_primaries;
    hdr.transfer_characteristic = frame->transfer_characteristic;
    hdr.matrix_coefficients = frame->matrix_coefficients;
    hdr.alpha = alpha;
    hdr.has_luma = cfg->has_luma_matrix != 0;
    hdr.has_chroma = cfg->has_chroma_matrix != 0;
    memcpy(hdr.luma_matrix, cfg->luma_matrix, 64);
    memcpy(hdr.chroma_matrix, cfg->chroma_matrix, 64);
    out.clear();
    write_frame_header(hdr, out);
    size_t target = cfg->target_frame_bytes >= 0 ? (size_t)cfg->target_frame_bytes
                                                 : target_frame_bytes(cfg->profile, frame->width, frame->height);
    out.reserve(target);
    size_t pictures = hdr.picture_count();
    size_t per_picture = (target > out.size() ? target - out.size() : 0) / pictures;
    g_last_qindices.clear();
    for (size_t index = 0; index < pictures; index++)
        encode_picture(hdr, index, frame, cfg->log2_slice_mbs, per_picture, cfg->threads, out);
    uint32_t size = (uint32_t)out.size();
    for (int i = 0; i < 4; i++) out[i] = (uint8_t)(size >> (24 - 8 * i));
    return {};
}

int report(const Error &e, char *msg, size_t cap) {
    if (msg && cap) {
        size_t n = std::min(cap - 1, e.msg.size());
        memcpy(msg, e.msg.data(), n);
        msg[n] = 0;
    }
    return e.kind;
}

Codebook book_by_id(int id) {
    if (id < 4) return DC_CODEBOOKS[id];
    if (id < 20) return RUN_CODEBOOKS[id - 4];
    if (id < 29) return LEVEL_CODEBOOKS[id - 20];
    return FIRST_DC_CODEBOOK;
}

int to_string(const std::vector<uint8_t> &v, size_t bits, char *out, size_t cap) {
    if (bits + 1 > cap) return -1;
    for (size_t i = 0; i < bits; i++) out[i] = (v[i / 8] >> (7 - i % 8)) & 1 ? '1' : '0';
    out[bits] = 0;
    return (int)bits;
}

}  // namespace

// ================================================================ C ABI

extern "C" {

int ora_decode(const uint8_t *data, size_t len, uint32_t out_bit_depth, uint32_t threads, ora_frame *out,
               char *msg, size_t msg_cap) {
    memset(out, 0, sizeof *out);
    Error e = decode_frame(data, len, out_bit_depth, threads, out);
    if (e) {
        ora_frame_free(out);
        return report(e, msg, msg_cap);
    }
    return ORA_OK;
}

void ora_frame_free(ora_frame *f) {
    free(f->data);
    free(f->alpha);
    f->data = nullptr;
    f->alpha = nullptr;
}

int ora_encode(const ora_config *cfg, const ora_frame *in, uint8_t **out, size_t *out_len, char *msg,
               size_t msg_cap) {
    std::vector<uint8_t> v;
    Error e = encode_frame(cfg, in, v);
    if (e) {
        *out = nullptr;
        *out_len = 0;
        return report(e, msg, msg_cap);
    }
    *out = (uint8_t *)malloc(v.size() ? v.size() : 1);
    memcpy(*out, v.data(), v.size());
    *out_len = v.size();
    return ORA_OK;
}

void ora_free(void *p) { free(p); }

size_t ora_last_qindices(int picture, uint8_t *out, size_t cap) {
    if (picture < 0 || (size_t)picture >= g_last_qindices.size()) return 0;
    const auto &q = g_last_qindices[picture];
    size_t n = std::min(cap, q.size());
    memcpy(out, q.data(), n);
    return q.size();
}

size_t ora_target_frame_bytes(int profile, uint32_t width, uint32_t height) {
    return target_frame_bytes(profile, width, height);
}

size_t ora_slice_sizes(uint32_t width_in_mb, uint32_t log2_slice_mbs, uint32_t *out, size_t cap) {
    auto v = slice_sizes(width_in_mb, log2_slice_mbs);
    for (size_t i = 0; i < v.size() && i < cap; i++) out[i] = v[i];
    return v.size();
}

int ora_codeword(int book, uint32_t n, char *bits, size_t cap) {
    std::vector<uint8_t> v;
    BitWriter w(&v);
    cb_put(book_by_id(book), w, n);
    size_t nb = w.bits();
    w.finish();
    return to_string(v, nb, bits, cap);
}

uint32_t ora_codeword_len(int book, uint32_t n) { return cb_len(book_by_id(book), n); }

int ora_codebook_read(int book, const uint8_t *data, size_t len, uint32_t *value, uint32_t *consumed) {
    BitReader r(data, len);
    int f = cb_read(book_by_id(book), r, value);
    *consumed = (uint32_t)r.pos;
    return f ? ORA_INVALID : ORA_OK;
}

int ora_alpha_run_code(uint32_t run, char *bits, size_t cap) {
    std::vector<uint8_t> v;
    BitWriter w(&v);
    put_alpha_run(w, run);
    size_t nb = w.bits();
    w.finish();
    return to_string(v, nb, bits, cap);
}

int ora_alpha_diff_code(int32_t diff, uint32_t bits, char *out, size_t cap) {
    std::vector<uint8_t> v;
    BitWriter w(&v);
    put_alpha_difference(w, diff, bits);
    size_t nb = w.bits();
    w.finish();
    return to_string(v, nb, out, cap);
}

uint16_t ora_rescale(uint32_t bits_in, uint32_t bits_out, uint16_t a) { return Rescale(bits_in, bits_out).apply(a); }
uint32_t ora_qscale(uint32_t qindex) { return qscale(qindex); }
void ora_scans(uint8_t progressive[64], uint8_t interlaced[64]) {
    memcpy(progressive, PROGRESSIVE_SCAN, 64);
    memcpy(interlaced, INTERLACED_SCAN, 64);
}
void ora_basis(float b[64]) { memcpy(b, basis().t, sizeof(float) * 64); }

void ora_idct_put(const int32_t coef[64], const float scale[64], uint32_t bit_depth, uint16_t out[64]) {
    idct_put(coef, scale, Output(bit_depth), out);
}
void ora_fdct_load(const uint16_t pix[64], float scale, float out[64]) { fdct_load(pix, scale, out); }
void ora_set_simd(int on) { g_simd.store(on != 0); }
void ora_quantise(const float *f, size_t n, const float inv[64], float ac_rounding, int32_t *out, uint64_t *mask) {
    quantise(f, n, inv, ac_rounding, out, mask);
}

size_t ora_encode_coefficients(const int32_t *scanned, size_t n_blocks, uint8_t *out, size_t cap, size_t *bits) {
    Quantised q;
    q.values.assign(scanned, scanned + n_blocks * 64);
    q.mask.assign(n_blocks, 0);
    for (size_t i = 0; i < n_blocks * 64; i++) q.mask[i / 64] |= (uint64_t)(scanned[i] != 0) << (i % 64);
    std::vector<uint8_t> v;
    BitWriter w(&v);
    encode_coefficients_masked(w, q, n_blocks);
    *bits = coefficient_bits(q, n_blocks);
    w.finish();
    memcpy(out, v.data(), std::min(cap, v.size()));
    return v.size();
}

int ora_decode_coefficients(const uint8_t *data, size_t len, size_t n_blocks, int32_t *scanned, char *msg,
                            size_t msg_cap) {
    for (size_t i = 0; i < n_blocks * 64; i++) scanned[i] = 0;
    int f = decode_scanned(data, len, n_blocks, [&](size_t n, int32_t v) { scanned[n] = v; });
    if (f) return report(invalid(fail_message(f)), msg, msg_cap);
    return ORA_OK;
}

size_t ora_encode_alpha(const uint16_t *values, size_t n, uint32_t bits, uint8_t *out, size_t cap) {
    std::vector<uint8_t> v;
    BitWriter w(&v);
    encode_alpha(w, values, n, bits);
    w.finish();
    memcpy(out, v.data(), std::min(cap, v.size()));
    return v.size();
}

int ora_decode_alpha(const uint8_t *data, size_t len, uint32_t bits, size_t count, size_t needed, uint16_t *out,
                     size_t *got) {
    std::vector<uint16_t> v;
    int f = decode_alpha(data, len, bits, count, needed, v);
    *got = v.size();
    if (f) return ORA_INVALID;
    memcpy(out, v.data(), v.size() * 2);
    return ORA_OK;
}

// tests/common/mod.rs:26-80
void ora_test_frame(uint32_t width, uint32_t height, int32_t chroma, uint32_t bit_depth, int32_t grain,
                    uint32_t seed, uint16_t *data) {
    Plane p[3];
    frame_layout(width, height, chroma, p);
    uint32_t rng = seed | 1;
    auto next = [&]() {
        rng ^= rng << 13;
        rng ^= rng >> 17;
        rng ^= rng << 5;
        return rng;
    };
    int shift = (int)bit_depth - 10;
    auto scale = [&](double v) -> uint16_t {
        v = std::min(std::max(v, 64.0), 940.0);
        double s = shift >= 0 ? v * (double)(1 << shift) : v / (double)(1 << -shift);
        return (uint16_t)round(s);
    };
    double w = width, h = height;
    for (int plane = 0; plane < 3; plane++) {
        double xs = plane == 0 ? 1.0 : (chroma == 2 ? 2.0 : 1.0);
        uint16_t *d = data + p[plane].offset;
        for (uint32_t y = 0; y < p[plane].height; y++)
            for (uint32_t x = 0; x < p[plane].width; x++) {
                double fx = (double)x * xs, fy = (double)y;
                double v;
                if (plane == 0)
                    v = 200.0 + 500.0 * fx / w + 120.0 * sin(fx / 37.0) * cos(fy / 23.0);
                else if (plane == 1)
                    v = 512.0 + 150.0 * (fx / w - 0.5) + 60.0 * sin(fy / 50.0);
                else
                    v = 512.0 - 120.0 * (fy / h - 0.5) + 50.0 * cos(fx / 70.0);
                if (fx > w * 0.15 && fx < w * 0.35 && fy > h * 0.2 && fy < h * 0.5) v = plane == 0 ? 900.0 : v + 150.0;
                if (fx > w * 0.6 && fx < w * 0.8 && fy > h * 0.55 && fy < h * 0.85) v = plane == 0 ? 90.0 : v - 150.0;
                if (fx < w * 0.25 && fy > h * 0.7) v += 150.0 * sin(fx * 1.3);
                if (grain > 0) v += (double)((int32_t)(next() % (uint32_t)(2 * grain + 1)) - grain);
                d[(size_t)y * p[plane].width + x] = scale(v);
            }
    }
}

}  // extern "C"
