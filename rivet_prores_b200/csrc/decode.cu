// decode.cu -- the RDD 36 decoding process (§7) as sm_100a kernels.
//
//   k_locate   one CTA per picture: the big-endian u16 slice table, scanned
//              into slice offsets (src/decode.rs:202-221), each slice's
//              place in the picture (src/header.rs:308-320), and the first
//              slice that runs past picture_size.
//   k_entropy  persistent; one lane per slice component (Y', Cb, Cr, alpha):
//              the slice header (src/decode.rs:301-338), then the DC and
//              run/level/sign codes of the interleaved scan (:484-540) as a
//              list of (position, value) entries, or the alpha
//              run/difference codes (:570-595) straight into the alpha plane.
//   k_idct     one CTA per slice: the entries placed in shared memory,
//              inverse quantisation, the 8x8 IDCT in the crate's exact
//              single-precision order (src/dct.rs:36-66,
//              src/dsp/scalar.rs:8-12) and the sample conversion, stored as
//              woven 16-byte rows (src/decode.rs:395-438).
//   k_status   one CTA per picture: the first failing slice component.
//
// The f32 arithmetic uses __fmul_rn/__fadd_rn so that nothing is contracted
// into an FMA: the decoded samples are bit-identical to the crate's.

#include <cuda_runtime.h>

#include <cstdint>

#include "codec_tables.h"
#include "device_types.h"
#include "pair_math.h"

namespace prores {

__constant__ uint8_t c_scan[2][64];
__constant__ float c_idct_basis[64];  // T[x][u] (dct_basis)

namespace {


// floor(v) clamped to [0, max] (max an integer below 2^16), as an integer:
// clamping before the floor gives the same value as after it for integer
// bounds, and adding 2^23 rounded down leaves floor(v) in the low bits.
__device__ __forceinline__ uint32_t floor_clamped(float v, float max) {
    const float c = fminf(fmaxf(v, 0.0f), max);
    return __float_as_uint(__fadd_rd(c, 8388608.0f)) & 0xFFFFu;
}

// q exactly, for |q| < 2^22: q added to the significand of 1.5 2^23.
__device__ __forceinline__ float small_int_to_float(int32_t q) {
    return __fadd_rn(__int_as_float(0x4B400000 + q), -12582912.0f);
}

__device__ __forceinline__ uint64_t bswap64(uint64_t v) {
    uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

__device__ __forceinline__ uint32_t be16(const uint8_t *p) { return ((uint32_t)p[0] << 8) | p[1]; }

// MSB-first reader over [start, end) bits of the bitstream buffer: a pair of
// aligned 64-bit words funnel-shifted to the position; bits past `end` read
// as zero (the crate's BitReader::peek64, src/bits.rs:30-40). The word after
// the pair is fetched one word ahead, so moving on to the next word never
// waits for memory. The buffer has at least 24 bytes of padding after the
// last data word, so the words read never leave it.
struct Bits {
    const uint64_t *w;
    uint64_t pos, end, idx, w0, w1, w2;

    __device__ __forceinline__ uint64_t ld(uint64_t i) const { return bswap64(__ldg(w + i)); }
    __device__ __forceinline__ void init(const uint8_t *base, uint64_t byte_off, uint64_t len) {
        w = reinterpret_cast<const uint64_t *>(base);
        pos = byte_off * 8;
        end = pos + len * 8;
        idx = pos >> 6;
        w0 = ld(idx);
        w1 = ld(idx + 1);
        w2 = ld(idx + 2);
    }
    __device__ __forceinline__ uint64_t remaining() const { return end - pos; }
    __device__ __forceinline__ uint64_t peek() {
        uint64_t i = pos >> 6;
        if (i != idx) {
            if (i == idx + 1) {
                w0 = w1;
                w1 = w2;
                w2 = ld(i + 2);
            } else {
                w0 = ld(i);
                w1 = ld(i + 1);
                w2 = ld(i + 2);
            }
            idx = i;
        }
        uint32_t sh = (uint32_t)(pos & 63);
        uint64_t v = sh ? (w0 << sh) | (w1 >> (64 - sh)) : w0;
        uint64_t rem = end - pos;
        if (rem < 64) v &= rem ? (~0ull << (64 - rem)) : 0ull;
        return v;
    }
    // `n` (1..57) bits as a number (src/bits.rs:61-72).
    __device__ __forceinline__ int read(uint32_t n, uint64_t &v) {
        if ((uint64_t)n > remaining()) return DE_PAST_END;
        v = peek() >> (64 - n);
        pos += n;
        return DE_OK;
    }
    // RDD 36 endOfData(): 31 or fewer bits remain, all zero (src/bits.rs:98-101).
    __device__ __forceinline__ bool end_of_data() {
        return remaining() <= 31 && peek() == 0;
    }
};

// One symbol of codebook `cb` (src/vlc.rs:207-230), read bit by bit as the
// crate reads it, naming any failure exactly as the crate does.
__device__ __forceinline__ int read_sym(Bits &b, Codebook cb, uint32_t &sym) {
    uint64_t w = b.peek();
    uint64_t rem = b.remaining();
    uint32_t lz = clz64(w);
    if (lz > kMaxPrefix) return DE_PREFIX;
    if ((uint64_t)lz >= rem) return DE_PAST_END;
    b.pos += lz;
    rem -= lz;
    w = b.peek();
    if (!cb.eg && lz <= cb.q) {
        uint32_t need = 1u + cb.r;
        if (need > rem) return DE_PAST_END;
        uint64_t v = (w >> (64 - need)) & ((1ull << cb.r) - 1);
        b.pos += need;
        sym = (uint32_t)(((uint64_t)lz << cb.r) | v);
        return DE_OK;
    }
    uint32_t qe = cb.eg ? lz : lz - (cb.q + 1u);
    uint32_t ke = cb.eg ? cb.r : cb.e;
    uint64_t off = cb.eg ? 0ull : ((uint64_t)(cb.q + 1u) << cb.r);
    uint32_t need = qe + ke + 1u;
    if (need > rem) return DE_PAST_END;
    uint64_t v = w >> (64 - need);
    b.pos += need;
    uint64_t n = v - (1ull << ke) + off;
    if (n > kMaxSymbol) return DE_RANGE;
    sym = (uint32_t)n;
    return DE_OK;
}

// A component's coefficient list, in a region of 2 cap 32-bit words (cap =
// 64 n_blocks, the component's positions): entries from the front, each
// (scanned index << 21) | value in 21-bit two's complement. Values outside
// [kListMin, 2^20) go to the back of the region, the k-th at 2 cap - 1 - k,
// and their entry holds -2^20 + k. Half the bytes of (index, value) pairs
// of 32-bit words, for values of any size.
constexpr int32_t kListMin = -(1 << 20) + 2048;

struct CoefList {
    uint32_t *w;
    uint32_t cap, big, count;
    __device__ __forceinline__ void put(uint32_t n, int32_t v) {
        if (v >= kListMin && v < (1 << 20)) {
            w[count++] = (n << 21) | ((uint32_t)v & 0x1FFFFFu);
        } else {
            w[2u * cap - 1u - big] = (uint32_t)v;
            w[count++] = (n << 21) | ((uint32_t)(-(1 << 20) + (int32_t)big) & 0x1FFFFFu);
            big++;
        }
    }
};

// A component's coefficients as one small integer (int8_t or int16_t) per
// scanned position in shared memory (zeroed beforehand: only the coded ones
// are written). A value the type cannot hold, other than its most negative
// one, is marked with that one (wide_mark<T>) and kept at the same position
// of a 32-bit array in global memory, which is otherwise never touched.
template <class T>
__device__ __forceinline__ constexpr int32_t wide_mark() {
    return sizeof(T) == 1 ? -128 : -32768;
}

template <class T>
struct SlotOut {
    T *slot;
    int32_t *wide;
    __device__ __forceinline__ void put(uint32_t n, int32_t v) {
        if (v > wide_mark<T>() && v <= -(wide_mark<T>() + 1)) {
            slot[n] = (T)v;
        } else {
            slot[n] = (T)wide_mark<T>();
            wide[n] = v;
        }
    }
};

// An entry's (index, value), reading a large value from the region's back.
__device__ __forceinline__ void list_entry(const uint32_t *w, uint32_t cap, uint32_t e, uint32_t &n, int32_t &v) {
    n = e >> 21;
    v = (int32_t)(e << 11) >> 11;
    if (v < kListMin) v = (int32_t)__ldg(w + 2u * cap - 1u - (uint32_t)(v + (1 << 20)));
}

// The read position as a 64-bit window consumed from the top: `cur` holds
// the bits [pos, pos + avail) MSB first with zeros below, and is refilled
// 32 bits at a time from the words after it, which are fetched two ahead
// and kept as loaded (byte-swapped only when they enter the window), so a
// refill never waits for the load it issues. A symbol costs shifts of the
// window rather than a fresh funnel shift of two words. Reads the same
// bits as Bits; only used while at least 32 bits of the component remain,
// so the top 32 bits are always data. The words fetched reach 12 bytes past
// the component's data at most, inside the bitstream buffer's padding.
struct Window {
    const uint32_t *w;
    uint64_t cur;
    uint32_t avail, left;  // valid bits in cur (>= 32); bits of the component from pos on
    uint64_t next;         // index of the word after those in cur
    uint32_t raw1, raw2;   // words next and next + 1, as loaded

    __device__ __forceinline__ static uint32_t be32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }
    __device__ __forceinline__ void init(const uint8_t *base, uint64_t pos, uint64_t end) {
        w = reinterpret_cast<const uint32_t *>(base);
        const uint64_t i = pos >> 5;
        const uint32_t skip = (uint32_t)(pos & 31);
        cur = (((uint64_t)be32(__ldg(w + i)) << 32) | be32(__ldg(w + i + 1))) << skip;
        avail = 64u - skip;
        next = i + 2;
        raw1 = __ldg(w + next);
        raw2 = __ldg(w + next + 1);
        left = (uint32_t)(end - pos);
    }
    __device__ __forceinline__ uint32_t top() const { return (uint32_t)(cur >> 32); }
    __device__ __forceinline__ void consume(uint32_t len) {
        cur <<= len;
        avail -= len;
        left -= len;
        if (avail < 32u) {
            cur |= (uint64_t)be32(raw1) << (32u - avail);
            avail += 32u;
            raw1 = raw2;
            raw2 = __ldg(w + ++next + 1);
        }
    }
};

// The codeword of codebook `cb` at the top of `t` (32 bits, all data), as
// read_sym's general path reads it, when it is no longer than 32 bits and
// its symbol is in range; false otherwise (read_sym then reads it, and
// names any failure).
__device__ __forceinline__ bool window_code(uint32_t t, Codebook cb, uint32_t &sym, uint32_t &len) {
    const uint32_t lz = __clz(t);
    if (!cb.eg && lz <= cb.q) {
        len = lz + 1u + cb.r;
        sym = (lz << cb.r) | (cb.r ? (t << (lz + 1u)) >> (32u - cb.r) : 0u);
        return true;
    }
    const uint32_t qe = cb.eg ? lz : lz - (cb.q + 1u);
    const uint32_t ke = cb.eg ? cb.r : cb.e;
    const uint32_t need = qe + ke + 1u;
    if (lz + need > 32u) return false;
    len = lz + need;
    const uint64_t n = (uint64_t)((t << lz) >> (32u - need)) - (1ull << ke) +
                       (cb.eg ? 0ull : (uint64_t)(cb.q + 1u) << cb.r);
    if (n > kMaxSymbol) return false;
    sym = (uint32_t)n;
    return true;
}

// scanned_coefficients() of one component (src/decode.rs:484-540): every
// coefficient the codes give, in scanned-index order, handed to `out.put`
// (position, value); the positions not handed over are zero. `run_tab` and
// `level_tab` are the packed prefix tables of build_book_tables (a row per
// distinct codebook). While 32 or more bits remain, codes are read from the
// window: a run, level and sign whose codewords are both in the tables in
// one go, any other codeword of up to 32 bits by window_code, a symbol at a
// time (all the bits they take are data, so they come out as the general
// reader would read them). A longer codeword and the last bits of the data
// go through the general reader, which also names every failure as the
// crate does.
// The DC part of decode_scanned() (src/decode.rs:486-498): the first
// DC by EG5, each next one as a difference by Table 9 on the previous
// difference, the sign flipped after a negative one.
template <class Out>
__device__ int decode_dc(Bits &b, uint32_t n_blocks, Out &out, Window &win, bool &in_win) {
    // Each code from the window while 32 or more bits remain (all of them
    // data, so a codeword of up to 32 bits reads as the general reader
    // would); otherwise, or for a longer one, the general reader, which
    // names any failure. The window is left at the first AC code.
    in_win = b.remaining() >= 32;
    if (in_win) win.init(reinterpret_cast<const uint8_t *>(b.w), b.pos, b.end);
    int32_t prev_dc = 0, prev_diff = 3;
    for (uint32_t i = 0; i < n_blocks; i++) {
        const Codebook cb = i == 0 ? kFirstDcBook : dc_book(prev_diff);
        uint32_t sym, len;
        if (in_win && win.left >= 32u && window_code(win.top(), cb, sym, len)) {
            win.consume(len);
        } else {
            if (in_win) b.pos = b.end - win.left;
            const int err = read_sym(b, cb, sym);
            if (err) return err;
            in_win = b.remaining() >= 32;
            if (in_win) win.init(reinterpret_cast<const uint8_t *>(b.w), b.pos, b.end);
        }
        if (i == 0) {
            prev_dc = symbol_to_signed(sym);
            out.put(0, prev_dc);
            continue;
        }
        int32_t n = symbol_to_signed(sym);
        int32_t diff = prev_diff < 0 ? -n : n;
        int64_t s = (int64_t)prev_dc + diff;
        if (s > INT32_MAX || s < INT32_MIN) return DE_DC_OVERFLOW;
        prev_dc = (int32_t)s;
        out.put(i, prev_dc);
        prev_diff = diff;
    }
    if (in_win) b.pos = b.end - win.left;
    return DE_OK;
}

template <class Out>
__device__ int decode_component(Bits &b, uint32_t n_blocks, Out &out, const uint16_t *run_tab,
                                const uint16_t *level_tab) {
    Window win;
    bool in_win;
    int err = decode_dc(b, n_blocks, out, win, in_win);
    if (err) return err;
    const uint32_t total = n_blocks * 64;
    uint32_t n = n_blocks, prev_run = 4, prev_level = 1;
    // One run, level and sign an iteration: from the window while it holds
    // the read position and 32 or more bits remain, else by the general
    // reader (which then hands the position back to a fresh window). A lane
    // that takes the general reader leaves the others only for that one
    // iteration.
    uint32_t rrow = run_book_row(prev_run) * kBookEntries, lrow = level_book_row(prev_level) * kBookEntries;
    for (;;) {
        bool level_next = false;  // the run is read; its level and sign are the general reader's
        if (in_win && win.left >= 32u) {
            const uint32_t t = win.top();
            const uint32_t e1 = run_tab[rrow + (t >> (32 - kBookBits))];
            uint32_t run = 0, l = 0;
            bool got = true;
            if (e1) {
                l = e1 & 15u;
                run = (e1 >> 4) & 63u;
                const uint32_t t2 = t << l;
                const uint32_t e2 = level_tab[lrow + (t2 >> (32 - kBookBits))];
                if (e2) {
                    // Run, level and sign in one go.
                    const uint32_t l2 = e2 & 15u;
                    prev_run = run;
                    prev_level = (e2 >> 4) & 63u;
                    n += run;
                    if (n >= total) return DE_RUN_PAST_END;
                    const int32_t level = (int32_t)prev_level + 1;
                    out.put(n, (t2 << l2) >> 31 ? -level : level);
                    n += 1;
                    rrow = (e1 >> 10) * kBookEntries;
                    lrow = (e2 >> 10) * kBookEntries;
                    win.consume(l + l2 + 1u);
                    continue;
                }
            } else {
                got = window_code(t, run_book(prev_run), run, l);
            }
            if (got) {
                prev_run = run;
                n += run;
                if (n >= total) return DE_RUN_PAST_END;
                win.consume(l);
                uint32_t lvl = 0;
                got = false;
                if (win.left >= 32u) {
                    const uint32_t u = win.top();
                    const uint32_t e2 = level_tab[lrow + (u >> (32 - kBookBits))];
                    if (e2) {
                        lvl = (e2 >> 4) & 63u;
                        l = e2 & 15u;
                        got = true;
                    } else {
                        got = window_code(u, level_book(prev_level), lvl, l);
                    }
                }
                if (got) {
                    win.consume(l);
                    prev_level = lvl;
                    if (win.left == 0) return DE_PAST_END;
                    const bool neg = win.top() >> 31;
                    win.consume(1u);
                    const int32_t level = (int32_t)lvl + 1;
                    out.put(n, neg ? -level : level);
                    n += 1;
                    rrow = run_book_row(prev_run) * kBookEntries;
                    lrow = level_book_row(prev_level) * kBookEntries;
                    continue;
                }
                level_next = true;
            }
        }
        // The general reader, from the window's position.
        if (in_win) b.pos = b.end - win.left;
        if (!level_next) {
            if (b.remaining() <= 31 && b.peek() == 0) break;  // endOfData()
            uint32_t run;
            if ((err = read_sym(b, run_book(prev_run), run))) return err;
            prev_run = run;
            n += run;
            if (n >= total) return DE_RUN_PAST_END;
        }
        uint32_t lvl;
        if ((err = read_sym(b, level_book(prev_level), lvl))) return err;
        prev_level = lvl;
        if (b.remaining() < 1) return DE_PAST_END;
        const bool neg = b.peek() >> 63;
        b.pos += 1;
        const int32_t level = (int32_t)lvl + 1;
        out.put(n, neg ? -level : level);
        n += 1;
        rrow = run_book_row(prev_run) * kBookEntries;
        lrow = level_book_row(prev_level) * kBookEntries;
        in_win = b.remaining() >= 32;
        if (in_win) win.init(reinterpret_cast<const uint8_t *>(b.w), b.pos, b.end);
    }
    return DE_OK;
}

__device__ __forceinline__ uint16_t rescale(uint32_t a, uint64_t m, bool identity) {
    return identity ? (uint16_t)a : (uint16_t)(((uint64_t)a * m + (1ull << 39)) >> 40);
}

// scanned_alpha() (src/decode.rs:570-595) and its placement (:365-389).
__device__ int decode_alpha(Bits &b, const FrameDesc &fd, const PicDesc &pd, const SliceDesc &sd, uint16_t *alpha) {
    const uint32_t bits = fd.alpha_bits;
    const uint32_t cols = 16u * sd.mbs;
    const uint32_t count = cols * 16u;
    const uint32_t rows = (uint32_t)sd.mb_y + 1u < pd.height_in_mb ? 16u : pd.height - 16u * (pd.height_in_mb - 1u);
    const uint32_t needed = cols * rows;
    const uint32_t width = fd.width;
    const uint32_t x0 = 16u * sd.mb_x;
    const uint32_t ncols = min(cols, width - x0);
    const int32_t mask = (int32_t)((1u << bits) - 1u);
    const uint32_t mag_bits = bits == 8 ? 3u : 6u;
    uint16_t *plane = fd.out_alpha ? fd.out_alpha : alpha + fd.alpha_off;
    const uint32_t cshift = (uint32_t)__ffs(cols) - 1u;  // cols is 16 times a power of two
    int32_t prev = -1;
    uint32_t n = 0;
    int err;
    while (n < count) {
        if (n >= needed && b.end_of_data()) break;
        uint64_t v;
        int32_t diff;
        uint32_t run;
        if (b.remaining() >= 64) {
            // A difference and a run take at most 34 bits: both from one
            // look at the next 64, all of them data.
            const uint64_t w = b.peek();
            uint32_t used;
            if (w >> 63) {
                diff = (int32_t)((w << 1) >> (64u - bits));
                used = 1u + bits;
            } else {
                const int32_t a = (int32_t)((w << 1) >> (64u - mag_bits)) + 1;
                diff = ((w << (1u + mag_bits)) >> 63) ? -a : a;
                used = 2u + mag_bits;
            }
            const uint64_t u = w << used;
            if (u >> 63) {
                run = 1;
                used += 1u;
            } else {
                const uint32_t r4 = (uint32_t)((u << 1) >> 60);
                if (r4) {
                    run = r4 + 1u;
                    used += 5u;
                } else {
                    run = (uint32_t)((u << 5) >> 53) + 1u;
                    used += 16u;
                }
            }
            b.pos += used;
        } else {
            if ((err = b.read(1, v))) return err;
            if (v == 1) {
                if ((err = b.read(bits, v))) return err;
                diff = (int32_t)v;
            } else {
                if ((err = b.read(mag_bits, v))) return err;
                int32_t a = (int32_t)v + 1;
                if ((err = b.read(1, v))) return err;
                diff = v ? -a : a;
            }
            if ((err = b.read(1, v))) return err;
            if (v == 1) {
                run = 1;
            } else {
                if ((err = b.read(4, v))) return err;
                if (v != 0) {
                    run = (uint32_t)v + 1;
                } else {
                    if ((err = b.read(11, v))) return err;
                    run = (uint32_t)v + 1;
                }
            }
        }
        int32_t value = (int32_t)((uint32_t)prev + (uint32_t)diff) & mask;
        prev = value;
        if (n + run > count) return DE_ALPHA_RUN;
        uint16_t out = rescale((uint32_t)value, fd.rescale_m, fd.rescale_identity != 0);
        uint32_t stop = min(n + run, needed);
        for (uint32_t i = n; i < stop;) {
            uint32_t r = i >> cshift, c = i & (cols - 1u);
            uint32_t seg_end = min(stop - i, cols - c);  // samples left in this row of the run
            uint16_t *row = plane + (uint64_t)(pd.first_row + pd.row_step * (16u * sd.mb_y + r)) * width + x0;
            for (uint32_t k = c; k < c + seg_end && k < ncols; k++) row[k] = out;
            i += seg_end;
        }
        n += run;
    }
    return DE_OK;
}

// The slice header (src/decode.rs:301-338) and where component `comp` (0
// Y', 1 Cb, 2 Cr, 3 alpha) lies in the slice. A header failure comes back
// (the Y' item reports it; the other components then report nothing).
__device__ int2 component_range(const uint8_t *sb, uint32_t size, bool has_alpha, uint32_t comp, uint32_t &start,
                                uint32_t &len) {
    const uint32_t min_header = has_alpha ? 8u : 6u;
    uint32_t hs = 0, ys = 0, cbs = 0, crs = 0;
    if (size < min_header) return make_int2(DE_SLICE_SHORT, 0);
    hs = sb[0] >> 3;
    const uint32_t qi = sb[1];
    if (hs < min_header || hs > size) return make_int2(DE_SLICE_HDR_SIZE, (int)hs);
    if (qi < 1 || qi > 224) return make_int2(DE_QINDEX, (int)qi);
    ys = be16(sb + 2);
    cbs = be16(sb + 4);
    const uint32_t body = size - hs;
    if (has_alpha) {
        crs = be16(sb + 6);
    } else {
        if (ys + cbs > body) return make_int2(DE_COMP_SIZES, 0);
        crs = body - ys - cbs;
    }
    if (ys + cbs + crs > body) return make_int2(DE_COMP_SIZES, 0);
    start = hs;
    if (comp == 0) {
        len = ys;
    } else if (comp == 1) {
        start += ys;
        len = cbs;
    } else if (comp == 2) {
        start += ys + cbs;
        len = crs;
    } else {
        start += ys + cbs + crs;
        len = size - start;
    }
    return make_int2(DE_OK, 0);
}

// One work item: component `comp` (0 Y', 1 Cb, 2 Cr, 3 alpha) of slice `s`.
__device__ void decode_item(const DecodeLaunch &d, uint32_t comp, uint32_t s, const uint16_t *run_tab,
                            const uint16_t *level_tab) {
    int2 *slot = d.slot_status + 4ull * s + comp;
    const SliceDesc sd = d.slices[s];
    const PicDesc &pd = d.pics[sd.pic];
    if (d.pic_status[sd.pic].locate_slice >= 0) return;  // never read: the picture failed before decoding
    // Every run writes every count of the slices it decodes (a failing
    // component's too), so k_idct never reads a stale one.
    if (comp < 3) d.coef_count[3ull * s + comp] = 0;
    const FrameDesc &fd = d.frames[pd.frame];
    const bool has_alpha = fd.alpha_bits != 0;
    if (comp == 3 && !has_alpha) {
        *slot = make_int2(DE_OK, 0);
        return;
    }
    uint32_t start = 0, len = 0;
    const int2 hdr_err = component_range(d.bits + sd.off, sd.size, has_alpha, comp, start, len);
    if (hdr_err.x != DE_OK) {
        *slot = comp == 0 ? hdr_err : make_int2(DE_OK, 0);
        return;
    }
    Bits b;
    b.init(d.bits, sd.off + start, len);
    int err;
    if (comp == 3) {
        err = decode_alpha(b, fd, pd, sd, d.alpha);
    } else {
        const uint32_t cpm = fd.chroma == 2 ? 2u : 4u;
        const uint32_t n_blocks = (comp == 0 ? 4u : cpm) * sd.mbs;
        const uint64_t base = sd.coef + (comp == 0 ? 0ull : 64ull * sd.mbs * (4u + (comp - 1u) * cpm));
        CoefList list{reinterpret_cast<uint32_t *>(d.coef + base), 64u * n_blocks, 0u, 0u};
        err = decode_component(b, n_blocks, list, run_tab, level_tab);
        d.coef_count[3ull * s + comp] = list.count;
    }
    *slot = make_int2(err, 0);
}

// ------------------------------------------------------------------ kernels

constexpr int kLocateThreads = 1024;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__global__ void __launch_bounds__(kLocateThreads) k_locate(DecodeLaunch d) {
    __shared__ uint32_t warp_sums[kLocateThreads / 32];
    __shared__ uint64_t carry;
    __shared__ int first_bad;
    const PicDesc p = d.pics[blockIdx.x];
    const FrameDesc &fd = d.frames[p.frame];
    const uint32_t cpm = fd.chroma == 2 ? 2u : 4u;
    const uint32_t coef_per_mb = 64u * (4u + 2u * cpm);
    const uint32_t S = 1u << p.log2_slice_mbs;
    const uint32_t full = p.width_in_mb >> p.log2_slice_mbs;
    const uint32_t rem_mbs = p.width_in_mb & (S - 1u);
    const uint8_t *table = d.bits + p.off + p.header_size;
    const uint64_t data_start = p.off + p.header_size + 2ull * p.n_slices;
    const uint64_t limit = p.off + p.picture_size;
    if (threadIdx.x == 0) {
        carry = 0;
        first_bad = INT32_MAX;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t chunk = 0; chunk < p.n_slices; chunk += kLocateThreads) {
        const uint32_t k = chunk + threadIdx.x;
        const uint32_t size = k < p.n_slices ? be16(table + 2ull * k) : 0u;
        uint32_t incl = warp_incl_scan(size);
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t ws = warp_sums[lane];
            warp_sums[lane] = warp_incl_scan(ws);
        }
        __syncthreads();
        const uint64_t excl = carry + (warp ? warp_sums[warp - 1] : 0u) + incl - size;
        if (k < p.n_slices) {
            const uint64_t off = data_start + excl;
            if (off + size > limit) atomicMin(&first_bad, (int)k);
            const uint32_t row = k / p.slices_per_row, j = k - row * p.slices_per_row;
            uint32_t mb_x, mbs;
            if (j < full) {
                mb_x = j * S;
                mbs = S;
            } else {
                // The slices after the full ones halve down the binary digits
                // of what is left (src/header.rs:308-320).
                uint32_t idx = j - full;
                mb_x = full * S;
                mbs = 1;
                for (int bit = (int)p.log2_slice_mbs - 1; bit >= 0; bit--) {
                    if (!(rem_mbs & (1u << bit))) continue;
                    if (idx == 0) {
                        mbs = 1u << bit;
                        break;
                    }
                    mb_x += 1u << bit;
                    idx--;
                }
            }
            SliceDesc sd;
            sd.off = off;
            sd.size = size;
            sd.pic = blockIdx.x;
            sd.mb_x = (uint16_t)mb_x;
            sd.mb_y = (uint16_t)row;
            sd.mbs = mbs;
            sd.coef = p.coef_base + ((uint64_t)row * p.width_in_mb + mb_x) * coef_per_mb;
            d.slices[p.slice_base + k] = sd;
        }
        __syncthreads();
        if (threadIdx.x == kLocateThreads - 1) carry += (warp ? warp_sums[warp - 1] : 0u) + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        PicStatus st;
        st.locate_slice = first_bad == INT32_MAX ? -1 : first_bad;
        st.slot = -1;
        st.code = 0;
        st.aux = 0;
        d.pic_status[blockIdx.x] = st;
    }
}

constexpr int kEntropyMaxThreads = 512;

// Persistent: each warp takes 32 x entropy_per_lane slice components per
// grab of the work counter, a lane each in turn, component-major, until the
// list runs out. The alpha components come first: where a frame has alpha,
// its run/difference codes take a lane several times as long as a colour
// component, and started last they would leave the launch waiting on them.
__global__ void __launch_bounds__(kEntropyMaxThreads) k_entropy(DecodeLaunch d) {
    __shared__ uint16_t run_tab[kBookTableWords];
    __shared__ uint16_t level_tab[kBookTableWords];
    for (uint32_t i = threadIdx.x; i < kBookTableWords / 2; i += blockDim.x) {
        reinterpret_cast<uint32_t *>(run_tab)[i] = reinterpret_cast<const uint32_t *>(d.tables.run_books)[i];
        reinterpret_cast<uint32_t *>(level_tab)[i] = reinterpret_cast<const uint32_t *>(d.tables.level_books)[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t items = 4u * d.n_slices;
    const uint32_t per_lane = d.entropy_per_lane > 0 ? d.entropy_per_lane : 1u;
    const uint32_t grab = 32u * per_lane;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(d.work_counter, grab);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= items) break;
        for (uint32_t k = 0; k < per_lane; k++) {
            const uint32_t item = base + 32u * k + lane;
            if (item < items) {
                const uint32_t kind = item / d.n_slices, s = item - kind * d.n_slices;
                decode_item(d, kind == 0 ? 3u : kind - 1u, s, run_tab, level_tab);
            }
        }
        __syncwarp();
    }
}

constexpr int kIdctThreads = 256;
constexpr int kMaxSliceCoefs = 64 * 12 * 8;  // 8 macroblocks of 4:4:4

// Placement of block b of macroblock m (src/decode.rs:395-413).
__device__ __forceinline__ void block_xy(uint32_t comp, uint32_t chroma, uint32_t mb_x, uint32_t mb_y, uint32_t m,
                                         uint32_t b, uint32_t &bx, uint32_t &by) {
    const uint32_t x = mb_x + m, y0 = 16u * mb_y;
    if (comp == 0) {
        bx = 16u * x + 8u * (b & 1u);
        by = y0 + 8u * (b >> 1);
    } else if (chroma == 2) {
        bx = 8u * x;
        by = y0 + 8u * b;
    } else {
        bx = 16u * x + 8u * (b >> 1);
        by = y0 + 8u * (b & 1u);
    }
}

__global__ void __launch_bounds__(kIdctThreads, 5) k_idct(DecodeLaunch d) {
    extern __shared__ __align__(16) unsigned char smem[];
    int32_t *cs = reinterpret_cast<int32_t *>(smem);                   // scanned coefficients
    float *tmp = reinterpret_cast<float *>(smem);  // row pass, over cs: [v][x][blk] per component
    uint8_t *nz = smem + 4 * kMaxSliceCoefs;       // non-zero rows, [blk][v]
    __shared__ float scale[2][64];
    __shared__ uint8_t scan[64];

    const SliceDesc sd = d.slices[blockIdx.x];
    const PicDesc &pd = d.pics[sd.pic];
    if (d.pic_status[sd.pic].locate_slice >= 0) return;
    const FrameDesc &fd = d.frames[pd.frame];
    const uint32_t cpm = fd.chroma == 2 ? 2u : 4u;
    const uint32_t mbs = sd.mbs;
    const uint32_t total = 64u * (4u + 2u * cpm) * mbs;
    const uint32_t tid = threadIdx.x;

    // The slice's coefficients: zero the block array, then place each
    // component's (position, value) entries.
    int4 *s4 = reinterpret_cast<int4 *>(cs);
    for (uint32_t i = tid; i < total / 4; i += kIdctThreads) s4[i] = make_int4(0, 0, 0, 0);
    __syncthreads();
    for (uint32_t c = 0; c < 3; c++) {
        const uint32_t cap = 64u * (c == 0 ? 4u : cpm) * mbs;
        const uint32_t start = c == 0 ? 0u : 64u * mbs * (4u + (c - 1u) * cpm);
        const uint32_t n = min(d.coef_count[3ull * blockIdx.x + c], cap);
        const uint32_t *list = reinterpret_cast<const uint32_t *>(d.coef + sd.coef + start);
        for (uint32_t i = tid; i < n; i += kIdctThreads) {
            uint32_t pos;
            int32_t v;
            list_entry(list, cap, __ldg(list + i), pos, v);
            if (pos < cap) cs[start + pos] = v;
        }
    }
    uint32_t qi = sd.size >= 2 ? d.bits[sd.off + 1] : 1u;
    qi = qi < 1u ? 1u : (qi > 224u ? 224u : qi);
    const uint32_t q = qscale(qi);
    if (tid < 128) {
        const uint32_t which = tid >> 6, k = tid & 63;
        // F = QF * (W * qScale / 8), one factor per raster position (src/decode.rs:356).
        scale[which][k] = (float)((uint32_t)d.weights[fd.weights * 128u + which * 64u + k] * q) / 8.0f;
    } else if (tid < 192) {
        scan[tid - 128] = c_scan[pd.interlaced_scan][tid - 128];
    }
    __syncthreads();

    // Row pass: tmp[v][x] = sum_u F[v][u] T[x][u], u in order, from 0
    // (src/dct.rs:38-53); all-zero rows are skipped, as the crate does.
    // Blocks of a component and its first coefficient in the slice (by
    // select, not an indexed array, which would live in local memory).
    const uint32_t luma_blocks = 4u * mbs, chroma_blocks = cpm * mbs;
    // Block counts are powers of two: task indices split by shifts, not by
    // divisions (which run on the conversion pipe this kernel is short of).
    const uint32_t luma_shift = 31u - __clz(luma_blocks), chroma_shift = 31u - __clz(chroma_blocks);
    const auto blocks_of = [&](uint32_t c) { return c == 0 ? luma_blocks : chroma_blocks; };
    const auto shift_of = [&](uint32_t c) { return c == 0 ? luma_shift : chroma_shift; };
    const auto start_of = [&](uint32_t c) { return c == 0 ? 0u : 64u * (luma_blocks + (c - 1u) * chroma_blocks); };
    const uint32_t all_blocks = luma_blocks + 2u * chroma_blocks;
    // The row results are held in registers until every thread has read
    // its coefficients, then written over them (the two arrays share the
    // shared memory, so that five CTAs fit on an SM).
    constexpr int kRowsPerThread = (kMaxSliceCoefs / 8 + kIdctThreads - 1) / kIdctThreads;
    float held[kRowsPerThread][8];
    bool held_any[kRowsPerThread];
#pragma unroll
    for (int k = 0; k < kRowsPerThread; k++) {
        const uint32_t t = tid + (uint32_t)k * kIdctThreads;
        held_any[k] = false;
        if (t >= all_blocks * 8u) continue;
        const uint32_t c = t < luma_blocks * 8u ? 0u : (t < (luma_blocks + chroma_blocks) * 8u ? 1u : 2u);
        const uint32_t tc = t - start_of(c) / 8u;  // 8 row tasks a block
        const uint32_t nb = blocks_of(c);
        const uint32_t blk = tc & (nb - 1u), v = tc >> shift_of(c);
        const int32_t *src = cs + start_of(c);
        const float *sc = scale[c > 0];
        float row[8];
        bool any = false;
        int32_t q[8];
        bool wide = false;
#pragma unroll
        for (int u = 0; u < 8; u++) {
            q[u] = src[nb * scan[8u * v + u] + blk];
            wide |= (uint32_t)(q[u] + (1 << 22)) >= (1u << 23);
        }
        // Values below 2^22 in magnitude convert exactly by an add (no
        // conversion instruction); a wider one, rare, takes the conversion.
        if (!wide) {
#pragma unroll
            for (int u = 0; u < 8; u++) row[u] = __fmul_rn(small_int_to_float(q[u]), sc[8u * v + u]);
        } else {
#pragma unroll
            for (int u = 0; u < 8; u++) row[u] = __fmul_rn(__int2float_rn(q[u]), sc[8u * v + u]);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) any |= row[u] != 0.0f;
        held_any[k] = any;
        if (any) {
            // Outputs x = 2 j, 2 j + 1 summed as a pair, each in the same
            // order; the products stay scalar (see pair_math.h).
#pragma unroll
            for (int j = 0; j < 4; j++) {
                uint64_t acc = 0;
#pragma unroll
                for (int u = 0; u < 8; u++)
                    acc = pair_add(acc, pair_of(__fmul_rn(row[u], c_idct_basis[8 * (2 * j) + u]),
                                                __fmul_rn(row[u], c_idct_basis[8 * (2 * j + 1) + u])));
                pair_split(acc, held[k][2 * j], held[k][2 * j + 1]);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kRowsPerThread; k++) {
        const uint32_t t = tid + (uint32_t)k * kIdctThreads;
        if (t >= all_blocks * 8u) continue;
        const uint32_t c = t < luma_blocks * 8u ? 0u : (t < (luma_blocks + chroma_blocks) * 8u ? 1u : 2u);
        const uint32_t tc = t - start_of(c) / 8u;  // 8 row tasks a block
        const uint32_t nb = blocks_of(c);
        const uint32_t blk = tc & (nb - 1u), v = tc >> shift_of(c);
        nz[(start_of(c) / 64u + blk) * 8u + v] = held_any[k];
        if (held_any[k]) {
            float *dst = tmp + start_of(c);
#pragma unroll
            for (int x = 0; x < 8; x++) dst[(v * 8u + x) * nb + blk] = held[k][x];
        }
    }
    __syncthreads();

    // Column pass and conversion: out[y][x] = sum_v T[y][v] tmp[v][x] in
    // order (src/dct.rs:54-64), then floor(v scale + bias) clamped
    // (src/dsp/scalar.rs:8-12). A task is two neighbouring columns of one
    // block, so each row result is read once; neighbouring threads take
    // neighbouring blocks (no bank conflicts). The samples go to shared
    // memory as pairs, [y][column pair][blk] per component.
    const float oscale = fd.out_scale, obias = fd.out_bias, omax = fd.out_max;
    uint32_t *stage = reinterpret_cast<uint32_t *>(smem + 4 * kMaxSliceCoefs + kMaxSliceCoefs / 8);
    // floor(v) clamped to [0, max] of the converted value v = a scale + bias.
    const auto convert = [&](float v) { return floor_clamped(v, omax); };
    for (uint32_t t = tid; t < all_blocks * 4u; t += kIdctThreads) {
        const uint32_t c = t < luma_blocks * 4u ? 0u : (t < (luma_blocks + chroma_blocks) * 4u ? 1u : 2u);
        const uint32_t tc = t - start_of(c) / 16u;  // 4 column tasks a block
        const uint32_t nb = blocks_of(c);
        const uint32_t blk = tc & (nb - 1u), j = tc >> shift_of(c);
        const float *src = tmp + start_of(c) + 2u * j * nb + blk;
        const uint64_t rows = *reinterpret_cast<const uint64_t *>(nz + (start_of(c) / 64u + blk) * 8u);
        // Outputs y = 2 i, 2 i + 1 of each column a pair.
        uint64_t a0[4], a1[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a0[i] = a1[i] = 0;
#pragma unroll
        for (int v = 0; v < 8; v++) {
            if (!((rows >> (8 * v)) & 0xffu)) continue;
            const float t0 = src[8u * v * nb], t1 = src[8u * v * nb + nb];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float w0 = c_idct_basis[8 * (2 * i) + v], w1 = c_idct_basis[8 * (2 * i + 1) + v];
                a0[i] = pair_add(a0[i], pair_of(__fmul_rn(w0, t0), __fmul_rn(w1, t0)));
                a1[i] = pair_add(a1[i], pair_of(__fmul_rn(w0, t1), __fmul_rn(w1, t1)));
            }
        }
        const uint64_t ob2 = pair_of(obias, obias);
        const auto scaled = [&](uint64_t a) {
            float lo, hi;
            pair_split(a, lo, hi);
            return pair_add(pair_of(__fmul_rn(lo, oscale), __fmul_rn(hi, oscale)), ob2);
        };
        uint32_t *dst = stage + start_of(c) / 2u + j * nb + blk;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float p0, p1, q0, q1;
            pair_split(scaled(a0[i]), p0, p1);
            pair_split(scaled(a1[i]), q0, q1);
            dst[4u * (2 * i) * nb] = convert(p0) | (convert(q0) << 16);
            dst[4u * (2 * i + 1) * nb] = convert(p1) | (convert(q1) << 16);
        }
    }
    __syncthreads();

    // Stores: a thread writes one 8-sample row of a block; neighbouring
    // threads write neighbouring row segments of the picture.
    for (uint32_t c = 0; c < 3; c++) {
        const uint32_t segs = (c == 0 || cpm == 4) ? 2u * mbs : mbs;
        const uint32_t per_mb = c == 0 ? 4u : cpm;
        const uint32_t nb = blocks_of(c);
        const uint32_t pw = fd.plane_w[c];
        uint16_t *plane = fd.out_planes ? fd.out_planes + (fd.plane_off[c] - fd.plane_off[0]) : d.planes + fd.plane_off[c];
        for (uint32_t t = tid; t < 16u * segs; t += kIdctThreads) {
            const uint32_t r = t >> (31u - __clz(segs)), sx = t & (segs - 1u);
            uint32_t m, bb;
            if (c == 0) {
                m = sx >> 1;
                bb = ((r >> 3) << 1) | (sx & 1u);
            } else if (cpm == 2) {
                m = sx;
                bb = r >> 3;
            } else {
                m = sx >> 1;
                bb = ((sx & 1u) << 1) | (r >> 3);
            }
            const uint32_t blk = m * per_mb + bb, y = r & 7u;
            uint32_t bx, by;
            block_xy(c, fd.chroma, sd.mb_x, sd.mb_y, m, bb, bx, by);
            if (bx >= pw || by + y >= pd.height) continue;
            const uint32_t *src = stage + start_of(c) / 2u + 4u * y * nb + blk;
            uint4 v;
            v.x = src[0];
            v.y = src[nb];
            v.z = src[2u * nb];
            v.w = src[3u * nb];
            const uint32_t cols = min(8u, pw - bx);
            uint16_t *dst = plane + (uint64_t)(pd.first_row + pd.row_step * (by + y)) * pw + bx;
            if (cols == 8u && ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0)) {
                *reinterpret_cast<uint4 *>(dst) = v;
            } else {
                for (uint32_t x = 0; x < cols; x++) {
                    const uint32_t w = x < 2u ? v.x : (x < 4u ? v.y : (x < 6u ? v.z : v.w));
                    dst[x] = (uint16_t)(w >> (16u * (x & 1u)));
                }
            }
        }
    }
}

// ------------------------------------------------------------ fused decode
//
// k_decode: the whole per-slice chain in one kernel (src/decode.rs:292-391).
// A CTA takes a group of consecutive slices of the flat list at a time
// (grabbed from a work counter) and
//   1. zeroes the group's coefficient slots in shared memory (one int16 per
//      scanned position of every component) and sets the slices up: where
//      their positions and blocks start, their dequantisation factors;
//   2. decodes every component of the group, one thread each (Y' of every
//      slice, then Cb, Cr, alpha), straight into the slots; alpha goes to
//      its plane as it is decoded;
//   3. transforms every block of the group, one thread each, in registers:
//      dequantise, the 8x8 IDCT in the crate's single-precision order,
//      conversion, and 16-byte row stores into the woven planes.
// No coefficient leaves the chip; the bitstream is read once and the planes
// written once.

constexpr int kDecodeThreads = 128;
constexpr uint32_t kMaxGroup = 32;  // slices a CTA decodes at once (4 items each <= 128 threads)

// Figures 4 and 5, folded into immediates in the unrolled transform:
// scan_at<IL>(8 v + u) is the scanned index of row v, column u.
struct ScanPair {
    uint8_t v[2][64];
};
__device__ constexpr ScanPair scan_pair() {
    ScanPair s{};
    for (int i = 0; i < 64; i++) {
        s.v[0][i] = kProgressiveScan[i];
        s.v[1][i] = kInterlacedScan[i];
    }
    return s;
}
template <int IL>
__device__ __forceinline__ constexpr uint32_t scan_at(int i) {
    constexpr ScanPair s = scan_pair();
    return s.v[IL][i];
}

// A slice of a CTA's group.
struct GroupSlice {
    uint32_t pos;         // its first position in the group's slots
    uint32_t blk;         // its first block in the group's list of blocks
    uint32_t nb_y, nb_c;  // blocks of Y' and of each chroma component
    uint32_t live;        // decoded at all (its picture's slices were located)
};



// One block: dequantise (F = QF scale, src/dsp/scalar.rs:8-12), the IDCT's
// row pass tmp[v][x] = sum_u F[v][u] T[x][u] and column pass
// f[y][x] = sum_v T[y][v] tmp[v][x], each sum in the crate's order
// (src/dct.rs:36-66), then floor(f s + b) clamped, stored row by row. Every
// term is computed: a zero term adds nothing to a non-zero sum and only
// flips the sign of a zero one, which the conversion cannot see, so the
// crate's skipped zero rows and its leading 0 + come out the same.
template <int IL, class T>
__device__ __forceinline__ void idct_block(const T *cs, const int32_t *wide, uint32_t nb, uint32_t blk,
                                           const float *sc, float oscale, float obias, float omax, uint16_t *row0,
                                           uint64_t row_pitch, uint32_t cols, uint32_t rows) {
    float t[64];
#pragma unroll
    for (int v = 0; v < 8; v++) {
        float f[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const uint32_t n = scan_at<IL>(8 * v + u) * nb + blk;
            const int32_t q = cs[n];
            const float fq = q == wide_mark<T>() ? __int2float_rn(wide[n]) : small_int_to_float(q);
            f[u] = __fmul_rn(fq, sc[8 * v + u]);
        }
#pragma unroll
        for (int x = 0; x < 8; x++) {
            float acc = __fmul_rn(f[0], c_idct_basis[8 * x]);
#pragma unroll
            for (int u = 1; u < 8; u++) acc = __fadd_rn(acc, __fmul_rn(f[u], c_idct_basis[8 * x + u]));
            t[8 * v + x] = acc;
        }
    }
#pragma unroll
    for (int y = 0; y < 8; y++) {
        uint32_t px[8];
#pragma unroll
        for (int x = 0; x < 8; x++) {
            float acc = __fmul_rn(c_idct_basis[8 * y], t[x]);
#pragma unroll
            for (int v = 1; v < 8; v++) acc = __fadd_rn(acc, __fmul_rn(c_idct_basis[8 * y + v], t[8 * v + x]));
            px[x] = floor_clamped(__fadd_rn(__fmul_rn(acc, oscale), obias), omax);
        }
        if ((uint32_t)y >= rows) continue;
        uint16_t *dst = row0 + (uint64_t)y * row_pitch;
        if (cols == 8u && (reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
            uint4 w;
            w.x = __byte_perm(px[0], px[1], 0x5410);
            w.y = __byte_perm(px[2], px[3], 0x5410);
            w.z = __byte_perm(px[4], px[5], 0x5410);
            w.w = __byte_perm(px[6], px[7], 0x5410);
            __stcs(reinterpret_cast<uint4 *>(dst), w);
        } else {
#pragma unroll
            for (int x = 0; x < 8; x++)
                if ((uint32_t)x < cols) dst[x] = (uint16_t)px[x];
        }
    }
}

template <class T>
__global__ void __launch_bounds__(kDecodeThreads) k_decode(DecodeLaunch d) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint16_t *run_tab = reinterpret_cast<uint16_t *>(smem);
    uint16_t *level_tab = run_tab + kBookTableWords;
    GroupSlice *gs = reinterpret_cast<GroupSlice *>(level_tab + kBookTableWords);  // kMaxGroup
    float *scale = reinterpret_cast<float *>(gs + kMaxGroup);                    // [group][luma, chroma][64]
    T *slots = reinterpret_cast<T *>(scale + 128u * d.group);                   // group_positions
    __shared__ uint32_t s_group, s_blocks;

    for (uint32_t i = threadIdx.x; i < kBookTableWords / 2; i += kDecodeThreads) {
        reinterpret_cast<uint32_t *>(run_tab)[i] = reinterpret_cast<const uint32_t *>(d.tables.run_books)[i];
        reinterpret_cast<uint32_t *>(level_tab)[i] = reinterpret_cast<const uint32_t *>(d.tables.level_books)[i];
    }
    const uint32_t n_groups = (d.n_slices + d.group - 1u) / d.group;
    int32_t *wide_all = reinterpret_cast<int32_t *>(d.coef);
    for (;;) {
        __syncthreads();  // the last group's blocks are all transformed (and the tables are in)
        if (threadIdx.x == 0) s_group = atomicAdd(d.work_counter, 1u);
        __syncthreads();
        const uint32_t g = s_group;
        if (g >= n_groups) break;
        const uint32_t first = g * d.group;
        const uint32_t count = min(d.group, d.n_slices - first);

        // 1. Zeroed slots; the slices' places in the group.
        for (uint32_t i = threadIdx.x; i < d.group_positions * sizeof(T) / 16u; i += kDecodeThreads)
            reinterpret_cast<int4 *>(slots)[i] = make_int4(0, 0, 0, 0);
        if (threadIdx.x < 32) {
            const uint32_t k = threadIdx.x;
            GroupSlice e{};
            uint32_t n_pos = 0, n_blk = 0;
            if (k < count) {
                const SliceDesc sd = d.slices[first + k];
                const uint32_t cpm = d.frames[d.pics[sd.pic].frame].chroma == 2 ? 2u : 4u;
                e.nb_y = 4u * sd.mbs;
                e.nb_c = cpm * sd.mbs;
                e.live = d.pic_status[sd.pic].locate_slice < 0;
                n_pos = 64u * (e.nb_y + 2u * e.nb_c);
                n_blk = e.live ? e.nb_y + 2u * e.nb_c : 0u;
            }
            const uint32_t ip = warp_incl_scan(n_pos), ib = warp_incl_scan(n_blk);
            e.pos = ip - n_pos;
            e.blk = ib - n_blk;
            if (k < count) gs[k] = e;
            if (k == 31) s_blocks = ib;
        }
        // F = QF W qScale / 8, one factor per raster position (src/decode.rs:356).
        for (uint32_t i = threadIdx.x; i < 128u * count; i += kDecodeThreads) {
            const uint32_t k = i >> 7, which = (i >> 6) & 1u, r = i & 63u;
            const SliceDesc sd = d.slices[first + k];
            const FrameDesc &fd = d.frames[d.pics[sd.pic].frame];
            uint32_t qi = sd.size >= 2 ? d.bits[sd.off + 1] : 1u;
            qi = qi < 1u ? 1u : (qi > 224u ? 224u : qi);
            scale[i] = (float)((uint32_t)d.weights[fd.weights * 128u + which * 64u + r] * qscale(qi)) / 8.0f;
        }
        __syncthreads();

        // 2. Entropy decoding. Thread i takes item kind i / count of slice
        // i % count: kind 0 its Y', kind 1 its Cb and then its Cr for 4:2:2
        // (together about as long as Y') or its Cb for 4:4:4, kind 2 the
        // Cr of a 4:4:4 slice, kind 3 its alpha; so the threads of a warp
        // mostly decode codes of about equal length.
        for (uint32_t i = threadIdx.x; i < 4u * count; i += kDecodeThreads) {
            const uint32_t kind = i / count, k = i - kind * count;
            const GroupSlice e = gs[k];
            if (!e.live) continue;  // never read: the picture failed before decoding
            const uint32_t s = first + k;
            const SliceDesc sd = d.slices[s];
            const PicDesc &pd = d.pics[sd.pic];
            const FrameDesc &fd = d.frames[pd.frame];
            const bool pair = fd.chroma == 2;  // 4:2:2: Cb and Cr on one thread
            uint32_t c = kind, last = kind;
            if (kind == 1 && pair) last = 2;
            if (kind == 2 && pair) continue;
            for (; c <= last; c++) {
                const bool has_alpha = fd.alpha_bits != 0;
                int2 *status = d.slot_status + 4ull * s + c;
                if (c == 3 && !has_alpha) {
                    *status = make_int2(DE_OK, 0);
                    continue;
                }
                uint32_t start = 0, len = 0;
                const int2 he = component_range(d.bits + sd.off, sd.size, has_alpha, c, start, len);
                if (he.x != DE_OK) {
                    *status = c == 0 ? he : make_int2(DE_OK, 0);
                    continue;
                }
                Bits b;
                b.init(d.bits, sd.off + start, len);
                int err;
                if (c == 3) {
                    err = decode_alpha(b, fd, pd, sd, d.alpha);
                } else {
                    const uint32_t nb = c == 0 ? e.nb_y : e.nb_c;
                    const uint32_t off = c == 0 ? 0u : 64u * (e.nb_y + (c - 1u) * e.nb_c);
                    SlotOut<T> out{slots + e.pos + off, wide_all + sd.coef + off};
                    err = decode_component(b, nb, out, run_tab, level_tab);
                }
                *status = make_int2(err, 0);
            }
        }
        __syncthreads();

        // 3. Every block: transform, convert, store.
        const uint32_t n_blocks = s_blocks;
        for (uint32_t bi = threadIdx.x; bi < n_blocks; bi += kDecodeThreads) {
            uint32_t k = 0;
            while (k + 1u < count && gs[k + 1u].blk <= bi) k++;
            const GroupSlice e = gs[k];
            const SliceDesc sd = d.slices[first + k];
            const PicDesc &pd = d.pics[sd.pic];
            const FrameDesc &fd = d.frames[pd.frame];
            uint32_t local = bi - e.blk, c = 0, nb = e.nb_y, off = 0;
            if (local >= e.nb_y) {
                local -= e.nb_y;
                c = local < e.nb_c ? 1u : 2u;
                local -= (c - 1u) * e.nb_c;
                nb = e.nb_c;
                off = 64u * (e.nb_y + (c - 1u) * e.nb_c);
            }
            const uint32_t per_mb = c == 0 ? 4u : (fd.chroma == 2 ? 2u : 4u);
            const uint32_t m = local / per_mb, bb = local - m * per_mb;
            uint32_t bx, by;
            block_xy(c, fd.chroma, sd.mb_x, sd.mb_y, m, bb, bx, by);
            const uint32_t pw = fd.plane_w[c];
            if (bx >= pw || by >= pd.height) continue;  // wholly outside the picture
            uint16_t *plane =
                fd.out_planes ? fd.out_planes + (fd.plane_off[c] - fd.plane_off[0]) : d.planes + fd.plane_off[c];
            uint16_t *row0 = plane + (uint64_t)(pd.first_row + pd.row_step * by) * pw + bx;
            const uint64_t pitch = (uint64_t)pd.row_step * pw;
            const float *sc = scale + (2u * k + (c > 0 ? 1u : 0u)) * 64u;
            const T *cs = slots + e.pos + off;
            const int32_t *wide = wide_all + sd.coef + off;
            const uint32_t cols = min(8u, pw - bx), rows = min(8u, pd.height - by);
            if (pd.interlaced_scan)
                idct_block<1>(cs, wide, nb, local, sc, fd.out_scale, fd.out_bias, fd.out_max, row0, pitch, cols, rows);
            else
                idct_block<0>(cs, wide, nb, local, sc, fd.out_scale, fd.out_bias, fd.out_max, row0, pitch, cols, rows);
        }
    }
}

constexpr int kStatusThreads = 256;

__global__ void __launch_bounds__(kStatusThreads) k_status(DecodeLaunch d) {
    __shared__ int best;
    const PicDesc p = d.pics[blockIdx.x];
    if (threadIdx.x == 0) best = INT32_MAX;
    __syncthreads();
    if (d.pic_status[blockIdx.x].locate_slice < 0) {
        const uint64_t first = 4ull * p.slice_base, n = 4ull * p.n_slices;
        for (uint64_t i = threadIdx.x; i < n; i += kStatusThreads) {
            if (d.slot_status[first + i].x != DE_OK) {
                atomicMin(&best, (int)i);
                break;  // later slots of this thread are further on
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && best != INT32_MAX) {
        const int2 st = d.slot_status[4ull * p.slice_base + best];
        d.pic_status[blockIdx.x].slot = best;
        d.pic_status[blockIdx.x].code = st.x;
        d.pic_status[blockIdx.x].aux = st.y;
    }
}

}  // namespace

cudaError_t upload_scans() {
    uint8_t s[2][64];
    for (int i = 0; i < 64; i++) {
        s[0][i] = kProgressiveScan[i];
        s[1][i] = kInterlacedScan[i];
    }
    return cudaMemcpyToSymbol(c_scan, s, sizeof s);
}

cudaError_t launch_locate(const DecodeLaunch &d, cudaStream_t s) {
    if (d.n_pics == 0) return cudaSuccess;
    k_locate<<<d.n_pics, kLocateThreads, 0, s>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_entropy(const DecodeLaunch &d, const EntropyShape &shape, cudaStream_t s) {
    if (d.n_slices == 0) return cudaSuccess;
    k_entropy<<<shape.grid, 32 * shape.warps_per_block, 0, s>>>(d);
    return cudaGetLastError();
}

// Coefficients (row results over them), non-zero row flags, sample pairs.
size_t idct_smem_bytes() { return 4 * kMaxSliceCoefs + kMaxSliceCoefs / 8 + 2 * kMaxSliceCoefs; }

cudaError_t launch_idct(const DecodeLaunch &d, cudaStream_t s) {
    if (d.n_slices == 0) return cudaSuccess;
    k_idct<<<d.n_slices, kIdctThreads, idct_smem_bytes(), s>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_status(const DecodeLaunch &d, cudaStream_t s) {
    if (d.n_pics == 0) return cudaSuccess;
    k_status<<<d.n_pics, kStatusThreads, 0, s>>>(d);
    return cudaGetLastError();
}

size_t decode_smem_bytes(uint32_t group, uint32_t group_positions, uint32_t slot_bytes) {
    return 2 * 2 * kBookTableWords + sizeof(GroupSlice) * kMaxGroup + 512u * group + slot_bytes * group_positions;
}

// The most shared memory a CTA of k_decode may take (a group of 8-macroblock
// 4:4:4 slices fills about a hundred kilobytes).
constexpr size_t kDecodeSmemMax = 200u << 10;

int decode_grid(int device, uint32_t group, uint32_t group_positions, uint32_t slot_bytes) {
    int sms = 0, fit = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t smem = decode_smem_bytes(group, group_positions, slot_bytes);
    if (slot_bytes == 1)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_decode<int8_t>, kDecodeThreads, smem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_decode<int16_t>, kDecodeThreads, smem);
    return sms * (fit > 0 ? fit : 1);
}

cudaError_t launch_decode(const DecodeLaunch &d, int grid, cudaStream_t s) {
    if (d.n_slices == 0) return cudaSuccess;
    const size_t smem = decode_smem_bytes(d.group, d.group_positions, d.slot_bytes);
    if (d.group < 1 || d.group > kMaxGroup || d.group_positions % 16u != 0 || smem > kDecodeSmemMax ||
        (d.slot_bytes != 1 && d.slot_bytes != 2))
        return cudaErrorInvalidValue;
    const uint32_t groups = (d.n_slices + d.group - 1u) / d.group;
    const int g = grid > 0 && (uint32_t)grid < groups ? grid : (int)groups;
    if (d.slot_bytes == 1)
        k_decode<int8_t><<<g, kDecodeThreads, smem, s>>>(d);
    else
        k_decode<int16_t><<<g, kDecodeThreads, smem, s>>>(d);
    return cudaGetLastError();
}

cudaError_t configure_decode_kernels() {
    cudaError_t e = cudaFuncSetAttribute(k_idct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)idct_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_decode<int16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecodeSmemMax);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_decode<int8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecodeSmemMax);
    if (e != cudaSuccess) return e;
    float basis[64];
    dct_basis(basis);
    if ((e = cudaMemcpyToSymbol(c_idct_basis, basis, sizeof basis)) != cudaSuccess) return e;
    return upload_scans();
}

int entropy_grid(int device, int warps_per_block, int blocks_per_sm) {
    int sms = 0, fit = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_entropy, 32 * warps_per_block, 0);
    if (fit < 1) fit = 1;
    const int per_sm = blocks_per_sm > 0 && blocks_per_sm < fit ? blocks_per_sm : fit;
    return sms * per_sm;
}

}  // namespace prores
