// encode.cu -- the encoder (the crate's src/encode.rs) as sm_100a kernels.
//
//   k_fdct        one CTA per slice: edge-replicated 8x8 gathers, p = s 512/2^b
//                 - 256 and the FDCT in the crate's exact single-precision
//                 order (src/encode.rs:488-555, src/dct.rs:70-93), written in
//                 the slice's scanned order once per frame.
//   k_alpha_size  one warp per slice: the lossless alpha codes' size
//                 (src/encode.rs:838-868, :457-470); it does not depend on
//                 the quantiser.
//   k_rc_init / k_cost / k_rc_step
//                 the rate control's probe sequence replayed exactly: 224,
//                 then mid = lo + (hi - lo) / 2 while lo < hi
//                 (src/encode.rs:685-713). k_cost sizes every slice of every
//                 picture still searching at that picture's probe, one warp
//                 per slice component (quantise + exact bit count,
//                 src/dsp/scalar.rs:19-39, src/encode.rs:398-409); k_rc_step
//                 sums a picture's slices and moves its interval.
//   k_cost_window the next kWindow finer quantisers below the uniform one.
//   k_shareout    one warp per picture: the sequential share-out of the slack
//                 (src/encode.rs:769-793), costing any deeper quantiser it
//                 needs itself.
//   k_layout / k_frame
//                 slice offsets (an exclusive scan per picture), picture and
//                 frame sizes, the frame and picture headers.
//   k_pack        one CTA per slice: the slice header, the table entry, and
//                 each component's codes bit-packed straight into the frame
//                 (src/encode.rs:413-437, :797-829), plus the alpha codes.
//
// Output bits are OR-ed into a zeroed buffer as big-endian 32-bit words, so
// writers that share a word never need to be ordered.

#include <cuda_runtime.h>

#include <cstdint>

#include "codec_tables.h"
#include "encode_types.h"
#include "pair_math.h"

namespace prores {

__constant__ uint8_t c_enc_scan[2][64];
__constant__ float c_fdct_basis[64];  // T[x][u], the same values as the decoder's

namespace {

constexpr float kAcRounding = 0.42f;  // src/encode.rs:204

__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

// ORs `value` into the bit field [bitpos, bitpos + len) (MSB first; the
// value's leading zeros are the field's) of a big-endian bit buffer.
__device__ __forceinline__ void put_field(uint32_t *out, uint64_t bitpos, uint64_t value, uint32_t len) {
    const uint32_t nb = bit_len64(value);
    if (nb == 0) return;
    const uint64_t start = bitpos + len - nb;
    uint32_t *w = out + (start >> 5);
    const uint32_t o = (uint32_t)(start & 31);
    const uint32_t first = 32 - o;
    if (nb <= first) {
        atomicOr(w, bswap32((uint32_t)(value << (first - nb))));
        return;
    }
    const uint32_t rest = nb - first;
    atomicOr(w, bswap32((uint32_t)(value >> rest)));
    if (rest <= 32) {
        atomicOr(w + 1, bswap32((uint32_t)(value << (32 - rest))));
    } else {
        atomicOr(w + 1, bswap32((uint32_t)(value >> (rest - 32))));
        atomicOr(w + 2, bswap32((uint32_t)(value << (64 - rest))));
    }
}

// floor(|x| + r) as an integer: |x| + r is positive, so truncation is the
// floor (and both saturate alike from 2^31 up).
__device__ __forceinline__ int32_t magnitude(float x, float r) { return __float2int_rz(__fadd_rn(fabsf(x), r)); }

__device__ __forceinline__ int32_t quantise1(float f, float inv, float r) {
    // x = F inv; QF = sign(x) floor(|x| + r) (src/dsp/scalar.rs:19-39).
    const float x = __fmul_rn(f, inv);
    const int32_t q = magnitude(x, r);
    return x < 0.0f ? -q : q;
}

// ---------------------------------------------------------------- fdct

constexpr int kFdctThreads = 128;
constexpr int kMaxSliceCoefs = 64 * 12 * 8;

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

// One warp per slice component, one lane per 8x8 block (a component has
// at most 32 blocks; lanes past the component's count idle). A lane loads
// its block's 8 rows, transforms them (rows, then columns, in the crate's
// order; the row results wait in shared memory, lane-minor, so no bank
// conflicts) and stores each coefficient at its scanned place
// n * scan[k] + blk: the lanes of a component store consecutive floats.
// The basis comes from constant memory, read by every lane at the same
// address. A chunk of 32 scanned coefficients is one scanned position of a
// 32-block component, or several positions of a smaller one; its largest
// |F| is reduced over the lanes as each position is stored and kept in
// shared memory until the component is done. (Cb and Cr of a 4:2:2 slice
// in one warp measured slower: fewer warps to hide the loads.)
__global__ void __launch_bounds__(kFdctThreads) k_fdct(EncodeLaunch e) {
    __shared__ uint32_t cmax_sh[kFdctThreads / 32][64];
    __shared__ float tmp_sh[kFdctThreads / 32][64][32];  // the row pass, [y * 8 + u][lane]
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t item = blockIdx.x * (kFdctThreads / 32) + warp;
    if (item >= 3u * e.n_slices) return;  // the whole warp
    const uint32_t s = item / 3u, c = item - 3u * s;
    const EncSliceDesc sd = e.slices[s];
    const EncPicDesc &pd = e.pics[sd.pic];
    const EncFrameDesc &fd = e.frames[pd.frame];
    const uint32_t cpm = fd.chroma == 2 ? 2u : 4u;
    const uint32_t per_mb = c == 0 ? 4u : cpm;
    const uint32_t nb = per_mb * sd.mbs;
    const uint32_t start = c == 0 ? 0u : 64u * sd.mbs * (4u + (c - 1u) * cpm);
    uint32_t *cm = cmax_sh[warp];
    cm[lane] = 0;
    cm[lane + 32] = 0;
    __syncwarp();
    if (lane < nb) {
        const uint8_t *scan = c_enc_scan[pd.interlaced_scan];
        float (*tmp)[32] = tmp_sh[warp];
        const uint32_t m = lane / per_mb, b = lane - m * per_mb;
        uint32_t bx, by;
        block_xy(c, fd.chroma, sd.mb_x, sd.mb_y, m, b, bx, by);
        const uint32_t w = fd.plane_w[c];
        const uint16_t *plane = e.in + fd.in_off[c];
        const float scale = fd.in_scale;
        // Rows: tmp[y][u] = sum_x p[y][x] T[x][u], x in order from 0.
#pragma unroll
        for (int y = 0; y < 8; y++) {
            // Edge replication: the last picture row and column repeat.
            const uint32_t py = min(by + (uint32_t)y, pd.height - 1u);
            const uint16_t *line = plane + (uint64_t)(pd.first_row + pd.row_step * py) * w;
            float p[8];
            if (bx + 8u <= w && ((reinterpret_cast<uintptr_t>(line + bx) & 15u) == 0)) {
                const uint4 v = __ldg(reinterpret_cast<const uint4 *>(line + bx));
                const uint32_t words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    p[2 * i] = __fsub_rn(__fmul_rn((float)(words[i] & 0xFFFFu), scale), 256.0f);
                    p[2 * i + 1] = __fsub_rn(__fmul_rn((float)(words[i] >> 16), scale), 256.0f);
                }
            } else {
#pragma unroll
                for (int x = 0; x < 8; x++) {
                    const uint32_t col = min(bx + (uint32_t)x, w - 1u);
                    p[x] = __fsub_rn(__fmul_rn((float)__ldg(line + col), scale), 256.0f);
                }
            }
            // Outputs u = 2 j, 2 j + 1 summed as a pair, each in the same
            // order; the products stay scalar (see pair_math.h).
#pragma unroll
            for (int j = 0; j < 4; j++) {
                uint64_t acc = 0;
#pragma unroll
                for (int x = 0; x < 8; x++)
                    acc = pair_add(acc, pair_of(__fmul_rn(p[x], c_fdct_basis[8 * x + 2 * j]),
                                                __fmul_rn(p[x], c_fdct_basis[8 * x + 2 * j + 1])));
                pair_split(acc, tmp[8 * y + 2 * j][lane], tmp[8 * y + 2 * j + 1][lane]);
            }
        }
        // Columns: F[v][u] = sum_y T[y][v] tmp[y][u], y in order from 0.
        float *out = e.coef + sd.coef + start;
        const uint32_t mask = nb >= 32u ? 0xffffffffu : (1u << nb) - 1u;
#pragma unroll 1
        for (int u = 0; u < 8; u++) {
            float col[8];
#pragma unroll
            for (int y = 0; y < 8; y++) col[y] = tmp[8 * y + u][lane];
            float res[8];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                // Outputs v = 2 j, 2 j + 1 summed as a pair.
                uint64_t acc = 0;
#pragma unroll
                for (int y = 0; y < 8; y++)
                    acc = pair_add(acc, pair_of(__fmul_rn(c_fdct_basis[8 * y + 2 * j], col[y]),
                                                __fmul_rn(c_fdct_basis[8 * y + 2 * j + 1], col[y])));
                pair_split(acc, res[2 * j], res[2 * j + 1]);
            }
#pragma unroll
            for (int v = 0; v < 8; v++) {
                const float acc = res[v];
                const uint32_t sp = scan[8 * v + u];
                out[nb * sp + lane] = acc;
                // Every active lane is at this position, in one chunk.
                const uint32_t big = __reduce_max_sync(mask, __float_as_uint(fabsf(acc)));
                if (lane == 0) {
                    const uint32_t j = (nb * sp) >> 5;
                    cm[j] = max(cm[j], big);
                }
            }
        }
    }
    __syncwarp();
    // The component's 2 nb chunk maxima.
    float *cmax = e.coef_max + ((sd.coef + start) >> 5);
    for (uint32_t j = lane; j < 2u * nb; j += 32) cmax[j] = __uint_as_float(cm[j]);
}

// ---------------------------------------------------------------- alpha

constexpr int kAlphaWarps = 4;
constexpr int kMaxAlphaValues = 16 * 16 * 8;

struct AlphaScratch {
    uint16_t start[kMaxAlphaValues + 1];
    uint16_t value[kMaxAlphaValues];
};

__device__ __forceinline__ uint32_t alpha_diff_len(int32_t diff, uint32_t bits) {
    const uint32_t a = diff < 0 ? 0u - (uint32_t)diff : (uint32_t)diff;
    const uint32_t mag = bits == 8 ? 3u : 6u, max = bits == 8 ? 8u : 64u;
    return (a >= 1u && a <= max) ? 2u + mag : 1u + bits;
}
__device__ __forceinline__ uint32_t alpha_run_len(uint32_t run) { return run == 1u ? 1u : (run <= 16u ? 5u : 16u); }

// The slice's alpha values (16 rows of 16 mbs, edges repeated, converted to
// the coded bits) into runs; returns the run count. A run cannot pass 2048
// values: a slice has at most 2048.
__device__ uint32_t alpha_runs(const EncodeLaunch &e, const EncSliceDesc &sd, const EncPicDesc &pd,
                               const EncFrameDesc &fd, AlphaScratch &sc) {
    const int lane = threadIdx.x & 31;
    const uint32_t cols = 16u * sd.mbs, count = 16u * cols;
    const uint32_t width = fd.width, x0 = 16u * sd.mb_x;
    const uint16_t max_in = (uint16_t)(0xFFFFu >> (16u - fd.bit_depth));
    const uint16_t *plane = e.alpha_in + fd.alpha_in_off;
    const uint32_t cshift = (uint32_t)__ffs(cols) - 1u;  // cols is 16 times a power of two
    uint32_t n_runs = 0;
    uint32_t prev = 0;
    // 256 values (count is a multiple) a round: their eight loads are all
    // issued before the first is used.
    for (uint32_t base = 0; base < count; base += 256) {
        uint32_t vals[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t i = base + 32u * k + lane;
            const uint32_t r = i >> cshift, n = i & (cols - 1u);
            const uint32_t row = pd.first_row + pd.row_step * min(16u * sd.mb_y + r, pd.height - 1u);
            vals[k] = __ldg(plane + (uint64_t)row * width + min(x0 + n, width - 1u));
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t i = base + 32u * k + lane;
            uint32_t a = vals[k] < max_in ? vals[k] : max_in;
            const uint32_t v = fd.rescale_identity ? a : (uint32_t)(((uint64_t)a * fd.rescale_m + (1ull << 39)) >> 40);
            const uint32_t before = __shfl_up_sync(0xffffffffu, v, 1);
            const uint32_t left = lane == 0 ? prev : before;
            const bool is_start = i == 0 || v != left;
            const uint32_t mask = __ballot_sync(0xffffffffu, is_start);
            if (is_start) {
                const uint32_t idx = n_runs + __popc(mask & ((1u << lane) - 1u));
                sc.start[idx] = (uint16_t)i;
                sc.value[idx] = (uint16_t)v;
            }
            n_runs += __popc(mask);
            prev = __shfl_sync(0xffffffffu, v, 31);
        }
    }
    if (lane == 0) sc.start[n_runs] = (uint16_t)count;
    __syncwarp();
    return n_runs;
}

__device__ __forceinline__ uint32_t alpha_run_bits(const AlphaScratch &sc, uint32_t j, uint32_t bits, uint32_t &dlen) {
    const int32_t prev = j ? (int32_t)sc.value[j - 1] : -1;
    dlen = alpha_diff_len((int32_t)sc.value[j] - prev, bits);
    return dlen + alpha_run_len((uint32_t)sc.start[j + 1] - sc.start[j]);
}

__global__ void __launch_bounds__(32 * kAlphaWarps) k_alpha_size(EncodeLaunch e) {
    __shared__ AlphaScratch scratch[kAlphaWarps];
    const uint32_t s = blockIdx.x * kAlphaWarps + (threadIdx.x >> 5);
    if (s >= e.n_slices) return;
    const int lane = threadIdx.x & 31;
    const EncSliceDesc sd = e.slices[s];
    const EncPicDesc &pd = e.pics[sd.pic];
    const EncFrameDesc &fd = e.frames[pd.frame];
    if (fd.alpha_bits == 0) {
        if (lane == 0) e.alpha_bytes[s] = 0;
        return;
    }
    AlphaScratch &sc = scratch[threadIdx.x >> 5];
    const uint32_t n_runs = alpha_runs(e, sd, pd, fd, sc);
    uint32_t bits = 0;
    for (uint32_t j = lane; j < n_runs; j += 32) {
        uint32_t dlen;
        bits += alpha_run_bits(sc, j, fd.alpha_bits, dlen);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bits += __shfl_xor_sync(0xffffffffu, bits, o);
    if (lane == 0) e.alpha_bytes[s] = (bits + 7u) / 8u;
}

__device__ void alpha_write(const EncodeLaunch &e, const EncSliceDesc &sd, const EncPicDesc &pd,
                            const EncFrameDesc &fd, AlphaScratch &sc, uint64_t bitpos) {
    const int lane = threadIdx.x & 31;
    const uint32_t n_runs = alpha_runs(e, sd, pd, fd, sc);
    const uint32_t bits = fd.alpha_bits;
    const uint32_t max = bits == 8 ? 8u : 64u;
    uint64_t carry = 0;
    for (uint32_t base = 0; base < n_runs; base += 32) {
        const uint32_t j = base + lane;
        uint32_t dlen = 0, len = 0;
        if (j < n_runs) len = alpha_run_bits(sc, j, bits, dlen);
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (j < n_runs) {
            const uint64_t at = bitpos + carry + incl - len;
            const int32_t prev = j ? (int32_t)sc.value[j - 1] : -1;
            const int32_t diff = (int32_t)sc.value[j] - prev;
            const uint32_t a = diff < 0 ? 0u - (uint32_t)diff : (uint32_t)diff;
            // Tables 13/14: `0`, |d| - 1, sign; or `1` and d mod 2^bits.
            if (a >= 1u && a <= max)
                put_field(e.out, at, ((uint64_t)(a - 1u) << 1) | (uint64_t)(diff < 0), dlen);
            else
                put_field(e.out, at, (1ull << bits) | ((uint32_t)diff & ((1u << bits) - 1u)), dlen);
            // Table 12: `1`; `0` and 4 bits of run - 1; or 5 zeros and 11 bits.
            const uint32_t run = (uint32_t)sc.start[j + 1] - sc.start[j];
            put_field(e.out, at + dlen, run == 1u ? 1u : run - 1u, len - dlen);
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// ---------------------------------------------------------------- costing

// Codeword lengths of run and level symbols below 32 by context, kept in
// shared memory by the kernels that count or write codes.
struct LenTables {
    uint8_t run[16][32];
    uint8_t level[9][32];
    __device__ void fill() {
        for (uint32_t i = threadIdx.x; i < 16 * 32; i += blockDim.x) run[i >> 5][i & 31] = (uint8_t)cb_len(run_book(i >> 5), i & 31);
        for (uint32_t i = threadIdx.x; i < 9 * 32; i += blockDim.x)
            level[i >> 5][i & 31] = (uint8_t)cb_len(level_book(i >> 5), i & 31);
    }
    __device__ __forceinline__ uint32_t run_len(uint32_t ctx, uint32_t r) const {
        const uint32_t c = ctx < 15u ? ctx : 15u;
        return r < 32u ? run[c][r] : cb_len(run_book(c), r);
    }
    __device__ __forceinline__ uint32_t level_len(uint32_t ctx, uint32_t lvl) const {
        const uint32_t c = ctx < 8u ? ctx : 8u;
        return lvl < 32u ? level[c][lvl] : cb_len(level_book(c), lvl);
    }
};

// The DC part of the bit count (src/encode.rs:383-395): EG5 of the first,
// then Table 9 by |previous difference|, the sign flipped after a negative
// one.
template <class Get>
__device__ __forceinline__ uint32_t dc_bits_of(Get get, uint32_t n_blocks, float inv0) {
    uint32_t bits = 0;
    int32_t prev_dc = 0, prev_diff = 3;
    for (uint32_t i = 0; i < n_blocks; i++) {
        const int32_t q = quantise1(get(i), inv0, 0.5f);
        if (i == 0) {
            bits += cb_len(kFirstDcBook, signed_to_symbol(q));
        } else {
            const int32_t diff = (int32_t)((uint32_t)q - (uint32_t)prev_dc);
            bits += cb_len(dc_book(prev_diff), signed_to_symbol(prev_diff < 0 ? -diff : diff));
            prev_diff = diff;
        }
        prev_dc = q;
    }
    return bits;
}

__device__ __forceinline__ uint32_t dc_bits(const float *f, uint32_t n_blocks, float inv0) {
    return dc_bits_of([&](uint32_t i) { return __ldg(f + i); }, n_blocks, inv0);
}

// One AC position of a lane's walk: x = F inv, m = floor(|x| + 0.42)
// (src/dsp/scalar.rs:19-39) as an integer; only a non-zero coefficient is
// coded (its run from the last one, its level, both by context).
struct AcWalk {
    uint32_t prev_run = 4, prev_level = 1, pos = 0;
};

template <class Emit>
__device__ __forceinline__ void ac_position(AcWalk &w, float f, float inv, uint32_t p, Emit emit) {
    const float x = __fmul_rn(f, inv);
    const int32_t m = magnitude(x, kAcRounding);
    if (m >= 1) {
        const uint32_t run = p - w.pos;
        const uint32_t level = (uint32_t)m - 1u;
        emit(w, run, level, x < 0.0f);
        w.prev_run = run;
        w.prev_level = level;
        w.pos = p + 1;
    }
}

// One component's view of a quantiser table (layout beside kQuantStride):
// inverse weights and non-zero bounds by scanned position, and the bound of
// each 32-coefficient chunk of a component of its block count.
struct CompQuant {
    const float *inv, *bound, *chunk;
};

__device__ __forceinline__ CompQuant comp_quant(const float *qb, uint32_t comp, uint32_t n_blocks) {
    const uint32_t g = comp > 0 ? 1u : 0u;
    CompQuant c;
    c.inv = qb + 64u * g;
    c.bound = qb + 128u + 64u * g;
    c.chunk = n_blocks >= 32u ? c.bound : qb + 256u + 60u * g + (2u * n_blocks - 4u);
    return c;
}

// Whether chunk j holds no coefficient that quantises to a non-zero: its
// largest |F| is below the least non-zero bound of its positions.
__device__ __forceinline__ bool chunk_is_zero(const float *cmax, const CompQuant &q, uint32_t j) {
    return __ldg(cmax + j) < __ldg(q.chunk + j);
}

// Walks a component's AC positions (n_blocks onwards) in order, position by
// position, skipping the chunks that quantise to zero; `emit` gets every
// position's coefficient and inverse weight.
template <class Emit>
__device__ __forceinline__ void ac_walk_dense(const float *f, const float *cmax, uint32_t n_blocks,
                                              const CompQuant &q, Emit emit) {
    const uint32_t total = 64u * n_blocks;
    const uint32_t shift = 31u - __clz(n_blocks);
    for (uint32_t c0 = n_blocks & ~31u; c0 < total; c0 += 32) {
        if (chunk_is_zero(cmax, q, c0 >> 5)) continue;
        if (n_blocks >= 4) {
            for (uint32_t p0 = max(c0, n_blocks); p0 < c0 + 32u; p0 += 4) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(f + p0));
                const float iv = __ldg(q.inv + (p0 >> shift));
                emit(v.x, iv, p0);
                emit(v.y, iv, p0 + 1);
                emit(v.z, iv, p0 + 2);
                emit(v.w, iv, p0 + 3);
            }
        } else {
            // Two blocks: positions 0 and 1 are the DCs; p and p + 1 share
            // scan position p / 2.
            for (uint32_t p0 = c0; p0 < c0 + 32u; p0 += 4) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(f + p0));
                const float ia = __ldg(q.inv + (p0 >> 1)), ib = __ldg(q.inv + (p0 >> 1) + 1);
                if (p0 > 0) {
                    emit(v.x, ia, p0);
                    emit(v.y, ia, p0 + 1);
                }
                emit(v.z, ib, p0 + 2);
                emit(v.w, ib, p0 + 3);
            }
        }
    }
}

// The same walk over candidates only: a chunk's candidate mask takes one
// compare per coefficient against the non-zero bound of its position (so
// it holds every non-zero, and each candidate is re-quantised exactly),
// and the lane then visits the candidates alone. Suited to heavy per-code
// work (the writer), where a position-by-position walk would make every
// lane wait out every other lane's codes.
template <class Emit>
__device__ __forceinline__ void ac_walk_sparse(const float *f, const float *cmax, uint32_t n_blocks,
                                               const CompQuant &q, Emit emit) {
    const uint32_t total = 64u * n_blocks;
    const uint32_t shift = 31u - __clz(n_blocks);
    AcWalk w;
    w.pos = n_blocks;
    for (uint32_t c0 = n_blocks & ~31u; c0 < total; c0 += 32) {
        if (chunk_is_zero(cmax, q, c0 >> 5)) continue;
        uint32_t mask = 0;
#pragma unroll
        for (uint32_t i = 0; i < 8; i++) {
            const uint32_t e0 = c0 + 4u * i;
            const float4 v = __ldg(reinterpret_cast<const float4 *>(f + e0));
            // With two blocks a load spans scan positions e0 / 2 and e0 / 2 + 1.
            const float ta = __ldg(q.bound + (e0 >> shift)), tb = __ldg(q.bound + ((e0 + 3u) >> shift));
            const uint32_t nib = (fabsf(v.x) >= ta ? 1u : 0u) | (fabsf(v.y) >= ta ? 2u : 0u) |
                                 (fabsf(v.z) >= tb ? 4u : 0u) | (fabsf(v.w) >= tb ? 8u : 0u);
            mask |= nib << (4u * i);
        }
        if (c0 == 0) mask &= ~0u << n_blocks;  // the DCs
        while (mask) {
            const uint32_t p = c0 + (uint32_t)__ffs(mask) - 1u;
            mask &= mask - 1u;
            ac_position(w, __ldg(f + p), __ldg(q.inv + (p >> shift)), p, emit);
        }
    }
}

// The AC part of a lane's bit count at one position: the position is
// quantised and its code length (run by the previous run's context, level
// by the previous level's, a sign bit) taken from the length tables
// whether or not it is a non-zero, and kept only if it is. Lanes that count
// different components so stay in step, with no branch per position; only
// a run or level past the tables (32 and above) takes a branch.
struct AcCount {
    uint32_t bits = 0, pos = 0, run_ctx = 4, level_ctx = 1;
};

__device__ __forceinline__ void count_position(AcCount &c, float f, float inv, uint32_t p, const LenTables &t) {
    const int32_t m = magnitude(__fmul_rn(f, inv), kAcRounding);
    const bool nz = m >= 1;
    const uint32_t run = p - c.pos;
    const uint32_t level = (uint32_t)m - 1u;
    uint32_t add = (uint32_t)t.run[c.run_ctx][min(run, 31u)] + (uint32_t)t.level[c.level_ctx][min(level, 31u)] + 1u;
    if (nz && (run | level) >= 32u)
        add = cb_len(run_book(c.run_ctx), run) + cb_len(level_book(c.level_ctx), level) + 1u;
    if (nz) {
        c.bits += add;
        c.run_ctx = min(run, 15u);
        c.level_ctx = min(level, 8u);
        c.pos = p + 1u;
    }
}

// Bits of one quantised component (src/encode.rs:398-409), one lane: the
// crate's own walk over the scanned positions.
__device__ uint32_t lane_component_bits(const float *f, const float *cmax, uint32_t n_blocks, const CompQuant &q,
                                        const LenTables &t) {
    AcCount c;
    c.pos = n_blocks;
    ac_walk_dense(f, cmax, n_blocks, q, [&](float v, float inv, uint32_t p) { count_position(c, v, inv, p, t); });
    return dc_bits(f, n_blocks, __ldg(q.inv)) + c.bits;
}

// The same count over the candidates of each chunk only (the writer's
// walk): the candidate masks cost a compare a coefficient, and only the
// candidates are quantised and coded. Faster than the position-by-position
// walk where most coefficients quantise to zero (coarse quantisers), slower
// where most do not.
__device__ uint32_t lane_component_bits_sparse(const float *f, const float *cmax, uint32_t n_blocks,
                                               const CompQuant &q, const LenTables &t) {
    uint32_t bits = 0;
    ac_walk_sparse(f, cmax, n_blocks, q, [&](AcWalk &w, uint32_t run, uint32_t level, bool) {
        bits += t.run_len(w.prev_run, run) + t.level_len(w.prev_level, level) + 1u;
    });
    return dc_bits(f, n_blocks, __ldg(q.inv)) + bits;
}

// Code lengths of a run and of a level by context, from the tables when
// they hold the symbol (src/vlc.rs:397-415).
__device__ __forceinline__ uint32_t run_len_of(const LenTables &t, uint32_t ctx, uint32_t r) {
    return r < 32u ? t.run[ctx][r] : cb_len(run_book(ctx), r);
}
__device__ __forceinline__ uint32_t level_len_of(const LenTables &t, uint32_t ctx, uint32_t l) {
    return l < 32u ? t.level[ctx][l] : cb_len(level_book(ctx), l);
}

// Bits of one quantised component (src/encode.rs:398-409), split over a
// group of kSeg lanes, for short launches bound by one lane's walk: lane r
// walks the r-th run of chunks as if the walk started there (previous run
// 4, previous level 1, last position its start), which gets every code
// right but the segment's first (run and level by the previous segment's
// state) and its second's run (by the first's run). Lanes past the first
// also find their segment's first two non-zeros, and the group's first
// lane puts the segments together in order, replacing those codes with the
// right ones: the sum is the one-lane walk's. Every lane of the warp takes
// part (the exchange is by shuffles); `active` is false for lanes past the
// work.
template <int kSeg>
__device__ uint32_t group_component_bits(bool active, const float *f, const float *cmax, uint32_t nb,
                                         const CompQuant &q, const LenTables &t) {
    const uint32_t lane = threadIdx.x & 31u, r = lane % (uint32_t)kSeg, base = lane - r;
    const uint32_t chunks = active ? 2u * nb : 0u;
    const uint32_t c_lo = chunks * r / kSeg, c_hi = chunks * (r + 1) / kSeg;
    const uint32_t shift = active ? 31u - __clz(nb) : 0u;
    const uint32_t start = r == 0 ? nb : 32u * c_lo;
    AcCount c;
    c.pos = start;
    for (uint32_t k = c_lo; k < c_hi; k++) {
        if (chunk_is_zero(cmax, q, k)) continue;
        const uint32_t c0 = 32u * k;
        if (nb >= 4) {
            for (uint32_t p0 = max(c0, nb); p0 < c0 + 32u; p0 += 4) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(f + p0));
                const float iv = __ldg(q.inv + (p0 >> shift));
                count_position(c, v.x, iv, p0, t);
                count_position(c, v.y, iv, p0 + 1, t);
                count_position(c, v.z, iv, p0 + 2, t);
                count_position(c, v.w, iv, p0 + 3, t);
            }
        } else {
            for (uint32_t p0 = c0; p0 < c0 + 32u; p0 += 4) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(f + p0));
                const float ia = __ldg(q.inv + (p0 >> 1)), ib = __ldg(q.inv + (p0 >> 1) + 1);
                if (p0 > 0) {
                    count_position(c, v.x, ia, p0, t);
                    count_position(c, v.y, ia, p0 + 1, t);
                }
                count_position(c, v.z, ib, p0 + 2, t);
                count_position(c, v.w, ib, p0 + 3, t);
            }
        }
    }
    // The segment's first two non-zeros (lanes past the first).
    uint32_t found = 0, q1 = 0, l1 = 0, q2 = 0;
    if (r > 0) {
        for (uint32_t k = c_lo; k < c_hi && found < 2u; k++) {
            if (chunk_is_zero(cmax, q, k)) continue;
            for (uint32_t p = 32u * k; p < 32u * k + 32u && found < 2u; p++) {
                const int32_t m = magnitude(__fmul_rn(__ldg(f + p), __ldg(q.inv + (p >> shift))), kAcRounding);
                if (m >= 1) {
                    if (found == 0) {
                        q1 = p;
                        l1 = (uint32_t)m - 1u;
                    } else {
                        q2 = p;
                    }
                    found++;
                }
            }
        }
    }
    // Put the segments together on the group's first lane.
    uint32_t bits = c.bits, pos = c.pos, rctx = c.run_ctx, lctx = c.level_ctx;
#pragma unroll
    for (int j = 1; j < kSeg; j++) {
        const uint32_t src = base + (uint32_t)j;
        const uint32_t s_bits = __shfl_sync(0xffffffffu, c.bits, src);
        const uint32_t s_found = __shfl_sync(0xffffffffu, found, src);
        const uint32_t s_q1 = __shfl_sync(0xffffffffu, q1, src);
        const uint32_t s_l1 = __shfl_sync(0xffffffffu, l1, src);
        const uint32_t s_q2 = __shfl_sync(0xffffffffu, q2, src);
        const uint32_t s_start = __shfl_sync(0xffffffffu, start, src);
        const uint32_t s_pos = __shfl_sync(0xffffffffu, c.pos, src);
        const uint32_t s_rctx = __shfl_sync(0xffffffffu, c.run_ctx, src);
        const uint32_t s_lctx = __shfl_sync(0xffffffffu, c.level_ctx, src);
        if (r == 0 && s_found > 0) {
            const uint32_t run1 = s_q1 - pos, run1_seg = s_q1 - s_start;
            // The first code: right contexts and run, in place of the
            // segment's own (unsigned arithmetic: the sum comes out right).
            bits += s_bits + run_len_of(t, rctx, run1) + level_len_of(t, lctx, s_l1) -
                    run_len_of(t, 4u, run1_seg) - level_len_of(t, 1u, s_l1);
            if (s_found == 1) {
                pos = s_q1 + 1u;
                rctx = min(run1, 15u);
                lctx = min(s_l1, 8u);
            } else {
                // The second code's run by the first's right run.
                const uint32_t run2 = s_q2 - s_q1 - 1u;
                bits += run_len_of(t, min(run1, 15u), run2) - run_len_of(t, min(run1_seg, 15u), run2);
                pos = s_pos;
                rctx = s_rctx;
                lctx = s_lctx;
            }
        }
    }
    return (r == 0 && active) ? dc_bits(f, nb, __ldg(q.inv)) + bits : 0u;
}

// The same count with a whole warp on one component, for when latency
// matters more than throughput (few items, or one slice the share-out
// needs): lane l takes scanned positions 32 k + l; a non-zero's run and its
// contexts (the previous non-zero's run and level symbol) come from the
// lanes below it or from what the last step carried.
// kShared: f and cmax point into shared memory (plain loads); else into
// global memory (read-only loads).
template <bool kShared>
__device__ __forceinline__ float coef_load(const float *f, uint32_t i) {
    if constexpr (kShared)
        return f[i];
    else
        return __ldg(f + i);
}

template <bool kShared = false>
__device__ uint32_t warp_component_bits(const float *f, const float *cmax, uint32_t n_blocks, const CompQuant &cq,
                                        const LenTables &t) {
    const float *inv = cq.inv;
    const int lane = threadIdx.x & 31;
    const uint32_t total = 64u * n_blocks;
    const uint32_t shift = 31u - __clz(n_blocks);
    uint32_t bits = 0;
    int32_t carry_pos = (int32_t)n_blocks - 1;
    uint32_t carry_run = 4, carry_level = 1;
    for (uint32_t base = 0; base < total; base += 32) {
        // Past the DCs a chunk that quantises to zero changes nothing.
        if (base > 0 && coef_load<kShared>(cmax, base >> 5) < __ldg(cq.chunk + (base >> 5))) continue;
        const uint32_t p = base + lane;
        const uint32_t sidx = p >> shift;
        const int32_t q = quantise1(coef_load<kShared>(f, p), __ldg(inv + sidx), sidx == 0 ? 0.5f : kAcRounding);
        if (base == 0) {
            // The DCs (n_blocks <= 32, all in this step).
            const int32_t left = __shfl_up_sync(0xffffffffu, q, 1);
            const int32_t diff = (int32_t)((uint32_t)q - (uint32_t)left);
            const int32_t prev_diff_raw = __shfl_up_sync(0xffffffffu, diff, 1);
            if (p < n_blocks) {
                if (p == 0) {
                    bits += cb_len(kFirstDcBook, signed_to_symbol(q));
                } else {
                    const int32_t prev_diff = p == 1 ? 3 : prev_diff_raw;
                    bits += cb_len(dc_book(prev_diff), signed_to_symbol(prev_diff < 0 ? -diff : diff));
                }
            }
        }
        const bool nz = q != 0 && p >= n_blocks;
        const uint32_t mask = __ballot_sync(0xffffffffu, nz);
        if (mask == 0) continue;
        const uint32_t below = mask & ((1u << lane) - 1u);
        const int src = below ? 31 - __clz(below) : lane;
        const int32_t prev_pos = below ? (int32_t)(base + src) : carry_pos;
        const uint32_t run = nz ? (uint32_t)((int32_t)p - prev_pos - 1) : 0u;
        const uint32_t level = nz ? (q < 0 ? 0u - (uint32_t)q : (uint32_t)q) - 1u : 0u;
        const uint32_t src_run = __shfl_sync(0xffffffffu, run, src);
        const uint32_t src_level = __shfl_sync(0xffffffffu, level, src);
        if (nz) bits += t.run_len(below ? src_run : carry_run, run) + t.level_len(below ? src_level : carry_level, level) + 1u;
        const int top = 31 - __clz(mask);
        carry_pos = (int32_t)(base + top);
        carry_run = __shfl_sync(0xffffffffu, run, top);
        carry_level = __shfl_sync(0xffffffffu, level, top);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bits += __shfl_xor_sync(0xffffffffu, bits, o);
    return bits;
}

// The quantiser table of quantization_index qi (layout beside kQuantStride).
__device__ __forceinline__ const float *quant_base(const EncodeLaunch &e, const EncPicDesc &pd, uint32_t qi) {
    return e.quant + ((uint64_t)pd.quant * 225u + qi) * kQuantStride;
}

__device__ __forceinline__ void comp_layout(const EncFrameDesc &fd, uint32_t mbs, uint32_t comp, uint32_t &n_blocks,
                                            uint32_t &offset) {
    const uint32_t cpm = fd.chroma == 2 ? 2u : 4u;
    n_blocks = (comp == 0 ? 4u : cpm) * mbs;
    offset = comp == 0 ? 0u : 64u * mbs * (4u + (comp - 1u) * cpm);
}

// From this quantiser index up, a lane costs a component over its chunks'
// candidates only (measured on UHD 4:2:2 10-bit: 1.5x faster at 56, 1.1x
// slower at 28).
constexpr uint32_t kSparseCostQi = 40;

// Bytes of one slice component at quantiser qi (one lane).
__device__ __forceinline__ uint32_t component_bytes(const EncodeLaunch &e, const EncSliceDesc &sd, const EncPicDesc &pd,
                                                    const EncFrameDesc &fd, uint32_t comp, uint32_t qi,
                                                    const LenTables &t) {
    uint32_t nb, off;
    comp_layout(fd, sd.mbs, comp, nb, off);
    const CompQuant q = comp_quant(quant_base(e, pd, qi), comp, nb);
    const float *f = e.coef + sd.coef + off, *cmax = e.coef_max + ((sd.coef + off) >> 5);
    const uint32_t bits = qi >= kSparseCostQi ? lane_component_bits_sparse(f, cmax, nb, q, t)
                                              : lane_component_bits(f, cmax, nb, q, t);
    return (bits + 7u) / 8u;
}

// Bytes of one slice component at quantiser qi, the whole warp.
__device__ __forceinline__ uint32_t warp_component_bytes(const EncodeLaunch &e, const EncSliceDesc &sd,
                                                         const EncPicDesc &pd, const EncFrameDesc &fd, uint32_t comp,
                                                         uint32_t qi, const LenTables &t) {
    uint32_t nb, off;
    comp_layout(fd, sd.mbs, comp, nb, off);
    const CompQuant q = comp_quant(quant_base(e, pd, qi), comp, nb);
    const uint32_t bits = warp_component_bits(e.coef + sd.coef + off, e.coef_max + ((sd.coef + off) >> 5), nb, q, t);
    return (bits + 7u) / 8u;
}

constexpr int kCostThreads = 256;

// Work items are (component, slice), component-major: a warp's lanes take
// the same component of 32 neighbouring slices, which cost about the same
// (and whose zero chunks mostly coincide, so the lanes skip them together).
// Persistent: as many CTAs as are resident, each warp taking 32 items at a
// time from the probe's counter, so no warp waits for the slowest of its
// CTA and the last wave is not left part-empty.
__global__ void __launch_bounds__(kCostThreads, 6) k_cost(EncodeLaunch e, int step) {
    __shared__ LenTables t;
    t.fill();
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t items = 3u * e.n_slices;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(e.cost_taken + step, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= items) break;
        const uint32_t item = base + lane;
        if (item >= items) continue;
        const uint32_t comp = item / e.n_slices, s = item - comp * e.n_slices;
        const EncSliceDesc sd = e.slices[s];
        const int32_t qi = e.state[sd.pic].probe_qi;
        if (qi == 0) continue;
        const EncPicDesc &pd = e.pics[sd.pic];
        const EncFrameDesc &fd = e.frames[pd.frame];
        e.probe_comp[((uint64_t)step * e.n_slices + s) * 3u + comp] =
            component_bytes(e, sd, pd, fd, comp, (uint32_t)qi, t);
    }
}

// k_cost with a warp per item, for batches too small to fill the GPU with
// one lane per item.
__global__ void __launch_bounds__(kCostThreads) k_cost_warp(EncodeLaunch e, int step) {
    __shared__ LenTables t;
    t.fill();
    __syncthreads();
    const uint32_t item = blockIdx.x * (kCostThreads / 32) + (threadIdx.x >> 5);
    if (item >= 3u * e.n_slices) return;
    const uint32_t s = item / 3u, comp = item - 3u * s;
    const EncSliceDesc sd = e.slices[s];
    const int32_t qi = e.state[sd.pic].probe_qi;
    if (qi == 0) return;
    const EncPicDesc &pd = e.pics[sd.pic];
    const EncFrameDesc &fd = e.frames[pd.frame];
    const uint32_t bytes = warp_component_bytes(e, sd, pd, fd, comp, (uint32_t)qi, t);
    if ((threadIdx.x & 31) == 0) e.probe_comp[((uint64_t)step * e.n_slices + s) * 3u + comp] = bytes;
}

// A slice's size from its component bytes, and whether every 16-bit size
// field holds it (src/encode.rs:671-681).
__device__ __forceinline__ uint64_t slice_total(uint32_t hdr, const uint32_t c[3], uint32_t alpha, bool &fits) {
    const uint64_t t = (uint64_t)hdr + c[0] + c[1] + c[2] + alpha;
    fits = t <= 65535u && c[0] <= 65535u && c[1] <= 65535u && c[2] <= 65535u;
    return t;
}

// Macroblocks from slice (mb_x, mb_y) to the end of the picture: the
// share-out's remaining_mbs (src/encode.rs:737-741, :771).
__device__ __forceinline__ uint64_t mbs_from(const EncPicDesc &pd, const EncSliceDesc &sd) {
    return (uint64_t)pd.width_in_mb * pd.height_in_mb - ((uint64_t)sd.mb_y * pd.width_in_mb + sd.mb_x);
}

// The probe step that costed quantiser qi for this picture, or -1. The crate
// reuses only the probe at uniform - 1 (src/encode.rs:743-749) and costs
// the later window levels afresh; a size is a function of the slice and
// the quantiser alone, so reusing any probe at a window's quantiser gives
// the same sizes and changes no choice.
__device__ __forceinline__ int probe_step_for(const EncPicState &st, int32_t qi) {
#pragma unroll
    for (int k = 0; k < kProbeSteps; k++)
        if (qi >= 1 && st.step_qi[k] == (uint32_t)qi) return k;
    return -1;
}

// Component sizes at window level j (quantiser uniform - 1 - j) of slice s:
// from a probe at that quantiser when there is one, else the window.
__device__ __forceinline__ const uint32_t *level_comp(const EncodeLaunch &e, const EncPicState &st, uint32_t j,
                                                      uint32_t s) {
    const int step = probe_step_for(st, st.uniform - 1 - (int32_t)j);
    if (step >= 0) return e.probe_comp + ((uint64_t)step * e.n_slices + s) * 3u;
    return e.win_comp + ((uint64_t)j * e.n_slices + s) * 3u;
}

// The slices whose window level is costed, as a list: level 0 takes every
// slice of a picture that has finer quantisers to share out; a later level
// the slices (at no level that a probe sized already)
// whose size at the level before fits and is within the most their share
// can come to (the crate's prefetch rule, src/encode.rs:741-767). The list
// order is the atomics' and steers nothing but speed.
__global__ void __launch_bounds__(kCostThreads) k_window_select(EncodeLaunch e, int level) {
    const uint32_t s = blockIdx.x * kCostThreads + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool take = false;
    if (s < e.n_slices) {
        const EncSliceDesc sd = e.slices[s];
        const EncPicState st = e.state[sd.pic];
        const int32_t qi = st.uniform - 1 - level;
        if (st.fits_at_all && st.uniform > 1 && qi >= 1 && probe_step_for(st, qi) < 0) {
            take = true;
            if (level > 0) {
                const EncPicDesc &pd = e.pics[sd.pic];
                const uint32_t *prev = level_comp(e, st, (uint32_t)level - 1u, s);
                take = prev[0] != kNotCosted;
                if (take) {
                    const uint32_t alpha = e.alpha_bytes[s];
                    const uint32_t pc[3] = {prev[0], prev[1], prev[2]};
                    bool fits, f2;
                    const uint64_t n = slice_total(pd.header_bytes, pc, alpha, fits);
                    const uint32_t *u = e.probe_comp + ((uint64_t)st.hi_probe * e.n_slices + s) * 3u;
                    const uint32_t uc[3] = {u[0], u[1], u[2]};
                    const uint64_t used = slice_total(pd.header_bytes, uc, alpha, f2);
                    const uint64_t slack = st.budget - st.hi_total;
                    const uint64_t most = used + slack * sd.mbs / mbs_from(pd, sd);
                    take = fits && n <= most;
                }
                if (!take) e.win_comp[((uint64_t)level * e.n_slices + s) * 3u] = kNotCosted;
            }
        }
    }
    const uint32_t m = __ballot_sync(0xffffffffu, take);
    if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t at = 0;
        if (lane == leader) at = atomicAdd(e.win_count + level, (uint32_t)__popc(m));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (take) e.win_list[at + __popc(m & ((1u << lane) - 1u))] = s;
    }
}

// Costs the listed slices at window level `level` (quantiser uniform - 1 -
// level): a lane per (component, slice), component-major, or a warp each.
// Lanes per component in the window levels' lane mode: these launches cover
// candidate lists, too short to fill the GPU, so a component's walk is
// split to cut the launch's length.
constexpr int kWindowSegments = 4;

template <bool kWarp>
__global__ void __launch_bounds__(kCostThreads) k_cost_window(EncodeLaunch e, int level) {
    __shared__ LenTables t;
    const uint32_t n = e.win_count[level];
    if (blockIdx.x * (kWarp ? kCostThreads / 32 : kCostThreads / kWindowSegments) >= 3u * n) return;  // the whole block
    t.fill();
    __syncthreads();
    if (kWarp) {
        const uint32_t item = blockIdx.x * (kCostThreads / 32) + (threadIdx.x >> 5);
        if (item >= 3u * n) return;
        const uint32_t comp = item % 3u, s = e.win_list[item / 3u];
        const EncSliceDesc sd = e.slices[s];
        const uint32_t qi = (uint32_t)(e.state[sd.pic].uniform - 1 - level);
        const EncPicDesc &pd = e.pics[sd.pic];
        const uint32_t bytes = warp_component_bytes(e, sd, pd, e.frames[pd.frame], comp, qi, t);
        if ((threadIdx.x & 31) == 0) e.win_comp[((uint64_t)level * e.n_slices + s) * 3u + comp] = bytes;
    } else {
        const uint32_t thread = blockIdx.x * kCostThreads + threadIdx.x;
        if ((thread & ~31u) / kWindowSegments >= 3u * n) return;  // the whole warp
        const uint32_t item = thread / kWindowSegments;
        const bool active = item < 3u * n;
        const uint32_t comp = active ? item / n : 0u;
        const uint32_t s = e.win_list[active ? item - comp * n : 0u];
        const EncSliceDesc sd = e.slices[s];
        const uint32_t qi = active ? (uint32_t)(e.state[sd.pic].uniform - 1 - level) : 1u;
        const EncPicDesc &pd = e.pics[sd.pic];
        const EncFrameDesc &fd = e.frames[pd.frame];
        uint32_t nb, off;
        comp_layout(fd, sd.mbs, comp, nb, off);
        const uint32_t bits = group_component_bits<kWindowSegments>(active, e.coef + sd.coef + off,
                                                                    e.coef_max + ((sd.coef + off) >> 5), nb,
                                                                    comp_quant(quant_base(e, pd, qi), comp, nb), t);
        if (active && thread % kWindowSegments == 0)
            e.win_comp[((uint64_t)level * e.n_slices + s) * 3u + comp] = (bits + 7u) / 8u;
    }
}

// The levels past the window, costed ahead of the share-out, a warp per
// slice, every slice at once: a slice whose last window level fits and is
// within its likely allowance goes on to the next finer quantiser, and so
// on while the size it just found fits and stays within that allowance,
// for up to kDeepLevels levels. A slice's ladder depends on nothing but its
// own sizes and its picture's slack, so the slices need not wait for one
// another; the share-out then reads these sizes instead of costing them one
// slice after another (which it still does for a level past the ladder).
//
// The likely allowance is the slice's share of the picture's slack in
// proportion to its macroblocks, plus a quarter, plus one step (its size
// change a finer quantiser, as estimated below), and never above the most
// its share can come to (the crate's prefetch rule: the whole slack from
// the slice on, if no slice before it took any). For a slice whose step is
// under a quarter of its share it is that most, and so it is, for at most
// kTailLevels levels, for a picture's last kTailSlices slices. The
// share-out's allowance for a slice is what the slices before it left,
// which stays near the proportional share but for the last slices of a
// picture; the most is far above it there (the last slice's is the whole
// slack), and a ladder to the most for every slice costed several
// quantisers of every slice of a picture's tail for nothing. What the
// ladder leaves out only moves work to the share-out, never changes a
// size.
constexpr uint32_t kTailSlices = 16;  // a picture's tail: slices within this many slices' macroblocks of its end
constexpr uint32_t kTailLevels = 4;

__global__ void __launch_bounds__(kCostThreads) k_cost_deep(EncodeLaunch e) {
    __shared__ LenTables t;
    t.fill();
    __syncthreads();
    const uint32_t s = blockIdx.x * (kCostThreads / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= e.n_slices) return;
    const EncSliceDesc sd = e.slices[s];
    const EncPicState st = e.state[sd.pic];
    uint32_t count = 0;
    if (st.fits_at_all && st.uniform - kWindow > 1) {
        const EncPicDesc &pd = e.pics[sd.pic];
        const EncFrameDesc &fd = e.frames[pd.frame];
        const uint32_t hb = pd.header_bytes, alpha = e.alpha_bytes[s];
        const uint32_t *u = e.probe_comp + ((uint64_t)st.hi_probe * e.n_slices + s) * 3u;
        const uint32_t uc[3] = {u[0], u[1], u[2]};
        bool f0;
        const uint64_t used = slice_total(hb, uc, alpha, f0);
        const uint64_t slack = st.budget - st.hi_total;
        const uint64_t most = used + slack * sd.mbs / mbs_from(pd, sd);
        const uint64_t share = slack * sd.mbs / ((uint64_t)pd.width_in_mb * pd.height_in_mb);
        const uint32_t *c = level_comp(e, st, kWindow - 1, s);
        bool fits = false;
        uint64_t n = ~0ull;
        if (c[0] != kNotCosted) {
            const uint32_t cc[3] = {c[0], c[1], c[2]};
            n = slice_total(hb, cc, alpha, fits);
        }
        // The slice's step: its size change a finer quantiser, the larger of
        // the first step and the mean of the window's next three (the first
        // can be far larger than the rest: above quantiser index 128 a step
        // of the index is 4 of qScale, below it 1).
        const uint32_t *c1 = level_comp(e, st, 0, s);
        uint64_t step = 0, n1 = 0;
        if (c1[0] != kNotCosted) {
            const uint32_t cc[3] = {c1[0], c1[1], c1[2]};
            bool f1;
            n1 = slice_total(hb, cc, alpha, f1);
            step = n1 > used ? n1 - used : 0u;
            if (c[0] != kNotCosted) step = min(step, n > n1 ? (n - n1) / (uint64_t)(kWindow - 1) : 0u);
        }
        // A slice whose step is small beside its share (a coarse quantiser,
        // where a step often changes no size) walks many levels wherever its
        // allowance lands: its ladder goes to the most. So do the last slices
        // of a picture, where what the slices before left gathers, for at
        // most kTailLevels levels.
        const bool coarse = 4u * step <= share;
        const bool tail = mbs_from(pd, sd) <= (uint64_t)kTailSlices * sd.mbs;
        const uint64_t likely = coarse || tail ? most : min(most, used + share + share / 4u + step);
        const uint32_t levels = coarse ? (uint32_t)kDeepLevels : (tail ? kTailLevels : (uint32_t)kDeepLevels);
        for (uint32_t j = 0; fits && n <= likely && j < levels; j++) {
            const int32_t qi = st.uniform - 1 - kWindow - (int32_t)j;
            if (qi < 1) break;
            uint32_t c3[3];
            for (uint32_t comp = 0; comp < 3; comp++) c3[comp] = warp_component_bytes(e, sd, pd, fd, comp, (uint32_t)qi, t);
            n = slice_total(hb, c3, alpha, fits);
            if (lane == 0)
                e.deep[(uint64_t)s * kDeepLevels + j] =
                    make_uint2(min(c3[0], 65535u) | (min(c3[1], 65535u) << 16), min(c3[2], 65535u) | ((fits ? 1u : 0u) << 16));
            count = j + 1;
        }
    }
    if (lane == 0) e.deep_count[s] = count;
}

constexpr int kRcThreads = 256;

__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v, uint64_t *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    uint64_t t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
    return t;
}

__global__ void __launch_bounds__(kRcThreads) k_rc_init(EncodeLaunch e) {
    __shared__ uint64_t sh[kRcThreads / 32];
    const EncPicDesc pd = e.pics[blockIdx.x];
    uint64_t a = 0;
    for (uint32_t k = threadIdx.x; k < pd.n_slices; k += kRcThreads) a += e.alpha_bytes[pd.slice_base + k];
    const uint64_t alpha = block_sum_u64(a, sh);
    if (threadIdx.x == 0) {
        // Alpha is lossless and comes on top of the rate; the picture
        // header and the slice table come out of it (src/encode.rs:686-689).
        const uint64_t overhead = 8u + 2ull * pd.n_slices;
        const uint64_t b = pd.budget_in + alpha;
        EncPicState st{};
        st.budget = b > overhead ? b - overhead : 0;
        st.lo = 1;
        st.hi = 224;
        st.probe_qi = 224;
        st.hi_probe = 0;
        st.lo_probe = -1;
        st.fits_at_all = 0;
        st.uniform = 224;
        e.state[blockIdx.x] = st;
        if (blockIdx.x == 0) {
            for (int j = 0; j < kWindow; j++) e.win_count[j] = 0;
            for (int j = 0; j < kProbeSteps; j++) e.cost_taken[j] = 0;
        }
    }
}

__global__ void __launch_bounds__(kRcThreads) k_rc_step(EncodeLaunch e, int step) {
    __shared__ uint64_t sh[kRcThreads / 32];
    __shared__ int all_fit;
    const EncPicDesc pd = e.pics[blockIdx.x];
    const EncPicState st0 = e.state[blockIdx.x];
    if (st0.probe_qi == 0) return;
    if (threadIdx.x == 0) all_fit = 1;
    __syncthreads();
    uint64_t sum = 0;
    bool fit = true;
    for (uint32_t k = threadIdx.x; k < pd.n_slices; k += kRcThreads) {
        const uint32_t s = pd.slice_base + k;
        const uint32_t *c = e.probe_comp + ((uint64_t)step * e.n_slices + s) * 3u;
        const uint32_t cc[3] = {c[0], c[1], c[2]};
        bool f;
        sum += slice_total(pd.header_bytes, cc, e.alpha_bytes[s], f);
        fit = fit && f;
    }
    if (!fit) all_fit = 0;
    const uint64_t total = block_sum_u64(sum, sh);
    if (threadIdx.x == 0) {
        EncPicState st = st0;
        st.step_qi[step] = (uint8_t)st.probe_qi;
        const bool ok = all_fit && total <= st.budget;
        if (step == 0) {
            // totals(224): if even the coarsest quantiser does not fit, it is
            // used throughout (src/encode.rs:701-713).
            st.fits_at_all = ok;
            st.hi_probe = 0;
            st.hi_total = total;
            if (!ok) {
                st.probe_qi = 0;
                st.uniform = 224;
            }
        } else if (ok) {
            st.hi = st.probe_qi;
            st.hi_probe = step;
            st.hi_total = total;
        } else {
            st.lo = st.probe_qi + 1;
            st.lo_probe = step;
        }
        if (st.fits_at_all) {
            if (st.lo < st.hi) {
                st.probe_qi = st.lo + (st.hi - st.lo) / 2;
            } else {
                st.probe_qi = 0;
                st.uniform = st.hi;
            }
        }
        e.state[blockIdx.x] = st;
    }
}

// The share-out (src/encode.rs:769-793). With D = remaining_budget -
// remaining_base, slice i steps from the uniform quantiser to the next finer
// one while that size n fits and n <= base + floor(D mbs / remaining_mbs),
// i.e. while n <= base or D >= ceil((n - base) remaining_mbs / mbs); D then
// falls by what the slice took over its base. Three kernels:
//   k_share_prep   every slice in parallel: its base and, for each window
//                  level, the threshold on D and the size over the base;
//   k_shareout     one warp per picture, the only serial part: D against
//                  the thresholds (the window's, then each slice's deep
//                  ladder from k_cost_deep), 32 slices at a time by ballot,
//                  each stepping slice settled by its own lane; the warp
//                  costs a deeper quantiser together when a slice gets past
//                  all of them;
//   k_share_final  every slice in parallel: its quantiser and sizes.
constexpr uint32_t kDeepFlag = 0x80000000u;  // share_steps: sizes are in final_comp already

__global__ void k_share_prep(EncodeLaunch e) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.n_slices) return;
    const EncSliceDesc sd = e.slices[s];
    const EncPicState st = e.state[sd.pic];
    SharePrep pr{};
    if (st.uniform > 1 && st.fits_at_all) {
        const EncPicDesc &pd = e.pics[sd.pic];
        const uint32_t hb = pd.header_bytes, alpha = e.alpha_bytes[s];
        const uint32_t *u = e.probe_comp + ((uint64_t)st.hi_probe * e.n_slices + s) * 3u;
        const uint32_t uc[3] = {u[0], u[1], u[2]};
        bool f;
        const uint64_t base = slice_total(hb, uc, alpha, f);
        const uint64_t rem = mbs_from(pd, sd);
        const uint32_t shift = 31u - __clz(sd.mbs);
        pr.base = (uint32_t)base;
        pr.hba = hb + alpha;
        pr.rem = (uint32_t)rem;
        pr.shift = shift;
        pr.deep_count = e.deep_count[s];
#pragma unroll
        for (int j = 0; j < kWindow; j++) {
            pr.thr[j] = ~0ull;
            if (st.uniform - j <= 1) continue;
            const uint32_t *c = level_comp(e, st, (uint32_t)j, s);
            if (c[0] == kNotCosted) continue;  // unknown: the walk costs it if reached
            const uint32_t cc[3] = {c[0], c[1], c[2]};
            bool fits;
            const uint64_t n = slice_total(hb, cc, alpha, fits);
            pr.known |= 1u << j;
            pr.delta[j] = (int32_t)((int64_t)n - (int64_t)base);
            if (fits) pr.thr[j] = n <= base ? 0ull : ((((n - base) * rem) + sd.mbs - 1) >> shift);
        }
    }
    e.share_prep[s] = pr;
}

// A level past the window from a slice's deep ladder: its size, and whether
// it fits.
__device__ __forceinline__ uint64_t deep_size(const SharePrep &p, uint2 v, bool &fits) {
    fits = (v.y >> 16) != 0;
    return (uint64_t)p.hba + (v.x & 0xFFFFu) + (v.x >> 16) + (v.y & 0xFFFFu);
}

// The steps a slice takes at D through its known levels (the walk of
// src/encode.rs:776-788 while the sizes are known: the window's, then its
// deep ladder, level j at deep[32 j]), as a table the share-out searches
// each time it settles the slice: at [32 k] the least D that lets the
// slice take k + 1 steps given that it took k (~0 where the level does not
// fit), made non-decreasing (a running maximum), so that the steps at D are
// the number of entries <= D; `len` is where the walk stops whatever D is,
// and `deep_at_end` whether it then needs a level nobody costed.
__device__ __forceinline__ void steps_table(const SharePrep &p, const uint2 *deep, int32_t uniform, uint64_t *tab,
                                            uint32_t &len, bool &deep_at_end) {
    uint64_t run = 0;
    uint32_t k = 0;
    deep_at_end = false;
#pragma unroll
    for (int j = 0; j < kWindow; j++) {
        // k == j steps so far: the quantiser is uniform - j.
        if (uniform - j <= 1) {
            len = k;
            return;
        }
        if (!((p.known >> j) & 1u)) {
            len = k;
            deep_at_end = true;
            return;
        }
        run = max(run, p.thr[j]);
        tab[32u * k] = run;
        k++;
    }
    for (uint32_t j = 0; j < p.deep_count; j++) {
        if (uniform - (int32_t)k <= 1) {
            len = k;
            return;
        }
        bool fits;
        const uint64_t n = deep_size(p, deep[32u * j], fits);
        const uint64_t thr =
            !fits ? ~0ull : (n <= p.base ? 0ull : (((n - p.base) * p.rem) + (1u << p.shift) - 1u) >> p.shift);
        run = max(run, thr);
        tab[32u * k] = run;
        k++;
    }
    len = k;
    deep_at_end = uniform - (int32_t)k > 1;
}

// The steps at D from steps_table(): a binary search.
__device__ __forceinline__ uint32_t steps_from(const uint64_t *tab, uint32_t len, bool deep_at_end, uint64_t D,
                                               bool &deep_needed) {
    uint32_t lo = 0, hi = len;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tab[32u * mid] <= D)
            lo = mid + 1u;
        else
            hi = mid;
    }
    deep_needed = lo == len && deep_at_end;
    return lo;
}

// The size over the base after `ks` steps (ks >= 1).
__device__ __forceinline__ int64_t delta_at(const SharePrep &p, const uint2 *deep, uint32_t ks) {
    if (ks <= (uint32_t)kWindow) {
        int32_t d = p.delta[0];
#pragma unroll
        for (int j = 1; j < kWindow; j++)
            if ((uint32_t)j + 1u == ks) d = p.delta[j];
        return d;
    }
    bool fits;
    return (int64_t)deep_size(p, deep[32u * (ks - 1u - kWindow)], fits) - (int64_t)p.base;
}

constexpr int kShareWarps = 1;
// A warp's staged ladders and steps tables.
constexpr uint32_t kShareLadderBytes = 32u * kDeepLevels * sizeof(uint2) + 32u * (kWindow + kDeepLevels) * sizeof(uint64_t);

__global__ void __launch_bounds__(32 * kShareWarps) k_shareout(EncodeLaunch e) {
    __shared__ LenTables t;
    // The slice a deep step costs, copied in once (its coefficients, then
    // its chunk maxima): the warp walks it for every quantiser it tries,
    // and from DRAM each of its chunks waited out a full load.
    __shared__ __align__(16) float stage[kShareWarps][kMaxSliceCoefs + kMaxSliceCoefs / 32];
    // The ladders of the 32 slices a warp settles, level j of lane l at
    // [32 j + l] (dynamic shared memory, kShareLadderBytes a warp): the
    // settling rounds walk them again and again, and from global memory
    // every level of the walk was a dependent load.
    extern __shared__ uint2 ladders_all[];
    uint2 *const ladders = ladders_all + (threadIdx.x >> 5) * (32u * kDeepLevels);
    // Each lane's steps_table(), [32 k + lane], after all warps' ladders.
    uint64_t *const tables = reinterpret_cast<uint64_t *>(ladders_all + kShareWarps * 32u * kDeepLevels) +
                             (threadIdx.x >> 5) * (32u * (kWindow + kDeepLevels));
    t.fill();
    __syncthreads();
    const uint32_t p = blockIdx.x * kShareWarps + (threadIdx.x >> 5);
    if (p >= e.n_pics) return;
    const int lane = threadIdx.x & 31;
    const EncPicDesc pd = e.pics[p];
    const EncPicState st = e.state[p];
    const bool refine = st.uniform > 1 && st.fits_at_all;
    if (!refine) {
        for (uint32_t k = lane; k < pd.n_slices; k += 32) e.share_steps[pd.slice_base + k] = 0;
        return;
    }
    const EncFrameDesc &fd = e.frames[pd.frame];
    const uint32_t hb = pd.header_bytes;
    uint64_t D = st.budget - st.hi_total;
    SharePrep next{};
    if ((uint32_t)lane < pd.n_slices) next = e.share_prep[pd.slice_base + lane];
    for (uint32_t k0 = 0; k0 < pd.n_slices; k0 += 32) {
        const SharePrep mine = next;
        const uint32_t k = k0 + lane;
        const bool live = k < pd.n_slices;
        uint2 *my_deep = ladders + lane;
        __syncwarp();  // the last chunk's walks are over
        if (live) {
            const uint2 *src = e.deep + (uint64_t)(pd.slice_base + k) * kDeepLevels;
#pragma unroll 4
            for (uint32_t j = 0; j < mine.deep_count; j++) my_deep[32u * j] = src[j];
        }
        uint32_t my_len = 0;
        bool my_deep_at_end = false;
        if (live) steps_table(mine, my_deep, st.uniform, tables + lane, my_len, my_deep_at_end);
        __syncwarp();
        // The next chunk's thresholds, fetched while this chunk is walked.
        if (k + 32 < pd.n_slices) next = e.share_prep[pd.slice_base + k + 32];
        uint32_t my_steps = 0;
        uint32_t done = 0;  // lanes below are settled
        while (done < 32u) {
            // The walk is sequential: a slice's slack D is what the slices
            // before it left. Each lane guesses its D, takes its steps there,
            // and the guesses are redone from the exclusive sum of the steps'
            // size changes until none moves. A lane's D depends only on the
            // lanes before it, so after t rounds the first t lanes are exact
            // and the fixed point reached (at most 33 rounds) is the
            // sequential walk's. Lanes from the first one that needs a level
            // nobody costed (`deep`) on wait for the warp to cost it.
            uint64_t myD = D;
            uint32_t ks = 0;
            int64_t dl = 0;
            uint32_t first_deep = 32;
            for (int round = 0; round < 34; round++) {
                bool deep = false;
                ks = live && (uint32_t)lane >= done ? steps_from(tables + lane, my_len, my_deep_at_end, myD, deep) : 0u;
                const uint32_t deep_mask = __ballot_sync(0xffffffffu, live && (uint32_t)lane >= done && deep);
                const uint32_t fd_lane = deep_mask ? (uint32_t)__ffs(deep_mask) - 1u : 32u;
                const int64_t mine_dl = ks ? delta_at(mine, my_deep, ks) : 0;
                dl = (uint32_t)lane < fd_lane ? mine_dl : 0;
                // Inclusive sum of dl over the lanes.
                int64_t incl = dl;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int64_t v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const uint64_t newD = (uint64_t)((int64_t)D - (incl - dl));
                const bool moved = (uint32_t)lane >= done && (uint32_t)lane <= fd_lane && newD != myD;
                myD = newD;
                const bool again = __any_sync(0xffffffffu, moved) || fd_lane != first_deep;
                first_deep = fd_lane;
                if (!again) break;
            }
            // Lanes done .. first_deep - 1 are settled at myD with ks steps.
            if ((uint32_t)lane >= done && (uint32_t)lane < first_deep) my_steps = ks;
            const int64_t settled = __shfl_sync(0xffffffffu, (int64_t)D - (int64_t)myD, first_deep < 32u ? first_deep : 31u);
            if (first_deep >= 32u) {
                // Every lane settled: D after the chunk.
                const int64_t total = __shfl_sync(0xffffffffu, (int64_t)D - (int64_t)myD + dl, 31);
                D = (uint64_t)((int64_t)D - total);
                break;
            }
            // The deep lane, at its exact D: the warp costs quantiser qi - 1
            // and the slice steps while it fits its allowance (fixed during
            // the slice's walk).
            D = (uint64_t)((int64_t)D - settled);
            const uint32_t f = first_deep;
            const uint32_t fk = __shfl_sync(0xffffffffu, ks, f);
            const int64_t my_delta = ks ? delta_at(mine, my_deep, ks) : 0;
            int64_t delta = __shfl_sync(0xffffffffu, my_delta, f);
            uint32_t steps = fk;
            {
                const uint32_t s = pd.slice_base + k0 + f;
                const EncSliceDesc fsd = e.slices[s];
                const uint32_t fbase = __shfl_sync(0xffffffffu, mine.base, f);
                const uint32_t alpha = e.alpha_bytes[s];
                const uint64_t allowed = fbase + D * fsd.mbs / mbs_from(pd, fsd);
                uint32_t c3[3] = {0, 0, 0};
                int32_t qi = st.uniform - (int32_t)fk;
                bool any = false;
                float *sf = stage[threadIdx.x >> 5], *smax = sf + kMaxSliceCoefs;
                const uint32_t cpm = fd.chroma == 2 ? 2u : 4u;
                const uint32_t total = 64u * (4u + 2u * cpm) * fsd.mbs;
                if (qi > 1) {
                    __syncwarp();  // the last deep slice's walks are over
                    const float4 *src = reinterpret_cast<const float4 *>(e.coef + fsd.coef);
#pragma unroll 4
                    for (uint32_t i = (uint32_t)lane; i < total / 4u; i += 32u)
                        reinterpret_cast<float4 *>(sf)[i] = __ldg(src + i);
                    const float *msrc = e.coef_max + (fsd.coef >> 5);
                    for (uint32_t i = (uint32_t)lane; i < total / 32u; i += 32u) smax[i] = __ldg(msrc + i);
                    __syncwarp();
                }
                while (qi > 1) {
                    uint32_t n3[3];
                    for (uint32_t c = 0; c < 3; c++) {
                        uint32_t nb, off;
                        comp_layout(fd, fsd.mbs, c, nb, off);
                        const CompQuant q = comp_quant(quant_base(e, pd, (uint32_t)(qi - 1)), c, nb);
                        n3[c] = (warp_component_bits<true>(sf + off, smax + (off >> 5), nb, q, t) + 7u) / 8u;
                    }
                    bool fits;
                    const uint64_t n = slice_total(hb, n3, alpha, fits);
                    if (!(fits && n <= allowed)) break;
                    qi -= 1;
                    steps++;
                    delta = (int64_t)n - (int64_t)fbase;
                    c3[0] = n3[0];
                    c3[1] = n3[1];
                    c3[2] = n3[2];
                    any = true;
                }
                if (any && lane == 0) {
                    e.final_comp[3ull * s] = c3[0];
                    e.final_comp[3ull * s + 1] = c3[1];
                    e.final_comp[3ull * s + 2] = c3[2];
                    steps |= kDeepFlag;
                }
                steps = __shfl_sync(0xffffffffu, steps, 0);
            }
            if (lane == (int)f) my_steps = steps;
            D = (uint64_t)((int64_t)D - delta);
            done = f + 1;
        }
        if (live) e.share_steps[pd.slice_base + k] = my_steps;
    }
}

__global__ void k_share_final(EncodeLaunch e) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.n_slices) return;
    const EncSliceDesc sd = e.slices[s];
    const EncPicState st = e.state[sd.pic];
    const uint32_t steps = e.share_steps[s];
    const uint32_t n = steps & ~kDeepFlag;
    e.final_qi[s] = (uint32_t)st.uniform - n;
    if (steps & kDeepFlag) return;  // written by the walk
    if (n > (uint32_t)kWindow) {
        // From the slice's deep ladder (a level the slice fits at, so no
        // size there is saturated).
        const uint2 v = e.deep[(uint64_t)s * kDeepLevels + (n - 1u - kWindow)];
        e.final_comp[3ull * s] = v.x & 0xFFFFu;
        e.final_comp[3ull * s + 1] = v.x >> 16;
        e.final_comp[3ull * s + 2] = v.y & 0xFFFFu;
        return;
    }
    const uint32_t *c = n == 0 ? e.probe_comp + ((uint64_t)st.hi_probe * e.n_slices + s) * 3u
                               : level_comp(e, st, n - 1u, s);
    e.final_comp[3ull * s] = c[0];
    e.final_comp[3ull * s + 1] = c[1];
    e.final_comp[3ull * s + 2] = c[2];
}

// ---------------------------------------------------------------- layout

constexpr int kLayoutThreads = 1024;

__device__ __forceinline__ uint64_t warp_incl_scan64(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Slice offsets within the picture (after its header and table) and the
// picture's size (src/encode.rs:820-829).
__global__ void __launch_bounds__(kLayoutThreads) k_layout(EncodeLaunch e) {
    __shared__ uint64_t warp_sums[kLayoutThreads / 32];
    __shared__ uint64_t carry;
    const EncPicDesc pd = e.pics[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 8u + 2ull * pd.n_slices;
    __syncthreads();
    for (uint32_t chunk = 0; chunk < pd.n_slices; chunk += kLayoutThreads) {
        const uint32_t k = chunk + threadIdx.x;
        uint64_t size = 0;
        if (k < pd.n_slices) {
            const uint32_t s = pd.slice_base + k;
            const uint32_t cc[3] = {e.final_comp[3ull * s], e.final_comp[3ull * s + 1], e.final_comp[3ull * s + 2]};
            bool f;
            size = slice_total(pd.header_bytes, cc, e.alpha_bytes[s], f);
        }
        const uint64_t incl = warp_incl_scan64(size);
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) warp_sums[lane] = warp_incl_scan64(warp_sums[lane]);
        __syncthreads();
        const uint64_t excl = carry + (warp ? warp_sums[warp - 1] : 0u) + incl - size;
        if (k < pd.n_slices) e.slice_off[pd.slice_base + k] = excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sums[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) e.state[blockIdx.x].pic_size = carry;
}

// Picture places and sizes, the frame header and frame_size, the picture
// headers (src/header.rs:174-199, :292-304). One thread per frame.
__global__ void k_frame(EncodeLaunch e) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= e.n_frames) return;
    const EncFrameDesc fd = e.frames[f];
    uint64_t pos = fd.header_len;
    for (uint32_t i = 0; i < fd.n_pics; i++) {
        e.state[fd.first_pic + i].pic_off = pos;
        pos += e.state[fd.first_pic + i].pic_size;
    }
    e.frame_size[f] = pos;
    const bool over = pos > fd.out_cap;
    e.frame_status[f] = over ? 1u : 0u;
    if (over) return;
    const uint64_t base = fd.out_base * 8u;
    const uint8_t *h = e.headers + (uint64_t)kHeaderSlot * fd.header_slot;
    put_field(e.out, base, (uint32_t)pos, 32);  // frame_size
    for (uint32_t b = 4; b < fd.header_len; b++) put_field(e.out, base + 8ull * b, h[b], 8);
    for (uint32_t i = 0; i < fd.n_pics; i++) {
        const EncPicDesc &pd = e.pics[fd.first_pic + i];
        const EncPicState &st = e.state[fd.first_pic + i];
        const uint64_t at = base + 8ull * st.pic_off;
        put_field(e.out, at, 8u << 3, 8);
        put_field(e.out, at + 8, (uint32_t)st.pic_size, 32);
        put_field(e.out, at + 40, pd.n_slices <= 65535u ? pd.n_slices : 0u, 16);
        put_field(e.out, at + 56, (pd.log2_slice_mbs & 3u) << 4, 8);
    }
}

// ---------------------------------------------------------------- packing

// An MSB-first writer into the big-endian output words from an absolute
// bit position. Words wholly inside the writer's bytes are stored; the
// partial words at either end, which a neighbour shares, are OR-ed.
struct BitOut {
    uint32_t *out;
    uint64_t cur;  // absolute position of the first bit held
    uint64_t acc;
    uint32_t nacc;
    __device__ __forceinline__ void init(uint32_t *o, uint64_t bitpos) {
        out = o;
        cur = bitpos;
        acc = 0;
        nacc = 0;
    }
    __device__ __forceinline__ void emit() {
        for (;;) {
            const uint32_t room = 32u - (uint32_t)(cur & 31u);
            if (nacc < room) return;
            const uint32_t chunk = (uint32_t)(acc >> (nacc - room)) & (room == 32u ? 0xFFFFFFFFu : ((1u << room) - 1u));
            uint32_t *w = out + (cur >> 5);
            if (room == 32u)
                *w = bswap32(chunk);
            else
                atomicOr(w, bswap32(chunk));
            nacc -= room;
            cur += room;
        }
    }
    // A field of n <= 32 bits holding v.
    __device__ __forceinline__ void put(uint64_t v, uint32_t n) {
        if (n == 0) return;
        acc = (acc << n) | v;
        nacc += n;
        emit();
    }
    // A field of any width holding v (its leading zeros included).
    __device__ __forceinline__ void put_long(uint64_t v, uint32_t n) {
        if (n > 64) {
            put(0, n - 64);
            n = 64;
        }
        if (n > 32) {
            put(v >> 32, n - 32);
            v &= 0xFFFFFFFFull;
            n = 32;
        }
        put(v, n);
    }
    // Zero bits to the next byte boundary, then the last partial word.
    __device__ __forceinline__ void finish() {
        const uint32_t pad = (uint32_t)((8u - ((cur + nacc) & 7u)) & 7u);
        put(0, pad);
        if (nacc) {
            const uint32_t room = 32u - (uint32_t)(cur & 31u);
            const uint32_t chunk = (uint32_t)(acc & ((1ull << nacc) - 1)) << (room - nacc);
            atomicOr(out + (cur >> 5), bswap32(chunk));
            cur += nacc;
            nacc = 0;
        }
    }
};

// The writer's tables: beside the code lengths, the codewords (their
// significant bits) of run and level symbols below 32 by context.
struct CodeTables : LenTables {
    uint32_t run_code[16][32];
    uint32_t level_code[9][32];
    __device__ void fill_all() {
        fill();
        for (uint32_t i = threadIdx.x; i < 16 * 32; i += blockDim.x)
            run_code[i >> 5][i & 31] = (uint32_t)cb_bits(run_book(i >> 5), i & 31);
        for (uint32_t i = threadIdx.x; i < 9 * 32; i += blockDim.x)
            level_code[i >> 5][i & 31] = (uint32_t)cb_bits(level_book(i >> 5), i & 31);
    }
};

// One quantised component's codes (src/encode.rs:413-437), one lane.
__device__ void lane_component_write(BitOut &w, const float *f, const float *cmax, uint32_t n_blocks,
                                     const CompQuant &q, const CodeTables &t) {
    const float inv0 = __ldg(q.inv);
    int32_t prev_dc = 0, prev_diff = 3;
    for (uint32_t i = 0; i < n_blocks; i++) {
        const int32_t q = quantise1(__ldg(f + i), inv0, 0.5f);
        Codebook cb;
        uint32_t sym;
        if (i == 0) {
            cb = kFirstDcBook;
            sym = signed_to_symbol(q);
        } else {
            const int32_t diff = (int32_t)((uint32_t)q - (uint32_t)prev_dc);
            cb = dc_book(prev_diff);
            sym = signed_to_symbol(prev_diff < 0 ? -diff : diff);
            prev_diff = diff;
        }
        w.put_long(cb_bits(cb, sym), cb_len(cb, sym));
        prev_dc = q;
    }
    ac_walk_sparse(f, cmax, n_blocks, q, [&](const AcWalk &a, uint32_t run, uint32_t level, bool neg) {
        // Run, level and sign in one field, from the tables, when they can.
        if (run < 32u && level < 32u) {
            const uint32_t rc = min(a.prev_run, 15u), lc = min(a.prev_level, 8u);
            const uint32_t rl = t.run[rc][run], ll = t.level[lc][level];
            if (rl + ll + 1u <= 32u) {
                w.put((((uint64_t)t.run_code[rc][run] << ll | t.level_code[lc][level]) << 1) | (uint64_t)neg,
                      rl + ll + 1u);
                return;
            }
        }
        const Codebook rb = run_book(a.prev_run), lb = level_book(a.prev_level);
        const uint32_t rl = t.run_len(a.prev_run, run), ll = t.level_len(a.prev_level, level);
        // Run, level and sign in one field when they fit.
        if (rl + ll + 1u <= 32u) {
            w.put((((cb_bits(rb, run) << ll) | cb_bits(lb, level)) << 1) | (uint64_t)neg, rl + ll + 1u);
        } else {
            w.put_long(cb_bits(rb, run), rl);
            w.put_long(cb_bits(lb, level), ll);
            w.put((uint64_t)neg, 1);
        }
    });
    w.finish();
}

// Each slice component's codes, one lane per (component, slice).
__global__ void __launch_bounds__(kCostThreads) k_pack(EncodeLaunch e) {
    __shared__ CodeTables t;
    t.fill_all();
    __syncthreads();
    const uint32_t item = blockIdx.x * kCostThreads + threadIdx.x;
    if (item >= 3u * e.n_slices) return;
    const uint32_t comp = item / e.n_slices, s = item - comp * e.n_slices;
    const EncSliceDesc sd = e.slices[s];
    const EncPicDesc &pd = e.pics[sd.pic];
    if (e.frame_status[pd.frame]) return;
    const EncFrameDesc &fd = e.frames[pd.frame];
    const EncPicState &st = e.state[sd.pic];
    uint64_t at = 8ull * (fd.out_base + st.pic_off + e.slice_off[s] + pd.header_bytes);
    for (uint32_t c = 0; c < comp; c++) at += 8ull * e.final_comp[3ull * s + c];
    uint32_t nb, off;
    comp_layout(fd, sd.mbs, comp, nb, off);
    BitOut w;
    w.init(e.out, at);
    lane_component_write(w, e.coef + sd.coef + off, e.coef_max + ((sd.coef + off) >> 5), nb,
                         comp_quant(quant_base(e, pd, e.final_qi[s]), comp, nb), t);
}

// Slice headers and table entries, one thread per slice; alpha codes, one
// warp per slice.
__global__ void k_pack_headers(EncodeLaunch e) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.n_slices) return;
    const EncSliceDesc sd = e.slices[s];
    const EncPicDesc &pd = e.pics[sd.pic];
    if (e.frame_status[pd.frame]) return;
    const EncFrameDesc &fd = e.frames[pd.frame];
    const EncPicState &st = e.state[sd.pic];
    const uint32_t comp[3] = {e.final_comp[3ull * s], e.final_comp[3ull * s + 1], e.final_comp[3ull * s + 2]};
    const uint32_t hb = pd.header_bytes;
    const uint64_t slice_bit = 8ull * (fd.out_base + st.pic_off + e.slice_off[s]);
    bool f;
    const uint64_t total = slice_total(hb, comp, e.alpha_bytes[s], f);
    // slice_header_size << 3, quantization_index, the component sizes (the
    // Cr size only with alpha); the slice table's entry.
    put_field(e.out, slice_bit, hb << 3, 8);
    put_field(e.out, slice_bit + 8, e.final_qi[s], 8);
    put_field(e.out, slice_bit + 16, comp[0] & 0xFFFFu, 16);
    put_field(e.out, slice_bit + 32, comp[1] & 0xFFFFu, 16);
    if (hb == 8) put_field(e.out, slice_bit + 48, comp[2] & 0xFFFFu, 16);
    const uint64_t table_bit = 8ull * (fd.out_base + st.pic_off + 8u + 2ull * (s - pd.slice_base));
    put_field(e.out, table_bit, (uint32_t)(total & 0xFFFFu), 16);
}

__global__ void __launch_bounds__(32 * kAlphaWarps) k_pack_alpha(EncodeLaunch e) {
    __shared__ AlphaScratch scratch[kAlphaWarps];
    const uint32_t s = blockIdx.x * kAlphaWarps + (threadIdx.x >> 5);
    if (s >= e.n_slices) return;
    const EncSliceDesc sd = e.slices[s];
    const EncPicDesc &pd = e.pics[sd.pic];
    const EncFrameDesc &fd = e.frames[pd.frame];
    if (!fd.alpha_bits || e.frame_status[pd.frame]) return;
    const EncPicState &st = e.state[sd.pic];
    const uint32_t *c = e.final_comp + 3ull * s;
    const uint64_t at = 8ull * (fd.out_base + st.pic_off + e.slice_off[s] + pd.header_bytes + c[0] + c[1] + c[2]);
    alpha_write(e, sd, pd, fd, scratch[threadIdx.x >> 5], at);
}

}  // namespace

cudaError_t launch_fdct(const EncodeLaunch &e, cudaStream_t s) {
    if (!e.n_slices) return cudaSuccess;
    const uint32_t warps = 3u * e.n_slices, per_block = kFdctThreads / 32;
    k_fdct<<<(warps + per_block - 1) / per_block, kFdctThreads, 0, s>>>(e);
    return cudaGetLastError();
}

cudaError_t launch_alpha_size(const EncodeLaunch &e, cudaStream_t s) {
    if (!e.n_slices) return cudaSuccess;
    if (!e.any_alpha) return cudaMemsetAsync(e.alpha_bytes, 0, 4ull * e.n_slices, s);
    k_alpha_size<<<(e.n_slices + kAlphaWarps - 1) / kAlphaWarps, 32 * kAlphaWarps, 0, s>>>(e);
    return cudaGetLastError();
}

cudaError_t launch_rc_init(const EncodeLaunch &e, cudaStream_t s) {
    if (!e.n_pics) return cudaSuccess;
    k_rc_init<<<e.n_pics, kRcThreads, 0, s>>>(e);
    return cudaGetLastError();
}

// One lane per item when the batch has enough items to fill the GPU that
// way (a lane's walk is long, so it needs the whole machine's worth of
// them); otherwise a warp per item.
// A lane per slice component needs enough of them to fill the GPU; below
// that, a warp per component.
static bool lane_mode(const EncodeLaunch &e) {
    return 3ull * e.n_slices >= (uint64_t)e.lane_items_per_sm * (uint64_t)e.sm_count;
}

cudaError_t launch_cost(const EncodeLaunch &e, int step, cudaStream_t s) {
    if (!e.n_slices) return cudaSuccess;
    const uint32_t items = 3u * e.n_slices;
    if (lane_mode(e)) {
        static int per_sm = 0;  // resident CTAs of k_cost per SM (the same for every device of a build)
        if (per_sm == 0) {
            int fit = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_cost, kCostThreads, 0);
            per_sm = fit > 0 ? fit : 1;
        }
        const uint32_t need = (items + kCostThreads - 1) / kCostThreads;
        const uint32_t grid = std::min<uint32_t>(need, (uint32_t)(per_sm * e.sm_count));
        k_cost<<<grid, kCostThreads, 0, s>>>(e, step);
    } else
        k_cost_warp<<<(items + kCostThreads / 32 - 1) / (kCostThreads / 32), kCostThreads, 0, s>>>(e, step);
    return cudaGetLastError();
}

cudaError_t launch_rc_step(const EncodeLaunch &e, int step, cudaStream_t s) {
    if (!e.n_pics) return cudaSuccess;
    k_rc_step<<<e.n_pics, kRcThreads, 0, s>>>(e, step);
    return cudaGetLastError();
}

cudaError_t launch_cost_window(const EncodeLaunch &e, int level, cudaStream_t s) {
    if (!e.n_slices) return cudaSuccess;
    const uint32_t items = 3u * e.n_slices;
    k_window_select<<<(e.n_slices + kCostThreads - 1) / kCostThreads, kCostThreads, 0, s>>>(e, level);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    // The grid covers every slice; blocks past the list's end return.
    if (lane_mode(e))
        k_cost_window<false><<<(items * kWindowSegments + kCostThreads - 1) / kCostThreads, kCostThreads, 0, s>>>(
            e, level);
    else
        k_cost_window<true><<<(items + kCostThreads / 32 - 1) / (kCostThreads / 32), kCostThreads, 0, s>>>(e, level);
    return cudaGetLastError();
}

cudaError_t launch_cost_deep(const EncodeLaunch &e, cudaStream_t s) {
    if (!e.n_slices) return cudaSuccess;
    k_cost_deep<<<(e.n_slices + kCostThreads / 32 - 1) / (kCostThreads / 32), kCostThreads, 0, s>>>(e);
    return cudaGetLastError();
}

cudaError_t launch_shareout(const EncodeLaunch &e, cudaStream_t s) {
    if (!e.n_pics) return cudaSuccess;
    k_share_prep<<<(e.n_slices + 255) / 256, 256, 0, s>>>(e);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    k_shareout<<<(e.n_pics + kShareWarps - 1) / kShareWarps, 32 * kShareWarps, kShareWarps * kShareLadderBytes, s>>>(e);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
    k_share_final<<<(e.n_slices + 255) / 256, 256, 0, s>>>(e);
    return cudaGetLastError();
}

cudaError_t launch_layout(const EncodeLaunch &e, cudaStream_t s) {
    if (e.n_pics) k_layout<<<e.n_pics, kLayoutThreads, 0, s>>>(e);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess || !e.n_frames) return err;
    k_frame<<<(e.n_frames + 127) / 128, 128, 0, s>>>(e);
    return cudaGetLastError();
}

cudaError_t launch_pack(const EncodeLaunch &e, cudaStream_t s) {
    if (!e.n_slices) return cudaSuccess;
    const uint32_t items = 3u * e.n_slices;
    k_pack<<<(items + kCostThreads - 1) / kCostThreads, kCostThreads, 0, s>>>(e);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    k_pack_headers<<<(e.n_slices + 255) / 256, 256, 0, s>>>(e);
    if ((err = cudaGetLastError()) != cudaSuccess || !e.any_alpha) return err;
    k_pack_alpha<<<(e.n_slices + kAlphaWarps - 1) / kAlphaWarps, 32 * kAlphaWarps, 0, s>>>(e);
    return cudaGetLastError();
}

cudaError_t configure_encode_kernels() {
    cudaError_t err0 = cudaFuncSetAttribute(k_shareout, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(kShareWarps * kShareLadderBytes));
    if (err0 != cudaSuccess) return err0;
    float basis[64];
    dct_basis(basis);
    cudaError_t err = cudaMemcpyToSymbol(c_fdct_basis, basis, sizeof basis);
    if (err != cudaSuccess) return err;
    uint8_t sc[2][64];
    for (int i = 0; i < 64; i++) {
        sc[0][i] = kProgressiveScan[i];
        sc[1][i] = kInterlacedScan[i];
    }
    return cudaMemcpyToSymbol(c_enc_scan, sc, sizeof sc);
}

}  // namespace prores
