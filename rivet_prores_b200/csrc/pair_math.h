// pair_math.h -- paired single-precision sums for the 8x8 transforms.
//
// sm_100a adds two f32 pairs in one instruction (add.rn.f32x2); each half
// is the IEEE round-to-nearest sum of its own operands, the value
// __fadd_rn gives. The transforms add their terms in pairs and keep every
// product scalar (__fmul_rn, mul.rn.f32), which is never contracted into a
// multiply-add: the crate's two roundings per term stay, with three
// instructions for two terms instead of four.
//
// Paired products (mul.rn.f32x2) are not used: measured on a B200, a
// paired product feeding a paired sum was at times fused into a paired
// multiply-add by the code generator, even with contraction turned off,
// which changes the last bit of the sum.
// A pair is a 64-bit value, low half first.
#pragma once

#include <cstdint>

namespace prores {

__device__ __forceinline__ uint64_t pair_of(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

__device__ __forceinline__ void pair_split(uint64_t v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ uint64_t pair_add(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

}  // namespace prores
