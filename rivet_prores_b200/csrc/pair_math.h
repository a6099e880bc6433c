// pair_math.h -- paired single-precision arithmetic for the 8x8 transforms.
//
// sm_100a multiplies or adds two f32 pairs in one instruction
// (mul.rn.f32x2 / add.rn.f32x2). Each half is the IEEE round-to-nearest
// product or sum of its own operands, the same value __fmul_rn / __fadd_rn
// give, and nothing is contracted into a multiply-add: the transforms keep
// the crate's two roundings per term while issuing half the instructions.
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

__device__ __forceinline__ uint64_t pair_mul(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ uint64_t pair_add(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

}  // namespace prores
