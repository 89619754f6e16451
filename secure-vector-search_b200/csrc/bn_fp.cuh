// bn_fp.cuh -- exact arithmetic in F_p, p = 2^61 - 1, for host and device.
//
// Field semantics follow scorer-bntm/src/crypto.rs:47-89 (canonical
// residues in [0, p)); the evaluation strategy is this project's own:
// products are formed from 32-bit x 21-bit limbs with IMAD.WIDE-style
// 32x32->64 multiply-adds so no 128-bit carry chain sits in the inner
// loop, and residues are folded (x mod 2^61 + x >> 61) only at tile ends.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define BN_HD __host__ __device__ __forceinline__
#else
#define BN_HD inline
#endif

namespace bn {

constexpr uint64_t P = (1ull << 61) - 1;
constexpr uint32_t N = 1024;          // ring dimension, params.rs:89-91
constexpr uint32_t LIMB_BITS = 21;    // v = b0 + b1*2^21 + b2*2^42
constexpr uint32_t LIMB_MASK = (1u << LIMB_BITS) - 1;

// 64-bit accumulate of a 32 x 32 -> 64 product (one IMAD.WIDE.U32).
BN_HD uint64_t mac(uint64_t acc, uint32_t a, uint32_t b) { return acc + (uint64_t)a * (uint64_t)b; }

// One Mersenne fold: x (< 2^64) -> congruent value < 2^61 + 8.
BN_HD uint64_t fold(uint64_t x) { return (x & P) + (x >> 61); }

// Canonical residue of any u64.
BN_HD uint64_t canon(uint64_t x) {
    x = fold(x);
    return x >= P ? x - P : x;
}

BN_HD uint64_t add_mod(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s >= P ? s - P : s;
}
BN_HD uint64_t sub_mod(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P - b; }

// x * 2^w mod p for 0 < w < 61 and x < 2^63 (result < 2^61 + 2^(w+2)).
BN_HD uint64_t rotl61(uint64_t x, uint32_t w) { return ((x << w) & P) + (x >> (61 - w)); }

// Canonical residue of the 128-bit value hi*2^64 + lo.
BN_HD uint64_t reduce128(uint64_t lo, uint64_t hi) {
    uint64_t t1 = lo & P;
    uint64_t t2 = (lo >> 61) | (hi << 3);   // low 64 bits of x >> 61
    uint64_t t3 = hi >> 61;                 // bits 64.. of x >> 61, weight 2^64 == 8
    uint64_t s = t1 + fold(t2) + (t3 << 3);
    return canon(s);
}

BN_HD uint64_t mul_mod(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return reduce128(a * b, __umul64hi(a, b));
#else
    unsigned __int128 x = (unsigned __int128)a * b;
    return reduce128((uint64_t)x, (uint64_t)(x >> 64));
#endif
}

// crypto.rs:128-135
BN_HD int64_t to_signed(uint64_t s) { return s < P / 2 ? (int64_t)s : (int64_t)s - (int64_t)P; }

// 21-bit limbs of a canonical residue (b2 < 2^19).
struct Limbs3 {
    uint32_t b0, b1, b2;
};
BN_HD Limbs3 limbs(uint64_t v) {
    return Limbs3{(uint32_t)(v & LIMB_MASK), (uint32_t)((v >> LIMB_BITS) & LIMB_MASK), (uint32_t)(v >> (2 * LIMB_BITS))};
}

// Pre-scaled limbs for the high 32-bit half of the other operand:
// m_hi * 2^32 * v == m_hi * (v * 2^32 mod p), so splitting v' = v*2^32 mod p
// into the same 21-bit limbs lets both halves of m share three accumulators
// (weights 2^0, 2^21, 2^42).
BN_HD Limbs3 limbs_hi(uint64_t v) { return limbs(canon(rotl61(v, 32))); }

// acc0 + acc1*2^21 + acc2*2^42 (each acc < 2^64) -> canonical residue.
BN_HD uint64_t combine3(uint64_t a0, uint64_t a1, uint64_t a2) {
    uint64_t s = fold(a0) + rotl61(fold(a1), 21) + rotl61(fold(a2), 42);
    return canon(s);
}

}  // namespace bn
