// bn_chacha.cuh -- ChaCha20 keystream for host and device.
//
// Stream semantics are those of rand_chacha 0.10's ChaCha20Rng as used by
// the reference (scorer-bntm/src/crypto.rs:142-162, 207-270, 1027): the
// RFC 8439 block function with a 64-bit block counter in words 12-13 and a
// 64-bit stream id (0) in words 14-15; output words are consumed in order;
// next_u64 takes two consecutive words, low word first.  Because every
// word has a fixed position in the keystream, the device generates any
// draw directly from its index (block = index / 16) instead of walking a
// sequential generator.
#pragma once
#include <stdint.h>
#include <string.h>

#include "bn_fp.cuh"

namespace bn {

struct ChaChaKey {
    uint32_t k[8];
};

BN_HD ChaChaKey chacha_key(const uint8_t seed[32]) {
    ChaChaKey key;
    for (int i = 0; i < 8; ++i)
        key.k[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                   ((uint32_t)seed[4 * i + 3] << 24);
    return key;
}

BN_HD uint32_t rotl32(uint32_t x, int r) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_l(x, x, r);
#else
    return (x << r) | (x >> (32 - r));
#endif
}

#define BN_QR(a, b, c, d)          \
    a += b; d ^= a; d = rotl32(d, 16); \
    c += d; b ^= c; b = rotl32(b, 12); \
    a += b; d ^= a; d = rotl32(d, 8);  \
    c += d; b ^= c; b = rotl32(b, 7);

// Block `counter` of the keystream (stream id 0): 16 output words.
BN_HD void chacha20_block(const ChaChaKey& key, uint64_t counter, uint32_t out[16]) {
    uint32_t x0 = 0x61707865u, x1 = 0x3320646eu, x2 = 0x79622d32u, x3 = 0x6b206574u;
    uint32_t x4 = key.k[0], x5 = key.k[1], x6 = key.k[2], x7 = key.k[3];
    uint32_t x8 = key.k[4], x9 = key.k[5], x10 = key.k[6], x11 = key.k[7];
    uint32_t x12 = (uint32_t)counter, x13 = (uint32_t)(counter >> 32), x14 = 0, x15 = 0;
#if defined(__CUDA_ARCH__)
#pragma unroll 2
#endif
    for (int i = 0; i < 10; ++i) {
        BN_QR(x0, x4, x8, x12) BN_QR(x1, x5, x9, x13) BN_QR(x2, x6, x10, x14) BN_QR(x3, x7, x11, x15)
        BN_QR(x0, x5, x10, x15) BN_QR(x1, x6, x11, x12) BN_QR(x2, x7, x8, x13) BN_QR(x3, x4, x9, x14)
    }
    out[0] = x0 + 0x61707865u; out[1] = x1 + 0x3320646eu; out[2] = x2 + 0x79622d32u; out[3] = x3 + 0x6b206574u;
    out[4] = x4 + key.k[0]; out[5] = x5 + key.k[1]; out[6] = x6 + key.k[2]; out[7] = x7 + key.k[3];
    out[8] = x8 + key.k[4]; out[9] = x9 + key.k[5]; out[10] = x10 + key.k[6]; out[11] = x11 + key.k[7];
    out[12] = x12 + (uint32_t)counter; out[13] = x13 + (uint32_t)(counter >> 32); out[14] = x14; out[15] = x15;
}

// Sequential generator for host code (keygen, query encoding).
struct HostRng {
    ChaChaKey key;
    uint64_t block = 0;
    uint32_t buf[16];
    uint32_t idx = 16;

    explicit HostRng(const uint8_t seed[32]) : key(chacha_key(seed)) {}
    uint32_t next_u32() {
        if (idx >= 16) {
            chacha20_block(key, block++, buf);
            idx = 0;
        }
        return buf[idx++];
    }
    uint64_t next_u64() {
        uint64_t lo = next_u32();
        uint64_t hi = next_u32();
        return lo | (hi << 32);
    }
    // crypto.rs:155-162
    uint64_t sample_fp() {
        for (;;) {
            uint64_t x = next_u64() & P;
            if (x < P) return x;
        }
    }
    // rand StandardUniform for [u8; 32]
    void bytes32(uint8_t out[32]) {
        for (int i = 0; i < 32; ++i) out[i] = (uint8_t)next_u32();
    }
};

// crypto.rs:142-150
inline void domain_separate(const uint8_t seed[32], const char* tag, uint8_t out[32]) {
    uint8_t s[32];
    memcpy(s, seed, 32);
    size_t n = strlen(tag);
    for (size_t i = 0; i < n; ++i) s[i % 32] ^= (uint8_t)tag[i];
    HostRng r(s);
    r.bytes32(out);
}

// ivf.rs:258-264
inline void derive_h_seed(uint64_t upload_seed, uint64_t cluster_idx, uint8_t out[32]) {
    uint8_t s[32] = {0};
    for (int i = 0; i < 8; ++i) {
        s[i] = (uint8_t)(upload_seed >> (8 * i));
        s[8 + i] = (uint8_t)(cluster_idx >> (8 * i));
    }
    HostRng r(s);
    r.bytes32(out);
}

}  // namespace bn
