// bn_host.cpp -- client-side half of the BN path (include/bn_host.h).
//
// The keystream generator evaluates 16 ChaCha20 blocks side by side in a
// structure-of-arrays layout so the compiler vectorises the rounds; the
// draws it hands out are the same words, in the same order, as a
// one-block-at-a-time ChaCha20Rng.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bn_host.h"

namespace {

constexpr uint64_t P = (1ull << 61) - 1;
constexpr int LANES = 16;

typedef unsigned __int128 u128;

inline uint64_t reduce128(u128 x) {
    u128 s1 = (x & P) + (x >> 61);
    uint64_t r = (uint64_t)(s1 & P) + (uint64_t)(s1 >> 61);
    if (r >= P) r -= P;
    if (r >= P) r -= P;
    return r;
}
inline uint64_t addm(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s >= P ? s - P : s;
}
inline uint64_t subm(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P - b; }

inline uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

// 16 consecutive keystream blocks starting at block0, written word-major
// per block: out[b * 16 + w].
void chacha_blocks16(const uint32_t key[8], uint64_t block0, uint32_t* out) {
    uint32_t x[16][LANES], s[16][LANES];
    static const uint32_t C[4] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
    for (int l = 0; l < LANES; ++l) {
        for (int w = 0; w < 4; ++w) s[w][l] = C[w];
        for (int w = 0; w < 8; ++w) s[4 + w][l] = key[w];
        const uint64_t b = block0 + (uint64_t)l;
        s[12][l] = (uint32_t)b;
        s[13][l] = (uint32_t)(b >> 32);
        s[14][l] = 0;
        s[15][l] = 0;
    }
    memcpy(x, s, sizeof x);
#define VQR(a, b, c, d)                                             \
    for (int l = 0; l < LANES; ++l) {                                 \
        x[a][l] += x[b][l]; x[d][l] ^= x[a][l]; x[d][l] = rotl(x[d][l], 16); \
        x[c][l] += x[d][l]; x[b][l] ^= x[c][l]; x[b][l] = rotl(x[b][l], 12); \
        x[a][l] += x[b][l]; x[d][l] ^= x[a][l]; x[d][l] = rotl(x[d][l], 8);  \
        x[c][l] += x[d][l]; x[b][l] ^= x[c][l]; x[b][l] = rotl(x[b][l], 7);  \
    }
    for (int i = 0; i < 10; ++i) {
        VQR(0, 4, 8, 12) VQR(1, 5, 9, 13) VQR(2, 6, 10, 14) VQR(3, 7, 11, 15)
        VQR(0, 5, 10, 15) VQR(1, 6, 11, 12) VQR(2, 7, 8, 13) VQR(3, 4, 9, 14)
    }
#undef VQR
    for (int l = 0; l < LANES; ++l)
        for (int w = 0; w < 16; ++w) out[l * 16 + w] = x[w][l] + s[w][l];
}

// ChaCha20Rng::from_seed(seed) with rand_core's word order.
struct Rng {
    uint32_t key[8];
    uint64_t block = 0;
    uint32_t buf[16 * LANES];
    uint32_t idx = 16 * LANES;

    explicit Rng(const uint8_t seed[32]) {
        for (int i = 0; i < 8; ++i)
            key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                     ((uint32_t)seed[4 * i + 3] << 24);
    }
    inline uint32_t next_u32() {
        if (idx >= 16 * LANES) {
            chacha_blocks16(key, block, buf);
            block += LANES;
            idx = 0;
        }
        return buf[idx++];
    }
    inline uint64_t next_u64() {
        uint64_t lo = next_u32();
        uint64_t hi = next_u32();
        return lo | (hi << 32);
    }
    inline uint64_t sample_fp() {  // crypto.rs:155-162
        for (;;) {
            uint64_t x = next_u64() & P;
            if (x < P) return x;
        }
    }
    void bytes32(uint8_t out[32]) {
        for (int i = 0; i < 32; ++i) out[i] = (uint8_t)next_u32();
    }
};

uint32_t threshold() {
    double t = bn_host_mu() * 4294967296.0;
    uint64_t u = t <= 0.0 ? 0 : (uint64_t)t;
    return (uint32_t)std::min<uint64_t>(u, 0xffffffffull);
}

// crypto.rs:207-223
uint32_t sparse_pm1(Rng& r, uint32_t n, uint32_t thr, uint32_t* idx, int8_t* sign) {
    uint32_t c = 0;
    for (uint32_t j = 0; j < n; ++j) {
        if (r.next_u32() < thr) {
            idx[c] = j;
            sign[c] = (r.next_u32() & 1u) == 0 ? (int8_t)-1 : (int8_t)1;
            ++c;
        }
    }
    return c;
}

// H then S for one seed; S rows appended at (*nnz) with rowptr offsets.
bool gen_h_s(const uint8_t seed[32], uint64_t m, uint32_t n, uint32_t n1, uint64_t* H, uint64_t* rowptr,
             uint64_t nnz0, uint32_t* s_idx, int8_t* s_sign, uint64_t s_cap, uint64_t* nnz_out) {
    Rng r(seed);
    for (uint64_t i = 0; i < m * n1; ++i) H[i] = r.sample_fp();
    const uint32_t thr = threshold();
    std::vector<uint32_t> ti(n);
    std::vector<int8_t> ts(n);
    uint64_t nnz = nnz0;
    bool ok = true;
    for (uint64_t i = 0; i < m; ++i) {
        uint32_t c = sparse_pm1(r, n, thr, ti.data(), ts.data());
        if (ok && nnz + c <= s_cap) {
            memcpy(s_idx + nnz, ti.data(), 4ull * c);
            memcpy(s_sign + nnz, ts.data(), c);
        } else {
            ok = false;
        }
        nnz += c;
        rowptr[i + 1] = nnz;
    }
    *nnz_out = nnz;
    return ok;
}

}  // namespace

extern "C" {

double bn_host_mu(void) { return pow(1024.0, 0.7 - 1.0); }

uint32_t bn_host_default_trials(void) { return (128 + 60 - 1) / 60; }

void bn_host_domain_separate(const uint8_t seed[32], const char* tag, uint8_t out[32]) {
    uint8_t s[32];
    memcpy(s, seed, 32);
    const size_t n = strlen(tag);
    for (size_t i = 0; i < n; ++i) s[i % 32] ^= (uint8_t)tag[i];
    Rng r(s);
    r.bytes32(out);
}

void bn_host_derive_h_seed(uint64_t upload_seed, uint64_t ci, uint8_t out[32]) {
    uint8_t s[32] = {0};
    for (int i = 0; i < 8; ++i) {
        s[i] = (uint8_t)(upload_seed >> (8 * i));
        s[8 + i] = (uint8_t)(ci >> (8 * i));
    }
    Rng r(s);
    r.bytes32(out);
}

void bn_host_generate_subspace(const uint8_t key_seed[32], uint32_t n, uint32_t n1, uint64_t* L) {
    Rng r(key_seed);
    for (uint64_t i = 0; i < (uint64_t)n * n1; ++i) L[i] = r.sample_fp();
}

int64_t bn_host_regenerate_h_s(const uint8_t h_seed[32], uint64_t m, uint32_t n, uint32_t n1, uint64_t* H,
                               uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign, uint64_t s_cap) {
    s_rowptr[0] = 0;
    uint64_t nnz = 0;
    bool ok = gen_h_s(h_seed, m, n, n1, H, s_rowptr, 0, s_idx, s_sign, s_cap, &nnz);
    return ok ? (int64_t)nnz : -(int64_t)nnz;
}

int64_t bn_host_regenerate_h_s_lists(uint64_t upload_seed, uint32_t nlist, const uint64_t* off, uint32_t n,
                                     uint32_t n1, uint64_t* H, uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign,
                                     uint64_t s_cap) {
    // Pass 1: per-list sparse sizes need the draws themselves, so each list
    // generates into private buffers, then lists are stitched in order.
    std::vector<std::vector<uint32_t>> idx(nlist);
    std::vector<std::vector<int8_t>> sgn(nlist);
    std::vector<std::vector<uint64_t>> rp(nlist);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)nlist; ++c) {
        const uint64_t m = off[c + 1] - off[c];
        uint8_t seed[32];
        bn_host_derive_h_seed(upload_seed, (uint64_t)c, seed);
        rp[c].assign(m + 1, 0);
        idx[c].resize(m * 160 + 64);
        sgn[c].resize(m * 160 + 64);
        uint64_t nnz = 0;
        while (!gen_h_s(seed, m, n, n1, H + off[c] * n1, rp[c].data(), 0, idx[c].data(), sgn[c].data(), idx[c].size(),
                        &nnz)) {
            idx[c].resize(nnz);
            sgn[c].resize(nnz);
        }
        idx[c].resize(nnz);
        sgn[c].resize(nnz);
    }
    uint64_t total = 0;
    for (uint32_t c = 0; c < nlist; ++c) total += idx[c].size();
    if (total > s_cap) return -(int64_t)total;
    uint64_t base = 0;
    s_rowptr[0] = 0;
    for (uint32_t c = 0; c < nlist; ++c) {
        const uint64_t m = off[c + 1] - off[c];
        for (uint64_t i = 0; i < m; ++i) s_rowptr[off[c] + i + 1] = base + rp[c][i + 1];
        memcpy(s_idx + base, idx[c].data(), 4 * idx[c].size());
        memcpy(s_sign + base, sgn[c].data(), sgn[c].size());
        base += idx[c].size();
    }
    return (int64_t)total;
}

void bn_host_quantise(const float* v, uint64_t count, uint32_t d, uint32_t n, uint64_t q, uint64_t* out) {
    const double qs = (double)q;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < (int64_t)count; ++r) {
        uint64_t* o = out + (uint64_t)r * n;
        memset(o, 0, 8ull * n);
        for (uint32_t i = 0; i < d && i < n; ++i) {
            const double rd = round((double)v[(uint64_t)r * d + i] * qs);
            int64_t k;
            if (rd >= 9223372036854775807.0) k = INT64_MAX;
            else if (rd <= -9223372036854775808.0) k = INT64_MIN;
            else k = (int64_t)rd;
            if (k >= 0) {
                o[i] = (uint64_t)k % P;
            } else {
                const uint64_t a = (uint64_t)0 - (uint64_t)k, rr = a % P;
                o[i] = rr == 0 ? 0 : P - rr;
            }
        }
    }
}

uint32_t bn_host_encode_query(const uint64_t* v_q, const uint64_t* L, uint32_t n, uint32_t n1, const uint8_t q_seed[32],
                              uint64_t* v_enc, uint64_t* g, uint32_t* t_idx, int8_t* t_sign) {
    Rng r(q_seed);
    for (uint32_t k = 0; k < n1; ++k) g[k] = r.sample_fp();
    const uint32_t tn = sparse_pm1(r, n, threshold(), t_idx, t_sign);
    for (uint32_t j = 0; j < n; ++j) {
        const uint64_t* l = L + (uint64_t)j * n1;
        u128 acc = 0;
        for (uint32_t k = 0; k < n1; ++k) {
            acc += (u128)l[k] * g[k];
            if ((k & 31) == 31) acc = reduce128(acc);
        }
        v_enc[j] = reduce128(acc);
    }
    for (uint32_t c = 0; c < tn; ++c) v_enc[t_idx[c]] = t_sign[c] == 1 ? addm(v_enc[t_idx[c]], 1) : subm(v_enc[t_idx[c]], 1);
    for (uint32_t j = 0; j < n; ++j) v_enc[j] = addm(v_enc[j], v_q[j]);
    return tn;
}

void bn_host_probe_route(const float* cents, uint32_t nlist, uint32_t d, const float* qs, uint64_t count,
                         uint32_t nprobe, uint32_t* out) {
    const uint32_t np = std::min(nprobe, nlist);
#pragma omp parallel
    {
        std::vector<std::pair<float, uint32_t>> ds(nlist);
#pragma omp for schedule(dynamic, 4)
        for (int64_t q = 0; q < (int64_t)count; ++q) {
            const float* x = qs + (uint64_t)q * d;
            for (uint32_t c = 0; c < nlist; ++c) {
                const float* y = cents + (uint64_t)c * d;
                float s = 0.0f;
                for (uint32_t i = 0; i < d; ++i) {
                    const float t = x[i] - y[i];
                    s += t * t;
                }
                ds[c] = {sqrtf(s), c};
            }
            std::partial_sort(ds.begin(), ds.begin() + np, ds.end());
            for (uint32_t i = 0; i < np; ++i) out[(uint64_t)q * np + i] = ds[i].second;
        }
    }
}

}  // extern "C"
