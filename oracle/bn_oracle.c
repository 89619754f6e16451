/*
 * bn_oracle.c -- CPU restatement of the reference BN scoring path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  See bn_oracle.h for the parity
 * status of each part.  Every function cites the reference file:line it
 * restates; paths are relative to the reference project root.
 */
#include "bn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__)
#include <immintrin.h>
#endif

typedef unsigned __int128 u128;
#define P BNO_P
#define P128 ((u128)BNO_P)

/* ------------------------------------------------------------------ */
/* F_p arithmetic -- scorer-bntm/src/crypto.rs:47-89                   */
/* ------------------------------------------------------------------ */

/* crypto.rs:47-65: two-stage Mersenne fold of a full u128, then at most
 * two conditional subtractions. */
static inline uint64_t reduce128(u128 x) {
    u128 s1 = (x & P128) + (x >> 61);
    uint64_t r = (uint64_t)(s1 & P128) + (uint64_t)(s1 >> 61);
    if (r >= P) r -= P;
    if (r >= P) r -= P;
    return r;
}
static inline uint64_t addm(uint64_t a, uint64_t b) { uint64_t s = a + b; return s >= P ? s - P : s; }
static inline uint64_t subm(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P - b; }

uint64_t bno_mersenne_reduce128(uint64_t lo, uint64_t hi) { return reduce128(((u128)hi << 64) | lo); }
uint64_t bno_add_mod(uint64_t a, uint64_t b) { return addm(a, b); }
uint64_t bno_sub_mod(uint64_t a, uint64_t b) { return subm(a, b); }
uint64_t bno_mul_mod(uint64_t a, uint64_t b) { return reduce128((u128)a * b); }

/* crypto.rs:128-135 */
int64_t bno_fp_to_signed(uint64_t s) { return s < P / 2 ? (int64_t)s : (int64_t)s - (int64_t)P; }

/* ------------------------------------------------------------------ */
/* ChaCha20 -- RFC 8439 block function with the 64-bit block counter   */
/* (words 12-13) and 64-bit stream id (words 14-15) used by            */
/* rand_chacha's ChaCha20Rng (dependency rand_chacha 0.10, Cargo.toml). */
/* ------------------------------------------------------------------ */

static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
#define QR(a, b, c, d)                      \
    a += b; d ^= a; d = rotl32(d, 16);      \
    c += d; b ^= c; b = rotl32(b, 12);      \
    a += b; d ^= a; d = rotl32(d, 8);       \
    c += d; b ^= c; b = rotl32(b, 7);

void bno_chacha20_block(const uint32_t key[8], uint64_t counter, uint64_t stream, uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      (uint32_t)counter, (uint32_t)(counter >> 32),
                      (uint32_t)stream, (uint32_t)(stream >> 32)};
    uint32_t x[16];
    memcpy(x, s, sizeof x);
    for (int i = 0; i < 10; ++i) {
        QR(x[0], x[4], x[8], x[12]) QR(x[1], x[5], x[9], x[13])
        QR(x[2], x[6], x[10], x[14]) QR(x[3], x[7], x[11], x[15])
        QR(x[0], x[5], x[10], x[15]) QR(x[1], x[6], x[11], x[12])
        QR(x[2], x[7], x[8], x[13]) QR(x[3], x[4], x[9], x[14])
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

void bno_rng_from_seed(bno_rng* r, const uint8_t seed[32]) {
    for (int i = 0; i < 8; ++i)
        r->key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
                    ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
    r->block = 0;
    r->stream = 0;
    r->idx = 64;
}

static void rng_refill(bno_rng* r) {
    for (int b = 0; b < 4; ++b) bno_chacha20_block(r->key, r->block + (uint64_t)b, r->stream, r->buf + 16 * b);
    r->block += 4;
    r->idx = 0;
}

uint32_t bno_next_u32(bno_rng* r) {
    if (r->idx >= 64) rng_refill(r);
    return r->buf[r->idx++];
}

/* rand_core BlockRng::next_u64: two consecutive words, low word first. */
uint64_t bno_next_u64(bno_rng* r) {
    uint64_t lo = bno_next_u32(r);
    uint64_t hi = bno_next_u32(r);
    return lo | (hi << 32);
}

/* rand_core SeedableRng::seed_from_u64: PCG32 output fills the seed. */
void bno_seed_from_u64(uint64_t state, uint8_t seed_out[32]) {
    for (int c = 0; c < 8; ++c) {
        state = state * 6364136223846793005ULL + 11634580027462260723ULL;
        uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
        seed_out[4 * c + 0] = (uint8_t)x;
        seed_out[4 * c + 1] = (uint8_t)(x >> 8);
        seed_out[4 * c + 2] = (uint8_t)(x >> 16);
        seed_out[4 * c + 3] = (uint8_t)(x >> 24);
    }
}

/* rand StandardUniform for [u8; 32]: element-wise, u8 = low byte of next_u32. */
void bno_random_bytes32(bno_rng* r, uint8_t out[32]) {
    for (int i = 0; i < 32; ++i) out[i] = (uint8_t)bno_next_u32(r);
}

/* rand StandardUniform for f32: 24 high bits of next_u32 scaled by 2^-24. */
float bno_random_f32(bno_rng* r) { return (float)(bno_next_u32(r) >> 8) * (1.0f / 16777216.0f); }

void bno_rng_u32s(const uint8_t seed[32], size_t count, uint32_t* out) {
    bno_rng r;
    bno_rng_from_seed(&r, seed);
    for (size_t i = 0; i < count; ++i) out[i] = bno_next_u32(&r);
}
void bno_rng_u64s(const uint8_t seed[32], size_t count, uint64_t* out) {
    bno_rng r;
    bno_rng_from_seed(&r, seed);
    for (size_t i = 0; i < count; ++i) out[i] = bno_next_u64(&r);
}

/* crypto.rs:142-150 */
void bno_domain_separate(const uint8_t seed[32], const uint8_t* tag, size_t tag_len, uint8_t out[32]) {
    uint8_t s[32];
    memcpy(s, seed, 32);
    for (size_t i = 0; i < tag_len; ++i) s[i % 32] ^= tag[i];
    bno_rng r;
    bno_rng_from_seed(&r, s);
    bno_random_bytes32(&r, out);
}

/* ivf.rs:258-264 */
void bno_derive_h_seed(uint64_t upload_seed, uint64_t cluster_idx, uint8_t out[32]) {
    uint8_t s[32] = {0};
    for (int i = 0; i < 8; ++i) {
        s[i] = (uint8_t)(upload_seed >> (8 * i));
        s[8 + i] = (uint8_t)(cluster_idx >> (8 * i));
    }
    bno_rng r;
    bno_rng_from_seed(&r, s);
    bno_random_bytes32(&r, out);
}

/* crypto.rs:155-162 */
uint64_t bno_sample_fp(bno_rng* r) {
    for (;;) {
        uint64_t x = bno_next_u64(r) & P;
        if (x < P) return x;
    }
}

/* ------------------------------------------------------------------ */
/* Parameters -- scorer-bntm/src/params.rs                             */
/* ------------------------------------------------------------------ */

/* params.rs:179-181: mu = n^(eps - 1), computed in f64 exactly as the
 * reference does (0.7 - 1.0 is -0.30000000000000004, so mu is a hair
 * below 1/8). */
double bno_mu(void) { return pow(1024.0, 0.7 - 1.0); }

/* crypto.rs:210-211 */
uint32_t bno_sparse_threshold(double mu) {
    double t = mu * 4294967296.0;
    uint64_t u = t <= 0.0 ? 0 : (uint64_t)t;
    if (u > 0xFFFFFFFFull) u = 0xFFFFFFFFull;
    return (uint32_t)u;
}

/* params.rs:102-120 (k outside 1..=4 panics in the reference; 0 here) */
uint32_t bno_n1(uint32_t k) { return (k >= 1 && k <= 4) ? (1024u >> k) : 0u; }

/* params.rs:198-205 */
uint32_t bno_verification_trials(void) { return (128 + (8 * 8 - 4) - 1) / (8 * 8 - 4); }

/* ------------------------------------------------------------------ */
/* Keygen / encrypt -- crypto.rs:207-270, 405-478                      */
/* ------------------------------------------------------------------ */

/* crypto.rs:207-223: returns nnz written (positions j ascending). */
static uint32_t sample_sparse_pm1(bno_rng* r, uint32_t n, uint32_t thr, uint32_t* idx, int8_t* sign) {
    uint32_t c = 0;
    for (uint32_t j = 0; j < n; ++j) {
        uint32_t x = bno_next_u32(r);
        if (x < thr) {
            idx[c] = j;
            sign[c] = (bno_next_u32(r) & 1u) == 0 ? (int8_t)-1 : (int8_t)1;
            ++c;
        }
    }
    return c;
}

/* crypto.rs:235-238 */
void bno_generate_subspace(const uint8_t key_seed[32], uint32_t n, uint32_t n1, uint64_t* L) {
    bno_rng r;
    bno_rng_from_seed(&r, key_seed);
    for (uint64_t i = 0; i < (uint64_t)n * n1; ++i) L[i] = bno_sample_fp(&r);
}

/* crypto.rs:258-270: H first (m*n1 draws), then S row by row. */
int64_t bno_regenerate_h_s(const uint8_t h_seed[32], uint64_t m, uint32_t n, uint32_t n1, double mu,
                           uint64_t* H, uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign,
                           uint64_t s_cap) {
    bno_rng r;
    bno_rng_from_seed(&r, h_seed);
    for (uint64_t i = 0; i < m * n1; ++i) H[i] = bno_sample_fp(&r);
    uint32_t thr = bno_sparse_threshold(mu);
    uint32_t* ti = (uint32_t*)malloc(sizeof(uint32_t) * n);
    int8_t* ts = (int8_t*)malloc(n);
    uint64_t nnz = 0;
    int overflow = 0;
    s_rowptr[0] = 0;
    for (uint64_t i = 0; i < m; ++i) {
        uint32_t c = sample_sparse_pm1(&r, n, thr, ti, ts);
        if (!overflow && nnz + c <= s_cap) {
            memcpy(s_idx + nnz, ti, sizeof(uint32_t) * c);
            memcpy(s_sign + nnz, ts, c);
        } else {
            overflow = 1;
        }
        nnz += c;
        s_rowptr[i + 1] = nnz;
    }
    free(ti);
    free(ts);
    return overflow ? -(int64_t)nnz : (int64_t)nnz;
}

/* crypto.rs:405-478: M_enc = M + H L^T + S ; AL = M L. */
int64_t bno_encrypt_cluster(const uint64_t* M, uint64_t m, uint32_t n, uint32_t n1, const uint64_t* L,
                            const uint8_t h_seed[32], double mu, uint64_t* M_enc, uint64_t* AL,
                            uint64_t* H, uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign,
                            uint64_t s_cap, int nthreads) {
    int64_t nnz = bno_regenerate_h_s(h_seed, m, n, n1, mu, H, s_rowptr, s_idx, s_sign, s_cap);
    if (nnz < 0) return nnz;
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)m; ++ii) {
        uint64_t i = (uint64_t)ii;
        const uint64_t* h_row = H + i * n1;
        const uint64_t* mat_row = M + i * n;
        uint64_t sp = s_rowptr[i], se = s_rowptr[i + 1];
        for (uint32_t j = 0; j < n; ++j) {
            const uint64_t* l_row = L + (uint64_t)j * n1;
            u128 acc = 0;
            for (uint32_t k = 0; k < n1; ++k) {
                acc += (u128)h_row[k] * l_row[k];
                if ((k & 31) == 31) acc = reduce128(acc);
            }
            uint64_t hl = reduce128(acc);
            /* sparse_lookup (crypto.rs:483-488): sorted idx, so advance. */
            int s_term = 0;
            while (sp < se && s_idx[sp] < j) ++sp;
            if (sp < se && s_idx[sp] == j) s_term = s_sign[sp];
            uint64_t mp = s_term == 1 ? addm(hl, 1) : (s_term == -1 ? subm(hl, 1) : hl);
            M_enc[i * n + j] = addm(mat_row[j], mp);
        }
        for (uint32_t k = 0; k < n1; ++k) {
            u128 acc = 0;
            for (uint32_t j = 0; j < n; ++j) {
                acc += (u128)mat_row[j] * L[(uint64_t)j * n1 + k];
                if ((j & 31) == 31) acc = reduce128(acc);
            }
            AL[i * n1 + k] = reduce128(acc);
        }
    }
    return nnz;
}

/* ------------------------------------------------------------------ */
/* Client encode -- crypto.rs:105-122, 508-553                         */
/* ------------------------------------------------------------------ */

void bno_quantise_vector(const float* v, uint32_t d, uint32_t n, uint64_t q, uint64_t* out) {
    memset(out, 0, sizeof(uint64_t) * n);
    double qs = (double)q;
    for (uint32_t i = 0; i < d && i < n; ++i) {
        double scaled = (double)v[i] * qs;
        double rd = round(scaled); /* f64::round: half away from zero */
        int64_t rounded;
        if (rd >= 9223372036854775807.0) rounded = INT64_MAX; /* `as i64` saturates */
        else if (rd <= -9223372036854775808.0) rounded = INT64_MIN;
        else rounded = (int64_t)rd;
        if (rounded >= 0) {
            out[i] = (uint64_t)rounded % P;
        } else {
            uint64_t k = (uint64_t)0 - (uint64_t)rounded;
            uint64_t rr = k % P;
            out[i] = rr == 0 ? 0 : P - rr;
        }
    }
}

uint32_t bno_encode_query(const uint64_t* v, const uint64_t* L, uint32_t n, uint32_t n1, double mu,
                          const uint8_t q_seed[32], uint64_t* v_enc, uint64_t* g, uint32_t* t_idx,
                          int8_t* t_sign) {
    bno_rng r;
    bno_rng_from_seed(&r, q_seed);
    for (uint32_t k = 0; k < n1; ++k) g[k] = bno_sample_fp(&r);
    uint32_t tn = sample_sparse_pm1(&r, n, bno_sparse_threshold(mu), t_idx, t_sign);
    for (uint32_t j = 0; j < n; ++j) {
        const uint64_t* l_row = L + (uint64_t)j * n1;
        u128 acc = 0;
        for (uint32_t k = 0; k < n1; ++k) {
            acc += (u128)l_row[k] * g[k];
            if ((k & 31) == 31) acc = reduce128(acc);
        }
        v_enc[j] = reduce128(acc);
    }
    for (uint32_t c = 0; c < tn; ++c) {
        uint32_t j = t_idx[c];
        v_enc[j] = t_sign[c] == 1 ? addm(v_enc[j], 1) : subm(v_enc[j], 1);
    }
    for (uint32_t j = 0; j < n; ++j) v_enc[j] = addm(v_enc[j], v[j]);
    return tn;
}

/* ------------------------------------------------------------------ */
/* Server scan -- crypto.rs:561-828                                    */
/* ------------------------------------------------------------------ */

static inline uint64_t row_dot_scalar(const uint64_t* row, const uint64_t* vec, uint32_t cols) {
    u128 acc = 0;
    for (uint32_t j = 0; j < cols; ++j) {
        acc += (u128)row[j] * vec[j];
        if ((j & 31) == 31) acc = reduce128(acc);
    }
    return reduce128(acc);
}

/* crypto.rs:606-626 */
void bno_matvec_scalar(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vec,
                       uint64_t* out, int nthreads) {
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < (int64_t)rows; ++i) out[i] = row_dot_scalar(mat + (uint64_t)i * cols, vec, cols);
}

int bno_have_avx512(void) {
#if defined(__x86_64__)
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx512f");
#else
    return 0;
#endif
}

#if defined(__x86_64__)
/* crypto.rs:659-739: lane-decomposed Mersenne MAC, four 32x32->64
 * partial products per u64 pair, 2^64 == 8 (mod p) for the high-high
 * partial, in-vector folds. */
__attribute__((target("avx512f"))) static inline __m512i fold512(__m512i v, __m512i mask) {
    return _mm512_add_epi64(_mm512_and_si512(v, mask), _mm512_srli_epi64(v, 61));
}

__attribute__((target("avx512f"))) static uint64_t avx512_row_dot(const uint64_t* row, const uint64_t* v,
                                                                  uint32_t cols) {
    const __m512i mask = _mm512_set1_epi64((long long)P);
    __m512i acc_ll = _mm512_setzero_si512(), acc_cross = _mm512_setzero_si512(), acc_hh = _mm512_setzero_si512();
    for (uint32_t j = 0; j < cols;) {
        __m512i a = _mm512_loadu_si512((const void*)(row + j));
        __m512i b = _mm512_loadu_si512((const void*)(v + j));
        __m512i a_hi = _mm512_srli_epi64(a, 32), b_hi = _mm512_srli_epi64(b, 32);
        __m512i p_ll = _mm512_mul_epu32(a, b);
        __m512i p_cross = _mm512_add_epi64(_mm512_mul_epu32(a, b_hi), _mm512_mul_epu32(a_hi, b));
        __m512i p_hh = _mm512_mul_epu32(a_hi, b_hi);
        acc_ll = _mm512_add_epi64(acc_ll, fold512(p_ll, mask));
        acc_cross = _mm512_add_epi64(acc_cross, fold512(p_cross, mask));
        acc_hh = _mm512_add_epi64(acc_hh, p_hh);
        acc_ll = fold512(acc_ll, mask);
        acc_cross = fold512(acc_cross, mask);
        j += 8;
        if (((j / 8) % 8) == 0) acc_hh = fold512(acc_hh, mask);
    }
    uint64_t bl[8], bc[8], bh[8];
    _mm512_storeu_si512((void*)bl, acc_ll);
    _mm512_storeu_si512((void*)bc, acc_cross);
    _mm512_storeu_si512((void*)bh, acc_hh);
    u128 sl = 0, sc = 0, sh = 0;
    for (int k = 0; k < 8; ++k) { sl += bl[k]; sc += bc[k]; sh += bh[k]; }
    u128 total = (u128)reduce128(sl) + ((u128)reduce128(sc) << 32) + (u128)reduce128(sh) * 8;
    return reduce128(total);
}
#endif

/* crypto.rs:643-657 (falls back to scalar where AVX-512F or cols%8 is missing) */
void bno_matvec_avx512(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vec,
                       uint64_t* out, int nthreads) {
#if defined(__x86_64__)
    if (bno_have_avx512() && cols > 0 && cols % 8 == 0) {
        if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int64_t i = 0; i < (int64_t)rows; ++i) out[i] = avx512_row_dot(mat + (uint64_t)i * cols, vec, cols);
        return;
    }
#endif
    bno_matvec_scalar(mat, rows, cols, vec, out, nthreads);
}

/* crypto.rs:753-769: out[j] = sum_i vec[i] * mat[i][j], column-parallel,
 * fold every 32 rows.  Eight adjacent columns share a thread so each
 * strided cache line is used fully; the per-column arithmetic and fold
 * cadence are the reference's. */
void bno_matvec_transpose(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vec,
                          uint64_t* out, int nthreads) {
    if (nthreads <= 0) nthreads = 1;
    int64_t ngroups = ((int64_t)cols + 7) / 8;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t gidx = 0; gidx < ngroups; ++gidx) {
        uint32_t j0 = (uint32_t)gidx * 8, jn = j0 + 8 <= cols ? 8 : cols - j0;
        u128 acc[8] = {0};
        for (uint64_t i = 0; i < rows; ++i) {
            const uint64_t* rowp = mat + i * cols + j0;
            for (uint32_t c = 0; c < jn; ++c) acc[c] += (u128)vec[i] * rowp[c];
            if ((i & 31) == 31)
                for (uint32_t c = 0; c < jn; ++c) acc[c] = reduce128(acc[c]);
        }
        for (uint32_t c = 0; c < jn; ++c) out[j0 + c] = reduce128(acc[c]);
    }
}

/* crypto.rs:782-828 */
void bno_matvec_batch(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vecs, uint32_t B,
                      uint64_t* out, int nthreads) {
    if (B == 0) return;
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        u128* accs = (u128*)malloc(sizeof(u128) * B);
#pragma omp for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)rows; ++ii) {
            const uint64_t* row = mat + (uint64_t)ii * cols;
            for (uint32_t q = 0; q < B; ++q) accs[q] = 0;
            for (uint32_t j = 0; j < cols; ++j) {
                u128 rj = row[j];
                for (uint32_t q = 0; q < B; ++q) {
                    accs[q] += rj * vecs[(uint64_t)q * cols + j];
                    if ((j & 31) == 31) accs[q] = reduce128(accs[q]);
                }
            }
            for (uint32_t q = 0; q < B; ++q) out[(uint64_t)q * rows + (uint64_t)ii] = reduce128(accs[q]);
        }
        free(accs);
    }
}

/* crypto.rs:1049-1059 */
uint64_t bno_dot_product(const uint64_t* a, const uint64_t* b, uint64_t len) {
    u128 acc = 0;
    for (uint64_t i = 0; i < len; ++i) {
        acc += (u128)a[i] * b[i];
        if ((i & 31) == 31) acc = reduce128(acc);
    }
    return reduce128(acc);
}

/* ------------------------------------------------------------------ */
/* Protocol 2 -- crypto.rs:1013-1046                                   */
/* ------------------------------------------------------------------ */

int32_t bno_verify_response(const uint64_t* r, const uint64_t* M_enc, uint64_t m, uint32_t n,
                            const uint64_t* v_enc, uint32_t trials, const uint8_t v_seed[32], uint64_t* ur,
                            uint64_t* zv, int nthreads) {
    bno_rng rng;
    bno_rng_from_seed(&rng, v_seed);
    uint64_t* u = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
    uint64_t* z = (uint64_t*)malloc(sizeof(uint64_t) * n);
    int32_t fail = -1;
    for (uint32_t t = 0; t < trials; ++t) {
        for (uint64_t i = 0; i < m; ++i) u[i] = bno_sample_fp(&rng);
        uint64_t a = bno_dot_product(u, r, m);
        bno_matvec_transpose(M_enc, m, n, u, z, nthreads);
        uint64_t b = bno_dot_product(z, v_enc, n);
        if (ur) ur[t] = a;
        if (zv) zv[t] = b;
        if (a != b) { fail = (int32_t)t; break; }
    }
    free(u);
    free(z);
    return fail;
}

/* Protocol 2 split over row shards (no counterpart in the reference): the
 * shard rows [row0, row0 + rows) of a corpus of `total` rows, every trial's
 * two partial sums u_t . r_shard and (u_t^T M_shard) . v_enc, where u_t is
 * verify_response's draw vector for the whole corpus (crypto.rs:1021-1036:
 * total draws per trial from one stream, rejection included) restricted to
 * the shard.  All trials, no early exit: the verdict needs every shard's
 * sums.  Summed over the shards mod p they are verify_response's ur / zv. */
void bno_verify_shard_partials(const uint64_t* r_shard, const uint64_t* M_shard, uint64_t rows, uint32_t n,
                               const uint64_t* v_enc, uint32_t trials, const uint8_t v_seed[32], uint64_t row0,
                               uint64_t total, uint64_t* ur, uint64_t* zv, int nthreads) {
    bno_rng rng;
    bno_rng_from_seed(&rng, v_seed);
    uint64_t* u = (uint64_t*)malloc(sizeof(uint64_t) * (rows ? rows : 1));
    uint64_t* z = (uint64_t*)malloc(sizeof(uint64_t) * n);
    for (uint32_t t = 0; t < trials; ++t) {
        for (uint64_t i = 0; i < total; ++i) {
            const uint64_t x = bno_sample_fp(&rng);
            if (i >= row0 && i < row0 + rows) u[i - row0] = x;
        }
        ur[t] = bno_dot_product(u, r_shard, rows);
        bno_matvec_transpose(M_shard, rows, n, u, z, nthreads);
        zv[t] = bno_dot_product(z, v_enc, n);
    }
    free(u);
    free(z);
}

/* ------------------------------------------------------------------ */
/* Decode -- crypto.rs:837-940                                         */
/* ------------------------------------------------------------------ */

/* crypto.rs:846-848 */
void bno_l_transpose_times_vec(const uint64_t* L, uint32_t n, uint32_t n1, const uint64_t* v, uint64_t* out) {
    bno_matvec_transpose(L, n, n1, v, out, 1);
}

void bno_decode_scores(const uint64_t* r, const uint64_t* AL, const uint64_t* M_plain, const uint64_t* H,
                       const uint64_t* s_rowptr, const uint32_t* s_idx, const int8_t* s_sign,
                       const uint64_t* L, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                       const int8_t* t_sign, uint32_t t_nnz, uint64_t m, uint32_t n, uint32_t n1,
                       uint64_t* out, int nthreads) {
    uint64_t* lt = (uint64_t*)malloc(sizeof(uint64_t) * n1);
    bno_l_transpose_times_vec(L, n, n1, v_enc, lt);
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)m; ++ii) {
        uint64_t i = (uint64_t)ii;
        /* M v' = AL G + M T   (crypto.rs:914-920, 852-873) */
        uint64_t al_g = row_dot_scalar(AL + i * n1, g, n1);
        uint64_t m_t = 0;
        for (uint32_t c = 0; c < t_nnz; ++c) {
            uint64_t x = M_plain[i * n + t_idx[c]];
            m_t = t_sign[c] == 1 ? addm(m_t, x) : subm(m_t, x);
        }
        uint64_t mvp = addm(al_g, m_t);
        /* M' v_enc = H (L^T v_enc) + S v_enc   (crypto.rs:925-932, 877-894) */
        uint64_t h_lt = row_dot_scalar(H + i * n1, lt, n1);
        uint64_t s_v = 0;
        for (uint64_t c = s_rowptr[i]; c < s_rowptr[i + 1]; ++c)
            s_v = s_sign[c] == 1 ? addm(s_v, v_enc[s_idx[c]]) : subm(s_v, v_enc[s_idx[c]]);
        uint64_t mpv = addm(h_lt, s_v);
        out[i] = subm(subm(r[i], mvp), mpv);
    }
    free(lt);
}

/* ------------------------------------------------------------------ */
/* Rank -- lib.rs:452-469 with a canonical tie-break                   */
/* ------------------------------------------------------------------ */

typedef struct { int64_t s; uint32_t id; } hit_t;
/* a "better" than b: higher score, then lower id */
static inline int better(hit_t a, hit_t b) { return a.s > b.s || (a.s == b.s && a.id < b.id); }

static void sift_down(hit_t* h, uint32_t n, uint32_t i) {
    /* min-heap on "better": root is the worst retained hit */
    for (;;) {
        uint32_t l = 2 * i + 1, r = l + 1, w = i;
        if (l < n && better(h[w], h[l])) w = l;
        if (r < n && better(h[w], h[r])) w = r;
        if (w == i) return;
        hit_t t = h[i]; h[i] = h[w]; h[w] = t;
        i = w;
    }
}

static int cmp_hits(const void* pa, const void* pb) {
    hit_t a = *(const hit_t*)pa, b = *(const hit_t*)pb;
    if (better(a, b)) return -1;
    if (better(b, a)) return 1;
    return 0;
}

uint32_t bno_topk(const int64_t* scores, const uint32_t* ids, uint64_t count, uint32_t k, uint32_t* out_ids,
                  int64_t* out_scores) {
    uint32_t kk = (uint64_t)k < count ? k : (uint32_t)count;
    if (kk == 0) return 0;
    hit_t* h = (hit_t*)malloc(sizeof(hit_t) * kk);
    uint32_t n = 0;
    for (uint64_t i = 0; i < count; ++i) {
        hit_t x = {scores[i], ids ? ids[i] : (uint32_t)i};
        if (n < kk) {
            h[n++] = x;
            if (n == kk)
                for (int64_t j = (int64_t)kk / 2 - 1; j >= 0; --j) sift_down(h, kk, (uint32_t)j);
        } else if (better(x, h[0])) {
            h[0] = x;
            sift_down(h, kk, 0);
        }
    }
    qsort(h, n, sizeof(hit_t), cmp_hits);
    for (uint32_t i = 0; i < n; ++i) { out_ids[i] = h[i].id; out_scores[i] = h[i].s; }
    free(h);
    return n;
}

/* ------------------------------------------------------------------ */
/* IVF routing -- ivf-index/src/distance.rs:29-36, ivf.rs:150-164,     */
/* kmeans.rs:15-132                                                    */
/* ------------------------------------------------------------------ */

float bno_l2_f32(const float* a, const float* b, uint32_t d) {
    float s = 0.0f;
    for (uint32_t i = 0; i < d; ++i) { float t = a[i] - b[i]; s += t * t; }
    return sqrtf(s);
}

typedef struct { float d; uint32_t i; } dist_t;
static int cmp_dist(const void* pa, const void* pb) {
    dist_t a = *(const dist_t*)pa, b = *(const dist_t*)pb;
    if (a.d < b.d) return -1;
    if (a.d > b.d) return 1;
    return a.i < b.i ? -1 : (a.i > b.i);
}

uint32_t bno_probe_route(const float* centroids, uint32_t nlist, uint32_t d, const float* q, uint32_t nprobe,
                         uint32_t* out) {
    dist_t* ds = (dist_t*)malloc(sizeof(dist_t) * nlist);
    for (uint32_t c = 0; c < nlist; ++c) { ds[c].d = bno_l2_f32(q, centroids + (uint64_t)c * d, d); ds[c].i = c; }
    qsort(ds, nlist, sizeof(dist_t), cmp_dist);
    uint32_t np = nprobe < nlist ? nprobe : nlist;
    for (uint32_t i = 0; i < np; ++i) out[i] = ds[i].i;
    free(ds);
    return np;
}

/* kmeans.rs:40-54: nearest centroid, first minimum wins. */
void bno_assign(const float* data, uint64_t count, uint32_t d, const float* centroids, uint32_t k,
                uint32_t* out, int nthreads) {
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        const float* v = data + (uint64_t)i * d;
        uint32_t best = 0;
        float bd = bno_l2_f32(v, centroids, d);
        for (uint32_t c = 1; c < k; ++c) {
            float dd = bno_l2_f32(v, centroids + (uint64_t)c * d, d);
            if (dd < bd) { bd = dd; best = c; }
        }
        out[i] = best;
    }
}

/* rand UniformInt<u64>::sample_single(0..n): Canon's widening-multiply
 * method, one extra draw when the low half could carry. */
static uint64_t random_range_u64(bno_rng* r, uint64_t n) {
    uint64_t range = n; /* high - low + 1 with low = 0, high = n - 1 */
    u128 p = (u128)bno_next_u64(r) * range;
    uint64_t result = (uint64_t)(p >> 64), lo = (uint64_t)p;
    if (lo > (uint64_t)0 - range) {
        u128 p2 = (u128)bno_next_u64(r) * range;
        uint64_t hi2 = (uint64_t)(p2 >> 64);
        if (lo + hi2 < lo) result += 1;
    }
    return result;
}

void bno_kmeans_train(const float* data, uint64_t count, uint32_t d, uint32_t k, uint64_t seed, uint32_t max_iter,
                      float* centroids, int nthreads) {
    uint8_t s[32];
    bno_seed_from_u64(seed, s);
    bno_rng rng;
    bno_rng_from_seed(&rng, s);
    /* k-means++ (kmeans.rs:76-128) */
    uint64_t first = random_range_u64(&rng, count);
    memcpy(centroids, data + first * d, sizeof(float) * d);
    float* mind = (float*)malloc(sizeof(float) * count);
    for (uint64_t i = 0; i < count; ++i) { float t = bno_l2_f32(data + i * d, centroids, d); mind[i] = t * t; }
    for (uint32_t ci = 1; ci < k; ++ci) {
        float total = 0.0f;
        for (uint64_t i = 0; i < count; ++i) total += mind[i];
        float thr = bno_random_f32(&rng) * total;
        uint64_t chosen = count - 1;
        for (uint64_t i = 0; i < count; ++i) {
            thr -= mind[i];
            if (thr <= 0.0f) { chosen = i; break; }
        }
        memcpy(centroids + (uint64_t)ci * d, data + chosen * d, sizeof(float) * d);
        for (uint64_t i = 0; i < count; ++i) {
            float t = bno_l2_f32(data + i * d, centroids + (uint64_t)ci * d, d);
            if (t * t < mind[i]) mind[i] = t * t;
        }
    }
    free(mind);
    /* Lloyd (kmeans.rs:24-36, 56-74) */
    uint32_t* asg = (uint32_t*)malloc(sizeof(uint32_t) * count);
    float* sums = (float*)malloc(sizeof(float) * (uint64_t)k * d);
    uint64_t* cnt = (uint64_t*)malloc(sizeof(uint64_t) * k);
    for (uint32_t it = 0; it < max_iter; ++it) {
        bno_assign(data, count, d, centroids, k, asg, nthreads);
        memset(sums, 0, sizeof(float) * (uint64_t)k * d);
        memset(cnt, 0, sizeof(uint64_t) * k);
        for (uint64_t i = 0; i < count; ++i) {
            float* sp = sums + (uint64_t)asg[i] * d;
            for (uint32_t t = 0; t < d; ++t) sp[t] += data[i * d + t];
            cnt[asg[i]]++;
        }
        int same = 1;
        for (uint32_t c = 0; c < k; ++c)
            for (uint32_t t = 0; t < d; ++t) {
                float nv = cnt[c] == 0 ? 0.0f : sums[(uint64_t)c * d + t] / (float)cnt[c];
                if (nv != centroids[(uint64_t)c * d + t]) same = 0;
                sums[(uint64_t)c * d + t] = nv;
            }
        if (same) break;
        memcpy(centroids, sums, sizeof(float) * (uint64_t)k * d);
    }
    free(asg);
    free(sums);
    free(cnt);
}

/* ------------------------------------------------------------------ */
/* Whole flat query -- lib.rs:326-475                                  */
/* ------------------------------------------------------------------ */

static double now_us(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e6 + ts.tv_nsec * 1e-3;
}

int32_t bno_score_flat(const uint64_t* M_enc, const uint64_t* AL, const uint64_t* M_plain, const uint64_t* H,
                       const uint64_t* s_rowptr, const uint32_t* s_idx, const int8_t* s_sign, const uint64_t* L,
                       uint64_t m, uint32_t n, uint32_t n1, const uint64_t* v_q, const uint8_t q_seed[32],
                       uint32_t trials, uint32_t k, uint32_t* out_ids, int64_t* out_scores, uint64_t* r_out,
                       double* timings_us, int nthreads, int use_avx512) {
    double t0 = now_us();
    double mu = bno_mu();
    uint64_t* v_enc = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint64_t* g = (uint64_t*)malloc(sizeof(uint64_t) * n1);
    uint32_t* t_idx = (uint32_t*)malloc(sizeof(uint32_t) * n);
    int8_t* t_sign = (int8_t*)malloc(n);
    uint32_t tn = bno_encode_query(v_q, L, n, n1, mu, q_seed, v_enc, g, t_idx, t_sign);
    double t1 = now_us();
    uint64_t* r = r_out ? r_out : (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
    if (use_avx512) bno_matvec_avx512(M_enc, m, n, v_enc, r, nthreads);
    else bno_matvec_scalar(M_enc, m, n, v_enc, r, nthreads);
    double t2 = now_us();
    int32_t fail = -1;
    if (trials > 0) {
        static const uint8_t tag[] = "protocol2";
        uint8_t vs[32];
        bno_domain_separate(q_seed, tag, 9, vs);
        fail = bno_verify_response(r, M_enc, m, n, v_enc, trials, vs, NULL, NULL, nthreads);
    }
    double t3 = now_us();
    if (fail < 0) {
        uint64_t* mv = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
        int64_t* sc = (int64_t*)malloc(sizeof(int64_t) * (m ? m : 1));
        bno_decode_scores(r, AL, M_plain, H, s_rowptr, s_idx, s_sign, L, v_enc, g, t_idx, t_sign, tn, m, n, n1, mv,
                          nthreads);
        for (uint64_t i = 0; i < m; ++i) sc[i] = bno_fp_to_signed(mv[i]);
        bno_topk(sc, NULL, m, k, out_ids, out_scores);
        free(mv);
        free(sc);
    }
    double t4 = now_us();
    if (timings_us) { timings_us[0] = t1 - t0; timings_us[1] = t2 - t1; timings_us[2] = t3 - t2; timings_us[3] = t4 - t3; }
    if (!r_out) free(r);
    free(v_enc); free(g); free(t_idx); free(t_sign);
    return fail;
}
