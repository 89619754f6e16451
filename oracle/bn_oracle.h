/*
 * bn_oracle.h -- CPU restatement of the reference Braverman-Newman (BN)
 * scoring path of sacs-epfl/secure-vector-search.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product (secure-vector-search_b200/) never links or calls it.
 *
 * Parity status
 *   - F_p arithmetic, matvec, batch matvec, transpose matvec, verify,
 *     decode: exact modular arithmetic, pinned by independent big-integer
 *     computation in tests/ (order-free, so any correct implementation
 *     agrees bit for bit).
 *   - ChaCha20 block function: pinned by the RFC 8439 test vectors.
 *   - rand/rand_chacha 0.10 stream conventions (u64 = two consecutive
 *     little-endian u32 words; seed_from_u64 via the PCG32 filler;
 *     random::<[u8;32]>() = low byte of 32 successive u32 draws;
 *     random::<f32>() = (u32 >> 8) * 2^-24):
 *     restated from the published crates, NOT pinned by any vector from
 *     the reference (the reference ships no golden outputs and its Rust
 *     toolchain is absent here).  Everything derived from ChaCha draws
 *     (L, H, S, G, T, Freivalds u) is therefore "parity unpinned" against
 *     the reference itself; it is pinned oracle <-> GPU.
 *   - Tie order of the reference's sort_unstable_by_key is unspecified;
 *     this oracle ranks by (score desc, id asc).
 */
#ifndef BN_ORACLE_H
#define BN_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BNO_P ((uint64_t)((1ULL << 61) - 1ULL))

/* ---- field (scorer-bntm/src/crypto.rs:47-89) ---- */
uint64_t bno_mersenne_reduce128(uint64_t lo, uint64_t hi);
uint64_t bno_add_mod(uint64_t a, uint64_t b);
uint64_t bno_sub_mod(uint64_t a, uint64_t b);
uint64_t bno_mul_mod(uint64_t a, uint64_t b);
int64_t bno_fp_to_signed(uint64_t s);

/* ---- ChaCha20 (rand_chacha 0.10 ChaCha20Rng; RFC 8439 block function) ---- */
typedef struct {
    uint32_t key[8];
    uint64_t block;      /* next block counter to generate */
    uint64_t stream;
    uint32_t buf[64];    /* 4 blocks of output words */
    uint32_t idx;        /* next unread word in buf; 64 = empty */
} bno_rng;

void bno_chacha20_block(const uint32_t key[8], uint64_t counter, uint64_t stream,
                        uint32_t out[16]);
void bno_rng_from_seed(bno_rng* r, const uint8_t seed[32]);
void bno_seed_from_u64(uint64_t state, uint8_t seed_out[32]);
uint32_t bno_next_u32(bno_rng* r);
uint64_t bno_next_u64(bno_rng* r);
void bno_random_bytes32(bno_rng* r, uint8_t out[32]);
float bno_random_f32(bno_rng* r);
/* Convenience: first `count` u32 / u64 draws of ChaCha20Rng::from_seed(seed). */
void bno_rng_u32s(const uint8_t seed[32], size_t count, uint32_t* out);
void bno_rng_u64s(const uint8_t seed[32], size_t count, uint64_t* out);

/* ---- seeds (crypto.rs:142-162, ivf.rs:258-264) ---- */
void bno_domain_separate(const uint8_t seed[32], const uint8_t* tag, size_t tag_len,
                         uint8_t out[32]);
void bno_derive_h_seed(uint64_t upload_seed, uint64_t cluster_idx, uint8_t out[32]);
uint64_t bno_sample_fp(bno_rng* r);

/* ---- params (params.rs:89-120,179-181,198-205) ---- */
double bno_mu(void);                 /* n^(eps-1) with n=1024, eps=0.7 */
uint32_t bno_sparse_threshold(double mu);
uint32_t bno_n1(uint32_t delta_pow2); /* 1024 >> k, k in 1..=4 else 0 */
uint32_t bno_verification_trials(void);

/* ---- keygen / encrypt (crypto.rs:170-270, 405-478) ---- */
void bno_generate_subspace(const uint8_t key_seed[32], uint32_t n, uint32_t n1, uint64_t* L);
/* H: m*n1; S in CSR (rowptr m+1, idx, sign).  Returns nnz, or -(needed)
 * when s_cap is too small (outputs then undefined). */
int64_t bno_regenerate_h_s(const uint8_t h_seed[32], uint64_t m, uint32_t n, uint32_t n1,
                           double mu, uint64_t* H, uint64_t* s_rowptr, uint32_t* s_idx,
                           int8_t* s_sign, uint64_t s_cap);
int64_t bno_encrypt_cluster(const uint64_t* M, uint64_t m, uint32_t n, uint32_t n1,
                            const uint64_t* L, const uint8_t h_seed[32], double mu,
                            uint64_t* M_enc, uint64_t* AL, uint64_t* H,
                            uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign,
                            uint64_t s_cap, int nthreads);

/* ---- client encode (crypto.rs:105-122, 508-553) ---- */
void bno_quantise_vector(const float* v, uint32_t d, uint32_t n, uint64_t q, uint64_t* out);
/* Returns |T|.  t_idx/t_sign need room for n entries. */
uint32_t bno_encode_query(const uint64_t* v, const uint64_t* L, uint32_t n, uint32_t n1,
                          double mu, const uint8_t q_seed[32], uint64_t* v_enc, uint64_t* g,
                          uint32_t* t_idx, int8_t* t_sign);

/* ---- server scan (crypto.rs:561-828) ---- */
void bno_matvec_scalar(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vec,
                       uint64_t* out, int nthreads);
int bno_have_avx512(void);
void bno_matvec_avx512(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vec,
                       uint64_t* out, int nthreads);
void bno_matvec_transpose(const uint64_t* mat, uint64_t rows, uint32_t cols,
                          const uint64_t* vec, uint64_t* out, int nthreads);
void bno_matvec_batch(const uint64_t* mat, uint64_t rows, uint32_t cols, const uint64_t* vecs,
                      uint32_t B, uint64_t* out /* B x rows */, int nthreads);
uint64_t bno_dot_product(const uint64_t* a, const uint64_t* b, uint64_t len);

/* ---- Protocol 2 (crypto.rs:1013-1059) ----
 * v_seed = domain_separate(q_seed, "protocol2").  Returns -1 when every
 * trial passes, else the first failing trial.  ur/zv (nullable) receive
 * the two sides of each trial that ran. */
void bno_verify_shard_partials(const uint64_t* r_shard, const uint64_t* M_shard, uint64_t rows, uint32_t n,
                               const uint64_t* v_enc, uint32_t trials, const uint8_t v_seed[32], uint64_t row0,
                               uint64_t total, uint64_t* ur, uint64_t* zv, int nthreads);
int32_t bno_verify_response(const uint64_t* r, const uint64_t* M_enc, uint64_t m, uint32_t n,
                            const uint64_t* v_enc, uint32_t trials, const uint8_t v_seed[32],
                            uint64_t* ur, uint64_t* zv, int nthreads);

/* ---- decode (crypto.rs:837-940) ---- */
void bno_l_transpose_times_vec(const uint64_t* L, uint32_t n, uint32_t n1, const uint64_t* v,
                               uint64_t* out);
void bno_decode_scores(const uint64_t* r, const uint64_t* AL, const uint64_t* M_plain,
                       const uint64_t* H, const uint64_t* s_rowptr, const uint32_t* s_idx,
                       const int8_t* s_sign, const uint64_t* L, const uint64_t* v_enc,
                       const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign,
                       uint32_t t_nnz, uint64_t m, uint32_t n, uint32_t n1, uint64_t* out,
                       int nthreads);

/* ---- rank (lib.rs:452-469): canonical (score desc, id asc) top-k ---- */
uint32_t bno_topk(const int64_t* scores, const uint32_t* ids /* nullable = 0..count-1 */,
                  uint64_t count, uint32_t k, uint32_t* out_ids, int64_t* out_scores);

/* ---- IVF routing (ivf-index/src/ivf.rs:150-164, distance.rs:29-36) ---- */
float bno_l2_f32(const float* a, const float* b, uint32_t d);
uint32_t bno_probe_route(const float* centroids, uint32_t nlist, uint32_t d, const float* q,
                         uint32_t nprobe, uint32_t* out);
void bno_assign(const float* data, uint64_t count, uint32_t d, const float* centroids,
                uint32_t k, uint32_t* out, int nthreads);
/* ivf-index/src/kmeans.rs:15-132 (k-means++ init + Lloyd), small sizes. */
void bno_kmeans_train(const float* data, uint64_t count, uint32_t d, uint32_t k, uint64_t seed,
                      uint32_t max_iter, float* centroids_out, int nthreads);

/* ---- whole flat query: encode -> scan -> verify -> decode -> top-k ----
 * lib.rs:326-475.  Returns -1 on success, or the failing Freivalds trial.
 * timings_us (nullable) = {encode, server, verify, decode}. */
int32_t bno_score_flat(const uint64_t* M_enc, const uint64_t* AL, const uint64_t* M_plain,
                       const uint64_t* H, const uint64_t* s_rowptr, const uint32_t* s_idx,
                       const int8_t* s_sign, const uint64_t* L, uint64_t m, uint32_t n,
                       uint32_t n1, const uint64_t* v_q, const uint8_t q_seed[32],
                       uint32_t trials, uint32_t k, uint32_t* out_ids, int64_t* out_scores,
                       uint64_t* r_out /* nullable */, double* timings_us, int nthreads,
                       int use_avx512);

#ifdef __cplusplus
}
#endif
#endif
