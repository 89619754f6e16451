/*
 * bn_host.h -- host-side (client) half of the BN path, in C++ above the
 * device ABI of bn_b200.h: key generation, quantisation and query encoding,
 * with the reference's exact RNG consumption so that the device sees the
 * same M_enc / v_enc the reference CPU scorer would build.
 *
 * Each function names the reference function it restates
 * (scorer-bntm/src/crypto.rs, lib.rs, ivf.rs).  All are CPU-only and need no
 * GPU; the device entry points are in bn_b200.h.
 */
#ifndef BN_HOST_H
#define BN_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* params.rs:179-181 mu = n^(eps-1); crypto.rs:210-211 32-bit threshold. */
double bn_host_mu(void);
/* params.rs:198-205 (3 trials for p = 2^61 - 1). */
uint32_t bn_host_default_trials(void);

/* crypto.rs:142-150 domain_separate(seed, tag). */
void bn_host_domain_separate(const uint8_t seed[32], const char* tag, uint8_t out[32]);
/* ivf.rs:258-264 derive_h_seed(upload_seed, cluster_idx). */
void bn_host_derive_h_seed(uint64_t upload_seed, uint64_t cluster_idx, uint8_t out[32]);

/* crypto.rs:235-238 generate_subspace: L, n x n1 row-major. */
void bn_host_generate_subspace(const uint8_t key_seed[32], uint32_t n, uint32_t n1, uint64_t* L);
/* crypto.rs:258-270 regenerate_h_s: H (m x n1) then S row by row (CSR).
 * Returns nnz(S), or -(needed) when s_cap is too small. */
int64_t bn_host_regenerate_h_s(const uint8_t h_seed[32], uint64_t m, uint32_t n, uint32_t n1, uint64_t* H,
                               uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign, uint64_t s_cap);
/* Per-list regenerate_h_s for an IVF index (ivf.rs:627-653): list c uses
 * derive_h_seed(upload_seed, c); outputs are the concatenation in list order
 * (rows list_offsets[c]..list_offsets[c+1]).  Lists run in parallel. */
int64_t bn_host_regenerate_h_s_lists(uint64_t upload_seed, uint32_t nlist, const uint64_t* list_offsets, uint32_t n,
                                     uint32_t n1, uint64_t* H, uint64_t* s_rowptr, uint32_t* s_idx, int8_t* s_sign,
                                     uint64_t s_cap);

/* crypto.rs:105-122 quantise_vector over `count` vectors of dimension d
 * (d <= n), zero-padded to n: out is count x n. */
void bn_host_quantise(const float* v, uint64_t count, uint32_t d, uint32_t n, uint64_t q, uint64_t* out);

/* crypto.rs:508-553 encode_query with ChaCha20Rng::from_seed(q_seed):
 * writes v_enc (n), g (n1), T (t_idx/t_sign, room for n) and returns |T|. */
uint32_t bn_host_encode_query(const uint64_t* v_q, const uint64_t* L, uint32_t n, uint32_t n1,
                              const uint8_t q_seed[32], uint64_t* v_enc, uint64_t* g, uint32_t* t_idx,
                              int8_t* t_sign);

/* ivf-index/src/ivf.rs:150-164 probe_route: the nprobe nearest centroids
 * by f32 L2 (scalar, in dimension order), ties by lower index.  Queries
 * run in parallel; out is count x min(nprobe, nlist). */
void bn_host_probe_route(const float* centroids, uint32_t nlist, uint32_t d, const float* queries, uint64_t count,
                         uint32_t nprobe, uint32_t* out);

/* ---------------------------------------------------------------- reference IVF cache files
 * Reader of the `.bntm-ivf-cache-<16 hex>.bin` files the reference's
 * BnTmIvfScorer writes (scorer-bntm/src/ivf.rs:440-560; its loader
 * load_bntm_ivf_cache, ivf.rs:1755-1901): the k-means index, and per list
 * the encrypted m_enc, a_l, the plaintext m_plain and H, plus L.  S is
 * not stored; regenerate it per list from the list's h_seed with
 * bn_host_regenerate_h_s, as the reference does.
 *
 * bn_host_cache_fingerprint: the header hash of scorer-core/src/cache.rs
 * (FNV-1a 64 over the parts, each prefixed by its u64 LE length); the
 * reference's parts for this cache are ivf.rs:321-331 ("bntm-ivf2",
 * n_centroids, train_seed, max_iter, number of vectors, upload_seed,
 * key_seed, n1, quantisation_q; integers as u64 LE, key_seed 32 bytes),
 * and the file name is ".bntm-ivf-cache-" + 16 lower-case hex digits of it
 * + ".bin". */
uint64_t bn_host_cache_fingerprint(const uint8_t* const* parts, const uint64_t* lens, uint32_t nparts);

typedef struct bn_ivf_cache bn_ivf_cache;
/* Maps and indexes the file.  fingerprint: the expected header hash, or 0
 * to accept any (the magic and version are always checked).  n, n1: the BN
 * dimensions the index was built with.  Returns BN_OK, or BN_EINVAL with
 * bn_last_error() naming the first inconsistency (the reference treats the
 * same conditions as a cache miss or as invalid data): bad magic, version
 * or fingerprint, a truncated region, or list sizes that differ between
 * the index and the encrypted part. */
int bn_host_ivf_cache_open(const char* path, uint64_t fingerprint, uint32_t n, uint32_t n1, bn_ivf_cache** out);
void bn_host_ivf_cache_close(bn_ivf_cache* c);
/* Lists, dimension of the index's f32 vectors, total rows. */
void bn_host_ivf_cache_info(const bn_ivf_cache* c, uint32_t* nlist, uint32_t* dim, uint64_t* rows);
/* list_offsets (nlist + 1), ids (rows, the vector ids in list order),
 * centroids (nlist x dim f32) and h_seeds (nlist x 32 bytes); each
 * nullable. */
void bn_host_ivf_cache_lists(const bn_ivf_cache* c, uint64_t* list_offsets, uint32_t* ids, float* centroids,
                             uint8_t* h_seeds);
/* The lists' arrays concatenated in list order, each nullable: m_enc and
 * m_plain rows x n, a_l and h rows x n1 (row-major), l_subspace n x n1. */
void bn_host_ivf_cache_arrays(const bn_ivf_cache* c, uint64_t* m_enc, uint64_t* a_l, uint64_t* m_plain, uint64_t* h,
                              uint64_t* l_subspace);

#ifdef __cplusplus
}
#endif
#endif /* BN_HOST_H */
