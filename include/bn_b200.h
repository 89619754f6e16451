/*
 * bn_b200.h -- C ABI of the B200 (sm_100a) backend for the Braverman-Newman
 * trapdoored-matrix scoring path of sacs-epfl/secure-vector-search.
 *
 * This is the drop-in boundary.  In the reference, the scorers reach the GPU
 * through `HandleInner::Gpu(Box<FlatGpuState>)` (scorer-bntm/src/lib.rs:118-127)
 * and `HandleInner::Gpu(Box<IvfGpuState>)` (scorer-bntm/src/ivf.rs:108-117);
 * every entry point below names the method it replaces.  Conventions:
 *
 *   - plain C types, host pointers unless a name starts with d_ (device);
 *   - every field element is a canonical residue mod p = 2^61 - 1, n = 1024;
 *   - every call returns BN_OK (0) or a negative status; bn_last_error()
 *     then describes the failure (thread-local string), mirroring the
 *     reference's GpuError (gpu/mod.rs:97-110);
 *   - handles are thread-safe: calls on one handle are serialised on its
 *     own CUDA stream, calls on distinct handles run concurrently;
 *   - host buffers are only borrowed for the duration of a call.
 */
#ifndef BN_B200_H
#define BN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BN_ABI_VERSION 1

/* Status codes (GpuError, gpu/mod.rs:97-110; BnTmError, lib.rs:178-196). */
#define BN_OK 0
#define BN_EINVAL (-1)       /* bad argument or shape (e.g. n != 1024, k > 1024)   */
#define BN_ECUDA (-2)        /* CUDA runtime failure      (GpuError::Driver)         */
#define BN_EBUDGET (-3)      /* payload exceeds budget    (GpuError::BudgetTooSmall) */
#define BN_ENODEV (-4)       /* no usable CUDA device                                */
#define BN_EUNSUPPORTED (-5) /* handle lacks the client state this call needs       */
#define BN_EAGAIN (-6)       /* bn_server_wait: the request is not complete yet;
                                bn_server_submit_*: the queue is full, retry later   */
/* A Protocol 2 draw equalled p.  The reference rejects that draw and takes
 * the next one (sample_fp, crypto.rs:155-162), which shifts every later draw
 * of the stream by one; the kernels here draw by stream position, so the
 * call reports the event instead of returning a verdict that could differ
 * from the reference's.  Odds: 2^-61 per draw (about 2^-37 per query at
 * N = 1M, 20 trials).  Retrying with another seed is the caller's choice. */
#define BN_EDRAW (-7)

#define BN_TOPK_MAX 1024
#define BN_MAX_TRIALS 64 /* Protocol 2 trials per call */

/* Protocol 2 engines (bn_ctx_set_engine).  Both compute z_t = u_t^T M_enc
 * exactly; TENSOR runs it as a u8-limb GEMM on tcgen05 tensor cores,
 * CUDA_CORE as 64-bit limb multiply-adds on the CUDA cores. */
#define BN_ENGINE_TENSOR 0
#define BN_ENGINE_CUDA_CORE 1

/* Last error message of the calling thread ("" when none). */
const char* bn_last_error(void);
/* Build description: ABI version, target architecture, compiler. */
const char* bn_build_info(void);
/* Number of visible CUDA devices (0 without a GPU). */
int bn_device_count(int* out);

typedef struct bn_ctx bn_ctx;
typedef struct bn_flat bn_flat;
typedef struct bn_ivf bn_ivf;
typedef struct bn_plan bn_plan;

/* Sparse {-1,0,+1} matrix in CSR form: rowptr has rows+1 entries, idx holds
 * sorted column indices, sign holds +1/-1 (crypto.rs:168-186 SparseMatrix). */
typedef struct bn_sparse_csr {
    const uint64_t* rowptr;
    const uint32_t* idx;
    const int8_t* sign;
} bn_sparse_csr;

/* ---------------------------------------------------------------- context
 * Replaces the process-wide cudarc context + PTX module (gpu/mod.rs:169-200)
 * and the VRAM budget resolution (scorer-gpu-common/src/budget.rs:132-150):
 * vram_budget_bytes = 0 takes 80 % of the device's free memory. */
int bn_ctx_create(int device, uint64_t vram_budget_bytes, bn_ctx** out);
int bn_ctx_destroy(bn_ctx* ctx);
/* Selects the Protocol 2 engine used by later calls on this context's
 * handles (default BN_ENGINE_TENSOR).  No counterpart in the reference, whose
 * verification runs on the host (lib.rs:419-437). */
int bn_ctx_set_engine(bn_ctx* ctx, int engine);
/* Budget, bytes currently held by handles, high-water mark
 * (FlatGpuState::{vram_budget_bytes, peak_vram_bytes}, gpu/mod.rs:334-340). */
int bn_ctx_memory(const bn_ctx* ctx, uint64_t* budget_bytes, uint64_t* used_bytes, uint64_t* peak_bytes);

/* ---------------------------------------------------------------- flat
 * FlatGpuState::build (gpu/mod.rs:300-332).  m_enc is m x n, a_l and h are
 * m x n1, all row-major host arrays; the corpus is uploaded eagerly and stays
 * resident (the reference uploads lazily through its LRU store). */
int bn_flat_build(bn_ctx* ctx, const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint64_t m,
                  uint32_t n, uint32_t n1, bn_flat** out);
/* Client-side state for on-device decode: L (n x n1 row-major), the
 * plaintext M (m x n row-major) and S (crypto.rs:353-392 EncryptedCluster
 * fields l_subspace/m_plain/s_mat).  Needed by bn_flat_query.  Besides the
 * uploaded arrays the decode keeps copies in 32-row blocks: 16 * n1 bytes
 * per row of [AL | H], plus 1024 bytes per row of M when every entry of M
 * is int8-valued (rows rounded up to a multiple of 32; counted in
 * bn_flat_info's device_bytes and against the context budget). */
int bn_flat_attach_client(bn_flat* h, const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat);
/* Encrypt on the device and build in one step (crypto.rs:405-478 +
 * gpu/mod.rs:300-332): M_enc = M + H L^T + S and AL = M L are computed
 * from the quantised plaintext m_q (m x n), L, H and S; the client state is
 * attached as by bn_flat_attach_client. */
int bn_flat_build_from_plain(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1,
                             const uint64_t* l_subspace, const uint64_t* h, bn_sparse_csr s_mat, bn_flat** out);
int bn_flat_destroy(bn_flat* h);
int bn_flat_info(const bn_flat* h, uint64_t* rows, uint64_t* device_bytes);
/* Device-resident m_enc (row-major m x 1024) of a flat handle. */
int bn_flat_device_m_enc(const bn_flat* h, const uint64_t** d_m_enc);

/* FlatGpuState::compute_products (gpu/mod.rs:362-379): r = M_enc v_enc. */
int bn_flat_compute_products(bn_flat* h, const uint64_t* v_enc, uint64_t* r);
/* Batched compute_products (crypto.rs:782-828): r is B x m. */
int bn_flat_compute_products_batch(bn_flat* h, const uint64_t* v_encs, uint32_t B, uint64_t* r);
/* FlatGpuState::decode_dense_terms (gpu/mod.rs:390-408): AL g + H lt_venc. */
int bn_flat_decode_dense_terms(bn_flat* h, const uint64_t* g, const uint64_t* lt_venc, uint64_t* out);
/* verify_response (crypto.rs:1013-1046) on the device for a claimed r.
 * v_seed is the seed of the verification RNG, i.e. domain_separate(q_seed,
 * "protocol2") in the reference (lib.rs:422).  *failed_trial = -1 when
 * every trial passes, else the first failing trial.  ur/zv (nullable, length
 * trials) receive both sides of every trial. */
int bn_flat_verify(bn_flat* h, const uint64_t* r, const uint64_t* v_enc, const uint8_t v_seed[32], uint32_t trials,
                   int32_t* failed_trial, uint64_t* ur, uint64_t* zv);
/* Allocation-free form of bn_flat_verify over device buffers, enqueued on
 * `stream` (no synchronisation).  No counterpart in the reference.  For
 * callers that cannot allocate device memory while scoring: services that
 * pre-reserve their whole memory budget and must not fail an allocation
 * mid-request, and latency-critical threads for which cudaMalloc / cudaFree
 * could synchronise the device.  Its scratch is a fixed array of about
 * 3 MiB in the library, held on every GPU that loads it until exit; trials
 * must be in 1..=BN_NOALLOC_MAX_TRIALS.  All calls share that array: calls
 * that overlap on the GPU race, so serialise them.  The array and the
 * kernels this call launches are loaded, and the array's address resolved,
 * by bn_ctx_create for that device (CUDA loads modules lazily, and loading
 * one allocates device memory): create the context before the memory budget
 * is handed out, and this call allocates nothing afterwards.
 *   d_r m, d_v_enc 1024, d_v_seed 32 bytes; outputs d_failed_trial (1),
 *   d_ur / d_zv (trials) as in bn_flat_verify, except that *d_failed_trial
 *   = -2 when a draw equalled p (the BN_EDRAW event, reported in the output
 *   because nothing is read back to the host).  An empty corpus gives -1 and
 *   zero sums, as bn_flat_verify does.  The calling thread's current device
 *   is left as it was. */
#define BN_NOALLOC_MAX_TRIALS 24
int bn_flat_verify_noalloc(bn_flat* h, const uint64_t* d_r, const uint64_t* d_v_enc, const uint8_t* d_v_seed,
                           uint32_t trials, int32_t* d_failed_trial, uint64_t* d_ur, uint64_t* d_zv, void* stream);
/* Whole server + client path of BnTmScorer::score / score_batch
 * (lib.rs:326-475, 522-624) for B encoded queries: scan, fused-launch
 * Protocol 2, decode, fp_to_signed and top-k, all on the device.
 *   v_enc  B x n, g  B x n1
 *   T      query b has t_nnz[b] entries starting at sum(t_nnz[0..b)) in
 *          t_idx (column) / t_sign (+1/-1)
 *   v_seeds B x 32 bytes (nullable when trials == 0)
 * Outputs: ids/scores B x k (score desc, id asc; n_hits[b] = min(k, m)
 * valid), failed_trial[b] (nullable; -1 = verified or not run), r_out and
 * mv_out (nullable, B x m: scan residues and decoded residues). */
int bn_flat_query(bn_flat* h, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                  const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
                  uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial, uint64_t* r_out,
                  uint64_t* mv_out);

/* One row shard of a flat corpus split over several GPUs (one process per
 * GPU).  No counterpart in the reference, whose GPU backend serves one card
 * per process.  The handle holds rows [shard_row0, shard_row0 + m) of a
 * corpus of total_rows rows; the call runs bn_flat_query's pipeline on them
 * with the Protocol 2 draws at those rows' positions in the whole corpus
 * (u_t[i] = draw t * total_rows + i of the query's stream, crypto.rs:1021-
 * 1036), and returns what the ranks exchange instead of a verdict:
 *   ids / scores / n_hits  the shard's top-k (ids are global row numbers);
 *   ur, zv (B x trials)    this shard's u_t . r and z_t . v_enc, canonical.
 * Summed over the shards (mod p), ur and zv are verify_response's two sides
 * for the whole corpus (z . v is linear in z), so query b is accepted iff
 * every trial's sums agree; the union of the shards' top-k lists holds the
 * global top-k.  The merge and the exact sums are the caller's
 * (bn_b200/shard.py does them over torch.distributed). */
int bn_flat_query_shard(bn_flat* h, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                        const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials,
                        uint32_t k, uint64_t shard_row0, uint64_t total_rows, uint32_t* ids, int64_t* scores,
                        uint32_t* n_hits, uint64_t* ur, uint64_t* zv);

/* Prepared, device-resident form of bn_flat_query for a fixed (B, trials,
 * k): bn_plan_enqueue only enqueues kernels on `stream` (no host work, no
 * allocation, no synchronisation), so it can be captured in a CUDA graph.
 *   d_v_enc B x 1024 u64, d_g B x n1 u64,
 *   d_t     B x 1024 u32 entries (col | 0x80000000 for -1), d_t_nnz B,
 *   d_v_seeds B x 32 bytes, outputs d_ids/d_scores B x k, d_n B,
 *   d_failed B (-1 = pass).  All device pointers. */
int bn_flat_plan(bn_flat* h, uint32_t B, uint32_t trials, uint32_t k, bn_plan** out);
int bn_plan_enqueue(bn_plan* p, const uint64_t* d_v_enc, const uint64_t* d_g, const uint32_t* d_t,
                    const uint32_t* d_t_nnz, const uint8_t* d_v_seeds, uint32_t* d_ids, int64_t* d_scores,
                    uint32_t* d_n, int32_t* d_failed, void* stream);
/* Scan-only enqueue of the same plan: d_r (B x m) = M_enc v_enc. */
int bn_plan_enqueue_scan(bn_plan* p, const uint64_t* d_v_enc, uint64_t* d_r, void* stream);
/* Device flags of the last enqueue of this plan (0 = healthy).  Bits
 * 0x1..0x40: a bounded device-side wait timed out; bit 0x1000
 * (BN_STATUS_DRAW_HIT_P): a Protocol 2 draw equalled p (see BN_EDRAW); block
 * plans add 0x100 when a T column sum left [-128, 127].  Any bit set means
 * the outputs must be discarded.  Synchronous: call after the enqueued work
 * has completed. */
#define BN_STATUS_DRAW_HIT_P 0x1000u
int bn_plan_status(bn_plan* p, uint32_t* device_flags);
/* Kernel timing for measurement: after bn_plan_profile(p, n), the next n
 * enqueues record CUDA events on their stream right before and after the
 * plan's dominant kernel (the one pass over m_enc: fused scan + Protocol 2 on
 * the tensor engine, the scan otherwise); bn_plan_profile_read waits for them
 * and returns their durations in ms (oldest first) and restarts the count.
 * No counterpart in the reference. */
int bn_plan_profile(bn_plan* p, uint32_t max_launches);
int bn_plan_profile_read(bn_plan* p, float* ms, uint32_t cap, uint32_t* n);
int bn_plan_destroy(bn_plan* p);

/* ---------------------------------------------------------------- block scoring
 * B queries per launch as tensor-core integer GEMMs over byte-planar copies of
 * the corpus: compute_products_batch (crypto.rs:782-828) + decode_scores
 * (crypto.rs:901-940) + top-k (lib.rs:452-469) for the whole block, with
 * Protocol 2 applied PER BLOCK: one 32-byte block seed, trial t's draws u_t
 * (draw t*m + i of ChaCha20Rng(block_seed), as verify_response draws them,
 * crypto.rs:1021-1036) shared by the block's queries, and query q accepted
 * iff u_t . r_q == (u_t^T M_enc) . v_q for every t.  No counterpart in the
 * reference, which verifies each query with its own seed (the per-query
 * entry points above keep that behaviour); the block form costs one pass of
 * M_enc per block instead of one per query.
 * Needs the client state with m_plain entries and S entries in [-128, 127]
 * (int8-quantised corpora; BN_EUNSUPPORTED otherwise).  The byte-planar
 * copies take 8 * (1024 + 2 * n1) + 2048 + 8 bytes per row of device memory,
 * built on first use or by bn_flat_block_prepare. */
#define BN_BLOCK_AUTOTUNE 1u /* bn_flat_block_plan: time the GEMM tilings on this corpus, keep the fastest */
int bn_flat_block_prepare(bn_flat* h);
/* Plan for blocks of exactly B queries (1..=8192).  Enqueue-only afterwards
 * (CUDA-graph capturable), like bn_flat_plan. */
int bn_flat_block_plan(bn_flat* h, uint32_t B, uint32_t trials, uint32_t k, uint32_t flags, bn_plan** out);
/* Chosen configuration: {W rows per tile (queries x 8), pipeline stages,
 * work order (0 = W tile fastest), A tiles resident in shared memory (0/1),
 * K panel of the u . r GEMM, K steps of 128 bytes per pipeline stage - 1};
 * tuned_ms
 * (nullable) = the autotuner's measured launch times of the r = M_enc v GEMM
 * and of the u . r GEMM with that configuration (0 when not autotuned). */
int bn_plan_block_config(const bn_plan* p, uint32_t config[6], float tuned_ms[2]);
/* Device buffers as bn_plan_enqueue, with one 32-byte d_block_seed.
 * bn_plan_status reports bit 8 when a T column sum left [-128, 127]. */
int bn_plan_enqueue_block(bn_plan* p, const uint64_t* d_v_enc, const uint64_t* d_g, const uint32_t* d_t,
                          const uint32_t* d_t_nnz, const uint8_t* d_block_seed, uint32_t* d_ids, int64_t* d_scores,
                          uint32_t* d_n, int32_t* d_failed, void* stream);
/* Host buffers, inputs and outputs as bn_flat_query (failed_trial[q] = first
 * failing trial of query q under the block seed, -1 if accepted); mv_out
 * (nullable) receives the decoded residues B x m. */
int bn_flat_query_block(bn_flat* h, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                        const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t block_seed[32], uint32_t trials,
                        uint32_t k, uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial,
                        uint64_t* mv_out);
/* Protocol 2 over claimed responses r (B x m) with the block seed:
 * failed_trial[q], and ur / zv (nullable, trials x B, [t][q]) = u_t . r_q and
 * z_t . v_q. */
int bn_flat_verify_block(bn_flat* h, uint32_t B, const uint64_t* r, const uint64_t* v_enc,
                         const uint8_t block_seed[32], uint32_t trials, int32_t* failed_trial, uint64_t* ur,
                         uint64_t* zv);

/* ---------------------------------------------------------------- IVF
 * IvfGpuState::build (gpu/mod.rs:423-474) over a device-resident CSR of the
 * inverted lists: list c owns rows [list_offsets[c], list_offsets[c+1]) of
 * the concatenated m_enc / a_l / h arrays; ids[row] is the global vector id
 * (ivf-index IvfIndex::clusters membership). */
int bn_ivf_build(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids, const uint64_t* m_enc,
                 const uint64_t* a_l, const uint64_t* h, uint32_t n, uint32_t n1, bn_ivf** out);
/* As bn_flat_attach_client, for the concatenated lists (the same decode
 * copies per row). */
int bn_ivf_attach_client(bn_ivf* h, const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat);
/* Device encryption of every list (crypto.rs:405-478 per cluster,
 * ivf.rs:627-653) followed by bn_ivf_build + bn_ivf_attach_client.  h and
 * s_mat are the concatenation of the per-list H / S (each list with its own
 * h_seed, ivf.rs:258-264). */
int bn_ivf_build_from_plain(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids,
                            const uint64_t* m_q, uint32_t n, uint32_t n1, const uint64_t* l_subspace,
                            const uint64_t* h, bn_sparse_csr s_mat, bn_ivf** out);
int bn_ivf_destroy(bn_ivf* h);
int bn_ivf_info(const bn_ivf* h, uint64_t* rows, uint64_t* device_bytes);
/* IvfGpuState::compute_products (gpu/mod.rs:506-536).  *m_out = list size;
 * 0 (and nothing written) for an empty or out-of-range list, the
 * reference's Ok(None). */
int bn_ivf_compute_products(bn_ivf* h, uint32_t ci, const uint64_t* v_enc, uint64_t* r, uint64_t* m_out);
/* IvfGpuState::decode_dense_terms (gpu/mod.rs:542-577). */
int bn_ivf_decode_dense_terms(bn_ivf* h, uint32_t ci, const uint64_t* g, const uint64_t* lt_venc, uint64_t* out,
                              uint64_t* m_out);
/* verify_response for one list and a claimed r (ivf.rs:791-806). */
int bn_ivf_verify(bn_ivf* h, uint32_t ci, const uint64_t* r, const uint64_t* v_enc, const uint8_t v_seed[32],
                  uint32_t trials, int32_t* failed_trial, uint64_t* ur, uint64_t* zv);
/* IVF routing on the device (ivf-index/src/ivf.rs:150-164 probe_route) for
 * a batch: bn_ivf_set_centroids keeps the nlist x d f32 centroids (row-major,
 * list order; d <= 8192, nlist <= 16384) on the handle; bn_ivf_route writes,
 * per query of the B x d f32 queries (B <= 65535), the min(nprobe, nlist) nearest lists
 * into probes (B x min(nprobe, nlist)), nearest first.  Distances are the
 * reference's scalar l2_f32 (distance.rs:30-36: sqrt of the in-order sum of
 * (x - y)^2, no fused multiply-add), ties to the lower list index, so the
 * result equals bn_host_probe_route bit for bit; the reference's AVX-512
 * build sums in 16 lanes and may order near-ties differently. */
int bn_ivf_set_centroids(bn_ivf* h, const float* centroids, uint32_t d);
int bn_ivf_route(bn_ivf* h, uint32_t B, const float* queries, uint32_t nprobe, uint32_t* probes);
/* BnTmIvfScorer::score / score_batch (ivf.rs:746-927, 1199-1366) for B
 * queries with nprobe routed lists each (probes B x nprobe, in probe
 * order): every probed list of every query is scanned, verified, decoded
 * and ranked in one persistent launch per stage.  Inputs as in
 * bn_flat_query.  failed_cluster[b]/failed_trial[b] (nullable) name the
 * first probed list (probe order) whose verification failed, -1 if none. */
int bn_ivf_query(bn_ivf* h, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc,
                 const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz,
                 const uint8_t* v_seeds, uint32_t trials, uint32_t k, uint32_t* ids, int64_t* scores, uint32_t* n_hits,
                 int32_t* failed_cluster, int32_t* failed_trial);

/* IVF block scoring: the batch's (query, list) pairs grouped by list, so
 * that every probed list is read once per batch (byte-planar GEMMs on the
 * tensor cores, one group per list).  Scores and ranking as bn_ivf_query
 * (ivf.rs:746-927: every probed list, empty ones skipped, global top-k).
 * Protocol 2 per block and list: list c's draws are verify_response's
 * (crypto.rs:1013-1059) on list c with block_seed as the seed (ivf.rs:791-806
 * seeds one fresh ChaCha20Rng per list), shared by every query that probes c;
 * failed_cluster / failed_trial as bn_ivf_query.  No counterpart in the
 * reference, which verifies each (query, list) with the query's own seed.
 * Needs the int8-quantised client state (as bn_flat_query_block;
 * BN_EUNSUPPORTED otherwise); bn_ivf_block_prepare builds the byte-planar
 * corpus copies ahead of the first call. */
int bn_ivf_block_prepare(bn_ivf* h);
int bn_ivf_query_block(bn_ivf* h, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc,
                       const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz,
                       const uint8_t block_seed[32], uint32_t trials, uint32_t k, uint32_t* ids, int64_t* scores,
                       uint32_t* n_hits, int32_t* failed_cluster, int32_t* failed_trial);
/* GEMM tiling of later block calls (and of a server's IVF block batches):
 * W rows per tile (a multiple of 16 up to 256; the MMA N) and pipeline stages
 * (2..=12, capped by shared memory); 0 = chosen per batch from its groups. */
int bn_ivf_block_tune(bn_ivf* h, uint32_t w_tile, uint32_t stages);
/* Stage timing of later bn_ivf_query_block calls (enable = 1) and its read:
 * ms[0] = host planning and packing, ms[1..10] = device time of the stages
 * (H2D + operand images, G1, G2, G3, top-k, Protocol 2's u draws, z passes
 * and u . r sums, z . v and verdicts, D2H) of the last call; with more than
 * 32 trials the earlier trial chunks count in the u draws; *n = 0 before the
 * first profiled call. */
int bn_ivf_block_profile(bn_ivf* h, int enable);
int bn_ivf_block_profile_read(bn_ivf* h, float* ms, uint32_t cap, uint32_t* n);
/* Protocol 2 of the block form over claimed responses: r holds every
 * (query, list) pair's m_c responses, pairs in probe order (query-major,
 * empty lists skipped), r_len entries in all.  ur / zv (nullable, pairs x
 * trials, [pair][t]) = u_t . r_pair and z_t^c . v_q. */
int bn_ivf_verify_block(bn_ivf* h, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* r,
                        uint64_t r_len, const uint64_t* v_enc, const uint8_t block_seed[32], uint32_t trials,
                        int32_t* failed_cluster, int32_t* failed_trial, uint64_t* ur, uint64_t* zv);

/* ---------------------------------------------------------------- serving loop
 * Continuous batching over device-resident corpora.  No counterpart in the
 * reference, whose scorers serve one query per call with every GPU call
 * synchronous on one stream (gpu/mod.rs:169-200); the scoring semantics per
 * query are BnTmScorer::score (lib.rs:326-475) and BnTmIvfScorer::score
 * (ivf.rs:746-927), so each result equals bn_flat_query / bn_ivf_query on the
 * same inputs, alone or in any mix of requests.
 * Requests are queued by submit; a scheduler thread keeps up to `slots`
 * batches in flight (one stream and one workspace each).  A free slot takes
 * up to max_batch queued requests of one corpus (IVF requests with different
 * nprobe share a batch) once the batch is full or its oldest request has
 * waited max_wait_us.  Admission is by device memory: a batch's workspace
 * plus the workspaces the other slots hold must fit in mem_budget (0 = no
 * limit beyond the context budget); a batch is cut shorter to fit, and a
 * request that cannot fit alone fails with BN_EBUDGET.  Admission is also
 * by queue: submit returns BN_EAGAIN (nothing queued) when max_queue requests
 * are waiting, or when the queue's expected wait (waiting requests over the
 * recent completion rate) exceeds queue_wait_us, so that the latency of
 * admitted requests stays bounded past saturation.
 * Hits (ids, scores) equal bn_flat_query / bn_ivf_query on the same inputs,
 * alone or in any mix.  Protocol 2 of a per-query batch uses each request's
 * own seed; a block batch (block_min) is verified per block with one seed
 * derived from all its members' seeds (domain_separate of their XOR with the
 * tag "serve-block"), so an honest response is accepted in any mix, while
 * the first failing trial of a rejected one depends on the batch. */
typedef struct bn_server bn_server;
#define BN_SERVER_FLAT 0
#define BN_SERVER_IVF 1
typedef struct bn_server_config {
    uint32_t max_batch;   /* queries per launch, 1..=4096 */
    uint32_t slots;       /* batches in flight, 1..=16 */
    uint64_t mem_budget;  /* device bytes for the slots' workspaces (0: unlimited) */
    uint32_t max_wait_us; /* batching window */
    uint32_t trials;      /* Protocol 2 trials per query (params.verification_trials()) */
    uint32_t k;           /* hits per query */
    uint32_t block_min;   /* batches of >= block_min requests run as block scoring: flat ones as
                             bn_flat_block_plan (one pass over the corpus for the batch), IVF ones as
                             bn_ivf_query_block (every probed list read once per batch); Protocol 2 per
                             block (and list) with the batch seed; 0 = every query verified with its
                             own seed */
    uint32_t max_queue;     /* waiting requests at which submit returns BN_EAGAIN (0: unbounded) */
    uint32_t queue_wait_us; /* expected queue wait at which submit returns BN_EAGAIN (0: off) */
} bn_server_config;
typedef struct bn_server_stats_t {
    uint64_t submitted, completed, batches;
    double mean_batch;                 /* queries per launched batch */
    double p50_us, p99_us, max_us;     /* submit -> result latency */
    double throughput_qps;             /* completed / (last completion - first submit) */
    uint64_t peak_workspace_bytes;
    uint64_t block_batches;            /* batches (flat or IVF) that ran as block scoring */
    uint64_t rejected;                 /* submits refused with BN_EAGAIN (queue admission) */
} bn_server_stats_t;
/* flat and/or ivf (nullable, not both), with client state, in one context. */
int bn_server_create(bn_flat* flat, bn_ivf* ivf, const bn_server_config* cfg, bn_server** out);
/* Inputs as one query of bn_flat_query / bn_ivf_query (copied); v_seed = the
 * query's Protocol 2 seed (32 bytes).  *ticket identifies the result. */
int bn_server_submit_flat(bn_server* s, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                          const int8_t* t_sign, uint32_t t_nnz, const uint8_t* v_seed, uint64_t* ticket);
int bn_server_submit_ivf(bn_server* s, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc,
                         const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign, uint32_t t_nnz,
                         const uint8_t* v_seed, uint64_t* ticket);
/* Waits up to timeout_ms; BN_EAGAIN when not complete by then.  On success
 * the ticket is released: ids / scores (k entries), *n_hits, the first failing
 * trial (and IVF list) or -1, and the request's latency. */
int bn_server_wait(bn_server* s, uint64_t ticket, uint32_t timeout_ms, uint32_t* ids, int64_t* scores,
                   uint32_t* n_hits, int32_t* failed_trial, int32_t* failed_cluster, double* latency_us);
/* Counters and latency percentiles since creation or the last reset. */
int bn_server_stats(bn_server* s, int reset, bn_server_stats_t* out);
/* Drains queued and in-flight requests, then frees the server. */
int bn_server_destroy(bn_server* s);

/* ---------------------------------------------------------------- testing
 * No counterpart in the reference.  While `on` is non-zero, every Protocol 2
 * run on this context's handles behaves as if one of its draws had equalled
 * p (BN_EDRAW from the host-buffer calls, BN_STATUS_DRAW_HIT_P in
 * bn_plan_status, failed_trial = -2 from bn_flat_verify_noalloc), so that a
 * caller can exercise its handling of that 2^-61 event. */
int bn_debug_plant_draw_hit(bn_ctx* ctx, int on);
/* No counterpart in the reference.  Every device-side pipeline wait (an
 * mbarrier wait between the copy, MMA and drain roles of the scan, fused
 * Protocol 2 and block GEMM kernels) gives up after about a second, records
 * the event in the launch's status word and winds the kernel down, so a lost
 * completion cannot hang the GPU.  This sets that limit, in clock cycles,
 * for later launches on this context's handles (0 restores the default), so
 * that a test can make the waits run out: the call then returns BN_ECUDA and
 * bn_plan_status reports the bits.  The wind-down waits for a CTA's own
 * copies and MMAs keep the full limit. */
int bn_debug_set_wait_limit(bn_ctx* ctx, uint64_t cycles);

/* ---------------------------------------------------------------- keygen
 * encrypt_cluster (crypto.rs:405-478) on the device with host in/out:
 * m_enc = m_q + H L^T + S, a_l = m_q L.  Used to cross-check the device
 * encryption against a CPU restatement. */
/* Key generation on the device (regenerate_h_s, crypto.rs:258-270): H
 * (m x n1, row-major) and S (CSR) drawn from the cluster's h_seed with the
 * same ChaCha20 stream positions as bn_host_regenerate_h_s, which they equal
 * bit for bit; S is parsed in parallel (the column / sign draw structure
 * scanned as a two-state machine).  S must fit in s_cap entries (*nnz gets
 * the count either way; BN_EINVAL when it does not fit).  BN_EDRAW when an H
 * draw equalled p (the reference redraws there; odds 2^-61 per draw): use the
 * host keygen for that seed. */
int bn_keygen_h_s(bn_ctx* ctx, const uint8_t h_seed[32], uint64_t m, uint32_t n1, uint64_t* H, uint64_t* s_rowptr,
                  uint32_t* s_idx, int8_t* s_sign, uint64_t s_cap, uint64_t* nnz);
/* bn_flat_build_from_plain with the keys drawn on the device from h_seed
 * instead of passed in (BnTmScorer::upload_cluster, lib.rs:223-324 +
 * crypto.rs:405-478, with only the plaintext and L crossing the bus). */
int bn_flat_build_keygen(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1,
                         const uint64_t* l_subspace, const uint8_t h_seed[32], bn_flat** out);
/* bn_ivf_build_from_plain with every list's keys drawn on the device from
 * its own h_seed = derive_h_seed(upload_seed, list) (ivf.rs:258-264,
 * 627-653). */
int bn_ivf_build_keygen(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids,
                        const uint64_t* m_q, uint32_t n, uint32_t n1, const uint64_t* l_subspace,
                        uint64_t upload_seed, bn_ivf** out);
int bn_encrypt_cluster(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1,
                       const uint64_t* l_subspace, const uint64_t* h, bn_sparse_csr s_mat, uint64_t* m_enc,
                       uint64_t* a_l);

/* ---------------------------------------------------------------- corpora larger than device memory
 * Replaces the streaming cluster store (ClusterStore::get_or_upload,
 * scorer-gpu-common/src/store.rs:247-395) as the flat scorer uses it
 * (FlatGpuState, scorer-bntm/src/gpu/mod.rs:279-376): the corpus is cut
 * into chunks of chunk_rows rows (a multiple of 32) whose device images stay
 * in pinned host memory; device memory holds budget_bytes / slot_bytes chunk
 * slots, kept least-recently-used, and a query uploads the chunks it misses
 * on an upload stream while the resident ones are scored.  Results (hits,
 * failed_trial) equal bn_flat_query's on the same corpus bit for bit: every
 * chunk is scored as a row shard with its rows' Protocol 2 draw positions in
 * the whole corpus.  BN_EBUDGET when the budget holds no slot (the
 * reference's BudgetTooSmall).  Calls on one handle are serialised. */
typedef struct bn_stream bn_stream;
/* The store's counters (store.rs:36-80 ClusterStoreStats; gets counts one
 * per chunk visited, uploads / bytes_uploaded the chunk images copied in). */
typedef struct bn_store_stats {
    uint64_t gets, uploads, evictions, bytes_uploaded;
    uint64_t resident_bytes, budget_bytes;
} bn_store_stats;
/* From the encrypted corpus and the client state, as bn_flat_build followed
 * by bn_flat_attach_client. */
int bn_stream_build(bn_ctx* ctx, const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint64_t m,
                    uint32_t n, uint32_t n1, const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat,
                    uint64_t chunk_rows, uint64_t budget_bytes, bn_stream** out);
/* From the quantised plaintext and the keys, as bn_flat_build_from_plain
 * (each chunk encrypted on the device). */
int bn_stream_build_from_plain(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1,
                               const uint64_t* l_subspace, const uint64_t* h, bn_sparse_csr s_mat,
                               uint64_t chunk_rows, uint64_t budget_bytes, bn_stream** out);
int bn_stream_info(const bn_stream* st, uint64_t* rows, uint32_t* chunks, uint32_t* slots, uint64_t* slot_bytes,
                   uint64_t* host_bytes);
/* bn_flat_query over the streamed corpus (same arguments and outputs). */
int bn_stream_query(bn_stream* st, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                    const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
                    uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial);
int bn_stream_stats(bn_stream* st, int reset, bn_store_stats* out);
int bn_stream_destroy(bn_stream* st);
/* The IVF form (the reference's per-cluster uploads, IvfGpuState,
 * gpu/mod.rs:423-577): chunks of whole lists up to chunk_rows rows (a
 * longer list is a chunk of its own); a call uploads only the chunks that
 * hold a probed list.  Arguments and results as bn_ivf_build +
 * bn_ivf_attach_client, bn_ivf_build_keygen and bn_ivf_query (failed_cluster
 * / failed_trial: the first failing list in probe order). */
typedef struct bn_ivf_stream bn_ivf_stream;
int bn_ivf_stream_build(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids,
                        const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint32_t n, uint32_t n1,
                        const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat, uint64_t chunk_rows,
                        uint64_t budget_bytes, bn_ivf_stream** out);
int bn_ivf_stream_build_keygen(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids,
                               const uint64_t* m_q, uint32_t n, uint32_t n1, const uint64_t* l_subspace,
                               uint64_t upload_seed, uint64_t chunk_rows, uint64_t budget_bytes, bn_ivf_stream** out);
int bn_ivf_stream_info(const bn_ivf_stream* st, uint64_t* rows, uint32_t* chunks, uint32_t* slots,
                       uint64_t* slot_bytes, uint64_t* host_bytes);
int bn_ivf_stream_query(bn_ivf_stream* st, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc,
                        const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz,
                        const uint8_t* v_seeds, uint32_t trials, uint32_t k, uint32_t* ids, int64_t* scores,
                        uint32_t* n_hits, int32_t* failed_cluster, int32_t* failed_trial);
int bn_ivf_stream_stats(bn_ivf_stream* st, int reset, bn_store_stats* out);
int bn_ivf_stream_destroy(bn_ivf_stream* st);

/* The store's LRU bookkeeping alone, with no CUDA (the reference's LruInner,
 * store.rs:133-245): touch bumps an entry's recency (hit = 1) or reports a
 * miss; pre_evict pops least-recently-used entries until `bytes` fits on top
 * of the resident total (BN_EBUDGET, nothing evicted, when bytes exceeds the
 * budget); insert adds an entry (inserted = 0 when the id is resident, which
 * keeps the existing entry, as on the reference's insert race). */
typedef struct bn_lru bn_lru;
int bn_lru_create(uint64_t budget_bytes, bn_lru** out);
int bn_lru_touch(bn_lru* l, uint64_t id, int* hit);
int bn_lru_pre_evict(bn_lru* l, uint64_t bytes, uint64_t* evicted, uint32_t cap, uint32_t* n_evicted);
int bn_lru_insert(bn_lru* l, uint64_t id, uint64_t bytes, int* inserted);
int bn_lru_stats(const bn_lru* l, bn_store_stats* out);
int bn_lru_destroy(bn_lru* l);

#ifdef __cplusplus
}
#endif
#endif /* BN_B200_H */
