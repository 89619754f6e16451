// bn_kernels.cuh -- launchers for the BN device kernels (sm_100a).
//
// Device data layout (one flat corpus, or the concatenation of all IVF
// lists in list order):
//   m_enc   u64 [rows][1024]   row-major, 8 KiB per row   (server state)
//   al_cm   u64 [128][rows]    AL, column-major           (client state)
//   h_cm    u64 [128][rows]    H,  column-major
//   mp_cm   u64 [1024][rows]   plaintext M, column-major  (M*T column sums)
//   s_ell   u16 sliced-ELL of S: 32-row slices, entry = col for +1,
//           ELL_NEG + col for -1, ELL_PAD = padding (an index into the
//           signed table [v, 0, p - v] of a query); s_off[slice] = u32
//           offset of the slice's data, s_w[slice] = width
//   ids     u32 [rows]         global vector id of each row (IVF), or null
// Decode copies of the client state, in blocks of 32 rows (rows32 = rows
// rounded up to 32; entries past the last row are 0):
//   alh_b   u64 [rows32/32][2*n1][32]  AL columns then H columns
//   m8_cm   s8  [1024][rows32]         plaintext M column-major, when every
//           entry is int8-valued (quantised corpora), else absent
// A warp that decodes 32 consecutive rows reads one 256-byte run per column
// of alh_b (a block's columns are contiguous) and one 32-byte run per T
// column of m8_cm.
// Column-major client arrays make the thread-per-row reads of the other
// kernels coalesced; the row-major m_enc makes the scan's warp-per-row reads
// coalesced.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bn_chacha.cuh"
#include "bn_fp.cuh"

namespace bn {

// Sliced-ELL entries of S (layout note above); ELL_TABLE entries of the
// decode's signed table, the last one a zero past every valid entry.
constexpr uint32_t ELL_PAD = 1024, ELL_NEG = 1025, ELL_TABLE = 2 * 1024 + 2;

// Per-query operand limbs for the scan: v = b0 + b1 2^21 + b2 2^42 and the
// same split of v * 2^32 mod p (c0..c2), padded to 32 bytes.
struct QLimb {
    uint32_t b0, b1, b2, c0, c1, c2, pad0, pad1;
};

// A contiguous run of rows scanned against one query; r lands at out0.
struct ScanSeg {
    uint64_t row0;
    uint64_t out0;
    uint32_t rows;
    uint32_t query;
};

// Rows per work item of the scan (one group of four warps).
constexpr int SCAN_ROWS = 4;

// Freivalds: per (segment, trial group) the u stream is ChaCha20Rng keyed
// by v_seed; u_t[i] is draw number t*m_seg + i of that stream (crypto.rs:
// 1026-1027).  A row shard of a larger corpus (bn_flat_query_shard) draws
// at its rows' positions in the whole corpus: t * draw_stride + draw_base + i.
struct VerifySeg {
    uint64_t row0;         // first row in m_enc
    uint64_t r0;           // first r value of this segment
    uint32_t rows;         // m of the list / flat corpus
    uint32_t query;        // index into v_enc / keys arrays
    uint64_t draw_stride;  // draws per trial (0: rows)
    uint64_t draw_base;    // draw position of the segment's first row within a trial
};
__host__ __device__ __forceinline__ uint64_t draw_index(const VerifySeg& vs, uint32_t t, uint64_t i) {
    return (uint64_t)t * (vs.draw_stride ? vs.draw_stride : vs.rows) + vs.draw_base + i;
}

// DRAW_HIT_P is or-ed into a Protocol 2 kernel's flag word if a draw hit the rejected
// value p (probability 2^-61 per draw), meaning later draws of the
// reference stream would be shifted by one (sample_fp redraws,
// crypto.rs:155-162); the host then fails the call with BN_EDRAW.  The bit
// is the public BN_STATUS_DRAW_HIT_P and stays clear of the wait-timeout
// bits (0x1..0x40) and the block path's T-range bit (0x100).
constexpr uint32_t DRAW_HIT_P = 0x1000u;

// *d_word |= bits on the stream (plants the draw flag for
// bn_debug_plant_draw_hit).
void launch_or_flag(uint32_t* d_word, uint32_t bits, cudaStream_t s);

// Loads the kernels launch_freivalds / launch_freivalds_finish use on the
// current device (CUDA loads modules lazily, on first use, and a load
// allocates device memory); the allocation-free verifier calls it at
// context set-up.
cudaError_t preload_freivalds_kernels();

void launch_query_limbs(const uint64_t* d_v, uint32_t nq, QLimb* d_limbs, cudaStream_t s);

// Segment scan: r[out0 + i] = sum_j m_enc[row0 + i][j] * v[query][j] mod p.
// seg_blk: exclusive prefix sum over ceil(rows / SCAN_ROWS), nseg + 1 entries.
// d_err (device u32): bit 0/1 set if a pipeline wait timed out (the scan
// result is then invalid); the kernel never waits without a bound.
// wait_cycles: limit of the pipeline waits (0 = about a second; shorter only
// to test the timeout path).
void launch_scan(const uint64_t* d_m_enc, const QLimb* d_limbs, const ScanSeg* d_segs, const uint64_t* d_seg_blk,
                 uint32_t nseg, uint64_t total_blocks, uint64_t* d_r, int num_sms, uint32_t* d_err, cudaStream_t s,
                 long long wait_cycles = 0);

// Freivalds partial sums for one segment list.  z_part: [nseg][chunks][T][1024],
// ur_part: [nseg][chunks][T].  chunk_rows: rows per chunk (multiple of 32).
struct FreivaldsPlan {
    uint32_t chunks;      // per segment
    uint32_t chunk_rows;
};
FreivaldsPlan plan_freivalds(uint64_t max_rows, uint32_t nseg, int num_sms);
void launch_freivalds(const uint64_t* d_m_enc, const uint64_t* d_r, const VerifySeg* d_vsegs, uint32_t nseg,
                      const ChaChaKey* d_keys, uint32_t trials, FreivaldsPlan plan, uint64_t* d_z_part,
                      uint64_t* d_ur_part, uint32_t* d_flags, cudaStream_t s);
// Per segment: ur[t], zv[t], first failing trial (-1 if none).
void launch_freivalds_finish(const uint64_t* d_z_part, const uint64_t* d_ur_part, const uint64_t* d_v_enc,
                             const VerifySeg* d_vsegs, uint32_t nseg, uint32_t trials, FreivaldsPlan plan,
                             uint64_t* d_ur, uint64_t* d_zv, int32_t* d_failed, cudaStream_t s);

// x = L^T v for nq queries: L is [1024][n1] row-major, x is [nq][n1].
void launch_lt_times_v(const uint64_t* d_L, uint32_t n1, const uint64_t* d_v, uint32_t nq, uint64_t* d_x,
                       cudaStream_t s);

// Dense decode terms only: out[i] = AL_i . g + H_i . x (FlatGpuState::
// decode_dense_terms, gpu/mod.rs:390-408).
void launch_dense_terms(const uint64_t* d_al_cm, const uint64_t* d_h_cm, uint64_t rows, uint32_t n1,
                        const uint64_t* d_g, const uint64_t* d_x, uint64_t* d_out, cudaStream_t s);

// Per-query segment range for decode + rank.  Query q's operands sit at
// fixed strides: v_enc at q*1024, g and x at q*n1, T entries at q*1024
// (t_nnz[q] of them, entry = col | 0x80000000 for -1).
struct DecodeQuery {
    uint32_t seg0;     // first segment of this query in the segment array
    uint32_t nseg;
    uint32_t cta0;     // the query's decode CTAs: [cta0, cta0 + ctas) of the launch
    uint32_t ctas;
};

// Resident decode_topk CTAs per SM (its register bound); the host sizes
// the decode grid to one wave of them.
constexpr int DECODE_CTAS_PER_SM = 3;

// Top-k candidate lists.
constexpr int TOPK_MAX = 1024;
constexpr int DECODE_CTAS_PER_QUERY_MAX = 148;

struct TopkScratch {
    int64_t* cand_s;    // [CTAs][k]
    uint32_t* cand_i;
    uint32_t* cand_n;   // [CTAs]
    uint32_t* done;     // [nq] CTAs finished (decode_topk only; zeroed by its launcher)
};

// The corpus arrays the decode reads (layouts above).
struct DecodeCorpus {
    const uint64_t* alh_b;
    const int8_t* m8_cm;    // null: M T from mp_cm
    const uint64_t* mp_cm;
    const uint16_t* s_ell;
    const uint32_t* s_off;
    const uint16_t* s_w;
    const uint32_t* ids;    // null: ids are row numbers
    uint64_t rows;
    uint32_t n1;
};

// Builds alh_b from al_cm / h_cm and m8_cm from mp_cm (m8_cm nullable, e.g.
// without client state); *d_bad (zeroed here) gets bit 0 if an entry of
// mp_cm is not int8-valued, in which case m8_cm must not be used.
void launch_decode_layout(const uint64_t* d_al_cm, const uint64_t* d_h_cm, const uint64_t* d_mp_cm, uint64_t rows,
                          uint32_t n1, uint64_t* d_alh_b, int8_t* d_m8_cm, uint32_t* d_bad, cudaStream_t s);

// Decode + fp_to_signed + top-k for every query: each CTA ranks its rows,
// and the last CTA of a query to finish merges the CTAs' lists into
// out_ids/out_scores [nq][k] (score desc, id asc) and out_n [nq].
// r is indexed like the scan output (segment out0).  mv_out (nullable)
// receives the decoded residues at the same offsets.  The work units are
// the aligned 32-row corpus blocks each segment touches: segment s owns
// units [d_seg_unit[s], d_seg_unit[s + 1]) (nseg + 1 entries).  The launch
// has total_ctas CTAs, query q owning d_q[q].cta0 .. + d_q[q].ctas (every
// query at least one; cta0 ascending); the scratch lists are indexed by CTA.
void launch_decode_topk(const uint64_t* d_r, const DecodeCorpus& dc, const ScanSeg* d_segs, const uint64_t* d_seg_unit,
                        const DecodeQuery* d_q, uint32_t nq, const uint64_t* d_v, const uint64_t* d_g, const uint64_t* d_x, const uint32_t* d_t,
                        const uint32_t* d_t_nnz, uint32_t k, uint32_t total_ctas, TopkScratch scratch,
                        uint64_t* d_mv_out, uint32_t* d_out_ids, int64_t* d_out_scores, uint32_t* d_out_n,
                        cudaStream_t s);

// Top-k over residues combined on the fly, mv = a + b - c at [q * ld + i]
// (i < rows; ld even; b, c nullable), ranked by to_signed, ids[i] or i;
// outputs as launch_decode_topk; d_mv_out (nullable) receives mv.
void launch_topk_rows(const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_c, uint64_t ld, uint64_t rows,
                      uint32_t nq, const uint32_t* d_ids, uint32_t k, int ctas_per_query, TopkScratch scratch,
                      uint32_t* d_out_ids, int64_t* d_out_scores, uint32_t* d_out_n, uint64_t* d_mv_out,
                      cudaStream_t s);

// The same over a segmented array: query q's entries are [qoff[q],
// qoff[q+1]) of a, b, c (each allocated to an even length), ids[i] per entry.
void launch_topk_segs(const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_c, const uint64_t* d_qoff,
                      uint32_t nq, const uint32_t* d_ids, uint32_t k, int ctas_per_query, TopkScratch scratch,
                      uint32_t* d_out_ids, int64_t* d_out_scores, uint32_t* d_out_n, cudaStream_t s);

// Keygen on the device (regenerate_h_s, crypto.rs:258-270) from a cluster's
// h_seed: H = the first `count` = m * n1 draws (sample_fp; DRAW_HIT_P in
// *d_flags if one equalled p), row-major.
void launch_keygen_h(const uint8_t seed[32], uint64_t count, uint64_t* d_H, uint32_t* d_flags, int num_sms,
                     cudaStream_t s);
// S as CSR: d_rowptr (m + 1, from 0), d_idx / d_sign (at most cap entries,
// in row order, columns ascending).  d_scratch: keygen_s_scratch_bytes(m, n).
// d_status[0] = 1 when the scanned keystream held all m * n column draws,
// d_status[1] = 1 when S had more than cap entries (both zeroed by the caller).
uint64_t keygen_s_scratch_bytes(uint64_t m, uint32_t n);
void launch_keygen_s(const uint8_t seed[32], uint64_t m, uint32_t n, uint32_t n1, uint32_t thr, void* d_scratch,
                     uint64_t cap, uint32_t* d_idx, int8_t* d_sign, uint64_t* d_rowptr, uint32_t* d_status,
                     cudaStream_t s);
// d_dst[i] = base + d_src[i], i < count (one list's row pointers in a concatenated CSR).
void launch_rowptr_shift(const uint64_t* d_src, uint64_t count, uint64_t base, uint64_t* d_dst, cudaStream_t s);

// Keygen-side dense F_p GEMM: C[i][j] = sum_k A[i][k] * B[j][k]  (A: rows x K,
// B: cols x K, both row-major), optionally C += D (same shape, row-major).
// K must be a multiple of 16 and at most 1024.
void launch_gemm_abt(const uint64_t* d_A, const uint64_t* d_B, const uint64_t* d_D, uint64_t rows, uint32_t cols,
                     uint32_t K, uint64_t* d_C, cudaStream_t s);
// Applies a CSR {-1,+1} matrix: C[i][idx] +-= 1 (mod p).
void launch_apply_sparse(const uint64_t* d_rowptr, const uint32_t* d_idx, const int8_t* d_sign, uint64_t rows,
                         uint32_t cols, uint64_t* d_C, cudaStream_t s);
// Row-major [rows][cols] -> column-major: out[c * out_ld + r].
void launch_transpose_u64(const uint64_t* d_in, uint64_t rows, uint32_t cols, uint64_t* d_out, uint64_t out_ld,
                          cudaStream_t s);
// CSR -> sliced ELL (see layout note above); s_off/s_w computed on host.
void launch_csr_to_ell(const uint64_t* d_rowptr, const uint32_t* d_idx, const int8_t* d_sign, uint64_t rows,
                       const uint32_t* d_s_off, const uint16_t* d_s_w, uint16_t* d_s_ell, cudaStream_t s);

}  // namespace bn
