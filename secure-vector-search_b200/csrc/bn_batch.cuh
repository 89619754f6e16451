// bn_batch.cuh -- block (many-query) scoring on the tensor cores.
//
// compute_products_batch (crypto.rs:782-828) as an exact integer GEMM.
// Every u64 operand is split into its 8 bytes and stored "byte-planar": the
// row of element (i, j) becomes 8 rows (i, a), a = byte index, each holding
// byte a of every element of the original row.  Then
//     r_q[i] = sum_j M[i][j] v_q[j]
//            = sum_{a,b} 2^(8(a+b)) sum_j Mp[(i,a)][j] Vp[(q,b)][j]
//            = sum_{a,b} 2^(8(a+b)) D[(i,a)][(q,b)],   D = Mp Vp^T,
// one u8 x u8 -> s32 GEMM (tcgen05.mma kind::i8, exact while K * 255^2 <
// 2^31) whose epilogue folds the 64 byte products of each (i, q) back into a
// residue mod p.  The same kernel computes the decode terms and the block's
// Freivalds dot products u_t . r_q (A = byte planes of r, K = corpus rows).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "bn_kernels.cuh"

namespace bn {

constexpr int BG_AROWS = 128;              // A rows per work item (TMEM lanes)
constexpr int BG_KSTEP = 128;              // K bytes per pipeline stage (one 128-byte swizzle atom)
constexpr int BG_MAX_STAGES = 12;
constexpr int BG_MAX_ASLOTS = 8;           // A-resident mode: K <= 8 * 128 bytes
constexpr uint32_t BG_MAX_SMEM = 232448;   // dynamic shared memory per CTA on sm_100
constexpr uint32_t BG_MAX_KPANEL = 16384;  // K bytes summed in s32 before a drain: 16384 * 255^2 < 2^31

enum BgMode : int {
    // u8 x u8; A rows (x, a), W rows (y, b); f(x, y) = sum 2^(8(a+b)) D mod p.
    // out[kp * out_pstride + y * out_ld + x] = f.
    // planar_out (nullable): byte a of f at planar_out[(y * 8 + a) * planar_ld + x].
    BG_PLANAR = 0,
    // s8 x s8; A rows x, W rows (y, b); f(x, y) = sum_b 2^(8b) D mod p.
    // out[y * out_ld + x] = f + corr[x].
    BG_S8 = 1,
};

// One work item of a grouped GEMM (an item table): the A tile (its TMA row,
// or its tile index when A is K-blocked) and the W tile's TMA row, the corpus
// rows x in [x0, x_lim) and the output slots y in [y0, y_lim) that the item's
// outputs may write (outputs go to out[pair_base[y] + x]).
struct BgItem {
    uint32_t a_y, w_y;
    uint32_t x0, x_lim;
    uint32_t y0, y_lim;
};

struct BgParams {
    int mode;
    uint32_t a_tiles;      // ceil(A rows / 128)
    uint32_t w_tiles;      // ceil(W rows / w_tile)
    uint32_t w_tile;       // W rows per item = MMA N (multiple of 16, 16..256)
    uint32_t k_bytes;      // K extent (multiple of 128)
    uint32_t k_panel;      // K bytes per item (multiple of 128, <= BG_MAX_KPANEL)
    uint32_t x_count;      // valid x (PLANAR: A rows / 8; S8: A rows)
    uint32_t y_count;      // valid y (W rows / 8)
    uint64_t* out;
    uint64_t out_ld;
    uint64_t out_pstride;  // per K panel (PLANAR)
    const uint64_t* corr;  // S8
    uint8_t* planar_out;   // PLANAR, nullable
    uint64_t planar_ld;
    int order_a_fast;      // work order: 0 = W tile fastest, 1 = A tile fastest
    int a_resident;        // keep each A tile (all of K, one K panel) in shared memory across its W tiles
    int a_blocked;         // A is K-blocked (launch_planar_rows with ks = k_bytes / 128): a_y = tile index
    int ksteps2;           // two K steps (256 bytes) per pipeline stage: needs k_panel a multiple of
                           // 256, tmap_w2, and (streaming A) a_blocked with tmap_a2
    // grouped mode (nullable): work items from a table instead of the a_tiles x
    // w_tiles grid (one K panel, no A-resident mode, no planar_out)
    const BgItem* item_tab;
    uint32_t n_items;
    const uint64_t* pair_base;  // grouped outputs: out[pair_base[y] + x]
    long long wait_cycles;      // limit of the pipeline waits (0 = about a second; shorter only in tests)
};

// tmap_a: A bytes {k_bytes, A rows}, box {128, 128}; tmap_w: W bytes
// {k_bytes, W rows}, box {128, w_tile}; both 128-byte swizzle.  stages in
// [2, BG_MAX_STAGES].  *err: bit 2/3/4 set when a bounded wait timed out,
// bit 64 when the wind-down wait for the CTA's own MMAs did.
// A-resident mode needs k_panel == k_bytes <= BG_MAX_ASLOTS * 128 and
// bgemm_smem_bytes(p, stages) <= BG_MAX_SMEM.
// With p.ksteps2: tmap_a2 = the K-blocked A with 256-row boxes (two K steps
// of a tile), tmap_w2 = make_tmap_u8_ksteps2 of the W bytes.
void launch_bgemm(const CUtensorMap& tmap_a, const CUtensorMap& tmap_w, const BgParams& p, uint32_t stages, int ctas,
                  uint32_t* d_err, cudaStream_t s, const CUtensorMap* tmap_a2 = nullptr,
                  const CUtensorMap* tmap_w2 = nullptr);
// Most pipeline stages whose shared memory fits one CTA (0 when even 2 do not).
uint32_t bgemm_max_stages(const BgParams& p);
uint32_t bgemm_stage_bytes(uint32_t w_tile, bool a_resident, uint32_t ksub = 1);
uint32_t bgemm_smem_bytes(const BgParams& p, uint32_t stages);

// Byte planes of a row-major u64 matrix: byte a of (negate ? p - src :
// src)[i * src_ld + j], j < k (k % 16 == 0), goes to plane row r = pi * 8 + a
// (pi = d_prow[i], or i when d_prow is null), column col0 + j: row-major at
// dst[r * dst_ld + col0 + j] (ks = 0), or K-blocked (ks > 0: tiles of 128
// plane rows stored as ks runs of 128 rows x 128 bytes, the layout of the
// corpus-side A operands, whose every (tile, K-step) TMA box is contiguous).
void launch_planar_rows(const uint64_t* d_src, uint64_t rows, uint32_t k, uint64_t src_ld, int negate, uint8_t* d_dst,
                        uint64_t dst_ld, uint32_t col0, cudaStream_t s, const uint32_t* d_prow = nullptr,
                        uint32_t ks = 0);
// Same from a column-major source: element (i, j) at src_cm[j * rows + i].
void launch_planar_cm(const uint64_t* d_src_cm, uint64_t rows, uint32_t k, uint8_t* d_dst, uint64_t dst_ld,
                      uint32_t col0, cudaStream_t s, const uint32_t* d_prow = nullptr, uint32_t ks = 0);
// [M | S] as signed bytes, 2n per row, K-blocked (16 K-steps per 128-row
// tile), corpus row i at row d_prow[i] (or i): M from mp_cm (residues of
// values in [-128, 127], else *bad |= 1), S from the sliced ELL; corr[i] =
// 128 * rowsum(S_i) * (2^64 - 1) / 255 mod p.
void launch_ms8(const uint64_t* d_mp_cm, const uint16_t* d_s_ell, const uint32_t* d_s_off, const uint16_t* d_s_w,
                uint64_t rows, int8_t* d_dst, uint64_t* d_corr, uint32_t* d_bad, cudaStream_t s,
                const uint32_t* d_prow = nullptr);
// W operand of the signed decode GEMM for nq queries: rows (q, b) of 2n
// bytes: [T_q if b == 0 else 0 | byte b of v_q - 128].  T entries as in
// DecodeQuery (col | 0x80000000 for -1); *bad |= 2 when a column sum leaves
// [-128, 127].
void launch_w_tv(const uint64_t* d_v, const uint32_t* d_t, const uint32_t* d_t_nnz, uint32_t nq, int8_t* d_dst,
                 uint32_t* d_bad, cudaStream_t s);
// z_t = sum over panels of z_part[panel][t_base + t][j] -> z[t_base + t][j].
void launch_zsum(const uint64_t* d_z_part, uint32_t npanels, uint32_t t_base, uint32_t t_cnt, uint32_t trials_total,
                 uint64_t* d_z, cudaStream_t s);
// zv[t][q] = z_t . v_q for t < trials, q < nq.
void launch_zv(const uint64_t* d_z, const uint64_t* d_v, uint32_t trials, uint32_t nq, uint64_t* d_zv, cudaStream_t s);
// ur[t][q] = sum over K panels of ur_part[kp][t][q]; failed[q] = first t with
// ur != zv, or -1.  d_ur (nullable) receives the sums.
void launch_ur_decide(const uint64_t* d_ur_part, uint32_t kpanels, uint32_t trials, uint32_t nq, const uint64_t* d_zv,
                      uint64_t* d_ur, int32_t* d_failed, cudaStream_t s);

}  // namespace bn
