// bn_tc.cuh -- tensor-core (tcgen05, kind::i8) kernels of the BN path.
//
// Protocol 2 on tensor cores.  With M_enc viewed as bytes Mb[i][c]
// (c = 8j + a, a = byte a of the u64 element j) and the Freivalds draws as
// bytes Ub[i][(t,b)] (byte b of u_t[i]),
//     z_t[j] = sum_i u_t[i] M[i][j] = sum_{a,b} 2^(8(a+b)) D[8j+a][(t,b)],
//     D      = Mb^T Ub                      (exact u8 x u8 -> s32 GEMM),
// so the 61-bit F_p products become one integer GEMM on the tensor cores
// followed by a cheap limb recombination mod p.  The M_enc tile that TMA
// brings into shared memory (128 rows x 128 bytes, 128-byte swizzle) is the
// MMA's A operand read MN-major; the U tile is the K-major B operand.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "bn_chacha.cuh"
#include "bn_kernels.cuh"

namespace bn {

constexpr int TC_ROWS = 128;         // rows (K) per stage
constexpr int TC_PANEL_ROWS = 4096;  // rows accumulated in TMEM before a drain (4096 * 255^2 < 2^31)
constexpr int TC_MAX_TRIALS = 20;    // per pass: N = 8 * trials_padded <= 160

// One panel of a verify segment: rows [row0, row0 + rows) of m_enc, whose U
// tiles start at row block `rb0` of the U buffer.
struct TcPanel {
    uint64_t row0;
    uint32_t rows;
    uint32_t rb0;
    uint32_t seg;
    uint32_t pad;
};

// Row block of the U generator: 128 rows of segment `seg` starting at local row `i0`.
struct TcBlock {
    uint32_t seg;
    uint32_t i0;
};

// Encodes the 2-D tensor maps (driver entry point; no -lcuda needed).
// Returns cudaSuccess or the failure.
cudaError_t make_tmap_u8(CUtensorMap* map, const void* base, uint64_t inner_bytes, uint64_t rows, uint32_t box_inner,
                         uint32_t box_rows);
// 3-D view {128 bytes, rows, row_bytes / 128 K steps} of a row-major byte
// matrix whose box {128, box_rows, 2} lands as two consecutive K steps'
// [box_rows x 128] tiles (128-byte swizzle); coordinates (0, row, k / 128).
cudaError_t make_tmap_u8_ksteps2(CUtensorMap* map, const void* base, uint64_t row_bytes, uint64_t rows,
                                 uint32_t box_rows);

// u generation: for each row block, U tile bytes [(t,b)][128 rows] (K-major
// B operand image, un-swizzled; TMA applies the swizzle) for trials
// [t_base, t_base + t_cnt), padded with zero rows up to n_rows = 8 * t_pad,
// and u_t . r partial sums per block.  *flags bit 0: a draw hit p.
// u_row_pitch = 0: per-block images (block b at d_u + b * n_rows * 128);
// otherwise one flat image, row (t,b) at d_u + (t*8+b) * u_row_pitch and the
// draw for r index x at byte column x (x = segment r0 + row).
void launch_tc_ugen(const VerifySeg* d_vsegs, const TcBlock* d_blocks, uint32_t nblocks, const ChaChaKey* d_keys,
                    const uint64_t* d_r, uint32_t t_base, uint32_t t_cnt, uint32_t n_rows, uint8_t* d_u,
                    uint64_t* d_ur_part, uint32_t trials_total, uint32_t* d_flags, cudaStream_t s,
                    uint64_t u_row_pitch = 0);

// The GEMM + drain: z_part[panel][t_base + t][j] (canonical residues) for
// t < t_cnt.  tmap_m: m_enc bytes {8192, rows}, box {128, 128}, swizzle 128B;
// tmap_u: U bytes {128, nblocks * n_rows}, box {128, n_rows}, swizzle 128B
// (u_flat = 0), or the flat image {row pitch, n_rows}, box {128, n_rows}
// (u_flat = 1; panel rb0 = first row / 128).
// *err: bit 2/3/4 set when a bounded pipeline wait timed out, bit 64 when
// the wind-down wait for the CTA's own MMAs did.  wait_cycles: limit of the
// pipeline waits (0 = about a second; shorter only to test the timeout path).
void launch_tc_freivalds(const CUtensorMap& tmap_m, const CUtensorMap& tmap_u, const TcPanel* d_panels,
                         uint32_t npanels, uint32_t t_base, uint32_t t_cnt, uint32_t n_rows, uint32_t trials_total,
                         uint64_t* d_z_part, uint32_t* d_err, int num_sms, cudaStream_t s, int u_flat = 0,
                         long long wait_cycles = 0);

// The same for panels [p_first, p_first + npanels) of at most
// TC_SMALL_PANEL_ROWS rows (short IVF lists): whole panels per CTA, the
// panel's U tiles resident in shared memory, one strip per work item into
// three rotating accumulators (n_rows <= 160) so drains overlap the MMAs.
constexpr uint32_t TC_SMALL_PANEL_ROWS = 3 * 128;
void launch_tc_freivalds_small(const CUtensorMap& tmap_m, const CUtensorMap& tmap_u, const TcPanel* d_panels,
                               uint32_t p_first, uint32_t npanels, uint32_t t_base, uint32_t t_cnt,
                               uint32_t n_rows, uint32_t trials_total, uint64_t* d_z_part, uint32_t* d_err,
                               int num_sms, cudaStream_t s, long long wait_cycles = 0);

// Fused single pass over m_enc for the first <= 20 trials, both products on
// the tensor cores: z_part as above plus r_part[group][r index] (3-strip
// group partial dots with the query, r_stride = total r entries, 22 groups),
// summed by launch_tc_rreduce.  tmap_w: the queries' diagonal byte images
// (launch_query_wimg) {128, nq * 1024}, box {128, 48}, swizzle 128B.
void launch_tc_fused(const CUtensorMap& tmap_m, const CUtensorMap& tmap_u, const CUtensorMap& tmap_w,
                     const TcPanel* d_panels, uint32_t npanels, const VerifySeg* d_vsegs, uint32_t t_cnt,
                     uint32_t n_rows, uint32_t trials_total, uint64_t* d_z_part, uint64_t* d_r_part, uint64_t r_stride,
                     uint32_t* d_err, int num_sms, cudaStream_t s, long long wait_cycles = 0);
inline uint32_t tc_groups(uint32_t) { return 22u; }  // strip groups of the fused pass (3 strips each)
constexpr uint32_t WIMG_BYTES_PER_QUERY = 64u * 16u * 128u;
constexpr uint32_t WIMG_BOX_ROWS = 48;  // one strip group's diagonal rows
// w[((q * 64 + strip) * 16 + s) * 128 + 8 j + a] = byte (s - a) of
// v[q][strip * 16 + j] (0 <= s - a <= 7), else 0.
void launch_query_wimg(const uint64_t* d_v, uint32_t nq, uint8_t* d_w, cudaStream_t s);
// r = sum of the group partials, and u_t . r partials for the pass's trials
// from the U byte image.
void launch_tc_rreduce(const VerifySeg* d_vsegs, const TcBlock* d_blocks, uint32_t nblocks, const uint64_t* d_r_part,
                       uint64_t r_stride, uint32_t groups, const uint8_t* d_u, uint32_t t_cnt, uint32_t n_rows,
                       uint32_t trials_total, uint64_t* d_r, uint64_t* d_ur_part, cudaStream_t s);

// Per segment: z_t = sum of its panels' partials, zv_t = z_t . v, ur_t =
// sum of its blocks' partials; failed = first t with ur_t != zv_t or -1.
// d_chunks: scratch of tc_finish_words(nseg, trials) words (the shares of z . v
// and u . r that the finish kernel's CTAs write and the decide kernel sums).
// With few segments each one's panels are split over tc_finish_split CTAs.
inline uint32_t tc_finish_split(uint32_t nseg) { return nseg <= 4 ? 16u : 1u; }
inline uint64_t tc_finish_words(uint32_t nseg, uint32_t trials) {
    return (uint64_t)nseg * trials * (N / 128 + 1) * tc_finish_split(nseg);
}
void launch_tc_finish(const uint64_t* d_z_part, const uint64_t* d_ur_part, const uint32_t* d_seg_panel0,
                      const uint32_t* d_seg_block0, const uint64_t* d_v_enc, const VerifySeg* d_vsegs, uint32_t nseg,
                      uint32_t trials, uint64_t* d_ur, uint64_t* d_zv, uint64_t* d_chunks, int32_t* d_failed,
                      cudaStream_t s);

}  // namespace bn
