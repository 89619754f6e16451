// bn_ivf_block.cu -- IVF block scoring: a batch's (query, list) pairs grouped
// by list, so that every probed list is read once per batch.
//
// The reference scores an IVF batch by looping its per-query path
// (BnTmIvfScorer::score_batch, ivf.rs:1199-1366; on GPU handles ivf.rs:1357-1364),
// which reads list c once for every query that probes it.  Here the pairs are
// sorted by list and list c, probed by n_c queries of the batch, becomes one
// group of the grouped byte-planar GEMM (bgemm item tables): its A tiles are
// the list's rows, its W tiles the n_c queries' operand images.  Per pair (q, c):
//   r_qc  = M_c v_q                        (G1: planes of m_enc x planes of v)
//   f2_qc = -(AL_c g_q + H_c L^T v_q)      (G2: planes of [AL | H] x planes of -[g | x])
//   f3_qc = M_c T_q + S_c v_q              (G3: signed bytes [M | S] x [T | bytes(v) - 128])
//   Mv_qc = r + f2 - f3                     (decode_scores, crypto.rs:901-940)
// in "r-space": query q's probed lists in probe order, empty lists skipped
// (ivf.rs:787-789), then a segmented top-k per query over all its lists
// (score desc, id asc; the global merge of ivf.rs:805-815).
//
// Protocol 2 per block and list: list c's draws are those of verify_response
// (crypto.rs:1013-1059) run on list c with the block seed in place of the
// query seed (ivf.rs:792-800 seeds a fresh ChaCha20Rng per list): u_t[i] =
// draw t*m_c + i of ChaCha20Rng(block_seed).  They are shared by the queries
// that probe c:
//   z_t^c = u_t^T M_c          (tc_freivalds over the batch's distinct lists, once each)
//   pair (q, c) passes trial t iff u_t . r_qc == z_t^c . v_q,
// and query q is rejected at its first failing list in probe order.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>

#include "bn_batch.cuh"
#include "bn_internal.cuh"
#include "bn_tc.cuh"

using namespace bn;
using namespace bn::api;

namespace bn {
namespace api {

namespace {

// One (query, list) pair, in q-major order (query q's probes in order).
struct IvPair {
    uint64_t out0;     // first r-space entry
    uint32_t q, list;  // query, list id
    uint32_t u;        // index of the list among the batch's distinct lists
    uint32_t ch0, nch; // its ur chunks
    uint32_t pad;
};

// Up to IV_CHUNK_ROWS rows of one pair (ids; u . r partial sums per chunk).
struct IvChunk {
    uint64_t r0;    // first r-space entry
    uint64_t row0;  // first corpus row
    uint32_t ublk;  // first 128-row block of the list's U image
    uint32_t rows;
};
constexpr uint32_t IV_CHUNK_ROWS = 2048;

// u . r work of one CTA: chunk c of a list (its U blocks from ublk0 on) for
// up to UR_SLAB of the list's pairs (list-major positions lp0 ...).
struct IvUrTask {
    uint32_t ublk0, rows;
    uint32_t lp0, npairs;
    uint32_t c;
};
constexpr uint32_t UR_SLAB = 8;
constexpr uint32_t UR_WARPS = 8;
constexpr uint32_t UR_PER_WARP = (UR_SLAB * TC_MAX_TRIALS + UR_WARPS - 1) / UR_WARPS;

// One distinct list of a batch: a group of the grouped GEMMs.
struct IvGroup {
    uint32_t row0, m;       // corpus rows of the list
    uint32_t lp0, n;        // its pairs, list-major
    uint32_t it_pl, it_s8;  // first item of the PLANAR (16-row A tiles) and S8 (128-row A tiles) tables
    uint32_t t16, t128;     // the list's first tile in the K-blocked planes / [M | S] bytes
};

// A list of several z panels: z[m][t][j] = sum of its panels' z_part[p][t][j].
struct IvZsum {
    uint32_t p0, p1;  // panels
    uint32_t m;       // slot in z
};

// ------------------------------------------------------------------ kernels
// dst block lp (8 rows of row_bytes) = src block map[lp]
__global__ void gather8_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst, const uint32_t* __restrict__ map,
                               uint32_t n, uint32_t row_bytes) {
    const uint32_t per = 8 * row_bytes / 16;
    const uint64_t total = (uint64_t)n * per;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t lp = (uint32_t)(e / per), c = (uint32_t)(e % per);
        dst[(uint64_t)lp * per + c] = src[(uint64_t)map[lp] * per + c];
    }
}

// The grouped GEMMs' item tables: group u owns PLANAR items [it_pl(u),
// it_pl(u + 1)), W tiles outer x 16-row A tiles inner, and S8 items likewise
// with 128-row A tiles (every group has at least one item of each).
__global__ void expand_items_kernel(const IvGroup* __restrict__ groups, uint32_t U, uint32_t n_pl, uint32_t n_s8,
                                    uint32_t wy, BgItem* __restrict__ items_pl, BgItem* __restrict__ items_s8) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_pl + n_s8) return;
    const bool s8 = e >= n_pl;
    const uint32_t it = s8 ? e - n_pl : e;
    uint32_t lo = 0, hi = U;  // first(lo) <= it < first(hi), first(U) = table size
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((s8 ? groups[mid].it_s8 : groups[mid].it_pl) <= it) lo = mid;
        else hi = mid;
    }
    const IvGroup g = groups[lo];
    const uint32_t rows_per = s8 ? (uint32_t)BG_AROWS : (uint32_t)BG_AROWS / 8;
    const uint32_t xt = (g.m + rows_per - 1) / rows_per;
    const uint32_t local = it - (s8 ? g.it_s8 : g.it_pl);
    const uint32_t xi = local % xt, x0 = g.row0 + xi * rows_per, y0 = g.lp0 + (local / xt) * wy;
    const BgItem item{(s8 ? g.t128 : g.t16) + xi, 8 * y0, x0, g.row0 + g.m, y0, g.lp0 + g.n};
    if (s8) items_s8[it] = item;
    else items_pl[it] = item;
}

// idmap[r-space entry] = corpus id of its row
__global__ void idmap_kernel(const IvChunk* __restrict__ chunks, const uint32_t* __restrict__ ids,
                             uint32_t* __restrict__ idmap) {
    const IvChunk c = chunks[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < c.rows; i += blockDim.x) idmap[c.r0 + i] = ids[c.row0 + i];
}

// 128-bit accumulation of a 61 x 61-bit product.
__device__ __forceinline__ void mac128(uint64_t& lo, uint64_t& hi, uint64_t a, uint64_t b) {
    const uint64_t pl = a * b, ph = __umul64hi(a, b);
    lo += pl;
    hi += ph + (lo < pl ? 1u : 0u);
}

// u_t . r for the pairs of one list chunk, trials [t_base, t_base + t_cnt):
// the chunk's U blocks (launch_tc_ugen, per-block images: byte a of u_t[i] at
// row 8t + a, column i) are read once each into shared memory and serve every
// pair of the slab.  Warp w owns the (pair, trial) combos w, w + 8, ... for
// the whole chunk; lane l takes rows 4l .. 4l + 3 of each block, reads one
// 32-bit word from each of the 8 byte rows of trial t and transposes them
// into the four u_t values.  16 blocks x 4 rows = 64 products (< 2^122 each)
// per lane and combo are summed in 128 bits.
__global__ void __launch_bounds__(UR_WARPS * 32)
ur_lists_kernel(const IvUrTask* __restrict__ tasks, const IvPair* __restrict__ pairs, const uint32_t* __restrict__ lmi,
                const uint8_t* __restrict__ ub, uint32_t n_rows, uint32_t t_base, uint32_t t_cnt,
                uint32_t trials_total, const uint64_t* __restrict__ r, uint64_t* __restrict__ ur_part) {
    extern __shared__ uint4 u_img[];  // one U block: 8 t_cnt rows x 128 bytes
    __shared__ uint64_t rbase_s[UR_SLAB];
    __shared__ uint32_t out_s[UR_SLAB];
    const IvUrTask tk = tasks[blockIdx.x];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x < tk.npairs) {
        const IvPair pr = pairs[lmi[tk.lp0 + threadIdx.x]];
        rbase_s[threadIdx.x] = pr.out0 + (uint64_t)tk.c * IV_CHUNK_ROWS;
        out_s[threadIdx.x] = pr.ch0 + tk.c;
    }
    const uint32_t combos = tk.npairs * t_cnt;
    uint64_t lo[UR_PER_WARP], hi[UR_PER_WARP];
#pragma unroll
    for (uint32_t ii = 0; ii < UR_PER_WARP; ++ii) lo[ii] = hi[ii] = 0;
    const uint32_t nblk = (tk.rows + TC_ROWS - 1) / TC_ROWS;
    const uint32_t img_words = 8 * t_cnt * TC_ROWS / 16;
    const uint8_t* img = reinterpret_cast<const uint8_t*>(u_img) + 4 * lane;
    for (uint32_t b = 0; b < nblk; ++b) {
        __syncthreads();  // the previous block's image is no longer read (and rbase_s is set)
        const uint4* src = reinterpret_cast<const uint4*>(ub + (uint64_t)(tk.ublk0 + b) * n_rows * TC_ROWS);
        for (uint32_t x = threadIdx.x; x < img_words; x += blockDim.x) u_img[x] = src[x];
        __syncthreads();
        const uint32_t i0 = b * TC_ROWS + 4 * lane;
#pragma unroll
        for (uint32_t ii = 0; ii < UR_PER_WARP; ++ii) {
            const uint32_t k = warp + UR_WARPS * ii;
            if (k < combos) {
                const uint32_t pk = k / t_cnt, t = k % t_cnt;
                const uint64_t rb = rbase_s[pk];
                uint64_t rv[4];
#pragma unroll
                for (int h = 0; h < 4; ++h) rv[h] = i0 + h < tk.rows ? r[rb + i0 + h] : 0;
                uint32_t w[8];
#pragma unroll
                for (int a = 0; a < 8; ++a) w[a] = *reinterpret_cast<const uint32_t*>(img + (8 * t + a) * TC_ROWS);
                // 8 x 4 byte transpose: byte a of u[h] = byte h of w[a]
                const uint32_t l01 = __byte_perm(w[0], w[1], 0x5140), h01 = __byte_perm(w[0], w[1], 0x7362);
                const uint32_t l23 = __byte_perm(w[2], w[3], 0x5140), h23 = __byte_perm(w[2], w[3], 0x7362);
                const uint32_t l45 = __byte_perm(w[4], w[5], 0x5140), h45 = __byte_perm(w[4], w[5], 0x7362);
                const uint32_t l67 = __byte_perm(w[6], w[7], 0x5140), h67 = __byte_perm(w[6], w[7], 0x7362);
                uint64_t u[4];
                u[0] = __byte_perm(l01, l23, 0x5410) | ((uint64_t)__byte_perm(l45, l67, 0x5410) << 32);
                u[1] = __byte_perm(l01, l23, 0x7632) | ((uint64_t)__byte_perm(l45, l67, 0x7632) << 32);
                u[2] = __byte_perm(h01, h23, 0x5410) | ((uint64_t)__byte_perm(h45, h67, 0x5410) << 32);
                u[3] = __byte_perm(h01, h23, 0x7632) | ((uint64_t)__byte_perm(h45, h67, 0x7632) << 32);
#pragma unroll
                for (int h = 0; h < 4; ++h) mac128(lo[ii], hi[ii], u[h], rv[h]);
            }
        }
    }
#pragma unroll
    for (uint32_t ii = 0; ii < UR_PER_WARP; ++ii) {
        const uint32_t k = warp + UR_WARPS * ii;
        if (k < combos) {  // warp-uniform
            uint64_t x = reduce128(lo[ii], hi[ii]);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x = add_mod(x, __shfl_xor_sync(0xffffffffu, x, off));
            if (lane == 0) ur_part[(uint64_t)out_s[k / t_cnt] * trials_total + t_base + k % t_cnt] = x;
        }
    }
}

__global__ void zsum_lists_kernel(const uint64_t* __restrict__ z_part, const IvZsum* __restrict__ lists,
                                  uint32_t trials, uint64_t* __restrict__ z) {
    const IvZsum l = lists[blockIdx.x / trials];
    const uint32_t t = blockIdx.x % trials;
    for (uint32_t j = threadIdx.x; j < N; j += blockDim.x) {
        uint64_t acc = 0;
        for (uint32_t p = l.p0; p < l.p1; ++p) acc = add_mod(acc, z_part[((uint64_t)p * trials + t) * N + j]);
        z[((uint64_t)l.m * trials + t) * N + j] = acc;
    }
}

// zv[i][t] = z_t^u . v_{q(i)} for pairs ZV_PAIRS * blockIdx.z, ... of list
// u = blockIdx.x and trials [ZV_TRIALS * blockIdx.y, + ZV_TRIALS): list u's z
// (at zbase + zoff[u]: its single panel's z_part, or its panel sum) is read
// into registers (thread x holds elements x + 128 e) and serves up to
// ZV_PAIRS of the list's pairs, whose v rows come from L2 (a list probed by
// many queries of the batch spreads over several CTAs).  8 products (< 2^122
// each) per thread and trial are summed in 128 bits.
constexpr uint32_t ZV_TRIALS = 4;
constexpr uint32_t ZV_PAIRS = 8;
__global__ void __launch_bounds__(128) zv_lists_kernel(const uint64_t* __restrict__ zbase,
                                                       const uint64_t* __restrict__ zoff,
                                                       const uint64_t* __restrict__ v,
                                                       const IvPair* __restrict__ pairs,
                                                       const IvGroup* __restrict__ groups,
                                                       const uint32_t* __restrict__ lmi, uint32_t trials,
                                                       uint64_t* __restrict__ zv) {
    const uint32_t u = blockIdx.x, t0 = blockIdx.y * ZV_TRIALS, k0 = blockIdx.z * ZV_PAIRS;
    const uint32_t tn = min(ZV_TRIALS, trials - t0);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const IvGroup g = groups[u];
    if (k0 >= g.n) return;  // CTA-uniform: this list has fewer pairs
    const uint32_t k1 = min(g.n, k0 + ZV_PAIRS);
    const uint64_t* zr = zbase + zoff[u] + (uint64_t)t0 * N;
    uint64_t z[ZV_TRIALS][N / 128];
#pragma unroll
    for (uint32_t tt = 0; tt < ZV_TRIALS; ++tt)
#pragma unroll
        for (uint32_t e = 0; e < N / 128; ++e) z[tt][e] = tt < tn ? zr[(uint64_t)tt * N + threadIdx.x + 128 * e] : 0;
    __shared__ uint64_t sh[4][ZV_TRIALS];
    for (uint32_t k = k0; k < k1; ++k) {
        const uint32_t i = lmi[g.lp0 + k];
        const uint64_t* vr = v + (uint64_t)pairs[i].q * N;
        uint64_t vv[N / 128];
#pragma unroll
        for (uint32_t e = 0; e < N / 128; ++e) vv[e] = vr[threadIdx.x + 128 * e];
#pragma unroll
        for (uint32_t tt = 0; tt < ZV_TRIALS; ++tt) {
            uint64_t lo = 0, hi = 0;
#pragma unroll
            for (uint32_t e = 0; e < N / 128; ++e) mac128(lo, hi, z[tt][e], vv[e]);
            uint64_t x = reduce128(lo, hi);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x = add_mod(x, __shfl_xor_sync(0xffffffffu, x, off));
            if (lane == 0) sh[warp][tt] = x;
        }
        __syncthreads();
        if (threadIdx.x < tn)
            zv[(uint64_t)i * trials + t0 + threadIdx.x] =
                add_mod(add_mod(sh[0][threadIdx.x], sh[1][threadIdx.x]), add_mod(sh[2][threadIdx.x], sh[3][threadIdx.x]));
        __syncthreads();  // sh is rewritten by the next pair
    }
}

// First failing trial of each pair (-1: accepted); ur_out (nullable) [i][t].
// One warp per pair: lanes sum its chunks' partials, trial by trial.
__global__ void pair_decide_kernel(const IvPair* __restrict__ pairs, uint32_t npairs,
                                   const uint64_t* __restrict__ ur_part, const uint64_t* __restrict__ zv,
                                   uint32_t trials, int32_t* __restrict__ pfail, uint64_t* __restrict__ ur_out) {
    const uint32_t i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= npairs) return;  // warp-uniform
    const IvPair pr = pairs[i];
    int32_t f = -1;
    for (uint32_t t = 0; t < trials; ++t) {
        uint64_t acc = 0;
        for (uint32_t c = pr.ch0 + lane; c < pr.ch0 + pr.nch; c += 32)
            acc = add_mod(acc, ur_part[(uint64_t)c * trials + t]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc = add_mod(acc, __shfl_xor_sync(0xffffffffu, acc, off));
        if (ur_out && lane == 0) ur_out[(uint64_t)i * trials + t] = acc;
        if (f < 0 && acc != zv[(uint64_t)i * trials + t]) {
            f = (int32_t)t;
            if (!ur_out) break;
        }
    }
    if (lane == 0) pfail[i] = f;
}

// Query q: its first failing pair in probe order -> (list, trial), else (-1, -1).
__global__ void query_decide_kernel(const IvPair* __restrict__ pairs, const uint32_t* __restrict__ q_pair0, uint32_t nq,
                                    const int32_t* __restrict__ pfail, int32_t* __restrict__ fc,
                                    int32_t* __restrict__ ft) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    int32_t c = -1, t = -1;
    for (uint32_t i = q_pair0[q]; i < q_pair0[q + 1]; ++i)
        if (pfail[i] >= 0) {
            c = (int32_t)pairs[i].list;
            t = pfail[i];
            break;
        }
    fc[q] = c;
    ft[q] = t;
}

unsigned grid_cap(uint64_t work, unsigned threads, unsigned cap) {
    const uint64_t g = (work + threads - 1) / threads;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

int tmap_u8(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint32_t box_rows, const char* what) {
    cudaError_t e = make_tmap_u8(m, base, inner, rows, 128, box_rows);
    if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map of %s: %s", what, cudaGetErrorString(e));
    return BN_OK;
}

}  // namespace

// One IVF block run: the host plan (pairs, groups, Protocol 2 layout), the
// workspace layout and the tensor maps of the gathered operands.
struct IvfBlockJob {
    uint32_t B = 0, trials = 0, k = 0;
    bool verify_only = false;
    uint32_t P = 0, U = 0, NB = 0, NP = 0, NCH = 0, n_pl = 0, n_s8 = 0, NZ = 0;
    uint32_t max_n = 0;   // most pairs of one list
    uint32_t NP_big = 0;  // panels [0, NP_big) belong to lists longer than TC_SMALL_PANEL_ROWS
    uint32_t NUR = 0;     // u . r tasks (list chunk x pair slab)
    uint64_t R = 0, max_q_rows = 0;
    uint32_t w_tile = 64, n_rows = 0, ctas = 1, st_g1 = 0, st_g2 = 0, st_g3 = 0;
    // host plan
    std::vector<IvPair> pairs;          // q-major
    std::vector<uint32_t> order;        // list-major position -> q-major pair
    std::vector<IvGroup> groups;        // distinct lists, by list id
    std::vector<uint32_t> block0, panel0;  // per group: first U block, first z panel
    std::vector<uint64_t> qoff;         // per query: first r-space entry (B + 1)
    std::vector<uint32_t> qp0;          // per query: first pair (B + 1)
    // inputs (one H2D from the staging buffer)
    uint64_t o_v, o_g, o_t, o_tn, o_seed, o_qoff, o_qp0, o_pairs, o_lmq, o_lmi, o_base, o_groups, o_vsegs, o_blocks,
        o_panels, o_zoff, o_zsum, o_chunks, o_urtasks, in_end;
    // outputs (one D2H)
    uint64_t o_ids, o_sc, o_n, o_fc, o_ft, o_err, out_end;
    // scratch
    uint64_t o_items_pl, o_items_s8, o_vp, o_gx, o_tv, o_x, o_wv, o_wgx, o_wtv, o_r, o_f2, o_f3, o_idmap, o_ub, o_zpart,
        o_z, o_urpart, o_zv, o_pfail, o_urout, o_cs, o_ci, o_cn, total;
    CUtensorMap tm_wv, tm_wgx, tm_wtv, tm_u;
    CUtensorMap tm_wv2, tm_wgx2, tm_wtv2;  // 3-D views: two K steps per box
};

void ivf_block_job_free(IvfBlockJob* j) { delete j; }
IvfBlockJob* ivf_block_job_new() { return new IvfBlockJob(); }
uint64_t ivf_block_job_bytes(const IvfBlockJob* j) { return j->total; }

namespace {

// W tile (MMA N) for the batch's groups: a group of n pairs spans 8n W rows;
// each A tile is re-streamed (from L2) once per W tile of its group, so pick
// the tile minimising sum over groups of A tiles x W tiles x (A + W rows +
// a fixed per-item cost).
uint32_t pick_w_tile(const std::vector<IvGroup>& groups, uint32_t B) {
    // Measured on 2M rows / 4096 k-means lists, batches of 64 (whole-batch
    // call times of each tiling in the same run): W = 128 ran nprobe 8 and 32
    // (1.6 and 2.8 queries per list on average) 5 % and 11 % faster than the
    // W = 64 the item-count model below picks there, and nprobe 128 (6.3 per
    // list) 2 % faster than the model's choice in three runs out of four; the
    // model keeps the batches too small to fill 128 W rows.
    if (B >= 16 && !groups.empty()) return 128;
    uint32_t best_w = 64;
    double best = 1e300;
    for (uint32_t w : {16u, 32u, 64u, 128u, 256u}) {
        double cost = 0;
        for (const IvGroup& g : groups)
            cost += (double)((g.m + 15) / 16) * (double)((8ull * g.n + w - 1) / w) * (128.0 + w + 64.0);
        if (cost < best) {
            best = cost;
            best_w = w;
        }
    }
    return best_w;
}

}  // namespace

// Host plan of one batch.  probe_off[B + 1] / probes: query q probes lists
// probes[probe_off[q] .. probe_off[q + 1]) in that order.  O(pairs log pairs
// + distinct lists); the per-block / per-panel / per-chunk tables are written
// by ivf_block_pack and the GEMM item tables on the device.
int ivf_block_plan(const bn_ivf& v, IvfBlockJob& j, uint32_t B, const uint32_t* probe_off, const uint32_t* probes,
                   uint32_t trials, uint32_t k, bool verify_only, int sms) {
    const Corpus& c = v.e.c;
    if (k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX = %d", k, BN_TOPK_MAX);
    if (trials > BN_MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %d", trials, BN_MAX_TRIALS);
    if (B > 65535) return fail(BN_EINVAL, "B = %u exceeds 65535 queries per call", B);
    if (c.rows * 8 >= (1ull << 31)) return fail(BN_EUNSUPPORTED, "IVF block scoring needs fewer than 2^28 corpus rows");
    if (probe_off[B] > (1u << 24)) return fail(BN_EINVAL, "%u probes exceed 2^24 per call", probe_off[B]);
    j.B = B;
    j.trials = trials;
    j.k = k;
    j.verify_only = verify_only;
    // pairs, q-major; empty lists skipped (ivf.rs:787-789)
    j.pairs.clear();
    j.pairs.reserve(probe_off[B]);
    j.qoff.assign(B + 1, 0);
    j.qp0.assign(B + 1, 0);
    j.max_q_rows = 0;
    uint64_t R = 0;
    for (uint32_t q = 0; q < B; ++q) {
        j.qoff[q] = R;
        j.qp0[q] = (uint32_t)j.pairs.size();
        for (uint32_t p = probe_off[q]; p < probe_off[q + 1]; ++p) {
            const uint32_t ci = probes[p];
            if (ci >= v.nlist)
                return fail(BN_EINVAL, "probe %u of query %u names list %u of %u", p - probe_off[q], q, ci, v.nlist);
            const uint64_t m = v.offsets[ci + 1] - v.offsets[ci];
            if (!m) continue;
            j.pairs.push_back(IvPair{R, q, ci, 0, 0, 0, 0});
            R += m;
        }
        j.max_q_rows = std::max(j.max_q_rows, R - j.qoff[q]);
    }
    j.qoff[B] = R;
    j.qp0[B] = (uint32_t)j.pairs.size();
    j.R = R;
    j.P = (uint32_t)j.pairs.size();
    // groups: pairs ordered by (list, pair), so a list's queries stay in
    // batch order (a counting sort over the lists: O(pairs + nlist))
    std::vector<uint32_t> keys(j.P), start(v.nlist + 1, 0);
    for (uint32_t i = 0; i < j.P; ++i) ++start[j.pairs[i].list + 1];
    for (uint32_t c = 0; c < v.nlist; ++c) start[c + 1] += start[c];
    for (uint32_t i = 0; i < j.P; ++i) keys[start[j.pairs[i].list]++] = i;
    j.order.resize(j.P);
    j.groups.clear();
    j.block0.clear();
    j.panel0.clear();
    uint32_t nb = 0, np = 0, nch = 0;
    for (uint32_t lp = 0; lp < j.P; ++lp) {
        const uint32_t i = keys[lp];
        j.order[lp] = i;
        IvPair& pr = j.pairs[i];
        if (lp == 0 || j.pairs[j.order[lp - 1]].list != pr.list) {
            const uint32_t m = (uint32_t)(v.offsets[pr.list + 1] - v.offsets[pr.list]);
            const bool tiles = !c.list_p16.empty();  // K-blocked copies exist (not needed to verify only)
            j.groups.push_back(IvGroup{(uint32_t)v.offsets[pr.list], m, lp, 0, 0, 0,
                                       tiles ? (uint32_t)(c.list_p16[pr.list] / 16) : 0u,
                                       tiles ? (uint32_t)(c.list_p128[pr.list] / 128) : 0u});
            j.block0.push_back(nb);
            nb += (m + TC_ROWS - 1) / TC_ROWS;
        }
        IvGroup& g = j.groups.back();
        pr.u = (uint32_t)j.groups.size() - 1;
        pr.ch0 = nch;
        pr.nch = (g.m + IV_CHUNK_ROWS - 1) / IV_CHUNK_ROWS;
        nch += pr.nch;
        ++g.n;
    }
    j.U = (uint32_t)j.groups.size();
    j.max_n = 0;
    for (const IvGroup& g : j.groups) j.max_n = std::max(j.max_n, g.n);
    // z panels: the long lists' first (tc_freivalds_kernel), then the short
    // lists' single panels (tc_freivalds_small_kernel)
    j.panel0.assign(j.U, 0);
    for (uint32_t u = 0; u < j.U; ++u)
        if (j.groups[u].m > TC_SMALL_PANEL_ROWS) {
            j.panel0[u] = np;
            np += (j.groups[u].m + TC_PANEL_ROWS - 1) / TC_PANEL_ROWS;
        }
    j.NP_big = np;
    for (uint32_t u = 0; u < j.U; ++u)
        if (j.groups[u].m <= TC_SMALL_PANEL_ROWS) j.panel0[u] = np++;
    j.NB = nb;
    j.NP = np;
    j.NCH = nch;
    j.NZ = 0;
    j.NUR = 0;
    for (uint32_t u = 0; u < j.U; ++u) {
        j.NZ += (j.groups[u].m > TC_PANEL_ROWS) ? 1u : 0u;
        j.NUR += ((j.groups[u].m + IV_CHUNK_ROWS - 1) / IV_CHUNK_ROWS) * ((j.groups[u].n + UR_SLAB - 1) / UR_SLAB);
    }
    // grouped GEMM item counts (the tables themselves are expanded on the device)
    j.n_pl = j.n_s8 = 0;
    if (!verify_only && j.P) {
        if (c.list_p16.size() != v.nlist) return fail(BN_EINVAL, "block scoring copies are not prepared");
        j.w_tile = v.blk_w ? v.blk_w : pick_w_tile(j.groups, B);
        const uint32_t wy = j.w_tile / 8;  // pairs per W tile
        for (IvGroup& g : j.groups) {
            const uint32_t yt = (g.n + wy - 1) / wy;
            g.it_pl = j.n_pl;
            g.it_s8 = j.n_s8;
            j.n_pl += yt * ((g.m + BG_AROWS / 8 - 1) / (BG_AROWS / 8));
            j.n_s8 += yt * ((g.m + BG_AROWS - 1) / BG_AROWS);
        }
        BgParams p{};
        p.w_tile = j.w_tile;
        p.ksteps2 = 1;
        j.st_g1 = j.st_g2 = j.st_g3 = bgemm_max_stages(p);
        if (!j.st_g1) return fail(BN_EUNSUPPORTED, "no pipeline depth fits W tile %u", j.w_tile);
        if (v.blk_stages) j.st_g1 = j.st_g2 = j.st_g3 = std::min(j.st_g1, v.blk_stages);
    }
    j.n_rows = pass_rows(std::min<uint32_t>(std::max<uint32_t>(trials, 1), TC_MAX_TRIALS));
    j.ctas = (uint32_t)pick_ctas(j.max_q_rows, std::max<uint32_t>(B, 1), sms);

    // workspace layout
    const uint32_t n1 = c.n1, ks = std::max<uint32_t>(k, 1), tt = std::max<uint32_t>(trials, 1);
    const uint64_t qb = verify_only ? 0 : B, pb = verify_only ? 0 : j.P;
    Layout L;
    j.o_v = L.take<uint64_t>((uint64_t)B * N);
    j.o_g = L.take<uint64_t>(qb * n1);
    j.o_t = L.take<uint32_t>(qb * N);
    j.o_tn = L.take<uint32_t>(qb);
    j.o_seed = L.take<uint8_t>(32);
    j.o_qoff = L.take<uint64_t>(B + 1);
    j.o_qp0 = L.take<uint32_t>(B + 1);
    j.o_pairs = L.take<IvPair>(j.P);
    j.o_lmq = L.take<uint32_t>(j.P);
    j.o_lmi = L.take<uint32_t>(j.P);
    j.o_base = L.take<uint64_t>(j.P);
    j.o_groups = L.take<IvGroup>(j.U);
    j.o_vsegs = L.take<VerifySeg>(j.U);
    j.o_blocks = L.take<TcBlock>(j.NB);
    j.o_panels = L.take<TcPanel>(j.NP);
    j.o_zoff = L.take<uint64_t>(j.U);
    j.o_zsum = L.take<IvZsum>(j.NZ);
    j.o_chunks = L.take<IvChunk>(j.NCH);
    j.o_urtasks = L.take<IvUrTask>(j.NUR);
    j.in_end = L.take<uint8_t>(0);
    j.o_ids = L.take<uint32_t>((uint64_t)B * ks);
    j.o_sc = L.take<int64_t>((uint64_t)B * ks);
    j.o_n = L.take<uint32_t>(B);
    j.o_fc = L.take<int32_t>(B);
    j.o_ft = L.take<int32_t>(B);
    j.o_err = L.take<uint32_t>(2);  // [0] pipeline flags, [1] operand range flags
    j.out_end = L.take<uint8_t>(0);
    j.o_items_pl = L.take<BgItem>(j.n_pl);
    j.o_items_s8 = L.take<BgItem>(j.n_s8);
    j.o_vp = L.take<uint8_t>(8 * qb * N);
    j.o_gx = L.take<uint8_t>(8 * qb * c.k_alh);
    j.o_tv = L.take<uint8_t>(8 * qb * 2 * N);
    j.o_x = L.take<uint64_t>(qb * n1);
    j.o_wv = L.take<uint8_t>(8 * pb * N);
    j.o_wgx = L.take<uint8_t>(8 * pb * c.k_alh);
    j.o_wtv = L.take<uint8_t>(8 * pb * 2 * N);
    const uint64_t re = R + 2;  // paired loads of the top-k may touch one entry past the end
    j.o_r = L.take<uint64_t>(re);
    j.o_f2 = L.take<uint64_t>(verify_only ? 0 : re);
    j.o_f3 = L.take<uint64_t>(verify_only ? 0 : re);
    j.o_idmap = L.take<uint32_t>(verify_only ? 0 : re);
    j.o_ub = L.take<uint8_t>(trials ? (uint64_t)j.NB * j.n_rows * TC_ROWS : 0);
    // z directly after z_part (zoff counts from z_part in elements)
    j.o_zpart = L.take<uint64_t>(trials ? (uint64_t)j.NP * tt * N + (uint64_t)j.NZ * tt * N : 0);
    j.o_z = j.o_zpart + (uint64_t)j.NP * tt * N * 8;
    j.o_urpart = L.take<uint64_t>(trials ? (uint64_t)j.NCH * tt : 0);
    j.o_zv = L.take<uint64_t>(trials ? (uint64_t)j.P * tt : 0);
    j.o_pfail = L.take<int32_t>(j.P);
    j.o_urout = L.take<uint64_t>(verify_only && trials ? (uint64_t)j.P * tt : 0);
    const uint64_t cand = (uint64_t)B * j.ctas * ks;
    j.o_cs = L.take<int64_t>(verify_only ? 0 : cand);
    j.o_ci = L.take<uint32_t>(verify_only ? 0 : cand);
    j.o_cn = L.take<uint32_t>(verify_only ? 0 : (uint64_t)B * j.ctas);
    j.total = L.off + 1024;
    return BN_OK;
}

// Validates and packs the query inputs and the plan's tables into the pinned
// staging buffer (grown as needed) and sizes ws (grown as needed,
// budget-accounted); encodes the tensor maps of this run's buffers.
int ivf_block_pack(Engine& e, IvfBlockJob& j, DevMem& ws, PinnedMem& host, const uint64_t* v_enc, const uint64_t* g,
                   const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* seed) {
    const Corpus& c = e.c;
    const uint32_t B = j.B;
    if (!v_enc) return fail(BN_EINVAL, "null v_enc");
    if (j.trials && !seed) return fail(BN_EINVAL, "block_seed is required when trials > 0");
    TRY(validate_residues(v_enc, (uint64_t)B * N, "v_enc"));
    TRY(ws.reserve_grow(e.ctx, j.total));
    TRY(host.reserve(j.out_end));  // inputs, then the outputs read back at the same offsets
    char* h = host.at<char>();
    memcpy(h + j.o_v, v_enc, (uint64_t)B * N * 8);
    if (!j.verify_only) {
        if (!g || !t_nnz) return fail(BN_EINVAL, "null query input");
        TRY(validate_residues(g, (uint64_t)B * c.n1, "g"));
        memcpy(h + j.o_g, g, (uint64_t)B * c.n1 * 8);
        uint32_t* ht = reinterpret_cast<uint32_t*>(h + j.o_t);
        uint64_t tp = 0;
        for (uint32_t q = 0; q < B; ++q) {
            if (t_nnz[q] > N) return fail(BN_EINVAL, "t_nnz[%u] = %u exceeds n", q, t_nnz[q]);
            if (t_nnz[q] && (!t_idx || !t_sign)) return fail(BN_EINVAL, "t_idx / t_sign are null");
            for (uint32_t i = 0; i < t_nnz[q]; ++i, ++tp) {
                if (t_idx[tp] >= N || (t_sign[tp] != 1 && t_sign[tp] != -1))
                    return fail(BN_EINVAL, "T entry %llu is not (col < n, sign +-1)", (unsigned long long)tp);
                ht[(uint64_t)q * N + i] = t_idx[tp] | (t_sign[tp] < 0 ? 0x80000000u : 0u);
            }
        }
        memcpy(h + j.o_tn, t_nnz, (uint64_t)B * 4);
    }
    if (seed) memcpy(h + j.o_seed, seed, 32);
    else memset(h + j.o_seed, 0, 32);
    // plan tables, written in place
    memcpy(h + j.o_qoff, j.qoff.data(), j.qoff.size() * 8);
    memcpy(h + j.o_qp0, j.qp0.data(), j.qp0.size() * 4);
    if (j.P) memcpy(h + j.o_pairs, j.pairs.data(), (uint64_t)j.P * sizeof(IvPair));
    if (j.U) memcpy(h + j.o_groups, j.groups.data(), (uint64_t)j.U * sizeof(IvGroup));
    uint32_t* lmq = reinterpret_cast<uint32_t*>(h + j.o_lmq);
    uint32_t* lmi = reinterpret_cast<uint32_t*>(h + j.o_lmi);
    uint64_t* base = reinterpret_cast<uint64_t*>(h + j.o_base);
    IvChunk* ch = reinterpret_cast<IvChunk*>(h + j.o_chunks);
    for (uint32_t lp = 0, nc = 0; lp < j.P; ++lp) {
        const uint32_t i = j.order[lp];
        const IvPair& pr = j.pairs[i];
        const IvGroup& gr = j.groups[pr.u];
        lmq[lp] = pr.q;
        lmi[lp] = i;
        base[lp] = pr.out0 - gr.row0;  // out[base + corpus row] (mod 2^64)
        for (uint32_t c0 = 0; c0 < gr.m; c0 += IV_CHUNK_ROWS)
            ch[nc++] = IvChunk{pr.out0 + c0, (uint64_t)gr.row0 + c0, j.block0[pr.u] + c0 / TC_ROWS,
                               std::min<uint32_t>(IV_CHUNK_ROWS, gr.m - c0)};
    }
    // Protocol 2 layout: one verify segment per distinct list (128-row U
    // blocks, 4096-row z panels); z of a single-panel list is its z_part,
    // several panels are summed into a z slot (after z_part)
    IvUrTask* ut = reinterpret_cast<IvUrTask*>(h + j.o_urtasks);
    for (uint32_t u = 0, nt = 0; u < j.U; ++u) {
        const IvGroup& gr = j.groups[u];
        for (uint32_t c = 0; c * IV_CHUNK_ROWS < gr.m; ++c)
            for (uint32_t p0 = 0; p0 < gr.n; p0 += UR_SLAB)
                ut[nt++] = IvUrTask{j.block0[u] + c * (IV_CHUNK_ROWS / TC_ROWS),
                                    std::min<uint32_t>(IV_CHUNK_ROWS, gr.m - c * IV_CHUNK_ROWS), gr.lp0 + p0,
                                    std::min<uint32_t>(UR_SLAB, gr.n - p0), c};
    }
    VerifySeg* vs = reinterpret_cast<VerifySeg*>(h + j.o_vsegs);
    TcBlock* bl = reinterpret_cast<TcBlock*>(h + j.o_blocks);
    TcPanel* pn = reinterpret_cast<TcPanel*>(h + j.o_panels);
    uint64_t* zoff = reinterpret_cast<uint64_t*>(h + j.o_zoff);
    IvZsum* zs = reinterpret_cast<IvZsum*>(h + j.o_zsum);
    const uint64_t tt = std::max<uint32_t>(j.trials, 1);
    for (uint32_t u = 0, nb = 0, nz = 0; u < j.U; ++u) {
        const IvGroup& gr = j.groups[u];
        vs[u] = VerifySeg{gr.row0, 0, gr.m, 0};
        for (uint32_t i0 = 0; i0 < gr.m; i0 += TC_ROWS) bl[nb++] = TcBlock{u, i0};
        const uint32_t p0 = j.panel0[u];
        uint32_t np = p0;
        for (uint32_t r0 = 0; r0 < gr.m; r0 += TC_PANEL_ROWS)
            pn[np++] = TcPanel{(uint64_t)gr.row0 + r0, std::min<uint32_t>(TC_PANEL_ROWS, gr.m - r0),
                               j.block0[u] + r0 / TC_ROWS, u, 0};
        if (np - p0 == 1) {
            zoff[u] = (uint64_t)p0 * tt * N;
        } else {
            zoff[u] = ((uint64_t)j.NP + nz) * tt * N;
            zs[nz] = IvZsum{p0, np, nz};
            ++nz;
        }
    }
    char* d = ws.at<char>();
    if (!j.verify_only && j.P) {
        TRY(tmap_u8(&j.tm_wv, d + j.o_wv, N, 8ull * j.P, j.w_tile, "gathered v planes"));
        TRY(tmap_u8(&j.tm_wgx, d + j.o_wgx, c.k_alh, 8ull * j.P, j.w_tile, "gathered [g | x] planes"));
        TRY(tmap_u8(&j.tm_wtv, d + j.o_wtv, 2 * N, 8ull * j.P, j.w_tile, "gathered [T | v] bytes"));
        const struct {
            CUtensorMap* m;
            uint64_t off, row_bytes;
        } w2[3] = {{&j.tm_wv2, j.o_wv, N}, {&j.tm_wgx2, j.o_wgx, c.k_alh}, {&j.tm_wtv2, j.o_wtv, 2 * N}};
        for (const auto& x : w2) {
            const cudaError_t e = make_tmap_u8_ksteps2(x.m, d + x.off, x.row_bytes, 8ull * j.P, j.w_tile);
            if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map of the W operands: %s", cudaGetErrorString(e));
        }
    }
    if (j.trials && j.NB) TRY(tmap_u8(&j.tm_u, d + j.o_ub, TC_ROWS, (uint64_t)j.NB * j.n_rows, j.n_rows, "u images"));
    return BN_OK;
}

// Enqueues the H2D of the packed inputs, the block pipeline and the D2H of
// the outputs on s.  r_in (verification only): the claimed responses, device
// copy already at o_r.
int ivf_block_launch(Engine& e, IvfBlockJob& j, DevMem& ws, PinnedMem& host, cudaStream_t s, cudaEvent_t* ev) {
    const Corpus& c = e.c;
    char* d = ws.at<char>();
    char* h = host.at<char>();
    const int sms = e.ctx->num_sms;
    const uint32_t B = j.B, n1 = c.n1;
    int last = -1;  // skipped stages are recorded with the next one (0 ms)
    auto mark = [&](int i) {
        if (ev)
            for (int x = last + 1; x <= i; ++x) cudaEventRecord(ev[x], s);
        last = i;
    };
    CU(cudaSetDevice(e.ctx->device));
    mark(0);
    CU(cudaMemcpyAsync(d, h, j.in_end, cudaMemcpyHostToDevice, s));
    uint32_t* err = reinterpret_cast<uint32_t*>(d + j.o_err);
    CU(cudaMemsetAsync(err, 0, 8, s));
    if (j.trials && e.ctx->debug_draw_hit) launch_or_flag(err, DRAW_HIT_P, s);
    auto U8 = [&](uint64_t o) { return reinterpret_cast<uint8_t*>(d + o); };
    auto U64 = [&](uint64_t o) { return reinterpret_cast<uint64_t*>(d + o); };
    auto U32 = [&](uint64_t o) { return reinterpret_cast<uint32_t*>(d + o); };
    const uint64_t* dv = U64(j.o_v);
    const IvPair* dpairs = reinterpret_cast<const IvPair*>(d + j.o_pairs);
    const IvChunk* dchunks = reinterpret_cast<const IvChunk*>(d + j.o_chunks);
    if (!j.verify_only) {
        if (j.P) {
            // per-query operand images, then one image per (list, query) pair, grouped by list
            if (c.k_alh != 2 * n1) CU(cudaMemsetAsync(d + j.o_gx, 0, 8ull * B * c.k_alh, s));
            launch_planar_rows(dv, B, N, N, 0, U8(j.o_vp), N, 0, s);
            launch_lt_times_v(c.L.at<uint64_t>(), n1, dv, B, U64(j.o_x), s);
            launch_planar_rows(U64(j.o_g), B, n1, n1, 1, U8(j.o_gx), c.k_alh, 0, s);
            launch_planar_rows(U64(j.o_x), B, n1, n1, 1, U8(j.o_gx), c.k_alh, n1, s);
            launch_w_tv(dv, U32(j.o_t), U32(j.o_tn), B, reinterpret_cast<int8_t*>(d + j.o_tv), err + 1, s);
            const uint32_t* lmq = U32(j.o_lmq);
            struct Img {
                uint64_t src, dst;
                uint32_t row_bytes;
            };
            const Img imgs[3] = {{j.o_vp, j.o_wv, N}, {j.o_gx, j.o_wgx, c.k_alh}, {j.o_tv, j.o_wtv, 2 * N}};
            for (const Img& im : imgs)
                gather8_kernel<<<grid_cap((uint64_t)j.P * im.row_bytes / 2, 256, (unsigned)sms * 8), 256, 0, s>>>(
                    reinterpret_cast<const uint4*>(d + im.src), reinterpret_cast<uint4*>(d + im.dst), lmq, j.P,
                    im.row_bytes);
            idmap_kernel<<<j.NCH, 256, 0, s>>>(dchunks, c.ids.at<uint32_t>(), U32(j.o_idmap));
            expand_items_kernel<<<(j.n_pl + j.n_s8 + 255) / 256, 256, 0, s>>>(
                reinterpret_cast<const IvGroup*>(d + j.o_groups), j.U, j.n_pl, j.n_s8, j.w_tile / 8,
                reinterpret_cast<BgItem*>(d + j.o_items_pl), reinterpret_cast<BgItem*>(d + j.o_items_s8));
            mark(1);
            // G1 r = M_c v_q, G2 f2 = -(AL_c g_q + H_c x_q), G3 f3 = M_c T_q + S_c v_q
            BgParams p{};
            p.mode = BG_PLANAR;
            p.a_tiles = p.w_tiles = 1;
            p.w_tile = j.w_tile;
            p.k_bytes = p.k_panel = N;
            p.out = U64(j.o_r);
            p.item_tab = reinterpret_cast<const BgItem*>(d + j.o_items_pl);
            p.n_items = j.n_pl;
            p.pair_base = U64(j.o_base);
            p.a_blocked = 1;
            p.ksteps2 = 1;  // two K steps per stage: half the producer / MMA handoffs per item
            p.wait_cycles = e.ctx->debug_wait_cycles;
            launch_bgemm(c.tmap_mp, j.tm_wv, p, j.st_g1, sms, err, s, &c.tmap_mp2, &j.tm_wv2);
            mark(2);
            p.k_bytes = p.k_panel = c.k_alh;
            p.out = U64(j.o_f2);
            launch_bgemm(c.tmap_alh, j.tm_wgx, p, j.st_g2, sms, err, s, &c.tmap_alh2, &j.tm_wgx2);
            mark(3);
            p.mode = BG_S8;
            p.k_bytes = p.k_panel = 2 * N;
            p.out = U64(j.o_f3);
            p.corr = c.corr.at<uint64_t>();
            p.item_tab = reinterpret_cast<const BgItem*>(d + j.o_items_s8);
            p.n_items = j.n_s8;
            launch_bgemm(c.tmap_ms, j.tm_wtv, p, j.st_g3, sms, err, s, &c.tmap_ms2, &j.tm_wtv2);
            mark(4);
        }
        if (j.k && j.P) {
            TopkScratch ts{reinterpret_cast<int64_t*>(d + j.o_cs), U32(j.o_ci), U32(j.o_cn)};
            launch_topk_segs(U64(j.o_r), U64(j.o_f2), U64(j.o_f3), U64(j.o_qoff), B, U32(j.o_idmap), j.k, (int)j.ctas,
                             ts, U32(j.o_ids), reinterpret_cast<int64_t*>(d + j.o_sc), U32(j.o_n), s);
        } else {
            CU(cudaMemsetAsync(d + j.o_n, 0, (uint64_t)B * 4, s));
        }
        mark(5);
    }
    if (j.trials && j.P) {
        const auto* vsegs = reinterpret_cast<const VerifySeg*>(d + j.o_vsegs);
        const auto* blocks = reinterpret_cast<const TcBlock*>(d + j.o_blocks);
        const auto* panels = reinterpret_cast<const TcPanel*>(d + j.o_panels);
        const auto* key = reinterpret_cast<const ChaChaKey*>(d + j.o_seed);
        for (uint32_t t0 = 0; t0 < j.trials; t0 += TC_MAX_TRIALS) {
            const uint32_t tc = std::min<uint32_t>(TC_MAX_TRIALS, j.trials - t0);
            const bool last_chunk = t0 + tc == j.trials;  // stage marks: the last trial chunk
            launch_tc_ugen(vsegs, blocks, j.NB, key, nullptr, t0, tc, j.n_rows, U8(j.o_ub), nullptr, j.trials, err, s);
            if (last_chunk) mark(6);
            launch_tc_freivalds(c.tmap_m, j.tm_u, panels, j.NP_big, t0, tc, j.n_rows, j.trials, U64(j.o_zpart), err,
                                sms, s, 0, e.ctx->debug_wait_cycles);
            launch_tc_freivalds_small(c.tmap_m, j.tm_u, panels, j.NP_big, j.NP - j.NP_big, t0, tc, j.n_rows, j.trials,
                                      U64(j.o_zpart), err, sms, s, e.ctx->debug_wait_cycles);
            if (last_chunk) mark(7);
            ur_lists_kernel<<<j.NUR, UR_WARPS * 32, 8 * tc * TC_ROWS, s>>>(
                reinterpret_cast<const IvUrTask*>(d + j.o_urtasks), dpairs, U32(j.o_lmi), U8(j.o_ub), j.n_rows, t0, tc,
                j.trials, U64(j.o_r), U64(j.o_urpart));
        }
        mark(8);
        if (j.NZ)
            zsum_lists_kernel<<<j.NZ * j.trials, 256, 0, s>>>(U64(j.o_zpart),
                                                              reinterpret_cast<const IvZsum*>(d + j.o_zsum), j.trials,
                                                              U64(j.o_z));
        zv_lists_kernel<<<dim3(j.U, (j.trials + ZV_TRIALS - 1) / ZV_TRIALS, (j.max_n + ZV_PAIRS - 1) / ZV_PAIRS), 128,
                          0, s>>>(
            U64(j.o_zpart), U64(j.o_zoff), dv, dpairs, reinterpret_cast<const IvGroup*>(d + j.o_groups), U32(j.o_lmi),
            j.trials, U64(j.o_zv));
        pair_decide_kernel<<<(j.P + 3) / 4, 128, 0, s>>>(dpairs, j.P, U64(j.o_urpart), U64(j.o_zv), j.trials,
                                                             reinterpret_cast<int32_t*>(d + j.o_pfail),
                                                             j.verify_only ? U64(j.o_urout) : nullptr);
        query_decide_kernel<<<(B + 127) / 128, 128, 0, s>>>(dpairs, U32(j.o_qp0), B,
                                                            reinterpret_cast<const int32_t*>(d + j.o_pfail),
                                                            reinterpret_cast<int32_t*>(d + j.o_fc),
                                                            reinterpret_cast<int32_t*>(d + j.o_ft));
    } else {
        CU(cudaMemsetAsync(d + j.o_fc, 0xff, (uint64_t)B * 4, s));
        CU(cudaMemsetAsync(d + j.o_ft, 0xff, (uint64_t)B * 4, s));
    }
    mark(9);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h + j.o_ids, d + j.o_ids, j.out_end - j.o_ids, cudaMemcpyDeviceToHost, s));
    mark(10);
    return BN_OK;
}

// After s has drained: flags, hits (k per query) and verdicts.
int ivf_block_finish(const IvfBlockJob& j, const PinnedMem& host, uint32_t* ids, int64_t* scores, uint32_t* n_hits,
                     int32_t* failed_cluster, int32_t* failed_trial) {
    const char* h = host.at<char>();
    const uint32_t* flags = reinterpret_cast<const uint32_t*>(h + j.o_err);
    TRY(device_flags_status(flags[0]));
    if (flags[1]) return fail(BN_EINVAL, "a T column sum leaves [-128, 127]");
    const uint32_t ks = std::max<uint32_t>(j.k, 1);
    const uint32_t* hid = reinterpret_cast<const uint32_t*>(h + j.o_ids);
    const int64_t* hsc = reinterpret_cast<const int64_t*>(h + j.o_sc);
    const uint32_t* hn = reinterpret_cast<const uint32_t*>(h + j.o_n);
    const int32_t* hfc = reinterpret_cast<const int32_t*>(h + j.o_fc);
    const int32_t* hft = reinterpret_cast<const int32_t*>(h + j.o_ft);
    for (uint32_t q = 0; q < j.B; ++q) {
        const uint32_t nh = (j.k && !j.verify_only) ? hn[q] : 0;
        if (n_hits) n_hits[q] = nh;
        for (uint32_t i = 0; i < nh; ++i) {
            if (ids) ids[(uint64_t)q * j.k + i] = hid[(uint64_t)q * ks + i];
            if (scores) scores[(uint64_t)q * j.k + i] = hsc[(uint64_t)q * ks + i];
        }
        if (failed_cluster) failed_cluster[q] = hfc[q];
        if (failed_trial) failed_trial[q] = hft[q];
    }
    return BN_OK;
}

int ivf_block_prepare(bn_ivf* v) {
    std::lock_guard<std::mutex> g(v->e.mu);
    return block_prepare_engine(v->e, &v->offsets);
}

}  // namespace api
}  // namespace bn

using namespace bn::api;

namespace {

std::vector<uint32_t> fixed_probe_off(uint32_t B, uint32_t nprobe) {
    std::vector<uint32_t> off(B + 1);
    for (uint32_t q = 0; q <= B; ++q) off[q] = q * nprobe;
    return off;
}

}  // namespace

extern "C" {

int bn_ivf_block_prepare(bn_ivf* v) {
    if (!v) return fail(BN_EINVAL, "null handle");
    return ivf_block_prepare(v);
}

int bn_ivf_query_block(bn_ivf* v, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc,
                       const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz,
                       const uint8_t* block_seed, uint32_t trials, uint32_t k, uint32_t* ids, int64_t* scores,
                       uint32_t* n_hits, int32_t* failed_cluster, int32_t* failed_trial) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (nprobe && !probes) return fail(BN_EINVAL, "null probes");
    if ((uint64_t)B * nprobe > (1u << 24)) return fail(BN_EINVAL, "B * nprobe exceeds 2^24");
    std::lock_guard<std::mutex> gd(v->e.mu);
    Engine& e = v->e;
    if (!e.c.client) return fail(BN_EUNSUPPORTED, "this handle has no client state (attach_client was not called)");
    TRY(block_prepare_engine(e, &v->offsets));
    const auto t0 = std::chrono::steady_clock::now();
    const std::vector<uint32_t> off = fixed_probe_off(B, nprobe);
    IvfBlockJob j;
    TRY(ivf_block_plan(*v, j, B, off.data(), probes, trials, k, false, e.ctx->num_sms));
    TRY(ivf_block_pack(e, j, e.ws, e.host, v_enc, g, t_idx, t_sign, t_nnz, block_seed));
    v->prof_host_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    v->prof_have = false;
    TRY(ivf_block_launch(e, j, e.ws, e.host, e.stream, v->prof ? v->prof_ev : nullptr));
    CU(cudaStreamSynchronize(e.stream));
    v->prof_have = v->prof;
    return ivf_block_finish(j, e.host, ids, scores, n_hits, failed_cluster, failed_trial);
}

int bn_ivf_block_tune(bn_ivf* v, uint32_t w_tile, uint32_t stages) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (w_tile && (w_tile % 16 || w_tile > 256)) return fail(BN_EINVAL, "w_tile = %u is not 0 or a multiple of 16 up to 256", w_tile);
    if (stages && (stages < 2 || stages > BG_MAX_STAGES)) return fail(BN_EINVAL, "stages = %u outside 2..=%d", stages, BG_MAX_STAGES);
    std::lock_guard<std::mutex> gd(v->e.mu);
    v->blk_w = w_tile;
    v->blk_stages = stages;
    return BN_OK;
}

int bn_ivf_block_profile(bn_ivf* v, int enable) {
    if (!v) return fail(BN_EINVAL, "null handle");
    std::lock_guard<std::mutex> gd(v->e.mu);
    CU(cudaSetDevice(v->e.ctx->device));
    if (enable)
        for (cudaEvent_t& ev : v->prof_ev)
            if (!ev) CU(cudaEventCreate(&ev));
    v->prof = enable != 0;
    v->prof_have = false;
    return BN_OK;
}

int bn_ivf_block_profile_read(bn_ivf* v, float* ms, uint32_t cap, uint32_t* n) {
    if (!v || !n) return fail(BN_EINVAL, "null argument");
    std::lock_guard<std::mutex> gd(v->e.mu);
    *n = 0;
    if (!v->prof_have) return BN_OK;
    const uint32_t total = bn_ivf::PROF_EVENTS;  // host plan + pack, then the 10 device stages
    for (uint32_t i = 0; i < total && i < cap; ++i) {
        if (i == 0) {
            ms[0] = v->prof_host_ms;
        } else {
            float x = 0.f;
            if (cudaEventElapsedTime(&x, v->prof_ev[i - 1], v->prof_ev[i]) != cudaSuccess) x = -1.f;
            ms[i] = x;
        }
        *n = i + 1;
    }
    cudaGetLastError();  // an unrecorded stage (skipped work) reports -1, not a sticky error
    return BN_OK;
}

int bn_ivf_verify_block(bn_ivf* v, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* r,
                        uint64_t r_len, const uint64_t* v_enc, const uint8_t* block_seed, uint32_t trials,
                        int32_t* failed_cluster, int32_t* failed_trial, uint64_t* ur, uint64_t* zv) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (!trials) return fail(BN_EINVAL, "trials must be at least 1");
    if (nprobe && !probes) return fail(BN_EINVAL, "null probes");
    if ((uint64_t)B * nprobe > (1u << 24)) return fail(BN_EINVAL, "B * nprobe exceeds 2^24");
    std::lock_guard<std::mutex> gd(v->e.mu);
    Engine& e = v->e;
    const std::vector<uint32_t> off = fixed_probe_off(B, nprobe);
    IvfBlockJob j;
    TRY(ivf_block_plan(*v, j, B, off.data(), probes, trials, 0, true, e.ctx->num_sms));
    if (r_len != j.R)
        return fail(BN_EINVAL, "r holds %llu entries; the probed lists hold %llu rows", (unsigned long long)r_len,
                    (unsigned long long)j.R);
    if (j.R && !r) return fail(BN_EINVAL, "null r");
    TRY(validate_residues(r, j.R, "r"));
    TRY(ivf_block_pack(e, j, e.ws, e.host, v_enc, nullptr, nullptr, nullptr, nullptr, block_seed));
    char* d = e.ws.at<char>();
    cudaStream_t s = e.stream;
    CU(cudaSetDevice(e.ctx->device));
    if (j.R) CU(cudaMemcpyAsync(d + j.o_r, r, j.R * 8, cudaMemcpyHostToDevice, s));
    TRY(ivf_block_launch(e, j, e.ws, e.host, s));
    if (ur && j.P) CU(cudaMemcpyAsync(ur, d + j.o_urout, (uint64_t)j.P * trials * 8, cudaMemcpyDeviceToHost, s));
    if (zv && j.P) CU(cudaMemcpyAsync(zv, d + j.o_zv, (uint64_t)j.P * trials * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return ivf_block_finish(j, e.host, nullptr, nullptr, nullptr, failed_cluster, failed_trial);
}

}  // extern "C"
