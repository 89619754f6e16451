// bn_tc.cu -- Protocol 2 (crypto.rs:1013-1046) on the 5th-generation tensor
// cores: z_t = u_t^T M_enc for up to 20 trials per pass as an exact u8 GEMM
// (tcgen05.mma kind::i8, s32 accumulators in TMEM), fed by TMA, drained by
// four epilogue warps that recombine the byte limbs modulo p = 2^61 - 1.
//
// Roles per CTA (one CTA per SM, persistent over 4096-row panels):
//   warp 0  TMA producer: per 128-row stage, S boxes of 128 rows x 128 bytes
//           of M_enc (S strips of 16 columns) + the 8T x 128 U tile
//   warp 1  MMA issuer: per stage S x 4 tcgen05.mma (M=128, N=8T, K=32),
//           tcgen05.commit frees the stage; after the panel's last stage a
//           commit hands the TMEM accumulators to the epilogue
//   warps 2-5 epilogue: tcgen05.ld, limb recombination, z partials to HBM
// Every mbarrier wait is bounded; on timeout the CTA flags *err and winds
// down (waits for its own copies and MMAs, frees TMEM) instead of hanging.
#include <cudaTypedefs.h>

#include <algorithm>

#include "bn_tc.cuh"
#include "bn_tcgen05.cuh"

namespace bn {

namespace {

using namespace tcg;

// ------------------------------------------------------------------ u draws
constexpr int UG_THREADS = 352;  // >= 20 trials x 17 keystream blocks: one block per thread
constexpr int UG_PAD = TC_ROWS + TC_ROWS / 16;  // one pad word per 16 keeps lanes off shared banks
__device__ __forceinline__ uint32_t ug_idx(uint32_t i) { return i + (i >> 4); }

// Byte transpose of four words: o_b = byte b of w[0], w[1], w[2], w[3] (in
// that order, low byte first), by byte permutes.
__device__ __forceinline__ void transpose_bytes4(const uint32_t w[4], uint32_t& o0, uint32_t& o1, uint32_t& o2,
                                                 uint32_t& o3) {
    const uint32_t t0 = __byte_perm(w[0], w[1], 0x5140), t1 = __byte_perm(w[2], w[3], 0x5140);
    const uint32_t t2 = __byte_perm(w[0], w[1], 0x7362), t3 = __byte_perm(w[2], w[3], 0x7362);
    o0 = __byte_perm(t0, t1, 0x5410);
    o1 = __byte_perm(t0, t1, 0x7632);
    o2 = __byte_perm(t2, t3, 0x5410);
    o3 = __byte_perm(t2, t3, 0x7632);
}

__global__ void __launch_bounds__(UG_THREADS)
tc_ugen_kernel(const VerifySeg* __restrict__ vsegs, const TcBlock* __restrict__ blocks, const ChaChaKey* __restrict__ keys,
               const uint64_t* __restrict__ r, uint32_t t_base, uint32_t t_cnt, uint32_t n_rows,
               uint8_t* __restrict__ u_out, uint64_t u_row_pitch, uint64_t* __restrict__ ur_part,
               uint32_t trials_total, uint32_t* __restrict__ flags) {
    const uint32_t blk = blockIdx.x;
    const TcBlock tb = blocks[blk];
    const VerifySeg vs = vsegs[tb.seg];
    const uint32_t here = min((uint32_t)TC_ROWS, vs.rows - tb.i0);
    const ChaChaKey key = keys[vs.query];
    __shared__ uint64_t us[TC_MAX_TRIALS][UG_PAD];

    // draws: 128 consecutive indices per trial span at most 17 keystream blocks
    for (uint32_t item = threadIdx.x; item < t_cnt * 17; item += blockDim.x) {
        const uint32_t tl = item / 17, bi = item % 17;
        const uint64_t first = draw_index(vs, t_base + tl, tb.i0);
        const uint64_t kb = first / 8 + bi;
        if (kb * 8 >= first + TC_ROWS) continue;
        uint32_t w[16];
        chacha20_block(key, kb, w);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint64_t idx = kb * 8 + q;
            if (idx >= first && idx < first + TC_ROWS) {
                const uint32_t ii = (uint32_t)(idx - first);
                uint64_t x = ((uint64_t)w[2 * q] | ((uint64_t)w[2 * q + 1] << 32)) & P;
                if (ii >= here) x = 0;  // rows past the segment end
                else if (x == P) { atomicOr(flags, DRAW_HIT_P); x = 0; }
                us[tl][ug_idx(ii)] = x;
            }
        }
    }
    __syncthreads();
    // U tile image: row (t, b) holds byte b of u_t[i] for the 128 rows i.
    // Thread (t, chunk) reads its 16 draws once and writes all 8 byte rows.
    // per-block image: rows of 128 bytes, blocks n_rows * 128 apart; flat
    // image: rows u_row_pitch apart, this block at byte column r0 + i0
    const uint64_t pitch = u_row_pitch ? u_row_pitch : TC_ROWS;
    uint8_t* dst = u_row_pitch ? u_out + vs.r0 + tb.i0 : u_out + (uint64_t)blk * n_rows * TC_ROWS;
    for (uint32_t c = threadIdx.x; c < t_cnt * (TC_ROWS / 16); c += blockDim.x) {
        const uint32_t tl = c / (TC_ROWS / 16), ch = c % (TC_ROWS / 16);
        uint32_t pl[8][4];  // pl[b][j]: byte b of draws 4j .. 4j + 3
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t lo[4], hi[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint64_t x = us[tl][ug_idx(ch * 16 + 4 * j + q)];
                lo[q] = (uint32_t)x;
                hi[q] = (uint32_t)(x >> 32);
            }
            transpose_bytes4(lo, pl[0][j], pl[1][j], pl[2][j], pl[3][j]);
            transpose_bytes4(hi, pl[4][j], pl[5][j], pl[6][j], pl[7][j]);
        }
#pragma unroll
        for (int b = 0; b < 8; ++b)
            reinterpret_cast<uint4*>(dst + (uint64_t)(tl * 8 + b) * pitch)[ch] =
                make_uint4(pl[b][0], pl[b][1], pl[b][2], pl[b][3]);
    }
    for (uint32_t c = threadIdx.x; c < (n_rows - 8 * t_cnt) * (TC_ROWS / 16); c += blockDim.x) {  // zero pad rows
        const uint32_t row = 8 * t_cnt + c / (TC_ROWS / 16), ch = c % (TC_ROWS / 16);
        reinterpret_cast<uint4*>(dst + (uint64_t)row * pitch)[ch] = make_uint4(0, 0, 0, 0);
    }
    // u_t . r over this block's rows (skipped when r is not known yet)
    if (!r) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t tl = warp; tl < t_cnt; tl += blockDim.x / 32) {
        uint64_t acc = 0;
        for (uint32_t ii = lane; ii < here; ii += 32)
            acc = add_mod(acc, mul_mod(us[tl][ug_idx(ii)], r[vs.r0 + tb.i0 + ii]));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc = add_mod(acc, __shfl_xor_sync(FULLMASK, acc, off));
        if (lane == 0) ur_part[(uint64_t)blk * trials_total + t_base + tl] = acc;
    }
}

// ------------------------------------------------------------------ GEMM + drain

constexpr int TC_THREADS = 320;  // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr uint32_t STRIP_BYTES = TC_ROWS * 128;  // one 128x128 M box
constexpr int TC_EPI_WARPS = 8;                // TMEM drain warps: 2 per lane quarter

// Drains one work item's accumulators into z partials.  TMEM holds, per strip
// s < sg (columns s * n_rows ...), lanes = the strip's 128 byte columns (j, a)
// (element j = lane / 8, byte a = lane % 8) and columns (t, b) (trial t, byte
// b of u_t).  Warp (lane quarter q, half) reads every other 64-column chunk:
// each lane folds its 8 trials' byte products to (lo + hi 2^32) 2^(8a) mod p,
// then a butterfly over the 8 lanes of one element leaves lane a with trial
// c0/8 + a's sum; 16-column remainders use a plain 3-level reduction.
// z_out[t * N + j] receives z_t[j] for t < t_cnt.
// (lo + hi 2^32) 2^w mod p, folded below 2^61 + 8 (so 8 of them sum below
// 2^64): lo, hi < 2^56 (byte sums of s32 accumulators), 0 <= w < 61.
__device__ __forceinline__ uint64_t fold_part(uint64_t lo, uint64_t hi, uint32_t w) {
    return fold(rotl61(lo + rotl61(hi, 32), w));
}

// One 32-column chunk (4 trials) of a strip: two butterfly levels leave
// lanes a and a ^ 1 with trial c0/8 + 2 (a >> 2 & 1) + (a >> 1 & 1).
__device__ __forceinline__ void z_drain32(uint32_t taddr, uint32_t lane, uint32_t j, uint32_t c0, uint32_t t_cnt,
                                          uint64_t* __restrict__ z_out) {
    const uint32_t a = lane & 7;
    const bool b2 = (a & 4) != 0, b1 = (a & 2) != 0;
    uint32_t v[32];
    tmem_ld32(taddr, v);
    uint64_t part[4];
#pragma unroll
    for (int tt = 0; tt < 4; ++tt) {
        uint64_t lo = 0, hi = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            lo += (uint64_t)v[8 * tt + b] << (8 * b);
            hi += (uint64_t)v[8 * tt + 4 + b] << (8 * b);
        }
        part[tt] = fold_part(lo, hi, 8 * a);
    }
    uint64_t k2[2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
        k2[i] = (b2 ? part[i + 2] : part[i]) + __shfl_xor_sync(FULLMASK, b2 ? part[i] : part[i + 2], 4);
    uint64_t k1 = (b1 ? k2[1] : k2[0]) + __shfl_xor_sync(FULLMASK, b1 ? k2[0] : k2[1], 2);
    k1 += __shfl_xor_sync(FULLMASK, k1, 1);
    const uint32_t t = c0 / 8 + (b2 ? 2u : 0u) + (b1 ? 1u : 0u);
    if ((a & 1) == 0 && t < t_cnt) z_out[(uint64_t)t * N + j] = canon(k1);
}

// One 64-column chunk (8 trials) of a strip: lane (xi, a) folds its 8
// trials' byte products to (lo + hi 2^32) 2^(8a) mod p, a butterfly over the
// 8 lanes of one element leaves lane a with trial c0/8 + a's sum.
__device__ __forceinline__ void z_drain64(uint32_t taddr, uint32_t lane, uint32_t j, uint32_t c0, uint32_t t_cnt,
                                          uint64_t* __restrict__ z_out) {
    const uint32_t a = lane & 7;
    const uint32_t w1 = 8 * a;
    const bool b2 = (a & 4) != 0, b1 = (a & 2) != 0, b0 = (a & 1) != 0;
    uint32_t v[64];
    tmem_ld64(taddr, v);
    uint64_t part[8];
#pragma unroll
    for (int tt = 0; tt < 8; ++tt) {
        uint64_t lo = 0, hi = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            lo += (uint64_t)v[8 * tt + b] << (8 * b);
            hi += (uint64_t)v[8 * tt + 4 + b] << (8 * b);
        }
        part[tt] = fold_part(lo, hi, w1);
    }
    uint64_t k4[4], k2[2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
        k4[i] = (b2 ? part[i + 4] : part[i]) + __shfl_xor_sync(FULLMASK, b2 ? part[i] : part[i + 4], 4);
#pragma unroll
    for (int i = 0; i < 2; ++i)
        k2[i] = (b1 ? k4[i + 2] : k4[i]) + __shfl_xor_sync(FULLMASK, b1 ? k4[i] : k4[i + 2], 2);
    const uint64_t z = canon((b0 ? k2[1] : k2[0]) + __shfl_xor_sync(FULLMASK, b0 ? k2[0] : k2[1], 1));
    const uint32_t t = c0 / 8 + a;
    if (t < t_cnt) z_out[(uint64_t)t * N + j] = z;
}

// One 16-column chunk (2 trials) of a strip: plain 3-level reduction.
__device__ __forceinline__ void z_drain16(uint32_t taddr, uint32_t lane, uint32_t j, uint32_t c0, uint32_t t_cnt,
                                          uint64_t* __restrict__ z_out) {
    const uint32_t a = lane & 7;
    const uint32_t w1 = 8 * a;
    uint32_t v[16];
    tmem_ld16(taddr, v);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t t = c0 / 8 + h;
        uint64_t lo = 0, hi = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            lo += (uint64_t)v[8 * h + b] << (8 * b);
            hi += (uint64_t)v[8 * h + 4 + b] << (8 * b);
        }
        uint64_t zc = fold_part(lo, hi, w1);
        zc += __shfl_xor_sync(FULLMASK, zc, 1);
        zc += __shfl_xor_sync(FULLMASK, zc, 2);
        zc += __shfl_xor_sync(FULLMASK, zc, 4);
        if (a == 0 && t < t_cnt) z_out[(uint64_t)t * N + j] = canon(zc);
    }
}

// Drains one work item's accumulators into z partials.  TMEM holds, per strip
// s < sg (columns s * n_rows ...), lanes = the strip's 128 byte columns (j, a)
// (element j = lane / 8, byte a = lane % 8) and columns (t, b) (trial t, byte
// b of u_t).  Warp (lane quarter q, half) reads every other 64-column chunk,
// then every other 16-column remainder chunk.
// z_out[t * N + j] receives z_t[j] for t < t_cnt.
__device__ __forceinline__ void z_drain(uint32_t tmem, uint32_t q, uint32_t half, uint32_t lane, uint32_t sg,
                                        uint32_t strip0, uint32_t n_rows, uint32_t t_cnt, uint64_t* __restrict__ z_out) {
    const uint32_t jl = q * 4 + (lane >> 3);
    const uint32_t wide = n_rows & ~63u;
    for (uint32_t s = 0; s < sg; ++s) {
        const uint32_t j = (strip0 + s) * 16 + jl;
        const uint32_t tbase = tmem + ((q * 32) << 16) + s * n_rows;
        for (uint32_t c0 = 64 * half; c0 < wide; c0 += 128) z_drain64(tbase + c0, lane, j, c0, t_cnt, z_out);
        for (uint32_t c0 = wide + 16 * half; c0 < n_rows; c0 += 32) z_drain16(tbase + c0, lane, j, c0, t_cnt, z_out);
    }
}

template <int S>
__global__ void __launch_bounds__(TC_THREADS, 1)
tc_freivalds_kernel(const __grid_constant__ CUtensorMap tmap_m, const __grid_constant__ CUtensorMap tmap_u,
                    const TcPanel* __restrict__ panels, uint32_t npanels, uint32_t t_base, uint32_t t_cnt,
                    uint32_t n_rows, uint32_t trials_total, uint32_t stages, uint32_t stage_bytes,
                    uint64_t* __restrict__ z_part, uint32_t* __restrict__ err, int u_flat, long long wait_limit) {
    extern __shared__ uint8_t tc_dyn[];
    __shared__ uint64_t full_b[4], empty_b[4], accf_b, acce_b, done_b;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const uint32_t base = (su32(tc_dyn) + 1023u) & ~1023u;  // 1024-byte aligned stage ring
    uint8_t* ring = tc_dyn + (base - su32(tc_dyn));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t u_off = S * STRIP_BYTES;
    const uint32_t u_bytes = n_rows * TC_ROWS;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            bar_init(&full_b[s], 1);
            bar_init(&empty_b[s], 1);
        }
        bar_init(&accf_b, 1);
        bar_init(&acce_b, TC_EPI_WARPS);
        bar_init(&done_b, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_s)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = tmem_base_s;
    const uint32_t groups = (64 + S - 1) / S;

    if (warp == 0) {
        // ---------------------------------------------------------- TMA producer
        if (lane == 0) {
            uint64_t it = 0;
            bool stop = false;
            for (uint32_t item = blockIdx.x; item < npanels * groups && !stop; item += gridDim.x) {
                const uint32_t p = item / groups, g = item % groups;
                const TcPanel pn = panels[p];
                const uint32_t nrb = (pn.rows + TC_ROWS - 1) / TC_ROWS;
                {
                    const uint32_t sg = min((uint32_t)S, 64u - g * S);
                    for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                        const uint32_t st = (uint32_t)(it % stages);
                        if (it >= stages && !bar_wait(&empty_b[st], (uint32_t)(((it / stages) - 1) & 1), wait_limit)) {
                            abort_s = 1;
                            atomicOr(err, 4u);
                            stop = true;
                            break;
                        }
                        if (abort_s) { stop = true; break; }
                        uint8_t* sb = ring + (uint64_t)st * stage_bytes;
                        bar_expect_tx(&full_b[st], sg * STRIP_BYTES + u_bytes);
                        for (uint32_t s = 0; s < sg; ++s)
                            tma_2d(sb + s * STRIP_BYTES, &tmap_m, (int)((g * S + s) * 128), (int)(pn.row0 + rb * TC_ROWS),
                                   &full_b[st]);
                            if (u_flat)
                            tma_2d(sb + u_off, &tmap_u, (int)((pn.rb0 + rb) * TC_ROWS), 0, &full_b[st]);
                        else
                            tma_2d(sb + u_off, &tmap_u, 0, (int)((pn.rb0 + rb) * n_rows), &full_b[st]);
                    }
                }
            }
            // no copy may still be landing in shared memory when the CTA exits
            for (uint64_t j = it > stages ? it - stages : 0; j < it; ++j)
                bar_wait(&full_b[j % stages], (uint32_t)((j / stages) & 1));
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = (2u << 4) | (1u << 15) | ((n_rows >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
            uint64_t it = 0, gc = 0;
            bool stop = false;
            for (uint32_t item = blockIdx.x; item < npanels * groups && !stop; item += gridDim.x, ++gc) {
                const uint32_t p = item / groups, g = item % groups;
                const TcPanel pn = panels[p];
                const uint32_t nrb = (pn.rows + TC_ROWS - 1) / TC_ROWS;
                {
                    const uint32_t sg = min((uint32_t)S, 64u - g * S);
                    if (gc > 0 && !bar_wait(&acce_b, (uint32_t)((gc - 1) & 1), wait_limit)) {
                        abort_s = 1;
                        atomicOr(err, 8u);
                        stop = true;
                        break;
                    }
                    tc_after();
                    for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                        const uint32_t st = (uint32_t)(it % stages);
                        if (!bar_wait(&full_b[st], (uint32_t)((it / stages) & 1), wait_limit) || abort_s) {
                            abort_s = 1;
                            atomicOr(err, 8u);
                            stop = true;
                            break;
                        }
                        tc_after();
                        const uint32_t sb = base + st * stage_bytes;
                        for (uint32_t s = 0; s < sg; ++s)
#pragma unroll
                            for (uint32_t ks = 0; ks < TC_ROWS / 32; ++ks) {
                                const uint64_t a = sdesc(sb + s * STRIP_BYTES + ks * 4096u, STRIP_BYTES, 1024);
                                const uint64_t b = sdesc(sb + u_off + ks * 32u, 16, 1024);
                                mma_i8(tmem + s * n_rows, a, b, idesc, (rb | ks) != 0);
                            }
                        mma_commit(&empty_b[st]);  // stage reusable once these MMAs have read it
                    }
                    if (stop) break;
                    mma_commit(&accf_b);  // accumulators complete for this group
                }
            }
            mma_commit(&done_b);
            if (!bar_wait(&done_b, 0)) atomicOr(err, 64u);  // every issued MMA has finished before TMEM is freed
        }
    } else {
        // ---------------------------------------------------------- epilogue
        const uint32_t q = (uint32_t)(warp & 3);            // TMEM lane quarter of this warp
        const uint32_t half = (uint32_t)(warp - 2) >> 2;    // which chunks of the item it drains
        uint64_t gc = 0;
        bool stop = false;
        for (uint32_t item = blockIdx.x; item < npanels * groups && !stop; item += gridDim.x, ++gc) {
            const uint32_t p = item / groups, g = item % groups;
            const uint32_t sg = min((uint32_t)S, 64u - g * S);
            const bool ok = __all_sync(FULLMASK, bar_wait(&accf_b, (uint32_t)(gc & 1), wait_limit));  // warp-uniform
            if (!ok && lane == 0) { abort_s = 1; atomicOr(err, 16u); }
            if (__any_sync(FULLMASK, !ok || abort_s)) { stop = true; break; }
            tc_after();
            z_drain(tmem, q, half, lane, sg, g * S, n_rows, t_cnt, z_part + ((uint64_t)p * trials_total + t_base) * N);
            tc_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&acce_b);
        }
    }
    tc_before();
    __syncthreads();
    if (warp == 1) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// ------------------------------------------------------------------ small panels
// tc_freivalds_kernel for panels of at most TC_SMALL_RB row blocks (the short
// inverted lists of an IVF batch, most of them a single 128-row block).  A
// CTA takes whole panels: the panel's U tiles are loaded once into one of two
// shared-memory regions (the next panel's load overlaps this one's MMAs) and
// stay there while the panel's 64 strips of m_enc stream through the stage
// ring, one strip per item, into three rotating TMEM accumulators (3 x n_rows
// <= 480 columns): the drain of a strip overlaps the MMAs of the next two.
// Roles: warp 0 TMA, warp 1 MMA issuer, warps 2-21 drain (5 per lane
// quarter; a strip's 32-column chunks, and a last 16-column one when n_rows
// is not a multiple of 32, are dealt out among them: one each at 20 trials).
// Every mbarrier wait is bounded; on timeout the CTA sets *err and winds down.
constexpr uint32_t TC_SMALL_RB = TC_SMALL_PANEL_ROWS / TC_ROWS;
constexpr uint32_t SM_STAGES = 6;
constexpr int SM_EPI_WARPS = 20;
constexpr uint32_t SM_DRAIN_PARTS = SM_EPI_WARPS / 4;
constexpr int SM_THREADS = 64 + 32 * SM_EPI_WARPS;

__global__ void __launch_bounds__(SM_THREADS, 1)
tc_freivalds_small_kernel(const __grid_constant__ CUtensorMap tmap_m, const __grid_constant__ CUtensorMap tmap_u,
                          const TcPanel* __restrict__ panels, uint32_t p_first, uint32_t npanels,
                          uint32_t t_base, uint32_t t_cnt, uint32_t n_rows, uint32_t trials_total,
                          uint64_t* __restrict__ z_part, uint32_t* __restrict__ err, long long wait_limit) {
    extern __shared__ uint8_t tc_dyn[];
    __shared__ uint64_t full_b[SM_STAGES], empty_b[SM_STAGES], accf_b[3], acce_b[3], ufull_b[2], ufree_b[2], done_b;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    // 1024-byte aligned: [U region 0][U region 1][stage ring]
    const uint32_t base = (su32(tc_dyn) + 1023u) & ~1023u;
    uint8_t* sm = tc_dyn + (base - su32(tc_dyn));
    const uint32_t u_tile = n_rows * TC_ROWS;  // one row block's U tile (a multiple of 2048 bytes)
    const uint32_t u_region = TC_SMALL_RB * u_tile;
    const uint32_t ring_off = 2 * u_region;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < SM_STAGES; ++s) {
            bar_init(&full_b[s], 1);
            bar_init(&empty_b[s], 1);
        }
        for (int b = 0; b < 3; ++b) {
            bar_init(&accf_b[b], 1);
            bar_init(&acce_b[b], SM_EPI_WARPS);
        }
        for (int b = 0; b < 2; ++b) {
            bar_init(&ufull_b[b], 1);
            bar_init(&ufree_b[b], 1);
        }
        bar_init(&done_b, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_s)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = tmem_base_s;

    if (warp == 0) {
        // ---------------------------------------------------------- TMA producer
        if (lane == 0) {
            uint64_t it = 0;
            uint32_t pc = 0;
            bool stop = false;
            for (uint32_t w = blockIdx.x; w < npanels && !stop; w += gridDim.x, ++pc) {
                const TcPanel pn = panels[p_first + w];
                const uint32_t nrb = min((pn.rows + TC_ROWS - 1) / TC_ROWS, TC_SMALL_RB);
                const uint32_t ub = pc & 1;
                // U region ub is free once the MMAs of panel pc - 2 have read it
                if (pc >= 2 && !bar_wait(&ufree_b[ub], ((pc >> 1) - 1) & 1, wait_limit)) {
                    abort_s = 1;
                    atomicOr(err, 4u);
                    break;
                }
                if (abort_s) break;
                bar_expect_tx(&ufull_b[ub], nrb * u_tile);
                for (uint32_t rb = 0; rb < nrb; ++rb)
                    tma_2d(sm + ub * u_region + rb * u_tile, &tmap_u, 0, (int)((pn.rb0 + rb) * n_rows), &ufull_b[ub]);
                for (uint32_t s = 0; s < 64 && !stop; ++s)
                    for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                        const uint32_t st = (uint32_t)(it % SM_STAGES);
                        if (it >= SM_STAGES && !bar_wait(&empty_b[st], (uint32_t)(((it / SM_STAGES) - 1) & 1), wait_limit)) {
                            abort_s = 1;
                            atomicOr(err, 4u);
                            stop = true;
                            break;
                        }
                        if (abort_s) { stop = true; break; }
                        bar_expect_tx(&full_b[st], STRIP_BYTES);
                        tma_2d(sm + ring_off + st * STRIP_BYTES, &tmap_m, (int)(s * 128), (int)(pn.row0 + rb * TC_ROWS),
                               &full_b[st]);
                    }
            }
            // no copy may still be landing in shared memory when the CTA exits:
            // the last ring stages and the U loads of the last two panels
            for (uint64_t j = it > SM_STAGES ? it - SM_STAGES : 0; j < it; ++j)
                bar_wait(&full_b[j % SM_STAGES], (uint32_t)((j / SM_STAGES) & 1));
            for (uint32_t x = pc > 2 ? pc - 2 : 0; x < pc; ++x) bar_wait(&ufull_b[x & 1], (x >> 1) & 1);
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = (2u << 4) | (1u << 15) | ((n_rows >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
            uint64_t it = 0, sc = 0;
            uint32_t pc = 0;
            bool stop = false;
            for (uint32_t w = blockIdx.x; w < npanels && !stop; w += gridDim.x, ++pc) {
                const TcPanel pn = panels[p_first + w];
                const uint32_t nrb = min((pn.rows + TC_ROWS - 1) / TC_ROWS, TC_SMALL_RB);
                const uint32_t ub = pc & 1;
                if (!bar_wait(&ufull_b[ub], (pc >> 1) & 1, wait_limit) || abort_s) {
                    abort_s = 1;
                    atomicOr(err, 8u);
                    break;
                }
                tc_after();
                for (uint32_t s = 0; s < 64 && !stop; ++s, ++sc) {
                    const uint32_t b = (uint32_t)(sc % 3), use = (uint32_t)(sc / 3);
                    if (use > 0 && !bar_wait(&acce_b[b], (use - 1) & 1, wait_limit)) {
                        abort_s = 1;
                        atomicOr(err, 8u);
                        stop = true;
                        break;
                    }
                    tc_after();
                    const uint32_t d = tmem + b * n_rows;
                    for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                        const uint32_t st = (uint32_t)(it % SM_STAGES);
                        if (!bar_wait(&full_b[st], (uint32_t)((it / SM_STAGES) & 1), wait_limit) || abort_s) {
                            abort_s = 1;
                            atomicOr(err, 8u);
                            stop = true;
                            break;
                        }
                        tc_after();
                        const uint32_t sa = base + ring_off + st * STRIP_BYTES;
                        const uint32_t su = base + ub * u_region + rb * u_tile;
#pragma unroll
                        for (uint32_t ks = 0; ks < TC_ROWS / 32; ++ks)
                            mma_i8(d, sdesc(sa + ks * 4096u, STRIP_BYTES, 1024), sdesc(su + ks * 32u, 16, 1024), idesc,
                                   (rb | ks) != 0);
                        mma_commit(&empty_b[st]);  // stage reusable once these MMAs have read it
                    }
                    if (stop) break;
                    mma_commit(&accf_b[b]);  // this strip's accumulator is complete
                }
                if (stop) break;
                mma_commit(&ufree_b[ub]);  // U region reusable once this panel's MMAs are done
            }
            mma_commit(&done_b);
            if (!bar_wait(&done_b, 0)) atomicOr(err, 64u);  // every issued MMA has finished before TMEM is freed
        }
    } else {
        // ---------------------------------------------------------- drain
        const uint32_t q = (uint32_t)(warp & 3);             // TMEM lane quarter of this warp
        const uint32_t part = (uint32_t)(warp - 2) >> 2;      // its share of each strip's chunks
        const uint32_t jl = q * 4 + (lane >> 3);
        const uint32_t tasks = (n_rows + 31) / 32;            // 32-column chunks (the last may be 16)
        uint64_t sc = 0;
        bool stop = false;
        for (uint32_t w = blockIdx.x; w < npanels && !stop; w += gridDim.x) {
            const uint32_t p = p_first + w;
            uint64_t* z_out = z_part + ((uint64_t)p * trials_total + t_base) * N;
            for (uint32_t s = 0; s < 64; ++s, ++sc) {
                const uint32_t b = (uint32_t)(sc % 3), use = (uint32_t)(sc / 3);
                const bool ok = __all_sync(FULLMASK, bar_wait(&accf_b[b], use & 1, wait_limit));  // warp-uniform
                if (!ok && lane == 0) { abort_s = 1; atomicOr(err, 16u); }
                if (__any_sync(FULLMASK, !ok || abort_s)) { stop = true; break; }
                tc_after();
                const uint32_t tbase = tmem + ((q * 32) << 16) + b * n_rows;
                const uint32_t j = s * 16 + jl;
                for (uint32_t k = part; k < tasks; k += SM_DRAIN_PARTS) {
                    if (32 * k + 32 <= n_rows) z_drain32(tbase + 32 * k, lane, j, 32 * k, t_cnt, z_out);
                    else z_drain16(tbase + 32 * k, lane, j, 32 * k, t_cnt, z_out);
                }
                tc_before();
                __syncwarp();
                if (lane == 0) bar_arrive(&acce_b[b]);
            }
        }
    }
    tc_before();
    __syncthreads();
    if (warp == 1) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// ------------------------------------------------------------------ fused scan + Protocol 2
// One pass over m_enc yields both products, all on the tensor cores.  Each
// stage's S strips (128 rows x 128 bytes of m_enc each) feed two MMAs:
//   z: D[c][(t,b)] += Mb^T Ub as in tc_freivalds_kernel (strip read
//      MN-major), accumulated over the 4096-row panel and drained by the
//      eight epilogue warps at the end of each work item;
//   r: E[i][s] = sum_{j,a} Mb[i][8j+a] W[s][8j+a], the same strip read
//      K-major against the query's diagonal byte image W[s][8j+a] = byte
//      (s - a) of v_j (16 rows per strip: s = a + b < 15), so that
//      sum_s 2^(8s) E[i][s] = sum_j M[i][j] v_j over the group's elements.
//      E is per stage (new rows every stage): two 16-column TMEM buffers at
//      column 480 alternate, and four drain warps turn each into r partials
//      r_part[group][r index] while the next stage accumulates.
// The z and r MMAs are issued by two warps (1 and FU_R_WARP), so neither
// instruction stream waits for the other; a stage is free once the z issuer
// has committed and a drain warp has seen the stage's r MMAs complete.  TMEM: z in columns [0, 3 n_rows) (n_rows <= 160), E in [480, 512).
constexpr int FU_S = 3;
constexpr int FU_DRAIN_WARPS = 4;
constexpr int FU_R_WARP = 2 + TC_EPI_WARPS + FU_DRAIN_WARPS;           // issues the r MMAs
constexpr int FU_THREADS = TC_THREADS + 32 * (FU_DRAIN_WARPS + 1);  // 480
constexpr uint32_t FU_E_COL = 480;
constexpr uint32_t W_STRIP_BYTES = 16 * 128;  // one strip's 16 diagonal rows

__global__ void __launch_bounds__(FU_THREADS, 1)
tc_fused_kernel(const __grid_constant__ CUtensorMap tmap_m, const __grid_constant__ CUtensorMap tmap_u,
                const __grid_constant__ CUtensorMap tmap_w, const TcPanel* __restrict__ panels, uint32_t npanels,
                const VerifySeg* __restrict__ vsegs, uint32_t t_cnt, uint32_t n_rows, uint32_t trials_total,
                uint32_t stages, uint32_t stage_bytes, uint64_t* __restrict__ z_part, uint64_t* __restrict__ r_part,
                uint64_t r_stride, uint32_t* __restrict__ err, long long wait_limit) {
    constexpr int S = FU_S;
    extern __shared__ uint8_t tc_dyn[];
    __shared__ uint64_t full_b[4], empty_b[4], accf_b, acce_b, done_b, racc_b[2], rfree_b[2], wfull_b[2], wfree_b[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const uint32_t base = (su32(tc_dyn) + 1023u) & ~1023u;
    uint8_t* ring = tc_dyn + (base - su32(tc_dyn));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t u_off = S * STRIP_BYTES;
    const uint32_t u_bytes = n_rows * TC_ROWS;
    // the query's diagonal image of an item's strip group: loaded once per item
    // into one of two buffers behind the stage ring (1024-aligned: stage_bytes
    // and w_bytes are multiples of 1024)
    const uint32_t w_bytes = S * W_STRIP_BYTES;
    const uint32_t w_ring = stages * stage_bytes;
    const uint32_t groups = (64 + S - 1) / S;
    const uint32_t items = npanels * groups;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            bar_init(&full_b[s], 1);
            bar_init(&empty_b[s], 2);  // z issuer's commit + r drain's arrival
        }
        bar_init(&accf_b, 1);
        bar_init(&acce_b, TC_EPI_WARPS);
        bar_init(&done_b, 2);
        for (int e = 0; e < 2; ++e) {
            bar_init(&racc_b[e], 1);
            bar_init(&rfree_b[e], FU_DRAIN_WARPS);
            bar_init(&wfull_b[e], 1);
            bar_init(&wfree_b[e], 1);
        }
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_s)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = tmem_base_s;

    if (warp == 0) {
        if (lane == 0) {  // ------------------------------------------ TMA producer
            uint64_t it = 0;
            uint32_t ic = 0, w_issued = 0;  // items started, W images loaded
            bool stop = false;
            for (uint32_t item = blockIdx.x; item < items && !stop; item += gridDim.x, ++ic) {
                const uint32_t p = item / groups, g = item % groups;
                const TcPanel pn = panels[p];
                const uint32_t query = vsegs[pn.seg].query;
                const uint32_t nrb = (pn.rows + TC_ROWS - 1) / TC_ROWS;
                const uint32_t sg = min((uint32_t)S, 64u - g * S);
                const uint32_t ib = ic & 1;  // W buffer of this item: free once item ic - 2's r MMAs are done
                if (ic >= 2 && !bar_wait(&wfree_b[ib], ((ic >> 1) - 1) & 1, wait_limit)) {
                    abort_s = 1;
                    atomicOr(err, 4u);
                    break;
                }
                if (abort_s) break;
                bar_expect_tx(&wfull_b[ib], w_bytes);
                tma_2d(ring + w_ring + ib * w_bytes, &tmap_w, 0, (int)((query * 64 + g * S) * 16), &wfull_b[ib]);
                ++w_issued;
                for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                    const uint32_t st = (uint32_t)(it % stages);
                    if (it >= stages && !bar_wait(&empty_b[st], (uint32_t)(((it / stages) - 1) & 1), wait_limit)) {
                        abort_s = 1;
                        atomicOr(err, 4u);
                        stop = true;
                        break;
                    }
                    if (abort_s) { stop = true; break; }
                    uint8_t* sb = ring + (uint64_t)st * stage_bytes;
                    bar_expect_tx(&full_b[st], sg * STRIP_BYTES + u_bytes);
                    for (uint32_t s = 0; s < sg; ++s)
                        tma_2d(sb + s * STRIP_BYTES, &tmap_m, (int)((g * S + s) * 128), (int)(pn.row0 + rb * TC_ROWS),
                               &full_b[st]);
                    tma_2d(sb + u_off, &tmap_u, 0, (int)((pn.rb0 + rb) * n_rows), &full_b[st]);
                }
            }
            // no copy may still be landing in shared memory when the CTA exits:
            // the last ring stages and the W images of the last two items
            for (uint64_t j = it > stages ? it - stages : 0; j < it; ++j)
                bar_wait(&full_b[j % stages], (uint32_t)((j / stages) & 1));
            for (uint32_t x = w_issued > 2 ? w_issued - 2 : 0; x < w_issued; ++x)
                bar_wait(&wfull_b[x & 1], (x >> 1) & 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {  // ------------------------------------------ z MMA issuer
            const uint32_t idesc_z = (2u << 4) | (1u << 15) | ((n_rows >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
            uint64_t it = 0, gc = 0;
            bool stop = false;
            for (uint32_t item = blockIdx.x; item < items && !stop; item += gridDim.x, ++gc) {
                const uint32_t p = item / groups, g = item % groups;
                const TcPanel pn = panels[p];
                const uint32_t nrb = (pn.rows + TC_ROWS - 1) / TC_ROWS;
                const uint32_t sg = min((uint32_t)S, 64u - g * S);
                if (gc > 0 && !bar_wait(&acce_b, (uint32_t)((gc - 1) & 1), wait_limit)) {
                    abort_s = 1;
                    atomicOr(err, 8u);
                    break;
                }
                tc_after();
                for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                    const uint32_t st = (uint32_t)(it % stages);
                    if (!bar_wait(&full_b[st], (uint32_t)((it / stages) & 1), wait_limit) || abort_s) {
                        abort_s = 1;
                        atomicOr(err, 8u);
                        stop = true;
                        break;
                    }
                    tc_after();
                    const uint32_t sb = base + st * stage_bytes;
                    for (uint32_t s = 0; s < sg; ++s)
#pragma unroll
                        for (uint32_t ks = 0; ks < TC_ROWS / 32; ++ks)  // strip read MN-major
                            mma_i8(tmem + s * n_rows, sdesc(sb + s * STRIP_BYTES + ks * 4096u, STRIP_BYTES, 1024),
                                   sdesc(sb + u_off + ks * 32u, 16, 1024), idesc_z, (rb | ks) != 0);
                    mma_commit(&empty_b[st]);  // this issuer is done with the stage
                }
                if (stop) break;
                mma_commit(&accf_b);
            }
            mma_commit(&done_b);
            if (!bar_wait(&done_b, 0)) atomicOr(err, 64u);  // every issued MMA has finished
        }
    } else if (warp == FU_R_WARP) {
        if (lane == 0) {  // ------------------------------------------ r MMA issuer
            const uint32_t idesc_r = (2u << 4) | ((16u >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
            uint64_t it = 0;
            uint32_t ic = 0;
            bool stop = false;
            for (uint32_t item = blockIdx.x; item < items && !stop; item += gridDim.x, ++ic) {
                const uint32_t p = item / groups, g = item % groups;
                const TcPanel pn = panels[p];
                const uint32_t nrb = (pn.rows + TC_ROWS - 1) / TC_ROWS;
                const uint32_t sg = min((uint32_t)S, 64u - g * S);
                const uint32_t ib = ic & 1;
                if (!bar_wait(&wfull_b[ib], (ic >> 1) & 1, wait_limit) || abort_s) {
                    abort_s = 1;
                    atomicOr(err, 8u);
                    break;
                }
                const uint32_t wb = base + w_ring + ib * w_bytes;
                for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                    const uint32_t st = (uint32_t)(it % stages), eb = (uint32_t)(it & 1);
                    if (!bar_wait(&full_b[st], (uint32_t)((it / stages) & 1), wait_limit) || abort_s ||
                        (it >= 2 && !bar_wait(&rfree_b[eb], (uint32_t)(((it >> 1) - 1) & 1), wait_limit))) {
                        abort_s = 1;
                        atomicOr(err, 8u);
                        stop = true;
                        break;
                    }
                    tc_after();
                    const uint32_t sb = base + st * stage_bytes;
                    for (uint32_t s = 0; s < sg; ++s)
#pragma unroll
                        for (uint32_t ks = 0; ks < TC_ROWS / 32; ++ks)  // strip read K-major
                            mma_i8(tmem + FU_E_COL + 16 * eb, sdesc(sb + s * STRIP_BYTES + ks * 32u, 16, 1024),
                                   sdesc(wb + s * W_STRIP_BYTES + ks * 32u, 16, 1024), idesc_r, (s | ks) != 0);
                    mma_commit(&racc_b[eb]);  // the stage's row products are ready (and its strips read)
                }
                if (stop) break;
                mma_commit(&wfree_b[ib]);  // W buffer reusable once this item's r MMAs have read it
            }
            mma_commit(&done_b);
            if (!bar_wait(&done_b, 0)) atomicOr(err, 64u);  // every issued MMA has finished
        }
    } else if (warp < 2 + TC_EPI_WARPS) {
        // ---------------------------------------------------------- TMEM epilogue (z)
        const uint32_t q = (uint32_t)(warp & 3);
        const uint32_t half = (uint32_t)(warp - 2) >> 2;
        uint64_t gc = 0;
        for (uint32_t item = blockIdx.x; item < items; item += gridDim.x, ++gc) {
            const uint32_t p = item / groups, g = item % groups;
            const uint32_t sg = min((uint32_t)S, 64u - g * S);
            const bool ok = __all_sync(FULLMASK, bar_wait(&accf_b, (uint32_t)(gc & 1), wait_limit));  // warp-uniform
            if (!ok && lane == 0) { abort_s = 1; atomicOr(err, 16u); }
            if (__any_sync(FULLMASK, !ok || abort_s)) break;
            tc_after();
            z_drain(tmem, q, half, lane, sg, g * S, n_rows, t_cnt, z_part + (uint64_t)p * trials_total * N);
            tc_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&acce_b);
        }
    } else if (warp < FU_R_WARP) {
        // ---------------------------------------------------------- r drain warps
        // Lane (quarter q) = stage row q*32 + lane: E[row][s] for s < 16 ->
        // sum_s 2^(8s) E[s] mod p, grouped by 4 (weights 2^0, 2^32, 2^64 =
        // 2^3, 2^96 = 2^35 mod p).  E < 48 * 8 * 255^2 < 2^25 per column.
        const uint32_t q = (uint32_t)(warp & 3);
        const uint32_t rr = q * 32 + lane;
        uint64_t it = 0;
        bool stop = false;
        for (uint32_t item = blockIdx.x; item < items && !stop; item += gridDim.x) {
            const uint32_t p = item / groups, g = item % groups;
            const TcPanel pn = panels[p];
            const VerifySeg vs = vsegs[pn.seg];
            const uint32_t nrb = (pn.rows + TC_ROWS - 1) / TC_ROWS;
            const uint64_t r0 = vs.r0 + (pn.row0 - vs.row0);  // r index of the panel's first row
            for (uint32_t rb = 0; rb < nrb; ++rb, ++it) {
                const uint32_t eb = (uint32_t)(it & 1);
                const bool ok = __all_sync(FULLMASK, bar_wait(&racc_b[eb], (uint32_t)((it >> 1) & 1), wait_limit));
                if (!ok && lane == 0) { abort_s = 1; atomicOr(err, 32u); }
                if (__any_sync(FULLMASK, !ok || abort_s)) { stop = true; break; }
                // the r MMAs of stage it have completed, so they no longer read its
                // strips: the r side's release of the stage (one commit fewer per
                // stage for the r issuer)
                if (q == 0 && lane == 0) bar_arrive(&empty_b[it % stages]);
                tc_after();
                uint32_t v[16];
                tmem_ld16(tmem + ((q * 32) << 16) + FU_E_COL + 16 * eb, v);
                tc_before();
                __syncwarp();
                if (lane == 0) bar_arrive(&rfree_b[eb]);  // the buffer may take stage it + 2
                uint64_t gsum[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    gsum[k] = (uint64_t)v[4 * k] + ((uint64_t)v[4 * k + 1] << 8) + ((uint64_t)v[4 * k + 2] << 16) +
                              ((uint64_t)v[4 * k + 3] << 24);
                const uint64_t rv = canon(gsum[0] + rotl61(gsum[1], 32) + rotl61(gsum[2], 3) + rotl61(gsum[3], 35));
                const uint32_t lr = rb * TC_ROWS + rr;
                if (lr < pn.rows) r_part[(uint64_t)g * r_stride + r0 + lr] = rv;
            }
        }
    }
    tc_before();
    __syncthreads();
    if (warp == 1) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// Diagonal byte image of each query for the fused scan MMA:
// w[((q * 64 + strip) * 16 + s) * 128 + 8 j + a] = byte (s - a) of
// v[q][strip * 16 + j] when 0 <= s - a <= 7, else 0.
__global__ void query_wimg_kernel(const uint64_t* __restrict__ v, uint32_t nq, uint8_t* __restrict__ w) {
    const uint64_t total = (uint64_t)nq * 64 * 16 * 16;  // (query, strip, s, j)
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(e & 15), s = (uint32_t)((e >> 4) & 15);
        const uint64_t qs = e >> 8;  // q * 64 + strip
        const uint64_t x = v[(qs >> 6) * N + (qs & 63) * 16 + j];
        uint64_t word = 0;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int b = (int)s - a;
            if (b >= 0 && b <= 7) word |= ((x >> (8 * b)) & 0xffull) << (8 * a);
        }
        *reinterpret_cast<uint64_t*>(w + (qs * 16 + s) * 128 + 8 * j) = word;
    }
}

// r[i] = sum over strip groups of r_part, then u_t . r for this pass's draws
// rebuilt from their byte image (one CTA per 128-row block).  For the dot
// products warp w takes trials w, w + 4, ... (at most 5) and lane l rows
// 4l .. 4l + 3, whose bytes of draw plane (t, b) are one 32-bit word of the
// image: all of a warp's words are loaded before the arithmetic.
__global__ void __launch_bounds__(TC_ROWS)
tc_rreduce_kernel(const VerifySeg* __restrict__ vsegs, const TcBlock* __restrict__ blocks,
                  const uint64_t* __restrict__ r_part, uint64_t r_stride, uint32_t groups,
                  const uint8_t* __restrict__ u_img, uint32_t t_cnt, uint32_t n_rows, uint32_t trials_total,
                  uint64_t* __restrict__ r, uint64_t* __restrict__ ur_part) {
    constexpr int TPW = TC_MAX_TRIALS / (TC_ROWS / 32);  // trials per warp
    const uint32_t blk = blockIdx.x;
    const TcBlock tb = blocks[blk];
    const VerifySeg vs = vsegs[tb.seg];
    const uint32_t i = threadIdx.x;
    const bool valid = tb.i0 + i < vs.rows;
    const uint64_t ri = vs.r0 + tb.i0 + i;
    __shared__ uint64_t rs[TC_ROWS];
    uint64_t rv = 0;
    if (valid) {
#pragma unroll 8
        for (uint32_t g = 0; g < groups; ++g) rv = add_mod(rv, r_part[(uint64_t)g * r_stride + ri]);
        r[ri] = rv;
    }
    rs[i] = rv;  // 0 past the segment's last row
    const int warp = i >> 5, lane = i & 31;
    const uint8_t* img = u_img + (uint64_t)blk * n_rows * TC_ROWS + 4 * lane;
    uint32_t w[TPW][8];
#pragma unroll
    for (int j = 0; j < TPW; ++j) {
        const uint32_t t = warp + 4 * j;
#pragma unroll
        for (int b = 0; b < 8; ++b)
            w[j][b] = t < t_cnt ? *reinterpret_cast<const uint32_t*>(img + (uint64_t)(8 * t + b) * TC_ROWS) : 0u;
    }
    __syncthreads();
    const uint64_t rr[4] = {rs[4 * lane], rs[4 * lane + 1], rs[4 * lane + 2], rs[4 * lane + 3]};
#pragma unroll
    for (int j = 0; j < TPW; ++j) {
        const uint32_t t = warp + 4 * j;
        if (t >= t_cnt) break;  // warp-uniform
        uint64_t part = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint64_t u = 0;
#pragma unroll
            for (int b = 0; b < 8; ++b) u |= (uint64_t)((w[j][b] >> (8 * q)) & 0xffu) << (8 * b);
            part = add_mod(part, mul_mod(u, rr[q]));
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) part = add_mod(part, __shfl_xor_sync(FULLMASK, part, off));
        if (lane == 0) ur_part[(uint64_t)blk * trials_total + t] = part;
    }
}

// CTA (trial t, y, segment, split sp): y < 8 sums z over every split-th
// panel of the segment (from its sp-th) for the 128 columns [128y, 128y+128)
// and writes that share of z_t . v (z . v is linear in z, so the shares of
// the splits add up); y == 8 sums every split-th row block's u_t . r
// partial.  Splitting the panels over more CTAs keeps enough loads in flight
// when a launch has few segments (one query: 245 panels at N = 1M).
constexpr int FIN_CHUNKS = N / 128;

__global__ void __launch_bounds__(128)
tc_finish_kernel(const uint64_t* __restrict__ z_part, const uint64_t* __restrict__ ur_part,
                 const uint32_t* __restrict__ seg_panel0, const uint32_t* __restrict__ seg_block0,
                 const uint64_t* __restrict__ v_enc, const VerifySeg* __restrict__ vsegs, uint32_t trials,
                 uint32_t split, uint64_t* __restrict__ chunks) {
    const uint32_t t = blockIdx.x, y = blockIdx.y, seg = blockIdx.z / split, sp = blockIdx.z % split;
    __shared__ uint64_t sh[4];
    uint64_t part = 0;
    if (y < FIN_CHUNKS) {
        const VerifySeg vs = vsegs[seg];
        const uint32_t j = y * 128 + threadIdx.x;
        const uint32_t p0 = seg_panel0[seg], p1 = seg_panel0[seg + 1];
        uint64_t z = 0;
#pragma unroll 4
        for (uint32_t p = p0 + sp; p < p1; p += split) z = add_mod(z, z_part[((uint64_t)p * trials + t) * N + j]);
        part = mul_mod(z, v_enc[(uint64_t)vs.query * N + j]);
    } else {
        const uint32_t b0 = seg_block0[seg], b1 = seg_block0[seg + 1];
        for (uint32_t b = b0 + sp + split * threadIdx.x; b < b1; b += split * blockDim.x)
            part = add_mod(part, ur_part[(uint64_t)b * trials + t]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) part = add_mod(part, __shfl_xor_sync(FULLMASK, part, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0)
        chunks[(((uint64_t)seg * trials + t) * (FIN_CHUNKS + 1) + y) * split + sp] =
            add_mod(add_mod(sh[0], sh[1]), add_mod(sh[2], sh[3]));
}

// One CTA per segment, a warp per trial: ur_t and zv_t from the finish
// kernel's shares, then the first trial whose sides differ (-1 if none).
constexpr int DECIDE_WARPS = 8;

__global__ void __launch_bounds__(DECIDE_WARPS * 32)
tc_decide_kernel(const uint64_t* __restrict__ chunks, uint32_t trials, uint32_t split, uint64_t* __restrict__ ur,
                 uint64_t* __restrict__ zv, int32_t* __restrict__ failed) {
    const uint32_t seg = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ int32_t first;
    if (threadIdx.x == 0) first = 0x7fffffff;
    __syncthreads();
    const uint32_t per = (FIN_CHUNKS + 1) * split;  // shares per trial; the last split of them are u . r
    for (uint32_t t = warp; t < trials; t += DECIDE_WARPS) {
        const uint64_t* c = chunks + ((uint64_t)seg * trials + t) * per;
        uint64_t a = 0, b = 0;
        for (uint32_t i = lane; i < per; i += 32) {
            if (i < FIN_CHUNKS * split) b = add_mod(b, c[i]);
            else a = add_mod(a, c[i]);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            a = add_mod(a, __shfl_xor_sync(FULLMASK, a, off));
            b = add_mod(b, __shfl_xor_sync(FULLMASK, b, off));
        }
        if (lane == 0) {
            ur[(uint64_t)seg * trials + t] = a;
            zv[(uint64_t)seg * trials + t] = b;
            if (a != b) atomicMin(&first, (int32_t)t);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) failed[seg] = first == 0x7fffffff ? -1 : first;
}

}  // namespace

cudaError_t make_tmap_u8(CUtensorMap* map, const void* base, uint64_t inner_bytes, uint64_t rows, uint32_t box_inner,
                         uint32_t box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {inner_bytes, rows};
    const cuuint64_t strides[1] = {inner_bytes};
    const cuuint32_t box[2] = {box_inner, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t make_tmap_u8_ksteps2(CUtensorMap* map, const void* base, uint64_t row_bytes, uint64_t rows,
                                 uint32_t box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[3] = {128, rows, row_bytes / 128};
    const cuuint64_t strides[2] = {row_bytes, 128};
    const cuuint32_t box[3] = {128, box_rows, 2};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

void launch_tc_ugen(const VerifySeg* d_vsegs, const TcBlock* d_blocks, uint32_t nblocks, const ChaChaKey* d_keys,
                    const uint64_t* d_r, uint32_t t_base, uint32_t t_cnt, uint32_t n_rows, uint8_t* d_u,
                    uint64_t* d_ur_part, uint32_t trials_total, uint32_t* d_flags, cudaStream_t s,
                    uint64_t u_row_pitch) {
    if (!nblocks) return;
    tc_ugen_kernel<<<nblocks, UG_THREADS, 0, s>>>(d_vsegs, d_blocks, d_keys, d_r, t_base, t_cnt, n_rows, d_u,
                                                  u_row_pitch, d_ur_part, trials_total, d_flags);
}

void launch_tc_freivalds(const CUtensorMap& tmap_m, const CUtensorMap& tmap_u, const TcPanel* d_panels,
                         uint32_t npanels, uint32_t t_base, uint32_t t_cnt, uint32_t n_rows, uint32_t trials_total,
                         uint64_t* d_z_part, uint32_t* d_err, int num_sms, cudaStream_t s, int u_flat,
                         long long wait_cycles) {
    if (!npanels) return;
    const long long wl = wait_cycles > 0 ? wait_cycles : TC_WAIT_CYCLES;
    const int S = n_rows <= 128 ? 4 : 3;
    const uint32_t stage_bytes = (uint32_t)S * STRIP_BYTES + ((n_rows * TC_ROWS + 1023u) & ~1023u);
    uint32_t stages = (220u * 1024u) / stage_bytes;
    stages = stages < 2 ? 2 : (stages > 4 ? 4 : stages);
    const int smem = (int)(stages * stage_bytes + 1024);
    const uint32_t items = npanels * ((64 + S - 1) / S);
    const unsigned grid = items < (uint32_t)num_sms ? items : (unsigned)num_sms;
    if (S == 4) {
        cudaFuncSetAttribute(tc_freivalds_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        tc_freivalds_kernel<4><<<grid, TC_THREADS, smem, s>>>(tmap_m, tmap_u, d_panels, npanels, t_base, t_cnt, n_rows,
                                                              trials_total, stages, stage_bytes, d_z_part, d_err, u_flat, wl);
    } else {
        cudaFuncSetAttribute(tc_freivalds_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        tc_freivalds_kernel<3><<<grid, TC_THREADS, smem, s>>>(tmap_m, tmap_u, d_panels, npanels, t_base, t_cnt, n_rows,
                                                              trials_total, stages, stage_bytes, d_z_part, d_err, u_flat, wl);
    }
}

void launch_tc_freivalds_small(const CUtensorMap& tmap_m, const CUtensorMap& tmap_u, const TcPanel* d_panels,
                               uint32_t p_first, uint32_t npanels, uint32_t t_base, uint32_t t_cnt,
                               uint32_t n_rows, uint32_t trials_total, uint64_t* d_z_part, uint32_t* d_err,
                               int num_sms, cudaStream_t s, long long wait_cycles) {
    if (!npanels) return;
    const long long wl = wait_cycles > 0 ? wait_cycles : TC_WAIT_CYCLES;
    const int smem = (int)(2 * TC_SMALL_RB * n_rows * TC_ROWS + SM_STAGES * STRIP_BYTES + 1024);
    cudaFuncSetAttribute(tc_freivalds_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const unsigned grid = npanels < (uint32_t)num_sms ? npanels : (unsigned)num_sms;
    tc_freivalds_small_kernel<<<grid, SM_THREADS, smem, s>>>(tmap_m, tmap_u, d_panels, p_first, npanels, t_base, t_cnt,
                                                             n_rows, trials_total, d_z_part, d_err, wl);
}

void launch_query_wimg(const uint64_t* d_v, uint32_t nq, uint8_t* d_w, cudaStream_t s) {
    if (!nq) return;
    const uint64_t total = (uint64_t)nq * 64 * 16 * 16;
    const unsigned grid = (unsigned)std::min<uint64_t>((total + 255) / 256, 148 * 16);
    query_wimg_kernel<<<grid, 256, 0, s>>>(d_v, nq, d_w);
}

void launch_tc_fused(const CUtensorMap& tmap_m, const CUtensorMap& tmap_u, const CUtensorMap& tmap_w,
                     const TcPanel* d_panels, uint32_t npanels, const VerifySeg* d_vsegs, uint32_t t_cnt,
                     uint32_t n_rows, uint32_t trials_total, uint64_t* d_z_part, uint64_t* d_r_part, uint64_t r_stride,
                     uint32_t* d_err, int num_sms, cudaStream_t s, long long wait_cycles) {
    if (!npanels) return;
    const long long wl = wait_cycles > 0 ? wait_cycles : TC_WAIT_CYCLES;
    const uint32_t stage_bytes = (uint32_t)FU_S * STRIP_BYTES + ((n_rows * TC_ROWS + 1023u) & ~1023u);
    const uint32_t w_two = 2u * FU_S * W_STRIP_BYTES;  // the two per-item W buffers
    uint32_t stages = (227u * 1024u - 2048u - w_two) / stage_bytes;
    stages = stages < 2 ? 2 : (stages > 4 ? 4 : stages);
    const int smem = (int)(stages * stage_bytes + w_two + 1024);
    const uint32_t items = npanels * ((64 + FU_S - 1) / FU_S);
    const unsigned grid = items < (uint32_t)num_sms ? items : (unsigned)num_sms;
    cudaFuncSetAttribute(tc_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    tc_fused_kernel<<<grid, FU_THREADS, smem, s>>>(tmap_m, tmap_u, tmap_w, d_panels, npanels, d_vsegs, t_cnt, n_rows,
                                                   trials_total, stages, stage_bytes, d_z_part, d_r_part, r_stride,
                                                   d_err, wl);
}

void launch_tc_rreduce(const VerifySeg* d_vsegs, const TcBlock* d_blocks, uint32_t nblocks, const uint64_t* d_r_part,
                       uint64_t r_stride, uint32_t groups, const uint8_t* d_u, uint32_t t_cnt, uint32_t n_rows,
                       uint32_t trials_total, uint64_t* d_r, uint64_t* d_ur_part, cudaStream_t s) {
    if (!nblocks) return;
    tc_rreduce_kernel<<<nblocks, TC_ROWS, 0, s>>>(d_vsegs, d_blocks, d_r_part, r_stride, groups, d_u, t_cnt, n_rows,
                                                  trials_total, d_r, d_ur_part);
}

void launch_tc_finish(const uint64_t* d_z_part, const uint64_t* d_ur_part, const uint32_t* d_seg_panel0,
                      const uint32_t* d_seg_block0, const uint64_t* d_v_enc, const VerifySeg* d_vsegs, uint32_t nseg,
                      uint32_t trials, uint64_t* d_ur, uint64_t* d_zv, uint64_t* d_chunks, int32_t* d_failed,
                      cudaStream_t s) {
    if (!nseg || !trials) return;
    const uint32_t split = tc_finish_split(nseg);
    const uint32_t per_launch = 65535u / split;  // grid.z limit
    for (uint32_t s0 = 0; s0 < nseg; s0 += per_launch) {
        const uint32_t ns = nseg - s0 < per_launch ? nseg - s0 : per_launch;
        tc_finish_kernel<<<dim3(trials, FIN_CHUNKS + 1, ns * split), 128, 0, s>>>(
            d_z_part, d_ur_part, d_seg_panel0 + s0, d_seg_block0 + s0, d_v_enc, d_vsegs + s0, trials, split,
            d_chunks + (uint64_t)s0 * trials * (FIN_CHUNKS + 1) * split);
    }
    tc_decide_kernel<<<nseg, DECIDE_WARPS * 32, 0, s>>>(d_chunks, trials, split, d_ur, d_zv, d_failed);
}

}  // namespace bn
