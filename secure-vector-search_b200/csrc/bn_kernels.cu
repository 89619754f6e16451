// bn_kernels.cu -- CUDA-core kernels of the BN path for sm_100a.
//
// scan_tma_kernel   r = M_enc . v (crypto.rs:561-626 / kernels.cu:100-178),
//                   4-row blocks streamed into shared memory by one bulk
//                   copy each; one work item = 4 rows x 1024 columns split
//                   over four warps (a quarter row each); per element 6
//                   IMAD.WIDE into three 64-bit limb accumulators, no carries,
//                   no per-product fold; a transposed warp reduction and one
//                   fold per row at the end.
// freivalds_kernel  Protocol 2 (crypto.rs:1013-1046): u drawn on device from
//                   the ChaCha20 keystream by index, z_t = u_t^T M_enc and
//                   u_t . r partials per row chunk.
// decode_topk       decode_scores (crypto.rs:901-940) + fp_to_signed + top-k
//                   (lib.rs:452-469) in one pass over the client arrays.
// gemm_abt          keygen-side F_p GEMMs (crypto.rs:419-467).
#include <cuda_runtime.h>
#include <stdint.h>

#include <cooperative_groups.h>
#include <type_traits>

#include "bn_kernels.cuh"

namespace cg = cooperative_groups;

namespace bn {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void named_bar(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__global__ void or_flag_kernel(uint32_t* w, uint32_t bits) { atomicOr(w, bits); }

// ------------------------------------------------------------------ limbs
__global__ void query_limbs_kernel(const uint64_t* __restrict__ v, uint64_t total, QLimb* __restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    uint64_t x = v[i];
    Limbs3 b = limbs(x), c = limbs_hi(x);
    out[i] = QLimb{b.b0, b.b1, b.b2, c.b0, c.b1, c.b2, 0u, 0u};
}

// ------------------------------------------------------------------ scan

__device__ __forceinline__ uint32_t find_seg(const uint64_t* __restrict__ seg_blk, uint32_t nseg, uint32_t hint,
                                             uint64_t blk) {
    if (blk >= seg_blk[hint] && blk < seg_blk[hint + 1]) return hint;
    uint32_t lo = 0, hi = nseg;  // find last s with seg_blk[s] <= blk
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (seg_blk[mid] <= blk) lo = mid; else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------------ scan, TMA pipeline
// One producer warp streams each 4-row block (up to 32 KiB, contiguous in
// m_enc) into a ring of shared-memory stages with a single cp.async.bulk;
// four consumer groups of four warps take the stages round-robin.  Every
// mbarrier wait is bounded: on timeout the CTA records an error in *err
// and stops, so a lost completion cannot hang the GPU.
constexpr int TS_STAGES = 6;
constexpr int TS_GROUPS = 4;
constexpr int TS_CONSUMERS = 32 * 4 * TS_GROUPS;   // 512
constexpr int TS_THREADS = TS_CONSUMERS + 32;      // + producer warp
constexpr uint32_t TS_STAGE_BYTES = SCAN_ROWS * N * 8;  // 32 KiB
constexpr long long WAIT_CYCLES = 2000000000ll;    // ~1 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: true when the phase with `parity` completed within `limit`
// cycles (pipeline waits take the kernel's wait_limit argument; the drain of
// the CTA's own copies keeps the full limit).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = WAIT_CYCLES) {
    const long long t0 = clock64();
    if (limit >= WAIT_CYCLES) {
        while (!mbar_try_wait(bar, parity))
            if (clock64() - t0 > limit) return false;
        return true;
    }
    // a shortened (test) limit polls with test_wait: try_wait may stay
    // suspended until the phase completes, which would outlast the limit
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
    }
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

struct ScanBlock {
    uint64_t row0;  // first m_enc row
    uint64_t out0;  // first r slot
    int nrows;
    uint32_t query;
};
__device__ __forceinline__ ScanBlock scan_block(const ScanSeg* __restrict__ segs, const uint64_t* __restrict__ seg_blk,
                                                uint32_t nseg, uint32_t& hint, uint64_t blk) {
    hint = find_seg(seg_blk, nseg, hint, blk);
    const ScanSeg sg = segs[hint];
    const uint64_t local = (blk - seg_blk[hint]) * SCAN_ROWS;
    const uint64_t left = (uint64_t)sg.rows - local;
    return ScanBlock{sg.row0 + local, sg.out0 + local, left < (uint64_t)SCAN_ROWS ? (int)left : SCAN_ROWS, sg.query};
}

__global__ void __launch_bounds__(TS_THREADS, 1)
scan_tma_kernel(const uint64_t* __restrict__ m_enc, const QLimb* __restrict__ qlimbs, const ScanSeg* __restrict__ segs,
                const uint64_t* __restrict__ seg_blk, uint32_t nseg, uint64_t total_blocks, uint64_t* __restrict__ r,
                uint32_t* __restrict__ err, long long wait_limit) {
    extern __shared__ __align__(1024) unsigned char ts_smem[];
    uint4* stage_base = reinterpret_cast<uint4*>(ts_smem);
    __shared__ uint64_t full_bar[TS_STAGES], empty_bar[TS_STAGES];
    __shared__ unsigned long long red[2][TS_GROUPS][4][SCAN_ROWS][3];
    __shared__ volatile int abort_flag;
    __shared__ volatile int group_stop[2][TS_GROUPS];  // per-iteration snapshot, double-buffered

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < TS_STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 4);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const uint64_t nblk = total_blocks > blockIdx.x ? (total_blocks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (warp == TS_CONSUMERS / 32) {  // ---------------- producer warp
        if (lane == 0) {
            uint32_t hint = 0;
            uint64_t i = 0;
            for (; i < nblk; ++i) {
                const int s = (int)(i % TS_STAGES);
                if (i >= TS_STAGES && !mbar_wait(&empty_bar[s], (uint32_t)(((i / TS_STAGES) - 1) & 1), wait_limit)) {
                    abort_flag = 1;
                    atomicOr(err, 1u);
                    break;
                }
                if (abort_flag) break;
                const ScanBlock b = scan_block(segs, seg_blk, nseg, hint, blockIdx.x + i * gridDim.x);
                const uint32_t bytes = (uint32_t)b.nrows * N * 8;
                mbar_expect_tx(&full_bar[s], bytes);
                bulk_g2s(stage_base + (uint64_t)s * (TS_STAGE_BYTES / 16), m_enc + b.row0 * N, bytes, &full_bar[s]);
            }
            // drain: no bulk copy may still be writing shared memory at exit
            for (uint64_t j = (i > TS_STAGES ? i - TS_STAGES : 0); j < i; ++j)
                mbar_wait(&full_bar[j % TS_STAGES], (uint32_t)((j / TS_STAGES) & 1));
        }
        return;
    }

    // ---------------------------------------------------- consumer groups
    const int group = warp >> 2, wq = warp & 3;
    const bool hi16 = (lane & 16) != 0, hi8 = (lane & 8) != 0;
    uint32_t b0[8], b1[8], b2[8], c0[8], c1[8], c2[8];
    uint32_t cur_q = 0xffffffffu, hint = 0;
    int parity = 0;
    for (uint64_t i = group; i < nblk; i += TS_GROUPS) {
        const int s = (int)(i % TS_STAGES);
        const ScanBlock b = scan_block(segs, seg_blk, nseg, hint, blockIdx.x + i * gridDim.x);
        if (b.query != cur_q) {
            cur_q = b.query;
            const QLimb* ql = qlimbs + (uint64_t)cur_q * N + wq * 256 + 2 * lane;
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const QLimb q = ql[64 * k + e];
                    b0[2 * k + e] = q.b0; b1[2 * k + e] = q.b1; b2[2 * k + e] = q.b2;
                    c0[2 * k + e] = q.c0; c1[2 * k + e] = q.c1; c2[2 * k + e] = q.c2;
                }
        }
        const bool ok = mbar_wait(&full_bar[s], (uint32_t)((i / TS_STAGES) & 1), wait_limit);
        if (!ok) { abort_flag = 1; atomicOr(err, 2u); }
        uint64_t acc[SCAN_ROWS][3];
        const uint4* base = stage_base + (uint64_t)s * (TS_STAGE_BYTES / 16) + wq * 128 + lane;
#pragma unroll
        for (int rr = 0; rr < SCAN_ROWS; ++rr) {
            uint64_t a0 = 0, a1 = 0, a2 = 0;
            if (ok && rr < b.nrows) {
                const uint4* rp = base + rr * (N / 2);
                uint4 x[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) x[k] = rp[32 * k];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int e0 = 2 * k, e1 = 2 * k + 1;
                    a0 = mac(mac(a0, x[k].x, b0[e0]), x[k].y, c0[e0]);
                    a1 = mac(mac(a1, x[k].x, b1[e0]), x[k].y, c1[e0]);
                    a2 = mac(mac(a2, x[k].x, b2[e0]), x[k].y, c2[e0]);
                    a0 = mac(mac(a0, x[k].z, b0[e1]), x[k].w, c0[e1]);
                    a1 = mac(mac(a1, x[k].z, b1[e1]), x[k].w, c1[e1]);
                    a2 = mac(mac(a2, x[k].z, b2[e1]), x[k].w, c2[e1]);
                }
            }
            acc[rr][0] = a0; acc[rr][1] = a1; acc[rr][2] = a2;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[s]);  // this warp is done with the stage
        uint64_t w[2][3];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                uint64_t send = hi16 ? acc[q][a] : acc[q + 2][a];
                uint64_t keep = hi16 ? acc[q + 2][a] : acc[q][a];
                w[q][a] = keep + __shfl_xor_sync(FULL, send, 16);
            }
        uint64_t xs[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            uint64_t send = hi8 ? w[0][a] : w[1][a];
            uint64_t keep = hi8 ? w[1][a] : w[0][a];
            xs[a] = keep + __shfl_xor_sync(FULL, send, 8);
        }
#pragma unroll
        for (int off = 4; off > 0; off >>= 1)
#pragma unroll
            for (int a = 0; a < 3; ++a) xs[a] += __shfl_xor_sync(FULL, xs[a], off);
        if ((lane & 7) == 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) red[parity][group][wq][lane >> 3][a] = xs[a];
        }
        // Stop decision: one snapshot per group and iteration, written before
        // the barrier and read after it, so the four warps agree.
        if (wq == 0 && lane == 0) group_stop[parity][group] = abort_flag;
        named_bar(1 + group, 128);
        if (group_stop[parity][group]) break;
        if (wq == 0 && lane < b.nrows) {
            uint64_t t[3];
#pragma unroll
            for (int a = 0; a < 3; ++a)
                t[a] = red[parity][group][0][lane][a] + red[parity][group][1][lane][a] +
                       red[parity][group][2][lane][a] + red[parity][group][3][lane][a];
            r[b.out0 + lane] = combine3(t[0], t[1], t[2]);
        }
        parity ^= 1;
    }
}

// ------------------------------------------------------------------ Freivalds
constexpr int FV_THREADS = 256;
constexpr int FV_TILE = 32;

template <int TMAX>
__global__ void __launch_bounds__(FV_THREADS)
freivalds_kernel(const uint64_t* __restrict__ m_enc, const uint64_t* __restrict__ r, const VerifySeg* __restrict__ vsegs,
                 const ChaChaKey* __restrict__ keys, uint32_t t_base, uint32_t t_cnt, uint32_t trials,
                 uint32_t chunks, uint32_t chunk_rows, uint64_t* __restrict__ z_part, uint64_t* __restrict__ ur_part,
                 uint32_t* __restrict__ flags, uint32_t seg_base) {
    const uint32_t seg = seg_base + blockIdx.z, chunk = blockIdx.y;
    const uint32_t j = blockIdx.x * FV_THREADS + threadIdx.x;
    const VerifySeg vs = vsegs[seg];
    const uint64_t row_begin = (uint64_t)chunk * chunk_rows;
    const uint64_t row_end = min((uint64_t)vs.rows, row_begin + chunk_rows);
    const ChaChaKey key = keys[vs.query];

    __shared__ uint32_t ul[FV_TILE][TMAX][6];
    __shared__ uint64_t uraw[TMAX][FV_TILE];

    uint64_t acc[TMAX][3];
#pragma unroll
    for (int t = 0; t < TMAX; ++t) acc[t][0] = acc[t][1] = acc[t][2] = 0;
    uint64_t urp = 0;
    uint32_t since_fold = 0;
    const uint32_t gen_t = threadIdx.x >> 3, gen_b = threadIdx.x & 7;

    for (uint64_t tile = row_begin; tile < row_end; tile += FV_TILE) {
        const uint32_t nt = (uint32_t)min((uint64_t)FV_TILE, row_end - tile);
        __syncthreads();
        if (gen_t < t_cnt) {
            const uint64_t first = draw_index(vs, t_base + gen_t, tile);  // draw index of row `tile`
            const uint64_t blk = first / 8 + gen_b;
            if (blk * 8 < first + nt) {
                uint32_t w[16];
                chacha20_block(key, blk, w);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const uint64_t idx = blk * 8 + q;
                    if (idx >= first && idx < first + nt) {
                        uint64_t x = ((uint64_t)w[2 * q] | ((uint64_t)w[2 * q + 1] << 32)) & P;
                        if (x == P) { atomicOr(flags, DRAW_HIT_P); x = 0; }
                        const uint32_t ii = (uint32_t)(idx - first);
                        Limbs3 b = limbs(x), c = limbs_hi(x);
                        ul[ii][gen_t][0] = b.b0; ul[ii][gen_t][1] = b.b1; ul[ii][gen_t][2] = b.b2;
                        ul[ii][gen_t][3] = c.b0; ul[ii][gen_t][4] = c.b1; ul[ii][gen_t][5] = c.b2;
                        uraw[gen_t][ii] = x;
                    }
                }
            }
        }
        __syncthreads();
        const uint64_t* mp = m_enc + (vs.row0 + tile) * N + j;
        for (uint32_t ii = 0; ii < nt; ++ii) {
            const uint64_t mv = __ldg(mp + (uint64_t)ii * N);
            const uint32_t mlo = (uint32_t)mv, mhi = (uint32_t)(mv >> 32);
#pragma unroll
            for (int t = 0; t < TMAX; ++t) {
                if (t < (int)t_cnt) {
                    const uint32_t* u = ul[ii][t];
                    acc[t][0] = mac(mac(acc[t][0], mlo, u[0]), mhi, u[3]);
                    acc[t][1] = mac(mac(acc[t][1], mlo, u[1]), mhi, u[4]);
                    acc[t][2] = mac(mac(acc[t][2], mlo, u[2]), mhi, u[5]);
                }
            }
        }
        if (blockIdx.x == 0 && threadIdx.x < t_cnt) {
            for (uint32_t ii = 0; ii < nt; ++ii)
                urp = add_mod(urp, mul_mod(uraw[threadIdx.x][ii], r[vs.r0 + tile + ii]));
        }
        since_fold += nt;
        if (since_fold >= 480) {  // 512 more rows would still fit below 2^63
#pragma unroll
            for (int t = 0; t < TMAX; ++t) { acc[t][0] = fold(acc[t][0]); acc[t][1] = fold(acc[t][1]); acc[t][2] = fold(acc[t][2]); }
            since_fold = 0;
        }
    }
    const uint64_t slot = (uint64_t)seg * chunks + chunk;
#pragma unroll
    for (int t = 0; t < TMAX; ++t)
        if (t < (int)t_cnt) z_part[(slot * trials + t_base + t) * N + j] = combine3(acc[t][0], acc[t][1], acc[t][2]);
    if (blockIdx.x == 0 && threadIdx.x < t_cnt) ur_part[slot * trials + t_base + threadIdx.x] = urp;
}

__device__ __forceinline__ uint64_t block_sum_mod(uint64_t v, uint64_t* sh) {
    // 256 threads
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = add_mod(v, __shfl_xor_sync(FULL, v, off));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    uint64_t t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = add_mod(t, sh[w]);
    return t;
}

__global__ void __launch_bounds__(256)
freivalds_finish_kernel(const uint64_t* __restrict__ z_part, const uint64_t* __restrict__ ur_part,
                        const uint64_t* __restrict__ v_enc, const VerifySeg* __restrict__ vsegs, uint32_t trials,
                        uint32_t chunks, uint64_t* __restrict__ ur, uint64_t* __restrict__ zv,
                        int32_t* __restrict__ failed) {
    const uint32_t seg = blockIdx.x;
    const VerifySeg vs = vsegs[seg];
    const uint64_t* v = v_enc + (uint64_t)vs.query * N;
    __shared__ uint64_t sh[32];
    int32_t fail = -1;
    for (uint32_t t = 0; t < trials; ++t) {
        uint64_t part = 0;
        for (uint32_t j = threadIdx.x; j < N; j += blockDim.x) {
            uint64_t z = 0;
            for (uint32_t c = 0; c < chunks; ++c) z = add_mod(z, z_part[(((uint64_t)seg * chunks + c) * trials + t) * N + j]);
            part = add_mod(part, mul_mod(z, v[j]));
        }
        const uint64_t zvt = block_sum_mod(part, sh);
        if (threadIdx.x == 0) {
            uint64_t urt = 0;
            for (uint32_t c = 0; c < chunks; ++c) urt = add_mod(urt, ur_part[((uint64_t)seg * chunks + c) * trials + t]);
            ur[(uint64_t)seg * trials + t] = urt;
            zv[(uint64_t)seg * trials + t] = zvt;
            if (fail < 0 && urt != zvt) fail = (int32_t)t;
        }
    }
    if (threadIdx.x == 0) failed[seg] = fail;
}

// ------------------------------------------------------------------ L^T v
// A cluster of 8 CTAs of 1024 threads per query (one CTA per query kept a
// single SM busy for ~34 us): column k = tid % n1, rows j of the CTA's
// range, slice, slice + slices, ... with v_j's limbs in shared memory, so
// each term is six multiply-adds into three accumulators and the column
// loads are independent (batches of 8 in flight).  Each thread sums at most
// 64 terms below 2^53.2 (hi < 2^29), so the accumulators stay below 2^64.
constexpr uint32_t LT_SPLIT = 8;  // CTAs per query (one cluster), N / LT_SPLIT terms each

__global__ void __cluster_dims__(1, LT_SPLIT, 1) __launch_bounds__(1024)
lt_times_v_kernel(const uint64_t* __restrict__ L, uint32_t n1, const uint64_t* __restrict__ v, uint64_t* __restrict__ x) {
    // CTA (q, s) of the query's cluster sums the terms j in [s N/8, (s+1) N/8)
    // for every output k; CTA 0 adds the 8 partial rows through distributed
    // shared memory.  A thread takes one k and every slices-th term of the range.
    constexpr uint32_t TERMS = N / LT_SPLIT;
    const uint32_t q = blockIdx.x, s = blockIdx.y;
    const uint32_t k = threadIdx.x % n1, slices = blockDim.x / n1, sl = threadIdx.x / n1;
    __shared__ uint4 vl[2 * TERMS];
    __shared__ uint64_t part[1024];
    __shared__ uint64_t row[512];  // this CTA's partial x (n1 <= 512)
    for (uint32_t jj = threadIdx.x; jj < TERMS; jj += blockDim.x) {
        const uint64_t w = v[(uint64_t)q * N + s * TERMS + jj];
        const Limbs3 b = limbs(w), c = limbs_hi(w);
        vl[2 * jj] = make_uint4(b.b0, b.b1, b.b2, c.b0);
        vl[2 * jj + 1] = make_uint4(c.b1, c.b2, 0u, 0u);
    }
    __syncthreads();
    uint64_t a0 = 0, a1 = 0, a2 = 0;
    const uint32_t terms = TERMS / slices;  // n1 / 8: a multiple of 8 for n1 >= 64
    for (uint32_t i0 = 0; i0 < terms; i0 += 8) {
        uint64_t xs[8];
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) xs[ii] = __ldg(L + (uint64_t)(s * TERMS + sl + (i0 + ii) * slices) * n1 + k);
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
            const uint32_t jj = sl + (i0 + ii) * slices;
            const uint4 l0 = vl[2 * jj], l1 = vl[2 * jj + 1];
            const uint32_t xl = (uint32_t)xs[ii], xh = (uint32_t)(xs[ii] >> 32);
            a0 = mac(mac(a0, xl, l0.x), xh, l0.w);
            a1 = mac(mac(a1, xl, l0.y), xh, l1.x);
            a2 = mac(mac(a2, xl, l0.z), xh, l1.y);
        }
    }
    part[threadIdx.x] = combine3(a0, a1, a2);
    __syncthreads();
    if (threadIdx.x < n1) {
        uint64_t t = 0;
        for (uint32_t i = 0; i < slices; ++i) t = add_mod(t, part[i * n1 + threadIdx.x]);
        row[threadIdx.x] = t;
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();  // every CTA's row is written
    if (s == 0 && threadIdx.x < n1) {
        uint64_t t = 0;
        for (uint32_t r = 0; r < LT_SPLIT; ++r) t = add_mod(t, cluster.map_shared_rank(row, r)[threadIdx.x]);
        x[(uint64_t)q * n1 + threadIdx.x] = t;
    }
    cluster.sync();  // no CTA leaves while CTA 0 still reads its row
}

// ------------------------------------------------------------------ decode
// Dot of a column-major row with a vector whose limbs sit in shared memory.
__device__ __forceinline__ uint64_t cm_dot(const uint64_t* __restrict__ a_cm, uint64_t rows, uint64_t row,
                                           const uint32_t (*vl)[6], uint32_t n1) {
    uint64_t a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 8
    for (uint32_t k = 0; k < n1; ++k) {
        const uint64_t x = __ldg(a_cm + (uint64_t)k * rows + row);
        const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
        a0 = mac(mac(a0, lo, vl[k][0]), hi, vl[k][3]);
        a1 = mac(mac(a1, lo, vl[k][1]), hi, vl[k][4]);
        a2 = mac(mac(a2, lo, vl[k][2]), hi, vl[k][5]);
    }
    return combine3(a0, a1, a2);
}

__global__ void dense_terms_kernel(const uint64_t* __restrict__ al_cm, const uint64_t* __restrict__ h_cm, uint64_t rows,
                                   uint32_t n1, const uint64_t* __restrict__ g, const uint64_t* __restrict__ x,
                                   uint64_t* __restrict__ out) {
    __shared__ uint32_t gl[512][6], xl[512][6];
    for (uint32_t k = threadIdx.x; k < n1; k += blockDim.x) {
        Limbs3 b = limbs(g[k]), c = limbs_hi(g[k]);
        gl[k][0] = b.b0; gl[k][1] = b.b1; gl[k][2] = b.b2; gl[k][3] = c.b0; gl[k][4] = c.b1; gl[k][5] = c.b2;
        b = limbs(x[k]); c = limbs_hi(x[k]);
        xl[k][0] = b.b0; xl[k][1] = b.b1; xl[k][2] = b.b2; xl[k][3] = c.b0; xl[k][4] = c.b1; xl[k][5] = c.b2;
    }
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = add_mod(cm_dot(al_cm, rows, i, gl, n1), cm_dot(h_cm, rows, i, xl, n1));
}

// Decode copies of the client state in 32-row blocks (layouts in
// bn_kernels.cuh); reads and writes are both coalesced along the rows.
__global__ void decode_layout_kernel(const uint64_t* __restrict__ al_cm, const uint64_t* __restrict__ h_cm,
                                     const uint64_t* __restrict__ mp_cm, uint64_t rows, uint32_t n1,
                                     uint64_t* __restrict__ alh_b, int8_t* __restrict__ m8_cm, uint32_t* __restrict__ bad) {
    const uint64_t rows32 = (rows + 31) / 32 * 32;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t n_alh = rows32 * 2 * n1;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_alh; e += stride) {
        const uint64_t col = (e >> 5) % (2 * n1), gr = ((e >> 5) / (2 * n1)) * 32 + (e & 31);
        uint64_t x = 0;
        if (gr < rows) x = col < n1 ? al_cm[col * rows + gr] : h_cm[(col - n1) * rows + gr];
        alh_b[e] = x;
    }
    if (!m8_cm) return;
    bool out_of_range = false;
    const uint64_t n_m = rows32 * N;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_m; e += stride) {
        const uint64_t col = e / rows32, gr = e - col * rows32;
        int64_t v = 0;
        if (gr < rows) v = to_signed(mp_cm[col * rows + gr]);
        out_of_range |= v < -128 || v > 127;
        m8_cm[e] = (int8_t)v;
    }
    if (out_of_range) atomicOr(bad, 1u);
}

constexpr int DT_THREADS = 256;
constexpr int CAND_CAP = 2048;

__device__ __forceinline__ bool better(int64_t s1, uint32_t i1, int64_t s2, uint32_t i2) {
    return s1 > s2 || (s1 == s2 && i1 < i2);
}

// In-place bitonic sort of n (power of two) entries, best first.
__device__ void bitonic_best_first(int64_t* s, uint32_t* id, int n) {
    for (int size = 2; size <= n; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int i = threadIdx.x; i < n / 2; i += blockDim.x) {
                const int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const bool sw = up ? better(s[hi], id[hi], s[lo], id[lo]) : better(s[lo], id[lo], s[hi], id[hi]);
                if (sw) {
                    int64_t ts = s[lo]; s[lo] = s[hi]; s[hi] = ts;
                    uint32_t ti = id[lo]; id[lo] = id[hi]; id[hi] = ti;
                }
            }
        }
    __syncthreads();
}

// Candidate buffer of one CTA: entries better than the current k-th best
// are appended; when the buffer nears capacity it is sorted and cut to k.
struct TopkBuf {
    int64_t s[CAND_CAP];
    uint32_t id[CAND_CAP];
    int cnt;
    int64_t thr_s;
    uint32_t thr_i;
    int have_thr;
};

// Compaction decision, uniform across the CTA: every thread reads the count
// between two barriers, so no thread can append (next iteration) before all
// have read it; then either all threads compact or none does (topk_compact
// holds __syncthreads).
__device__ __forceinline__ bool topk_full(TopkBuf& b, int limit) {
    __syncthreads();
    const bool full = b.cnt > limit;
    __syncthreads();
    return full;
}

__device__ void topk_compact(TopkBuf& b, int k) {
    __syncthreads();
    const int cnt = b.cnt;
    int n = 1;
    while (n < cnt) n <<= 1;
    for (int i = cnt + threadIdx.x; i < n; i += blockDim.x) { b.s[i] = INT64_MIN; b.id[i] = 0xffffffffu; }
    bitonic_best_first(b.s, b.id, n);
    if (threadIdx.x == 0) {
        if (cnt >= k) {
            b.cnt = k;
            b.thr_s = b.s[k - 1];
            b.thr_i = b.id[k - 1];
            b.have_thr = 1;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void topk_offer(TopkBuf& b, bool valid, int64_t s, uint32_t id, int64_t thr_s, uint32_t thr_i,
                                           int have_thr) {
    if (valid && (!have_thr || better(s, id, thr_s, thr_i))) {
        const int pos = atomicAdd(&b.cnt, 1);
        b.s[pos] = s;
        b.id[pos] = id;
    }
}

// Sum of +-x (sign in bit 31 of the entry) over a gathered column list,
// folded lazily: every term is < 2^61, three terms fit below 2^63.
__device__ __forceinline__ uint64_t signed_term(uint64_t x, bool neg) { return neg ? P - x : x; }

// AL_i . g + H_i . x for corpus row gr from the 32-row-blocked alh_b: the
// 2 n1 columns of the row's block are contiguous, so a warp's batch of 32
// column loads is one 8 KB run.  lim[2k], lim[2k+1] hold the limbs of g_k
// (k < n1) and of x_(k-n1) (k >= n1).  Every column adds lo*b + hi*c <
// 2^53 + 2^50 (hi < 2^29: residues are < 2^61) to an accumulator, so the
// 2 n1 <= 1024 columns stay below 2^64 with no fold.
__device__ __forceinline__ uint64_t dense_terms_row(const uint64_t* __restrict__ alh_b, uint32_t n1, uint64_t gr,
                                                    const uint4* __restrict__ lim) {
    const uint64_t* p = alh_b + (gr >> 5) * (2ull * n1) * 32 + (gr & 31);
    uint64_t a0 = 0, a1 = 0, a2 = 0;
    for (uint32_t k0 = 0; k0 < 2 * n1; k0 += 32) {  // 2 n1 is a multiple of 32 (n1 >= 64)
        uint64_t xs[32];
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) xs[kk] = __ldg(p + (uint64_t)(k0 + kk) * 32);
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) {
            const uint4 l0 = lim[2 * (k0 + kk)], l1 = lim[2 * (k0 + kk) + 1];  // {b0,b1,b2,c0}, {c1,c2,-,-}
            const uint32_t xl = (uint32_t)xs[kk], xh = (uint32_t)(xs[kk] >> 32);
            a0 = mac(mac(a0, xl, l0.x), xh, l0.w);
            a1 = mac(mac(a1, xl, l0.y), xh, l1.x);
            a2 = mac(mac(a2, xl, l0.z), xh, l1.y);
        }
    }
    return combine3(a0, a1, a2);
}

// Two zero-extended 16-bit halves from bytes 0, 1 (sel 0x4140) or 2, 3
// (sel 0x4342) of x (selector nibble 4 picks a zero byte).
__device__ __forceinline__ uint32_t zext_pair(uint32_t x, uint32_t sel) {
    uint32_t d;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(d) : "r"(x), "r"(sel));
    return d;
}

// M . T for the warp's 32-row block (lane l = row 32 blk + l): the T
// columns go 32 at a time, one per lane; a lane loads its column's 32 row
// bytes (one 32-byte run of the column-major int8 copy: the warps decoding
// neighbouring blocks at the same time read neighbouring runs of the same
// columns, so DRAM pages serve many of them).  Each byte m becomes the
// unsigned m + 128 (xor 0x80) for a +1 entry or 127 - m (xor 0x7f) for a -1
// entry, widened to 16-bit halves; a reduce-scatter over the lanes (lane bit
// 4 keeps rows 0-15 or 16-31, then bits 3..0) with plain 32-bit adds (32
// terms <= 255 stay below 2^16, so no carry crosses a half) leaves lane l
// the biased sum of row l over those 32 columns.  The bias, 128 per +1
// entry and 127 per -1 entry, is taken off at the end.  Four groups of
// loads are in flight at a time.  Returns the exact integer.
__device__ __forceinline__ int32_t m_times_t_warp(const int8_t* __restrict__ m8_cm, uint64_t rows32, uint64_t blk,
                                                  const uint32_t* __restrict__ tl, uint32_t tn, uint32_t lane) {
    const int8_t* base = m8_cm + blk * 32;  // column c's run: base + c * rows32, 32-byte aligned
    int32_t acc = 0, bias = 0;
    for (uint32_t g0 = 0; g0 < tn; g0 += 4 * 32) {
        uint4 lo[4], hi[4];
        uint32_t mask[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t c = g0 + u * 32 + lane;
            lo[u] = hi[u] = make_uint4(0u, 0u, 0u, 0u);
            mask[u] = 0;  // past tn: zero bytes, no bias
            if (c < tn) {
                const uint32_t e = tl[c];
                const uint4* run = reinterpret_cast<const uint4*>(base + (uint64_t)(e & 0x3ffu) * rows32);
                lo[u] = __ldg(run);
                hi[u] = __ldg(run + 1);
                mask[u] = (e >> 31) ? 0x7f7f7f7fu : 0x80808080u;
            }
            const uint32_t pos = __ballot_sync(FULL, mask[u] == 0x80808080u), neg = __ballot_sync(FULL, mask[u] == 0x7f7f7f7fu);
            bias += 128 * __popc(pos) + 127 * __popc(neg);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (g0 + u * 32 >= tn) break;  // warp-uniform
            const uint32_t wds[8] = {lo[u].x ^ mask[u], lo[u].y ^ mask[u], lo[u].z ^ mask[u], lo[u].w ^ mask[u],
                                     hi[u].x ^ mask[u], hi[u].y ^ mask[u], hi[u].z ^ mask[u], hi[u].w ^ mask[u]};
            uint32_t v[16];  // v[w]: rows 2w (low half), 2w + 1 (high half)
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                v[2 * i] = zext_pair(wds[i], 0x4140u);
                v[2 * i + 1] = zext_pair(wds[i], 0x4342u);
            }
            // reduce-scatter: after the step over lane bit b the lane keeps
            // the half of its words that its bit b selects
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                const bool up = lane & 16;
                const uint32_t send = up ? v[w] : v[w + 8], keep = up ? v[w + 8] : v[w];
                v[w] = keep + __shfl_xor_sync(FULL, send, 16);
            }
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const bool up = lane & 8;
                const uint32_t send = up ? v[w] : v[w + 4], keep = up ? v[w + 4] : v[w];
                v[w] = keep + __shfl_xor_sync(FULL, send, 8);
            }
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const bool up = lane & 4;
                const uint32_t send = up ? v[w] : v[w + 2], keep = up ? v[w + 2] : v[w];
                v[w] = keep + __shfl_xor_sync(FULL, send, 4);
            }
            {
                const bool up = lane & 2;
                const uint32_t send = up ? v[0] : v[1], keep = up ? v[1] : v[0];
                v[0] = keep + __shfl_xor_sync(FULL, send, 2);
            }
            const uint32_t pair = v[0] + __shfl_xor_sync(FULL, v[0], 1);
            acc += (int32_t)((lane & 1) ? (pair >> 16) : (pair & 0xffffu));
        }
    }
    return acc - bias;
}

// M_i . T from the column-major residues (plaintext not int8-valued): one
// row per lane, gathers lazily folded.
__device__ __forceinline__ uint64_t m_times_t_cm(const uint64_t* __restrict__ mp_cm, uint64_t rows, uint64_t gr,
                                                 const uint32_t* __restrict__ tl, uint32_t tn) {
    uint64_t m_t = 0;
    uint32_t c = 0;
    for (; c + 8 <= tn; c += 8) {  // 8 gathers in flight, folded two terms at a time
        uint64_t x[8];
        uint32_t e[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            e[q] = tl[c + q];
            x[q] = __ldg(mp_cm + (uint64_t)(e[q] & 0x3ffu) * rows + gr);
        }
#pragma unroll
        for (int q = 0; q < 8; q += 2)
            m_t = fold(m_t) + signed_term(x[q], e[q] >> 31) + signed_term(x[q + 1], e[q + 1] >> 31);
    }
    for (; c < tn; ++c) {
        const uint32_t e = tl[c];
        m_t = fold(m_t) + signed_term(__ldg(mp_cm + (uint64_t)(e & 0x3ffu) * rows + gr), e >> 31);
    }
    return canon(m_t);
}

// S . v_enc for the warp's 32-row block, which is exactly one sliced-ELL
// slice ([width][32 rows] u16).  The slice is read as 16-byte chunks, chunk
// j = lane + 32 i holding entries of column slot j / 4 for rows 8 (j % 4) ..
// + 7, so a lane always sees the same 8 rows (8 (lane % 4) + 0..7) and
// keeps 8 partial sums; a reduce-scatter over lane bits 4, 3, 2 then leaves
// one row's sum per lane, and a shuffle hands row l to lane l.  Every entry
// is an index into vt = [v_enc, 0, p - v_enc] (ELL_NEG, ELL_PAD), so a term
// is one shared load and one add; the sums fold every 4 terms (4 terms
// below 2^61 on top of a folded value stay below 2^64).
__device__ __forceinline__ uint64_t s_times_v_warp(const DecodeCorpus& dc, uint64_t blk, const uint64_t* __restrict__ vt,
                                                   uint32_t lane) {
    const uint32_t off = dc.s_off[blk], wdt = dc.s_w[blk];
    const uint4* base = reinterpret_cast<const uint4*>(dc.s_ell + off);  // slice data is 64 * wdt bytes
    const uint32_t chunks = wdt * 4;
    constexpr uint32_t PAD2 = ELL_PAD | (ELL_PAD << 16);
    uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t j0 = 0; j0 < chunks; j0 += 8 * 32) {
        uint4 ch[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t j = j0 + u * 32 + lane;
            ch[u] = j < chunks ? __ldg(base + j) : make_uint4(PAD2, PAD2, PAD2, PAD2);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t w[4] = {ch[u].x, ch[u].y, ch[u].z, ch[u].w};
#pragma unroll
            for (int h = 0; h < 8; ++h)  // clamped into the table (ELL_TABLE - 1 holds 0)
                acc[h] += vt[min((h & 1) ? (w[h >> 1] >> 16) : (w[h >> 1] & 0xffffu), ELL_TABLE - 1)];
            if ((u & 3) == 3) {
#pragma unroll
                for (int h = 0; h < 8; ++h) acc[h] = fold(acc[h]);
            }
        }
    }
    // each step adds two values below 2^61 + 8 and folds the sum
#pragma unroll
    for (int h = 0; h < 4; ++h) {  // lane bit 4: keep rows h + 4 * bit
        const bool up = lane & 16;
        const uint64_t send = up ? acc[h] : acc[h + 4], keep = up ? acc[h + 4] : acc[h];
        acc[h] = fold(keep + __shfl_xor_sync(FULL, send, 16));
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // lane bit 3
        const bool up = lane & 8;
        const uint64_t send = up ? acc[h] : acc[h + 2], keep = up ? acc[h + 2] : acc[h];
        acc[h] = fold(keep + __shfl_xor_sync(FULL, send, 8));
    }
    {  // lane bit 2
        const bool up = lane & 4;
        const uint64_t send = up ? acc[0] : acc[1], keep = up ? acc[1] : acc[0];
        acc[0] = fold(keep + __shfl_xor_sync(FULL, send, 4));
    }
    // lane l now holds row 8 (l & 3) + 4 b4 + 2 b3 + b2 (b = bits of l); lane
    // r fetches its row from the lane that holds it
    const uint32_t src = (lane >> 3) | ((lane & 1) << 2) | (((lane >> 1) & 1) << 3) | (((lane >> 2) & 1) << 4);
    return canon(__shfl_sync(FULL, acc[0], src));
}

// A warp's running top-k (k <= 32) as a list sorted best first across the
// lanes: lane i holds the i-th best (score, id), lanes >= k the empty entry
// (INT64_MIN never occurs as a score: fp_to_signed lies in (-p/2, p/2)).
// Every lane offers one candidate; those better than the k-th best are
// inserted one at a time, each at the rank the ballot of the list entries
// better than it gives, the entries below it moving down one lane.  No
// shared memory and no block barrier.
constexpr int WARP_TOPK_MAX = 32;

__device__ __forceinline__ void warp_topk_offer(int64_t& ls, uint32_t& li, int k, bool valid, int64_t s, uint32_t id,
                                                uint32_t lane) {
    const int64_t ts = __shfl_sync(FULL, ls, k - 1);
    const uint32_t ti = __shfl_sync(FULL, li, k - 1);
    uint32_t m = __ballot_sync(FULL, valid && better(s, id, ts, ti));
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const int64_t cs = __shfl_sync(FULL, s, src);
        const uint32_t ci = __shfl_sync(FULL, id, src);
        const int pos = __popc(__ballot_sync(FULL, (int)lane < k && better(ls, li, cs, ci)));
        const int64_t up_s = __shfl_up_sync(FULL, ls, 1);
        const uint32_t up_i = __shfl_up_sync(FULL, li, 1);
        if (pos < k) {  // warp-uniform
            if ((int)lane > pos) { ls = up_s; li = up_i; }
            if ((int)lane == pos) { ls = cs; li = ci; }
            if ((int)lane >= k) { ls = INT64_MIN; li = 0xffffffffu; }
        }
    }
}

// Merges n (score, id) entries of shared memory into every warp's list
// (entry e goes to warp e / 32 % warps), then the warps' lists into warp 0
// through `xs`, `xi` (32 * warps entries).  Returns in warp 0's lanes.
__device__ __forceinline__ void warp_topk_reduce(int64_t& ls, uint32_t& li, int k, int64_t* xs, uint32_t* xi,
                                                 uint32_t warp, uint32_t lane) {
    xs[warp * 32 + lane] = ls;
    xi[warp * 32 + lane] = li;
    __syncthreads();
    if (warp == 0) {
        for (uint32_t w = 1; w < DT_THREADS / 32; ++w) {
            const int64_t s = xs[w * 32 + lane];
            const uint32_t id = xi[w * 32 + lane];
            warp_topk_offer(ls, li, k, s != INT64_MIN, s, id, lane);
        }
    }
    __syncthreads();
}

// A warp decodes one unit: a segment's rows inside one aligned 32-row block
// of the corpus (lane l = row 32 blk + l; lanes outside the segment idle in
// the row work but join the block-wide M T and S v).  A CTA takes tiles of
// 8 units of its query in turn (the host gives each query CTAs in
// proportion to its units).  Mv = r - (AL g + H x) - M T - S v, ranked by
// fp_to_signed into the CTA's candidate buffer (WARP_LISTS: k <= 32, every
// warp's own list, merged at the end with no barrier in the loop); the CTA's
// best k go to the scratch lists, and the last CTA of the query to finish (a
// ticket taken after a device-scope fence, no waiting) merges them.
constexpr uint32_t DT_WARPS = DT_THREADS / 32;

template <bool WARP_LISTS>
__global__ void __launch_bounds__(DT_THREADS, DECODE_CTAS_PER_SM)
decode_topk_kernel(const uint64_t* __restrict__ r, DecodeCorpus dc, const ScanSeg* __restrict__ segs,
                   const uint64_t* __restrict__ seg_unit, const DecodeQuery* __restrict__ queries,
                   const uint64_t* __restrict__ vv, const uint64_t* __restrict__ gg, const uint64_t* __restrict__ xx,
                   const uint32_t* __restrict__ t_ent, const uint32_t* __restrict__ t_nnz, uint32_t k, TopkScratch ts,
                   uint64_t* __restrict__ mv_out, uint32_t* __restrict__ out_ids, int64_t* __restrict__ out_scores,
                   uint32_t* __restrict__ out_n, uint32_t nq) {
    uint32_t lo = 0, hi = nq;  // the query owning this CTA: last one with cta0 <= blockIdx.x
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (queries[mid].cta0 <= blockIdx.x) lo = mid; else hi = mid;
    }
    const uint32_t q = lo;
    const DecodeQuery dq = queries[q];
    const uint32_t cta = blockIdx.x - dq.cta0;
    const uint32_t n1 = dc.n1;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    extern __shared__ uint4 dyn_limbs[];  // 2 x uint4 per column: g's n1 columns, then x's
    __shared__ uint64_t vt[ELL_TABLE];  // [v_enc, 0, p - v_enc, 0]: the S . v table
    __shared__ uint32_t tl[N];
    struct WarpXchg {  // the warps' lists on their way to warp 0
        int64_t s[DT_THREADS];
        uint32_t id[DT_THREADS];
    };
    __shared__ typename std::conditional<WARP_LISTS, WarpXchg, TopkBuf>::type buf;
    __shared__ int last_s;
    const uint32_t tn = min(t_nnz[q], (uint32_t)N);
    for (uint32_t kk = threadIdx.x; kk < 2 * n1; kk += blockDim.x) {
        const uint64_t w = kk < n1 ? gg[(uint64_t)q * n1 + kk] : xx[(uint64_t)q * n1 + (kk - n1)];
        const Limbs3 b = limbs(w), c = limbs_hi(w);
        dyn_limbs[2 * kk] = make_uint4(b.b0, b.b1, b.b2, c.b0);
        dyn_limbs[2 * kk + 1] = make_uint4(c.b1, c.b2, 0u, 0u);
    }
    for (uint32_t j = threadIdx.x; j < N; j += blockDim.x) {
        const uint64_t x = vv[(uint64_t)q * N + j];
        vt[j] = x;
        vt[ELL_NEG + j] = x ? P - x : 0;
    }
    if (threadIdx.x == 0) vt[ELL_PAD] = vt[ELL_TABLE - 1] = 0;
    for (uint32_t c = threadIdx.x; c < tn; c += blockDim.x) tl[c] = t_ent[(uint64_t)q * N + c];
    if constexpr (!WARP_LISTS)
        if (threadIdx.x == 0) { buf.cnt = 0; buf.have_thr = 0; buf.thr_s = INT64_MIN; buf.thr_i = 0xffffffffu; }
    __syncthreads();
    int64_t ls = INT64_MIN;  // WARP_LISTS: this warp's list (lane i: i-th best)
    uint32_t li = 0xffffffffu;

    uint64_t u_begin = 0, u_count = 0;  // nseg == 0: every probed list of this query was empty
    if (dq.nseg) {
        u_begin = seg_unit[dq.seg0];
        u_count = seg_unit[dq.seg0 + dq.nseg] - u_begin;
    }
    const uint64_t tiles = (u_count + DT_WARPS - 1) / DT_WARPS;
    // The buffer is checked (two CTA barriers) every DT_CHECK tiles, not
    // every tile, so the warps may drift apart within that window; between
    // checks at most DT_CHECK * 256 rows append, and a check compacts above
    // CAND_CAP - DT_CHECK * 256 = 1024 >= k entries.
    constexpr uint32_t DT_CHECK = 4;
    static_assert(CAND_CAP - DT_CHECK * DT_THREADS >= TOPK_MAX, "candidate buffer too small for the check interval");
    uint32_t it = 0;
    for (uint64_t tile = cta; tile < tiles; tile += dq.ctas, ++it) {
        const uint64_t u = tile * DT_WARPS + warp;
        bool valid = false;
        int64_t score = 0;
        uint32_t id = 0;
        if (u < u_count) {  // warp-uniform
            const uint64_t gu = u_begin + u;
            uint32_t sa = dq.seg0, sb = dq.seg0 + dq.nseg;  // last segment with seg_unit <= gu
            while (sb - sa > 1) {
                const uint32_t mid = (sa + sb) >> 1;
                if (seg_unit[mid] <= gu) sa = mid; else sb = mid;
            }
            const ScanSeg sg = segs[sa];
            const uint64_t blk = (sg.row0 >> 5) + (gu - seg_unit[sa]);
            const uint64_t gr = blk * 32 + lane;
            valid = gr >= sg.row0 && gr < sg.row0 + sg.rows;
            const uint64_t ridx = sg.out0 + (gr - sg.row0);
            uint64_t rv = 0;
            if (valid) {
                rv = r[ridx];
                id = dc.ids ? dc.ids[gr] : (uint32_t)gr;
            }
            uint64_t m_t = 0;
            if (dc.m8_cm) {
                const int32_t mt = m_times_t_warp(dc.m8_cm, (dc.rows + 31) & ~31ull, blk, tl, tn, lane);
                m_t = mt >= 0 ? (uint64_t)mt : P - (uint64_t)(-(int64_t)mt);
            }
            const uint64_t s_v = s_times_v_warp(dc, blk, vt, lane);
            if (valid) {
                if (!dc.m8_cm) m_t = m_times_t_cm(dc.mp_cm, dc.rows, gr, tl, tn);
                const uint64_t dense = dense_terms_row(dc.alh_b, n1, gr, dyn_limbs);
                const uint64_t mv = sub_mod(sub_mod(rv, add_mod(dense, m_t)), s_v);
                if (mv_out) mv_out[ridx] = mv;
                score = to_signed(mv);
            }
        }
        if constexpr (WARP_LISTS) {
            warp_topk_offer(ls, li, (int)k, valid, score, id, lane);
        } else {
            const int64_t th_s = buf.thr_s;
            const uint32_t th_i = buf.thr_i;
            const int ht = buf.have_thr;
            topk_offer(buf, valid, score, id, th_s, th_i, ht);
            if (it % DT_CHECK == DT_CHECK - 1 && topk_full(buf, CAND_CAP - DT_CHECK * DT_THREADS))
                topk_compact(buf, (int)k);
        }
    }
    const uint32_t ctas = dq.ctas;
    const uint64_t slot = blockIdx.x;
    if constexpr (WARP_LISTS) {
        warp_topk_reduce(ls, li, (int)k, buf.s, buf.id, warp, lane);
        if (warp == 0) {
            const uint32_t keep = __popc(__ballot_sync(FULL, lane < k && ls != INT64_MIN));
            if (lane < keep) {
                ts.cand_s[slot * k + lane] = ls;
                ts.cand_i[slot * k + lane] = li;
            }
            if (lane == 0) ts.cand_n[slot] = keep;
        }
    } else {
        topk_compact(buf, (int)k);
        const int keep = min(buf.cnt, (int)k);
        for (int i = threadIdx.x; i < keep; i += blockDim.x) {
            ts.cand_s[slot * k + i] = buf.s[i];
            ts.cand_i[slot * k + i] = buf.id[i];
        }
        if (threadIdx.x == 0) ts.cand_n[slot] = (uint32_t)keep;
    }
    __threadfence();  // this CTA's lists are visible device-wide before its ticket
    __syncthreads();
    if (threadIdx.x == 0) last_s = atomicAdd(&ts.done[q], 1u) == ctas - 1;
    __syncthreads();
    if (!last_s) return;

    // ---------------------------------------------------------- merge (last CTA of the query)
    __threadfence();
    const uint64_t total = (uint64_t)ctas * k;
    if constexpr (WARP_LISTS) {
        // warp w takes entries w * 32 + lane + 256 i into its list; then warp 0 merges the lists
        ls = INT64_MIN;
        li = 0xffffffffu;
        for (uint64_t t0 = (uint64_t)warp * 32; t0 < total; t0 += DT_THREADS) {
            const uint64_t e = t0 + lane;
            bool v = false;
            int64_t sc = 0;
            uint32_t id = 0;
            if (e < total) {
                const uint64_t sl = (uint64_t)dq.cta0 + e / k;
                const uint32_t i = (uint32_t)(e % k);
                v = i < __ldcg(ts.cand_n + sl);
                if (v) {
                    sc = __ldcg(ts.cand_s + sl * k + i);
                    id = __ldcg(ts.cand_i + sl * k + i);
                }
            }
            warp_topk_offer(ls, li, (int)k, v, sc, id, lane);
        }
        warp_topk_reduce(ls, li, (int)k, buf.s, buf.id, warp, lane);
        if (warp == 0) {
            const uint32_t keep = __popc(__ballot_sync(FULL, lane < k && ls != INT64_MIN));
            if (lane < keep) {
                out_ids[(uint64_t)q * k + lane] = li;
                out_scores[(uint64_t)q * k + lane] = ls;
            }
            if (lane == 0) {
                out_n[q] = keep;
                ts.done[q] = 0;
            }
        }
        return;
    } else {
        if (threadIdx.x == 0) { buf.cnt = 0; buf.have_thr = 0; buf.thr_s = INT64_MIN; buf.thr_i = 0xffffffffu; }
        __syncthreads();
    // Four tiles of entries per round: their loads (written by other CTAs
    // during this launch, so read through L2) are all in flight before the
    // offers; entries past a list's count are loaded and ignored.
    for (uint64_t t0 = 0; t0 < total; t0 += 4 * DT_THREADS) {
        bool valid[4];
        int64_t sc[4];
        uint32_t id[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t e = t0 + u * DT_THREADS + threadIdx.x;
            valid[u] = false;
            sc[u] = 0;
            id[u] = 0;
            if (e < total) {
                const uint64_t sl = (uint64_t)dq.cta0 + e / k;
                const uint32_t i = (uint32_t)(e % k);
                const uint32_t n = __ldcg(ts.cand_n + sl);
                sc[u] = __ldcg(ts.cand_s + sl * k + i);
                id[u] = __ldcg(ts.cand_i + sl * k + i);
                valid[u] = i < n;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t th_s = buf.thr_s;
            const uint32_t th_i = buf.thr_i;
            const int ht = buf.have_thr;
            topk_offer(buf, valid[u], sc[u], id[u], th_s, th_i, ht);
            if (topk_full(buf, CAND_CAP - DT_THREADS)) topk_compact(buf, (int)k);
        }
    }
    topk_compact(buf, (int)k);
    const int out_keep = min(buf.cnt, (int)k);
    for (int i = threadIdx.x; i < out_keep; i += blockDim.x) {
        out_ids[(uint64_t)q * k + i] = buf.id[i];
        out_scores[(uint64_t)q * k + i] = buf.s[i];
    }
    if (threadIdx.x == 0) {
        out_n[q] = (uint32_t)out_keep;
        ts.done[q] = 0;
    }
    }
}

__global__ void __launch_bounds__(DT_THREADS)
topk_merge_kernel(const int64_t* __restrict__ cand_s, const uint32_t* __restrict__ cand_i,
                  const uint32_t* __restrict__ cand_n, uint32_t ctas, uint32_t k, uint32_t* __restrict__ out_ids,
                  int64_t* __restrict__ out_scores, uint32_t* __restrict__ out_n) {
    const uint32_t q = blockIdx.x;
    __shared__ TopkBuf buf;
    if (threadIdx.x == 0) { buf.cnt = 0; buf.have_thr = 0; buf.thr_s = INT64_MIN; buf.thr_i = 0xffffffffu; }
    __syncthreads();
    const uint64_t total = (uint64_t)ctas * k;
    for (uint64_t tile = 0; tile < total; tile += DT_THREADS) {
        const uint64_t e = tile + threadIdx.x;
        bool valid = false;
        int64_t s = 0;
        uint32_t id = 0;
        if (e < total) {
            const uint32_t c = (uint32_t)(e / k), i = (uint32_t)(e % k);
            const uint64_t slot = (uint64_t)q * ctas + c;
            if (i < cand_n[slot]) { valid = true; s = cand_s[slot * k + i]; id = cand_i[slot * k + i]; }
        }
        const int64_t ts = buf.thr_s;
        const uint32_t ti = buf.thr_i;
        const int ht = buf.have_thr;
        topk_offer(buf, valid, s, id, ts, ti, ht);
        if (topk_full(buf, CAND_CAP - DT_THREADS)) topk_compact(buf, (int)k);
    }
    topk_compact(buf, (int)k);
    const int keep = min(buf.cnt, (int)k);
    for (int i = threadIdx.x; i < keep; i += blockDim.x) {
        out_ids[(uint64_t)q * k + i] = buf.id[i];
        out_scores[(uint64_t)q * k + i] = buf.s[i];
    }
    if (threadIdx.x == 0) out_n[q] = (uint32_t)keep;
}

// Top-k of residues combined on the fly: query q's row i scores
// to_signed(a + b - c) (b, c nullable) with a = ra[q * ld + i] etc., ids[i]
// (or i); mv_out (nullable) receives the combined residues at the same
// offsets.  Same per-CTA candidate buffers as decode_topk_kernel, merged by
// topk_merge_kernel.
__global__ void __launch_bounds__(DT_THREADS)
topk_rows_kernel(const uint64_t* __restrict__ ra, const uint64_t* __restrict__ rb, const uint64_t* __restrict__ rc,
                 uint64_t ld, uint64_t rows, const uint64_t* __restrict__ qoff, const uint32_t* __restrict__ ids,
                 uint32_t k, int64_t* __restrict__ cand_s, uint32_t* __restrict__ cand_i, uint32_t* __restrict__ cand_n,
                 uint64_t* __restrict__ mv_out) {
    const uint32_t q = blockIdx.y;
    __shared__ TopkBuf buf;
    if (threadIdx.x == 0) { buf.cnt = 0; buf.have_thr = 0; buf.thr_s = INT64_MIN; buf.thr_i = 0xffffffffu; }
    __syncthreads();
    // rows of this query: [lo, hi) of row q (ld apart), or of the flat
    // segmented array [qoff[q], qoff[q+1]) (lo rounded down to even so the
    // paired loads stay 16-byte aligned; the extra entry is masked)
    const uint64_t base = qoff ? 0 : (uint64_t)q * ld;
    const uint64_t first = qoff ? qoff[q] : 0, hi = qoff ? qoff[q + 1] : rows;
    const uint64_t lo = first & ~1ull, span = hi > lo ? hi - lo : 0;
    const uint64_t per = ((span + gridDim.x - 1) / gridDim.x + 1) & ~1ull;
    const uint64_t v_begin = lo + min(span, (uint64_t)blockIdx.x * per);
    const uint64_t v_end = min(hi, v_begin + per);
    for (uint64_t tile = v_begin; tile < v_end; tile += 2 * DT_THREADS) {
        const uint64_t i0 = tile + 2 * threadIdx.x;
        const bool valid[2] = {i0 < v_end && i0 >= first, i0 + 1 < v_end};
        uint64_t mv[2] = {0, 0};
        if (i0 < v_end) {  // v_begin, per and ld are even: the pair is 16-byte aligned and inside the row of ld
            const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(ra + base + i0);
            mv[0] = x.x;
            mv[1] = x.y;
            if (rb) {
                const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(rb + base + i0);
                mv[0] = add_mod(mv[0], y.x);
                mv[1] = add_mod(mv[1], y.y);
            }
            if (rc) {
                const ulonglong2 z = *reinterpret_cast<const ulonglong2*>(rc + base + i0);
                mv[0] = sub_mod(mv[0], z.x);
                mv[1] = sub_mod(mv[1], z.y);
            }
            if (mv_out) {
                if (valid[0]) mv_out[base + i0] = mv[0];
                if (valid[1]) mv_out[base + i0 + 1] = mv[1];
            }
        }
        int64_t sc[2];
        uint32_t id[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            sc[h] = to_signed(mv[h]);
            id[h] = valid[h] ? (ids ? ids[i0 + h] : (uint32_t)(i0 + h)) : 0;
        }
        const int64_t ts = buf.thr_s;
        const uint32_t ti = buf.thr_i;
        const int ht = buf.have_thr;
        topk_offer(buf, valid[0], sc[0], id[0], ts, ti, ht);
        topk_offer(buf, valid[1], sc[1], id[1], ts, ti, ht);
        if (topk_full(buf, CAND_CAP - 2 * DT_THREADS)) topk_compact(buf, (int)k);
    }
    topk_compact(buf, (int)k);
    const int keep = min(buf.cnt, (int)k);
    const uint64_t slot = (uint64_t)q * gridDim.x + blockIdx.x;
    for (int i = threadIdx.x; i < keep; i += blockDim.x) {
        cand_s[slot * k + i] = buf.s[i];
        cand_i[slot * k + i] = buf.id[i];
    }
    if (threadIdx.x == 0) cand_n[slot] = (uint32_t)keep;
}

// ------------------------------------------------------------------ keygen GEMM
constexpr int GT = 64;   // output tile
constexpr int GK = 16;   // K chunk

__global__ void __launch_bounds__(256)
gemm_abt_kernel(const uint64_t* __restrict__ A, const uint64_t* __restrict__ B, const uint64_t* __restrict__ D,
                uint64_t rows, uint32_t cols, uint32_t K, uint64_t* __restrict__ C) {
    __shared__ uint64_t As[GT][GK + 1];
    __shared__ uint32_t Bs[GK][GT][6];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const uint64_t row0 = (uint64_t)blockIdx.x * GT;
    const uint32_t col0 = blockIdx.y * GT;
    uint64_t acc[4][4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = acc[a][b][2] = 0;
    for (uint32_t kk = 0; kk < K; kk += GK) {
        for (int e = threadIdx.x; e < GT * GK; e += 256) {
            const int rr = e / GK, k = e % GK;
            const uint64_t gr = row0 + rr;
            As[rr][k] = gr < rows ? A[gr * K + kk + k] : 0;
            const uint32_t gc = col0 + rr;
            const uint64_t bv = gc < cols ? B[(uint64_t)gc * K + kk + k] : 0;
            Limbs3 lb = limbs(bv), lc = limbs_hi(bv);
            Bs[k][rr][0] = lb.b0; Bs[k][rr][1] = lb.b1; Bs[k][rr][2] = lb.b2;
            Bs[k][rr][3] = lc.b0; Bs[k][rr][4] = lc.b1; Bs[k][rr][5] = lc.b2;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < GK; ++k) {
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const uint64_t m = As[ty + 16 * a][k];
                const uint32_t lo = (uint32_t)m, hi = (uint32_t)(m >> 32);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const uint32_t* l = Bs[k][tx + 16 * b];
                    acc[a][b][0] = mac(mac(acc[a][b][0], lo, l[0]), hi, l[3]);
                    acc[a][b][1] = mac(mac(acc[a][b][1], lo, l[1]), hi, l[4]);
                    acc[a][b][2] = mac(mac(acc[a][b][2], lo, l[2]), hi, l[5]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const uint64_t gr = row0 + ty + 16 * a;
            const uint32_t gc = col0 + tx + 16 * b;
            if (gr < rows && gc < cols) {
                uint64_t v = combine3(acc[a][b][0], acc[a][b][1], acc[a][b][2]);
                if (D) v = add_mod(v, D[gr * cols + gc]);
                C[gr * cols + gc] = v;
            }
        }
}

__global__ void apply_sparse_kernel(const uint64_t* __restrict__ rowptr, const uint32_t* __restrict__ idx,
                                    const int8_t* __restrict__ sign, uint64_t rows, uint32_t cols,
                                    uint64_t* __restrict__ C) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * blockDim.x)
        for (uint64_t c = rowptr[i]; c < rowptr[i + 1]; ++c) {
            uint64_t* p = C + i * cols + idx[c];
            *p = sign[c] > 0 ? add_mod(*p, 1) : sub_mod(*p, 1);
        }
}

__global__ void transpose_u64_kernel(const uint64_t* __restrict__ in, uint64_t rows, uint32_t cols,
                                     uint64_t* __restrict__ out, uint64_t out_ld) {
    __shared__ uint64_t t[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.x * 32;
    const uint32_t c0 = blockIdx.y * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const uint64_t r = r0 + yy;
        const uint32_t c = c0 + threadIdx.x;
        t[yy][threadIdx.x] = (r < rows && c < cols) ? in[r * cols + c] : 0;
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const uint32_t c = c0 + yy;
        const uint64_t r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[(uint64_t)c * out_ld + r] = t[threadIdx.x][yy];
    }
}

__global__ void csr_to_ell_kernel(const uint64_t* __restrict__ rowptr, const uint32_t* __restrict__ idx,
                                  const int8_t* __restrict__ sign, uint64_t rows, const uint32_t* __restrict__ s_off,
                                  const uint16_t* __restrict__ s_w, uint16_t* __restrict__ ell) {
    // every row position of every slice is written: the positions past the
    // last row of the last slice hold padding
    const uint64_t rows32 = (rows + 31) & ~31ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows32; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t slice = i >> 5;
        const uint32_t sl = (uint32_t)(i & 31), off = s_off[slice], w = s_w[slice];
        const uint64_t b = i < rows ? rowptr[i] : 0, e = i < rows ? rowptr[i + 1] : 0;
        for (uint32_t c = 0; c < w; ++c) {
            uint16_t v = (uint16_t)ELL_PAD;
            if (b + c < e) v = (uint16_t)(idx[b + c] + (sign[b + c] < 0 ? ELL_NEG : 0u));
            ell[off + (uint64_t)c * 32 + sl] = v;
        }
    }
}

inline unsigned grid_for(uint64_t n, unsigned threads, unsigned cap = 65535u * 16u) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

}  // namespace

// ------------------------------------------------------------------ launchers
void launch_query_limbs(const uint64_t* d_v, uint32_t nq, QLimb* d_limbs, cudaStream_t s) {
    const uint64_t total = (uint64_t)nq * N;
    query_limbs_kernel<<<grid_for(total, 256), 256, 0, s>>>(d_v, total, d_limbs);
}

void launch_scan(const uint64_t* d_m_enc, const QLimb* d_limbs, const ScanSeg* d_segs, const uint64_t* d_seg_blk,
                 uint32_t nseg, uint64_t total_blocks, uint64_t* d_r, int num_sms, uint32_t* d_err, cudaStream_t s,
                 long long wait_cycles) {
    if (total_blocks == 0) return;
    const int smem = TS_STAGES * TS_STAGE_BYTES;
    cudaFuncSetAttribute(scan_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);  // per device
    unsigned grid = (unsigned)(total_blocks < (uint64_t)num_sms ? total_blocks : (uint64_t)num_sms);
    scan_tma_kernel<<<grid, TS_THREADS, smem, s>>>(d_m_enc, d_limbs, d_segs, d_seg_blk, nseg, total_blocks, d_r, d_err,
                                                   wait_cycles > 0 ? wait_cycles : WAIT_CYCLES);
}

FreivaldsPlan plan_freivalds(uint64_t max_rows, uint32_t nseg, int num_sms) {
    // aim for ~2 waves of 4-column-block CTAs over all segments
    uint64_t target_ctas = (uint64_t)num_sms * 4;
    uint64_t per_seg = target_ctas / (4ull * (nseg ? nseg : 1));
    if (per_seg < 1) per_seg = 1;
    uint64_t chunk_rows = (max_rows + per_seg - 1) / per_seg;
    chunk_rows = ((chunk_rows + FV_TILE - 1) / FV_TILE) * FV_TILE;
    if (chunk_rows < FV_TILE) chunk_rows = FV_TILE;
    uint64_t chunks = (max_rows + chunk_rows - 1) / chunk_rows;
    if (chunks < 1) chunks = 1;
    return FreivaldsPlan{(uint32_t)chunks, (uint32_t)chunk_rows};
}

void launch_or_flag(uint32_t* d_word, uint32_t bits, cudaStream_t s) { or_flag_kernel<<<1, 1, 0, s>>>(d_word, bits); }

cudaError_t preload_freivalds_kernels() {
    cudaFuncAttributes a;
    const void* fns[] = {reinterpret_cast<const void*>(freivalds_kernel<24>),
                         reinterpret_cast<const void*>(freivalds_kernel<8>),
                         reinterpret_cast<const void*>(freivalds_kernel<4>),
                         reinterpret_cast<const void*>(freivalds_finish_kernel),
                         reinterpret_cast<const void*>(or_flag_kernel)};
    for (const void* f : fns) {
        const cudaError_t e = cudaFuncGetAttributes(&a, f);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void launch_freivalds(const uint64_t* d_m_enc, const uint64_t* d_r, const VerifySeg* d_vsegs, uint32_t nseg,
                      const ChaChaKey* d_keys, uint32_t trials, FreivaldsPlan plan, uint64_t* d_z_part,
                      uint64_t* d_ur_part, uint32_t* d_flags, cudaStream_t s) {
    for (uint32_t s0 = 0; s0 < nseg; s0 += 65535u) {
        const uint32_t ns = nseg - s0 < 65535u ? nseg - s0 : 65535u;
        dim3 grid(N / FV_THREADS, plan.chunks, ns);
        for (uint32_t t0 = 0; t0 < trials;) {
            const uint32_t left = trials - t0;
            if (left > 8) {
                const uint32_t c = left < 24 ? left : 24;
                freivalds_kernel<24><<<grid, FV_THREADS, 0, s>>>(d_m_enc, d_r, d_vsegs, d_keys, t0, c, trials, plan.chunks,
                                                                 plan.chunk_rows, d_z_part, d_ur_part, d_flags, s0);
                t0 += c;
            } else if (left > 4) {
                freivalds_kernel<8><<<grid, FV_THREADS, 0, s>>>(d_m_enc, d_r, d_vsegs, d_keys, t0, left, trials,
                                                                plan.chunks, plan.chunk_rows, d_z_part, d_ur_part, d_flags, s0);
                t0 += left;
            } else {
                freivalds_kernel<4><<<grid, FV_THREADS, 0, s>>>(d_m_enc, d_r, d_vsegs, d_keys, t0, left, trials,
                                                                plan.chunks, plan.chunk_rows, d_z_part, d_ur_part, d_flags, s0);
                t0 += left;
            }
        }
    }
}

void launch_freivalds_finish(const uint64_t* d_z_part, const uint64_t* d_ur_part, const uint64_t* d_v_enc,
                             const VerifySeg* d_vsegs, uint32_t nseg, uint32_t trials, FreivaldsPlan plan,
                             uint64_t* d_ur, uint64_t* d_zv, int32_t* d_failed, cudaStream_t s) {
    freivalds_finish_kernel<<<nseg, 256, 0, s>>>(d_z_part, d_ur_part, d_v_enc, d_vsegs, trials, plan.chunks, d_ur, d_zv,
                                                 d_failed);
}

void launch_lt_times_v(const uint64_t* d_L, uint32_t n1, const uint64_t* d_v, uint32_t nq, uint64_t* d_x,
                       cudaStream_t s) {
    lt_times_v_kernel<<<dim3(nq, LT_SPLIT), (1024 / n1) * n1, 0, s>>>(d_L, n1, d_v, d_x);
}

void launch_dense_terms(const uint64_t* d_al_cm, const uint64_t* d_h_cm, uint64_t rows, uint32_t n1,
                        const uint64_t* d_g, const uint64_t* d_x, uint64_t* d_out, cudaStream_t s) {
    dense_terms_kernel<<<grid_for(rows, 256, 148 * 8), 256, 0, s>>>(d_al_cm, d_h_cm, rows, n1, d_g, d_x, d_out);
}

void launch_decode_layout(const uint64_t* d_al_cm, const uint64_t* d_h_cm, const uint64_t* d_mp_cm, uint64_t rows,
                          uint32_t n1, uint64_t* d_alh_b, int8_t* d_m8_cm, uint32_t* d_bad, cudaStream_t s) {
    cudaMemsetAsync(d_bad, 0, 4, s);
    if (!rows) return;
    decode_layout_kernel<<<148 * 16, 256, 0, s>>>(d_al_cm, d_h_cm, d_mp_cm, rows, n1, d_alh_b, d_m8_cm, d_bad);
}

void launch_decode_topk(const uint64_t* d_r, const DecodeCorpus& dc, const ScanSeg* d_segs, const uint64_t* d_seg_unit,
                        const DecodeQuery* d_q, uint32_t nq, const uint64_t* d_v, const uint64_t* d_g, const uint64_t* d_x, const uint32_t* d_t,
                        const uint32_t* d_t_nnz, uint32_t k, uint32_t total_ctas, TopkScratch scratch,
                        uint64_t* d_mv_out, uint32_t* d_out_ids, int64_t* d_out_scores, uint32_t* d_out_n,
                        cudaStream_t s) {
    if (!nq) return;
    cudaMemsetAsync(scratch.done, 0, (uint64_t)nq * 4, s);
    const unsigned dyn = 2 * 2 * dc.n1 * 16;
    if (k >= 1 && k <= (uint32_t)WARP_TOPK_MAX) {  // every warp keeps its own list
        cudaFuncSetAttribute(decode_topk_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 2 * 512 * 16);
        decode_topk_kernel<true><<<total_ctas, DT_THREADS, dyn, s>>>(d_r, dc, d_segs, d_seg_unit, d_q, d_v, d_g, d_x,
                                                                     d_t, d_t_nnz, k, scratch, d_mv_out, d_out_ids,
                                                                     d_out_scores, d_out_n, nq);
    } else {
        cudaFuncSetAttribute(decode_topk_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 2 * 512 * 16);
        decode_topk_kernel<false><<<total_ctas, DT_THREADS, dyn, s>>>(d_r, dc, d_segs, d_seg_unit, d_q, d_v, d_g, d_x,
                                                                      d_t, d_t_nnz, k, scratch, d_mv_out, d_out_ids,
                                                                      d_out_scores, d_out_n, nq);
    }
}

void launch_topk_rows(const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_c, uint64_t ld, uint64_t rows,
                      uint32_t nq, const uint32_t* d_ids, uint32_t k, int ctas_per_query, TopkScratch scratch,
                      uint32_t* d_out_ids, int64_t* d_out_scores, uint32_t* d_out_n, uint64_t* d_mv_out,
                      cudaStream_t s) {
    if (!nq) return;
    topk_rows_kernel<<<dim3(ctas_per_query, nq), DT_THREADS, 0, s>>>(d_a, d_b, d_c, ld, rows, nullptr, d_ids, k,
                                                                   scratch.cand_s, scratch.cand_i, scratch.cand_n,
                                                                   d_mv_out);
    topk_merge_kernel<<<nq, DT_THREADS, 0, s>>>(scratch.cand_s, scratch.cand_i, scratch.cand_n, ctas_per_query, k,
                                                d_out_ids, d_out_scores, d_out_n);
}

void launch_topk_segs(const uint64_t* d_a, const uint64_t* d_b, const uint64_t* d_c, const uint64_t* d_qoff,
                      uint32_t nq, const uint32_t* d_ids, uint32_t k, int ctas_per_query, TopkScratch scratch,
                      uint32_t* d_out_ids, int64_t* d_out_scores, uint32_t* d_out_n, cudaStream_t s) {
    if (!nq) return;
    topk_rows_kernel<<<dim3(ctas_per_query, nq), DT_THREADS, 0, s>>>(d_a, d_b, d_c, 0, 0, d_qoff, d_ids, k,
                                                                   scratch.cand_s, scratch.cand_i, scratch.cand_n,
                                                                   nullptr);
    topk_merge_kernel<<<nq, DT_THREADS, 0, s>>>(scratch.cand_s, scratch.cand_i, scratch.cand_n, ctas_per_query, k,
                                                d_out_ids, d_out_scores, d_out_n);
}

void launch_gemm_abt(const uint64_t* d_A, const uint64_t* d_B, const uint64_t* d_D, uint64_t rows, uint32_t cols,
                     uint32_t K, uint64_t* d_C, cudaStream_t s) {
    dim3 grid((unsigned)((rows + GT - 1) / GT), (cols + GT - 1) / GT);
    gemm_abt_kernel<<<grid, 256, 0, s>>>(d_A, d_B, d_D, rows, cols, K, d_C);
}

void launch_apply_sparse(const uint64_t* d_rowptr, const uint32_t* d_idx, const int8_t* d_sign, uint64_t rows,
                         uint32_t cols, uint64_t* d_C, cudaStream_t s) {
    apply_sparse_kernel<<<grid_for(rows, 256, 148 * 16), 256, 0, s>>>(d_rowptr, d_idx, d_sign, rows, cols, d_C);
}

void launch_transpose_u64(const uint64_t* d_in, uint64_t rows, uint32_t cols, uint64_t* d_out, uint64_t out_ld,
                          cudaStream_t s) {
    dim3 grid((unsigned)((rows + 31) / 32), (cols + 31) / 32);
    transpose_u64_kernel<<<grid, dim3(32, 8), 0, s>>>(d_in, rows, cols, d_out, out_ld);
}

void launch_csr_to_ell(const uint64_t* d_rowptr, const uint32_t* d_idx, const int8_t* d_sign, uint64_t rows,
                       const uint32_t* d_s_off, const uint16_t* d_s_w, uint16_t* d_s_ell, cudaStream_t s) {
    csr_to_ell_kernel<<<grid_for((rows + 31) & ~31ull, 256, 148 * 16), 256, 0, s>>>(d_rowptr, d_idx, d_sign, rows, d_s_off,
                                                                                   d_s_w, d_s_ell);
}

}  // namespace bn
