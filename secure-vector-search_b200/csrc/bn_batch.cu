// bn_batch.cu -- tensor-core block scoring: the byte-planar u8/s8 GEMM with
// F_p recombination epilogues, and the layout / operand builders around it.
//
// bgemm_kernel roles per CTA (one CTA per SM, persistent over work items;
// an item is 128 A rows x w_tile W rows x one K panel):
//   warp 0    TMA producer: per 128-byte K step, the A box (128 rows) and the
//             W box (w_tile rows) into a ring of shared-memory stages
//   warp 1    MMA issuer: 4 x tcgen05.mma (M=128, N=w_tile, K=32) per stage
//             into one of two TMEM accumulators (double-buffered across
//             items), tcgen05.commit frees the stage / hands over the item
//   warps 2-9 epilogue: tcgen05.ld, byte-weight recombination mod p, stores
// Every mbarrier wait is bounded; on timeout the CTA sets *err and winds down
// (waits for its own copies and MMAs, frees TMEM) instead of hanging.
#include <cudaTypedefs.h>

#include <algorithm>

#include "bn_batch.cuh"
#include "bn_fp.cuh"
#include "bn_tcgen05.cuh"

namespace bn {

namespace {

using namespace tcg;

constexpr int BG_EPI_WARPS = 8;
constexpr int BG_THREADS = 64 + 32 * BG_EPI_WARPS;  // TMA warp, MMA warp, epilogue warps

// A work item: K panel, TMA rows of the A and W tiles, and the output range.
struct ItemIdx {
    uint32_t kp, tw;  // tw: W tile (A-resident mode reloads A when it wraps to 0)
    uint32_t a_y, w_y, x0, x_lim, y0, y_lim;
};
__device__ __forceinline__ ItemIdx grid_item(const BgParams& p, uint32_t kp, uint32_t ta, uint32_t tw) {
    const uint32_t x0 = p.mode == BG_S8 ? ta * BG_AROWS : ta * (BG_AROWS / 8);
    return ItemIdx{kp, tw, p.a_blocked ? ta : ta * BG_AROWS, tw * p.w_tile, x0, p.x_count, tw * p.w_tile / 8, p.y_count};
}
__device__ __forceinline__ ItemIdx item_idx(const BgParams& p, uint32_t item) {
    const uint32_t per = p.a_tiles * p.w_tiles;
    const uint32_t kp = item / per, rem = item % per;
    if (p.order_a_fast) return grid_item(p, kp, rem % p.a_tiles, rem / p.a_tiles);
    return grid_item(p, kp, rem / p.w_tiles, rem % p.w_tiles);
}

// The j-th work item of this CTA.  Streaming mode: global items blockIdx.x +
// j * gridDim.x.  A-resident mode: this CTA owns A tiles blockIdx.x + t *
// gridDim.x and visits every W tile of each (j = t * w_tiles + tw).
__device__ __forceinline__ bool item_at(const BgParams& p, uint32_t items, uint32_t j, ItemIdx& ix) {
    if (p.item_tab) {
        const uint32_t item = blockIdx.x + j * gridDim.x;
        if (item >= p.n_items) return false;
        const BgItem t = p.item_tab[item];
        ix = ItemIdx{0, 1, t.a_y, t.w_y, t.x0, t.x_lim, t.y0, t.y_lim};
        return true;
    }
    if (p.a_resident) {
        const uint32_t ta = blockIdx.x + (j / p.w_tiles) * gridDim.x;
        if (ta >= p.a_tiles) return false;
        ix = grid_item(p, 0, ta, j % p.w_tiles);
        return true;
    }
    const uint32_t item = blockIdx.x + j * gridDim.x;
    if (item >= items) return false;
    ix = item_idx(p, item);
    return true;
}

// This CTA's items in order, the next item's entry fetched one item ahead (in
// grouped mode an item-table load, whose latency then overlaps the current item).
struct ItemCursor {
    const BgParams& p;
    uint32_t items, j = 0;
    ItemIdx cur, nxt;
    bool have_cur, have_nxt;
    __device__ __forceinline__ ItemCursor(const BgParams& p_, uint32_t items_) : p(p_), items(items_) {
        have_cur = item_at(p, items, 0, cur);
        have_nxt = have_cur && item_at(p, items, 1, nxt);
    }
    __device__ __forceinline__ void advance() {
        ++j;
        cur = nxt;
        have_cur = have_nxt;
        if (have_cur) have_nxt = item_at(p, items, j + 1, nxt);
    }
};

__global__ void __launch_bounds__(BG_THREADS, 1)
bgemm_kernel(const __grid_constant__ CUtensorMap tmap_a, const __grid_constant__ CUtensorMap tmap_w,
             const __grid_constant__ CUtensorMap tmap_a2, const __grid_constant__ CUtensorMap tmap_w2, const BgParams p,
             uint32_t stages, uint32_t stage_bytes, uint32_t* __restrict__ err) {
    extern __shared__ uint8_t bg_dyn[];
    __shared__ uint64_t full_b[BG_MAX_STAGES], empty_b[BG_MAX_STAGES], accf_b[2], acce_b[2], done_b;
    __shared__ uint64_t afull_b[BG_MAX_ASLOTS], aempty_b[BG_MAX_ASLOTS];  // A-resident slots
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    // 1024-byte aligned (128-byte swizzle atoms): [A slots (A-resident)] [stage ring]
    const uint32_t sbase = (su32(bg_dyn) + 1023u) & ~1023u;
    uint8_t* sptr = bg_dyn + (sbase - su32(bg_dyn));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long wait_limit = p.wait_cycles > 0 ? p.wait_cycles : TC_WAIT_CYCLES;
    constexpr uint32_t A_BYTES = BG_AROWS * BG_KSTEP;
    const uint32_t w_bytes = p.w_tile * BG_KSTEP;
    const uint32_t ksub = p.ksteps2 ? 2u : 1u, kstage = ksub * BG_KSTEP;  // K steps / bytes per stage
    const uint32_t kpanels = (p.k_bytes + p.k_panel - 1) / p.k_panel;
    const uint32_t items = p.item_tab ? p.n_items : kpanels * p.a_tiles * p.w_tiles;
    const uint32_t a_slots = p.a_resident ? p.k_bytes / BG_KSTEP : 0;
    const uint32_t base = sbase + a_slots * A_BYTES;  // stage ring
    uint8_t* ring = sptr + a_slots * A_BYTES;
    // TMA coordinates of A's K step at byte k: row-major (x = k, y = row), or
    // K-blocked (x = 0, y = (tile * K steps + k / 128) * 128)
    const uint32_t a_ksteps = p.k_bytes / BG_KSTEP;
    auto a_x = [&](uint32_t k) -> int { return p.a_blocked ? 0 : (int)k; };
    auto a_row = [&](const ItemIdx& ix, uint32_t k) -> int {
        return p.a_blocked ? (int)((ix.a_y * a_ksteps + k / BG_KSTEP) * BG_AROWS) : (int)ix.a_y;
    };

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            bar_init(&full_b[s], 1);
            bar_init(&empty_b[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            bar_init(&accf_b[b], 1);
            bar_init(&acce_b[b], BG_EPI_WARPS);
        }
        for (uint32_t k = 0; k < a_slots; ++k) {
            bar_init(&afull_b[k], 1);
            bar_init(&aempty_b[k], 1);
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
        if (lane == 0) {  // ---------------------------------------------- TMA producer
            // stage ring: A + W boxes per K step (streaming) or W boxes only
            // (A-resident: the A tile's K slices stay in their slots for all
            // W tiles of the tile and are reloaded for the next one once the
            // MMAs of its last item have read them)
            uint64_t it = 0;
            // A loads issued last: slots [0, a_n) for tile a_t, the rest for a_t - 1
            uint32_t a_t = 0xffffffffu, a_n = 0;
            bool stop = false;
            for (ItemCursor cs(p, items); !stop && cs.have_cur; cs.advance()) {
                const ItemIdx& ix = cs.cur;
                const uint32_t j = cs.j;
                const uint32_t t = a_slots ? j / p.w_tiles : 0;
                const bool load_a = a_slots && ix.tw == 0;
                const uint32_t k0 = ix.kp * p.k_panel, k1 = min(p.k_bytes, k0 + p.k_panel);
                for (uint32_t k = k0; k < k1; k += kstage, ++it) {
                    const uint32_t ks = (k - k0) / BG_KSTEP;
                    if (load_a) {
                        for (uint32_t sub = 0; sub < ksub && !stop; ++sub) {
                            if (t > 0 && !bar_wait(&aempty_b[ks + sub], (t - 1) & 1, wait_limit)) {
                                abort_s = 1;
                                atomicOr(err, 4u);
                                stop = true;
                                break;
                            }
                            const uint32_t kq = k + sub * BG_KSTEP;
                            bar_expect_tx(&afull_b[ks + sub], A_BYTES);
                            tma_2d(sptr + (ks + sub) * A_BYTES, &tmap_a, a_x(kq), a_row(ix, kq), &afull_b[ks + sub]);
                            a_t = t;
                            a_n = ks + sub + 1;
                        }
                        if (stop) break;
                    }
                    const uint32_t st = (uint32_t)(it % stages);
                    if (it >= stages && !bar_wait(&empty_b[st], (uint32_t)(((it / stages) - 1) & 1), wait_limit)) {
                        abort_s = 1;
                        atomicOr(err, 4u);
                        stop = true;
                        break;
                    }
                    if (abort_s) { stop = true; break; }
                    uint8_t* sb = ring + (uint64_t)st * stage_bytes;
                    if (a_slots && ksub == 2) {  // [W step k | W step k+1]
                        bar_expect_tx(&full_b[st], 2 * w_bytes);
                        tma_3d(sb, &tmap_w2, 0, (int)ix.w_y, (int)(k / BG_KSTEP), &full_b[st]);
                    } else if (a_slots) {
                        bar_expect_tx(&full_b[st], w_bytes);
                        tma_2d(sb, &tmap_w, (int)k, (int)ix.w_y, &full_b[st]);
                    } else if (ksub == 2) {  // [A step k | A step k+1 | W step k | W step k+1]
                        bar_expect_tx(&full_b[st], 2 * (A_BYTES + w_bytes));
                        tma_2d(sb, &tmap_a2, 0, a_row(ix, k), &full_b[st]);
                        tma_3d(sb + 2 * A_BYTES, &tmap_w2, 0, (int)ix.w_y, (int)(k / BG_KSTEP), &full_b[st]);
                    } else {
                        bar_expect_tx(&full_b[st], A_BYTES + w_bytes);
                        tma_2d(sb, &tmap_a, a_x(k), a_row(ix, k), &full_b[st]);
                        tma_2d(sb + A_BYTES, &tmap_w, (int)k, (int)ix.w_y, &full_b[st]);
                    }
                }
            }
            // no copy may still be landing in shared memory when the CTA exits
            for (uint64_t j = it > stages ? it - stages : 0; j < it; ++j)
                bar_wait(&full_b[j % stages], (uint32_t)((j / stages) & 1));
            if (a_t != 0xffffffffu)
                for (uint32_t k = 0; k < a_slots; ++k) {
                    const uint32_t tk = k < a_n ? a_t : a_t - 1;  // the last tile slot k was loaded for
                    if (k < a_n || a_t > 0) bar_wait(&afull_b[k], tk & 1);
                }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // ---------------------------------------------- MMA issuer
            const uint32_t sgn = p.mode == BG_S8 ? 1u : 0u;
            const uint32_t idesc = (2u << 4) | (sgn << 7) | (sgn << 10) | ((p.w_tile >> 3) << 17) |
                                   ((uint32_t)(BG_AROWS >> 4) << 24);
            uint64_t it = 0;
            bool stop = false;
            for (ItemCursor cs(p, items); !stop && cs.have_cur; cs.advance()) {
                const ItemIdx& ix = cs.cur;
                const uint32_t j = cs.j;
                const uint64_t n = j;
                const uint32_t t = a_slots ? j / p.w_tiles : 0;
                const bool last_of_a = a_slots && ix.tw == p.w_tiles - 1;
                const uint32_t buf = (uint32_t)(n & 1), use = (uint32_t)(n >> 1);
                if (use > 0 && !bar_wait(&acce_b[buf], (use - 1) & 1, wait_limit)) {
                    abort_s = 1;
                    atomicOr(err, 8u);
                    break;
                }
                tc_after();
                const uint32_t d = tmem + buf * 256u;
                const uint32_t k0 = ix.kp * p.k_panel, k1 = min(p.k_bytes, k0 + p.k_panel);
                bool first = true;
                for (uint32_t k = k0; k < k1; k += kstage, ++it) {
                    const uint32_t st = (uint32_t)(it % stages);
                    const uint32_t ks = (k - k0) / BG_KSTEP;
                    bool a_ok = true;
                    for (uint32_t sub = 0; a_slots && sub < ksub; ++sub) a_ok = a_ok && bar_wait(&afull_b[ks + sub], t & 1, wait_limit);
                    if (!a_ok || !bar_wait(&full_b[st], (uint32_t)((it / stages) & 1), wait_limit) || abort_s) {
                        abort_s = 1;
                        atomicOr(err, 8u);
                        stop = true;
                        break;
                    }
                    tc_after();
                    const uint32_t sa = a_slots ? sbase + ks * A_BYTES : base + st * stage_bytes;
                    const uint32_t sw = a_slots ? base + st * stage_bytes : sa + ksub * A_BYTES;
                    for (uint32_t sub = 0; sub < ksub; ++sub)
#pragma unroll
                        for (uint32_t kk = 0; kk < BG_KSTEP / 32; ++kk)
                            mma_i8(d, sdesc(sa + sub * A_BYTES + kk * 32u, 16, 1024),
                                   sdesc(sw + sub * w_bytes + kk * 32u, 16, 1024), idesc,
                                   (first && sub == 0 && kk == 0) ? 0u : 1u);
                    first = false;
                    mma_commit(&empty_b[st]);                // stage reusable once these MMAs have read it
                    if (last_of_a)
                        for (uint32_t sub = 0; sub < ksub; ++sub)
                            mma_commit(&aempty_b[ks + sub]);  // A slots reusable for the next A tile
                }
                if (stop) break;
                mma_commit(&accf_b[buf]);  // accumulator complete for this item
            }
            mma_commit(&done_b);
            if (!bar_wait(&done_b, 0)) atomicOr(err, 64u);  // every issued MMA has finished before TMEM is freed
        }
    } else {
        // -------------------------------------------------------------- epilogue
        // 8 warps: warp w reads TMEM lane quarter w % 4 and every other
        // 64-column chunk (half = (w - 2) / 4) of each item.
        const uint32_t q = (uint32_t)(warp & 3);
        const uint32_t half = (uint32_t)(warp - 2) >> 2;
        const uint32_t wide = p.w_tile & ~63u;  // columns handled in 64-column chunks
        for (ItemCursor cs(p, items); cs.have_cur; cs.advance()) {
            const ItemIdx& ix = cs.cur;
            const uint64_t n = cs.j;
            const uint32_t buf = (uint32_t)(n & 1), use = (uint32_t)(n >> 1);
            // output bases of the y this lane stores, loaded before the wait:
            // PLANAR lane (xi, a) stores y = chunk + a (wide chunks) and
            // chunk + {0, 1} (16-column chunks); S8 lanes share every y, so
            // lane l holds chunk + (l & 7) and the stores shuffle it out
            const uint32_t ybase = ix.y0;
            auto obase = [&](uint32_t y) -> uint64_t {
                return y < ix.y_lim ? (p.pair_base ? p.pair_base[y] : (uint64_t)y * p.out_ld) : 0;
            };
            const uint32_t ysel = lane & 7;  // PLANAR: a; S8: the y this lane holds for the shuffles
            uint64_t ob_w[2], ob_r[2][2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const uint32_t cw = 64 * half + 128 * k, cr = wide + 16 * half + 32 * k;
                ob_w[k] = cw < wide ? obase(ybase + cw / 8 + ysel) : 0;
#pragma unroll
                for (int h = 0; h < 2; ++h) ob_r[k][h] = cr < p.w_tile ? obase(ybase + cr / 8 + h) : 0;
            }
            const bool ok = __all_sync(FULLMASK, bar_wait(&accf_b[buf], use & 1, wait_limit));  // warp-uniform
            if (!ok && lane == 0) { abort_s = 1; atomicOr(err, 16u); }
            if (__any_sync(FULLMASK, !ok || abort_s)) break;
            tc_after();
            const uint32_t taddr = tmem + ((q * 32u) << 16) + buf * 256u;
            if (p.mode == BG_PLANAR) {
                const uint32_t a = lane & 7, xi = lane >> 3;
                const uint32_t x4 = ix.x0 + q * 4;  // first x of this warp
                const uint32_t x = x4 + xi;
                const uint32_t w1 = 8 * a;
                uint64_t* out = p.out + (uint64_t)ix.kp * p.out_pstride;
                for (uint32_t c0 = 64 * half, k = 0; c0 < wide; c0 += 128, ++k) {
                    uint32_t v[64];
                    tmem_ld64(taddr + c0, v);
                    uint64_t part[8];  // (lo + hi 2^32) 2^(8a) mod p for the chunk's 8 y
#pragma unroll
                    for (int yy = 0; yy < 8; ++yy) {
                        uint64_t lo = 0, hi = 0;
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            lo += (uint64_t)v[8 * yy + b] << (8 * b);
                            hi += (uint64_t)v[8 * yy + 4 + b] << (8 * b);
                        }
                        part[yy] = fold(rotl61(lo + rotl61(hi, 32), w1));  // < 2^61 + 8: 8 sum below 2^64
                    }
                    // butterfly over the 8 lanes of one x: each level halves the
                    // y values a lane carries; lane a ends with y = a
                    const bool b2 = (a & 4) != 0, b1 = (a & 2) != 0, b0 = (a & 1) != 0;
                    uint64_t k4[4], k2[2];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        k4[i] = (b2 ? part[i + 4] : part[i]) + __shfl_xor_sync(FULLMASK, b2 ? part[i] : part[i + 4], 4);
#pragma unroll
                    for (int i = 0; i < 2; ++i)
                        k2[i] = (b1 ? k4[i + 2] : k4[i]) + __shfl_xor_sync(FULLMASK, b1 ? k4[i] : k4[i + 2], 2);
                    const uint64_t f =
                        canon((b0 ? k2[1] : k2[0]) + __shfl_xor_sync(FULLMASK, b0 ? k2[0] : k2[1], 1));  // < 8p
                    const uint32_t y = ybase + c0 / 8 + a;
                    if (y < ix.y_lim && x < ix.x_lim) out[(k ? ob_w[1] : ob_w[0]) + x] = f;
                    if (p.planar_out) {
                        // 4 x 8 byte transpose across the lanes of one y: lane
                        // (xi, a) ends with planes 4(xi&1) + 2(xi>>1) + {0, 1}
                        // of f(x4..x4+3, y) as two 32-bit words
                        const bool e0 = (xi & 1) != 0, e1 = (xi & 2) != 0;
                        const uint32_t flo = (uint32_t)f, fhi = (uint32_t)(f >> 32);
                        const uint32_t keep1 = e0 ? fhi : flo;
                        const uint32_t recv1 = __shfl_xor_sync(FULLMASK, e0 ? flo : fhi, 8);
                        const uint32_t ev = e0 ? recv1 : keep1, od = e0 ? keep1 : recv1;
                        const uint32_t pa = __byte_perm(ev, od, 0x5140), pb = __byte_perm(ev, od, 0x7362);
                        const uint32_t keep2 = e1 ? pb : pa;
                        const uint32_t recv2 = __shfl_xor_sync(FULLMASK, e1 ? pa : pb, 16);
                        const uint32_t p0 = e1 ? recv2 : keep2, p1 = e1 ? keep2 : recv2;
                        if (y < ix.y_lim && x4 < ix.x_lim) {
                            const uint32_t plane = 4 * (xi & 1) + 2 * (xi >> 1);
                            uint8_t* dst = p.planar_out + ((uint64_t)y * 8 + plane) * p.planar_ld + x4;
                            *reinterpret_cast<uint32_t*>(dst) = __byte_perm(p0, p1, 0x5410);
                            *reinterpret_cast<uint32_t*>(dst + p.planar_ld) = __byte_perm(p0, p1, 0x7632);
                        }
                    }
                }
                // remaining columns (w_tile not a multiple of 64): 16 at a time
                for (uint32_t c0 = wide + 16 * half, k = 0; c0 < p.w_tile; c0 += 32, ++k) {
                    uint32_t v[16];
                    tmem_ld16(taddr + c0, v);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t y = ybase + c0 / 8 + h;
                        const uint64_t ob = k ? ob_r[1][h] : ob_r[0][h];
                        uint64_t lo = 0, hi = 0;
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            lo += (uint64_t)v[8 * h + b] << (8 * b);
                            hi += (uint64_t)v[8 * h + 4 + b] << (8 * b);
                        }
                        uint64_t f = fold(rotl61(lo + rotl61(hi, 32), w1));
                        f += __shfl_xor_sync(FULLMASK, f, 1);
                        f += __shfl_xor_sync(FULLMASK, f, 2);
                        f += __shfl_xor_sync(FULLMASK, f, 4);
                        f = canon(f);
                        uint32_t packed = (uint32_t)((f >> (8 * a)) & 0xffu) << (8 * xi);
                        packed |= __shfl_xor_sync(FULLMASK, packed, 8);
                        packed |= __shfl_xor_sync(FULLMASK, packed, 16);
                        if (y < ix.y_lim) {
                            if (a == 0 && x < ix.x_lim) out[ob + x] = f;
                            if (p.planar_out && lane < 8 && x4 < ix.x_lim)
                                *reinterpret_cast<uint32_t*>(p.planar_out + ((uint64_t)y * 8 + lane) * p.planar_ld +
                                                             x4) = packed;
                        }
                    }
                }
            } else {
                const uint32_t x = ix.x0 + q * 32 + lane;
                const bool xv = x < ix.x_lim;
                const uint64_t corr = xv ? p.corr[x] : 0;
                for (uint32_t c0 = 64 * half, k = 0; c0 < wide; c0 += 128, ++k) {
                    uint32_t v[64];
                    tmem_ld64(taddr + c0, v);
                    const uint64_t obk = k ? ob_w[1] : ob_w[0];
#pragma unroll
                    for (int yy = 0; yy < 8; ++yy) {
                        const uint64_t ob = __shfl_sync(FULLMASK, obk, yy);
                        int64_t lo = 0, hi = 0;
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            lo += (int64_t)(int32_t)v[8 * yy + b] * (int64_t)(1ll << (8 * b));
                            hi += (int64_t)(int32_t)v[8 * yy + 4 + b] * (int64_t)(1ll << (8 * b));
                        }
                        const uint64_t lr = lo < 0 ? (uint64_t)(lo + (int64_t)P) : (uint64_t)lo;
                        const uint64_t hr = hi < 0 ? (uint64_t)(hi + (int64_t)P) : (uint64_t)hi;
                        const uint32_t y = ybase + c0 / 8 + yy;
                        if (xv && y < ix.y_lim) p.out[ob + x] = add_mod(canon(lr + rotl61(hr, 32)), corr);
                    }
                }
                for (uint32_t c0 = wide + 16 * half, k = 0; c0 < p.w_tile; c0 += 32, ++k) {
                    uint32_t v[16];
                    tmem_ld16(taddr + c0, v);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint64_t ob = k ? ob_r[1][h] : ob_r[0][h];
                        int64_t lo = 0, hi = 0;
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            lo += (int64_t)(int32_t)v[8 * h + b] * (int64_t)(1ll << (8 * b));
                            hi += (int64_t)(int32_t)v[8 * h + 4 + b] * (int64_t)(1ll << (8 * b));
                        }
                        const uint64_t lr = lo < 0 ? (uint64_t)(lo + (int64_t)P) : (uint64_t)lo;
                        const uint64_t hr = hi < 0 ? (uint64_t)(hi + (int64_t)P) : (uint64_t)hi;
                        const uint32_t y = ybase + c0 / 8 + h;
                        if (xv && y < ix.y_lim) p.out[ob + x] = add_mod(canon(lr + rotl61(hr, 32)), corr);
                    }
                }
            }
            tc_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&acce_b[buf]);
        }
    }
    tc_before();
    __syncthreads();
    if (warp == 1) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// ------------------------------------------------------------------ layouts and operands
// Byte offset of byte column c of row pr in a K-blocked operand: tiles of 128
// rows, each stored as its ks K-steps of 128 rows x 128 bytes, so that every
// (tile, K-step) TMA box is one contiguous 16 KB run.
__device__ __forceinline__ uint64_t blk_off(uint64_t pr, uint32_t c, uint32_t ks) {
    return ((((pr >> 7) * ks + (c >> 7)) << 7) + (pr & 127)) * 128 + (c & 127);
}

// Byte planes of rows of src: row i's byte a lands in row (prow[i] or i) * 8 + a,
// row-major with dst_ld (ks = 0) or K-blocked with ks K-steps per tile.
__global__ void planar_rows_kernel(const uint64_t* __restrict__ src, uint64_t rows, uint32_t k, uint64_t src_ld,
                                   int negate, uint8_t* __restrict__ dst, uint64_t dst_ld, uint32_t col0,
                                   const uint32_t* __restrict__ prow, uint32_t ks) {
    const uint32_t chunks = k / 16;
    const uint64_t total = rows * chunks;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = e / chunks;
        const uint32_t jc = (uint32_t)(e % chunks);
        uint64_t x[16];
        const uint64_t* s = src + i * src_ld + jc * 16;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const uint64_t y = s[t];
            x[t] = negate ? (y == 0 ? 0 : P - y) : y;
        }
        const uint64_t pi = prow ? prow[i] : i;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
            for (int t = 0; t < 16; ++t) w[t >> 2] |= (uint32_t)((x[t] >> (8 * a)) & 0xffu) << (8 * (t & 3));
            uint8_t* d = ks ? dst + blk_off(pi * 8 + a, col0 + jc * 16, ks) : dst + (pi * 8 + a) * dst_ld + col0 + jc * 16;
            *reinterpret_cast<uint4*>(d) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

__global__ void planar_cm_kernel(const uint64_t* __restrict__ src_cm, uint64_t rows, uint32_t k,
                                 uint8_t* __restrict__ dst, uint64_t dst_ld, uint32_t col0,
                                 const uint32_t* __restrict__ prow, uint32_t ks) {
    const uint32_t chunks = k / 16;
    const uint64_t total = rows * chunks;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t jc = (uint32_t)(e / rows);
        const uint64_t i = e % rows;  // consecutive threads: consecutive rows (coalesced column reads)
        uint64_t x[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) x[t] = src_cm[(uint64_t)(jc * 16 + t) * rows + i];
        const uint64_t pi = prow ? prow[i] : i;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
            for (int t = 0; t < 16; ++t) w[t >> 2] |= (uint32_t)((x[t] >> (8 * a)) & 0xffu) << (8 * (t & 3));
            uint8_t* d = ks ? dst + blk_off(pi * 8 + a, col0 + jc * 16, ks) : dst + (pi * 8 + a) * dst_ld + col0 + jc * 16;
            *reinterpret_cast<uint4*>(d) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// [M | S] rows as signed bytes, K-blocked (16 K-steps of 128 bytes per
// 128-row tile), corpus row i at row prow[i] (or i).
__global__ void ms8_m_kernel(const uint64_t* __restrict__ mp_cm, uint64_t rows, int8_t* __restrict__ dst,
                             uint32_t* __restrict__ bad, const uint32_t* __restrict__ prow) {
    const uint32_t chunks = N / 16;
    const uint64_t total = rows * chunks;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t jc = (uint32_t)(e / rows);
        const uint64_t i = e % rows;
        uint32_t w[4] = {0, 0, 0, 0};
        bool out_of_range = false;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const int64_t sv = to_signed(mp_cm[(uint64_t)(jc * 16 + t) * rows + i]);
            out_of_range |= sv < -128 || sv > 127;
            w[t >> 2] |= (uint32_t)((uint8_t)(int8_t)sv) << (8 * (t & 3));
        }
        if (out_of_range) atomicOr(bad, 1u);
        *reinterpret_cast<uint4*>(dst + blk_off(prow ? prow[i] : i, jc * 16, 2 * N / 128)) =
            make_uint4(w[0], w[1], w[2], w[3]);
    }
}

__global__ void ms8_s_kernel(const uint16_t* __restrict__ s_ell, const uint32_t* __restrict__ s_off,
                             const uint16_t* __restrict__ s_w, uint64_t rows, int8_t* __restrict__ dst,
                             uint64_t* __restrict__ corr, uint32_t* __restrict__ bad, const uint32_t* __restrict__ prow) {
    const uint64_t c_mod = canon(0x0101010101010101ull);  // sum_b 2^(8b)
    constexpr uint32_t KS = 2 * N / 128;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pi = prow ? prow[i] : i;
        for (uint32_t c = 0; c < N / 16; ++c)
            *reinterpret_cast<uint4*>(dst + blk_off(pi, N + 16 * c, KS)) = make_uint4(0, 0, 0, 0);
        const uint64_t slice = i >> 5;
        const uint32_t sl = (uint32_t)(i & 31), off = s_off[slice], wdt = s_w[slice];
        int rs = 0;
        for (uint32_t cc = 0; cc < wdt; ++cc) {
            const uint16_t f = s_ell[off + (uint64_t)cc * 32 + sl];
            if (f == ELL_PAD) continue;
            const int sgn = f >= ELL_NEG ? -1 : 1;
            int8_t* e = dst + blk_off(pi, N + (f >= ELL_NEG ? f - ELL_NEG : f), KS);
            const int nv = (int)*e + sgn;
            if (nv < -128 || nv > 127) atomicOr(bad, 1u);
            *e = (int8_t)nv;
            rs += sgn;
        }
        const uint64_t m = mul_mod((uint64_t)(128 * (rs < 0 ? -rs : rs)), c_mod);
        corr[i] = rs < 0 ? (m ? P - m : 0) : m;
    }
}

__global__ void w_tv_kernel(const uint64_t* __restrict__ v, uint32_t nq, int8_t* __restrict__ dst) {
    const uint32_t chunks = N / 16;
    const uint64_t total = (uint64_t)nq * 8 * chunks;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t qb = e / chunks;
        const uint32_t jc = (uint32_t)(e % chunks);
        const uint32_t q = (uint32_t)(qb >> 3), b = (uint32_t)(qb & 7);
        int8_t* row = dst + qb * (2 * N);
        reinterpret_cast<uint4*>(row)[jc] = make_uint4(0, 0, 0, 0);  // T part (b = 0 filled below)
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const int byte = (int)((v[(uint64_t)q * N + jc * 16 + t] >> (8 * b)) & 0xffu) - 128;
            w[t >> 2] |= (uint32_t)((uint8_t)(int8_t)byte) << (8 * (t & 3));
        }
        reinterpret_cast<uint4*>(row + N)[jc] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// T part of row (q, b = 0): column sums of query q's +-1 entries, one CTA per
// query (shared-memory counters, so repeated columns add up).
__global__ void __launch_bounds__(256) w_t_kernel(const uint32_t* __restrict__ t_ent, const uint32_t* __restrict__ t_nnz,
                                                  int8_t* __restrict__ dst, uint32_t* __restrict__ bad) {
    const uint32_t q = blockIdx.x;
    __shared__ int acc[N];
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) acc[i] = 0;
    __syncthreads();
    const uint32_t tn = min(t_nnz[q], (uint32_t)N);
    for (uint32_t c = threadIdx.x; c < tn; c += blockDim.x) {
        const uint32_t e = t_ent[(uint64_t)q * N + c];
        atomicAdd(&acc[e & 0x3ffu], (e >> 31) ? -1 : 1);
    }
    __syncthreads();
    int8_t* row = dst + (uint64_t)q * 8 * (2 * N);  // row (q, b = 0)
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        const int v = acc[i];
        if (v < -128 || v > 127) atomicOr(bad, 2u);
        row[i] = (int8_t)v;
    }
}

__global__ void zsum_kernel(const uint64_t* __restrict__ z_part, uint32_t npanels, uint32_t t_base,
                            uint32_t trials_total, uint64_t* __restrict__ z) {
    const uint32_t t = t_base + blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    uint64_t acc = 0;
    for (uint32_t pn = 0; pn < npanels; ++pn) acc = add_mod(acc, z_part[((uint64_t)pn * trials_total + t) * N + j]);
    z[(uint64_t)t * N + j] = acc;
}

__global__ void __launch_bounds__(128) zv_kernel(const uint64_t* __restrict__ z, const uint64_t* __restrict__ v,
                                                 uint32_t nq, uint64_t* __restrict__ zv) {
    const uint32_t q = blockIdx.x, t = blockIdx.y;
    __shared__ uint64_t sh[4];
    uint64_t acc = 0;
    for (uint32_t j = threadIdx.x; j < N; j += blockDim.x)
        acc = add_mod(acc, mul_mod(z[(uint64_t)t * N + j], v[(uint64_t)q * N + j]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc = add_mod(acc, __shfl_xor_sync(0xffffffffu, acc, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) zv[(uint64_t)t * nq + q] = add_mod(add_mod(sh[0], sh[1]), add_mod(sh[2], sh[3]));
}

__global__ void ur_decide_kernel(const uint64_t* __restrict__ ur_part, uint32_t kpanels, uint32_t trials, uint32_t nq,
                                 const uint64_t* __restrict__ zv, uint64_t* __restrict__ ur, int32_t* __restrict__ failed) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    int32_t f = -1;
    for (uint32_t t = 0; t < trials; ++t) {
        uint64_t acc = 0;
        for (uint32_t kp = 0; kp < kpanels; ++kp) acc = add_mod(acc, ur_part[((uint64_t)kp * trials + t) * nq + q]);
        if (ur) ur[(uint64_t)t * nq + q] = acc;
        if (f < 0 && acc != zv[(uint64_t)t * nq + q]) f = (int32_t)t;
    }
    failed[q] = f;
}

unsigned grid_for(uint64_t work, unsigned threads, unsigned cap) {
    const uint64_t g = (work + threads - 1) / threads;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

uint32_t bgemm_stage_bytes(uint32_t w_tile, bool a_resident, uint32_t ksub) {
    return ksub * ((a_resident ? 0u : (uint32_t)(BG_AROWS * BG_KSTEP)) + ((w_tile * BG_KSTEP + 1023u) & ~1023u));
}

uint32_t bgemm_smem_bytes(const BgParams& p, uint32_t stages) {
    const uint32_t a = p.a_resident ? (p.k_bytes / BG_KSTEP) * BG_AROWS * BG_KSTEP : 0u;
    return a + stages * bgemm_stage_bytes(p.w_tile, p.a_resident != 0, p.ksteps2 ? 2u : 1u) + 1024u;
}

uint32_t bgemm_max_stages(const BgParams& p) {
    for (uint32_t st = BG_MAX_STAGES; st >= 2; --st)
        if (bgemm_smem_bytes(p, st) + 1024 <= BG_MAX_SMEM) return st;
    return 0;
}

void launch_bgemm(const CUtensorMap& tmap_a, const CUtensorMap& tmap_w, const BgParams& p, uint32_t stages, int ctas,
                  uint32_t* d_err, cudaStream_t s, const CUtensorMap* tmap_a2, const CUtensorMap* tmap_w2) {
    if (p.ksteps2 && (p.k_panel % (2 * BG_KSTEP) || !tmap_w2 || (!p.a_resident && (!p.a_blocked || !tmap_a2)))) {
        BgParams q = p;  // two K steps per stage do not apply: one per stage
        q.ksteps2 = 0;
        launch_bgemm(tmap_a, tmap_w, q, stages, ctas, d_err, s);
        return;
    }
    const uint32_t kpanels = (p.k_bytes + p.k_panel - 1) / p.k_panel;
    const uint64_t items = p.item_tab ? p.n_items : (uint64_t)kpanels * p.a_tiles * p.w_tiles;
    if (!items) return;
    const uint32_t stage_bytes = bgemm_stage_bytes(p.w_tile, p.a_resident != 0, p.ksteps2 ? 2u : 1u);
    // at least half the SM's shared memory: one CTA per SM, so the second
    // never waits in tcgen05.alloc for the first one's 512 TMEM columns
    const int smem = (int)std::max<uint32_t>(bgemm_smem_bytes(p, stages), 116u * 1024u);
    cudaFuncSetAttribute(bgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const uint64_t units = p.item_tab ? p.n_items : p.a_resident ? p.a_tiles : items;
    const unsigned grid = units < (uint64_t)ctas ? (unsigned)units : (unsigned)ctas;
    bgemm_kernel<<<grid, BG_THREADS, smem, s>>>(tmap_a, tmap_w, tmap_a2 ? *tmap_a2 : tmap_a, tmap_w2 ? *tmap_w2 : tmap_w,
                                                p, stages, stage_bytes, d_err);
}

void launch_planar_rows(const uint64_t* d_src, uint64_t rows, uint32_t k, uint64_t src_ld, int negate, uint8_t* d_dst,
                        uint64_t dst_ld, uint32_t col0, cudaStream_t s, const uint32_t* d_prow, uint32_t ks) {
    if (!rows) return;
    planar_rows_kernel<<<grid_for(rows * (k / 16), 256, 148 * 16), 256, 0, s>>>(d_src, rows, k, src_ld, negate, d_dst,
                                                                              dst_ld, col0, d_prow, ks);
}

void launch_planar_cm(const uint64_t* d_src_cm, uint64_t rows, uint32_t k, uint8_t* d_dst, uint64_t dst_ld,
                      uint32_t col0, cudaStream_t s, const uint32_t* d_prow, uint32_t ks) {
    if (!rows) return;
    planar_cm_kernel<<<grid_for(rows * (k / 16), 256, 148 * 16), 256, 0, s>>>(d_src_cm, rows, k, d_dst, dst_ld, col0,
                                                                            d_prow, ks);
}

void launch_ms8(const uint64_t* d_mp_cm, const uint16_t* d_s_ell, const uint32_t* d_s_off, const uint16_t* d_s_w,
                uint64_t rows, int8_t* d_dst, uint64_t* d_corr, uint32_t* d_bad, cudaStream_t s,
                const uint32_t* d_prow) {
    if (!rows) return;
    ms8_m_kernel<<<grid_for(rows * (N / 16), 256, 148 * 16), 256, 0, s>>>(d_mp_cm, rows, d_dst, d_bad, d_prow);
    ms8_s_kernel<<<grid_for(rows, 128, 148 * 16), 128, 0, s>>>(d_s_ell, d_s_off, d_s_w, rows, d_dst, d_corr, d_bad,
                                                               d_prow);
}

void launch_w_tv(const uint64_t* d_v, const uint32_t* d_t, const uint32_t* d_t_nnz, uint32_t nq, int8_t* d_dst,
                 uint32_t* d_bad, cudaStream_t s) {
    if (!nq) return;
    w_tv_kernel<<<grid_for((uint64_t)nq * 8 * (N / 16), 256, 148 * 8), 256, 0, s>>>(d_v, nq, d_dst);
    w_t_kernel<<<nq, 256, 0, s>>>(d_t, d_t_nnz, d_dst, d_bad);
}

void launch_zsum(const uint64_t* d_z_part, uint32_t npanels, uint32_t t_base, uint32_t t_cnt, uint32_t trials_total,
                 uint64_t* d_z, cudaStream_t s) {
    if (!t_cnt) return;
    zsum_kernel<<<dim3(N / 256, t_cnt), 256, 0, s>>>(d_z_part, npanels, t_base, trials_total, d_z);
}

void launch_zv(const uint64_t* d_z, const uint64_t* d_v, uint32_t trials, uint32_t nq, uint64_t* d_zv, cudaStream_t s) {
    if (!trials || !nq) return;
    zv_kernel<<<dim3(nq, trials), 128, 0, s>>>(d_z, d_v, nq, d_zv);
}

void launch_ur_decide(const uint64_t* d_ur_part, uint32_t kpanels, uint32_t trials, uint32_t nq, const uint64_t* d_zv,
                      uint64_t* d_ur, int32_t* d_failed, cudaStream_t s) {
    if (!nq) return;
    ur_decide_kernel<<<(nq + 127) / 128, 128, 0, s>>>(d_ur_part, kpanels, trials, nq, d_zv, d_ur, d_failed);
}

}  // namespace bn
