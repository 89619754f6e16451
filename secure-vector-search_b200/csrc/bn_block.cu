// bn_block.cu -- block scoring: B queries per launch on the tensor cores.
//
// The reference scores a batch by looping its per-query path on GPU handles
// (lib.rs:615-622) and, on the CPU, by compute_products_batch
// (crypto.rs:782-828), which reads M_enc once for the batch.  Here a block of
// B queries becomes a handful of integer GEMMs over byte-planar copies of the
// corpus (bn_batch.cuh):
//   G1  r_q   = M_enc v_q                  (u8 planes of m_enc x u8 planes of v)
//   G2  r_q  += -(AL g_q + H L^T v_q)      (u8 planes of [AL | H] x planes of -[g | x])
//   G3  r_q  -= M T_q + S v_q              (s8 [M | S] x s8 [T | bytes(v) - 128])
//       -> r_q = Mv_q (decode_scores, crypto.rs:901-940), then top-k
// and Protocol 2 is applied per block: one seed for the block, trial t's
// draws u_t (ChaCha20Rng(block_seed), draw t*m + i) shared by the B queries,
//   z_t = u_t^T M_enc                       (tc_freivalds_kernel, one pass of M_enc)
//   u_t . r_q                               (G4: u8 planes of r x u8 planes of u_t)
// and query q is accepted iff u_t . r_q == z_t . v_q for every t (the
// verify_response check, crypto.rs:1013-1059, with the block's u).
#include <cuda_runtime.h>

#include <cstring>

#include "bn_batch.cuh"
#include "bn_internal.cuh"
#include "bn_tc.cuh"

using namespace bn;
using namespace bn::api;

namespace bn {
namespace api {

struct BlockPlan {
    bn_flat* h = nullptr;
    uint32_t B = 0, trials = 0, k = 0;
    bool verify_only = false;  // Protocol 2 over claimed responses only
    uint64_t rows = 0, nld = 0, npad = 0;
    uint32_t t_pass = 0, n_rows = 0;   // trials per Freivalds pass, U rows (8 * even trials)
    uint32_t nblocks = 0, npanels = 0;  // U row blocks, z panels (4096 rows)
    // tuned GEMM configuration
    uint32_t w_tile = 256, stages = 4, order = 0, a_res = 0, k_panel4 = 16384;
    uint32_t ks2 = 1;  // two K steps per pipeline stage in G1-G3
    float tuned_ms[2] = {0.f, 0.f};  // autotuner's best G1 and G4 launch times
    int topk_ctas = 1;
    // workspace
    DevMem ws;
    uint64_t o_err, o_bad, o_vseg, o_blocks, o_panels, o_vp, o_gx, o_tv, o_x, o_r, o_f2, o_f3, o_rp, o_ub, o_zpart, o_z, o_zv,
        o_urpart, o_ur, o_fail, o_cs, o_ci, o_cn, o_in, o_in_v, o_in_g, o_in_t, o_in_tn, o_in_seed, o_out_ids,
        o_out_sc, o_out_n, o_out_end;
    CUtensorMap tm_vp, tm_gx, tm_tv, tm_rp, tm_ub;
    CUtensorMap tm_vp2, tm_gx2, tm_tv2;  // 3-D views of the W operands: two K steps per box
    PinnedMem host;  // staging for the host-buffer entry points
};

void block_plan_free(BlockPlan* b) { delete b; }

namespace {

uint32_t kpanels_of(const BlockPlan& b) { return (uint32_t)((b.npad + b.k_panel4 - 1) / b.k_panel4); }

uint32_t stages_for(const BgParams& p) { return bgemm_max_stages(p); }

// The u . r GEMM's stage count (W = the U planes, streaming A).
uint32_t stages_u(uint32_t n_rows) {
    BgParams p{};
    p.w_tile = n_rows;
    return stages_for(p);
}

int tmap(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint32_t box_rows, const char* what) {
    cudaError_t e = make_tmap_u8(m, base, inner, rows, 128, box_rows);
    if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map of %s: %s", what, cudaGetErrorString(e));
    return BN_OK;
}

// Byte-planar operands of the corpus (once per handle), K-blocked, each list
// (the whole corpus when offsets is null) starting on a tile boundary.
int block_prepare_locked(Engine& e, const std::vector<uint64_t>* offsets) {
    Corpus& c = e.c;
    if (c.block_ready) return BN_OK;
    if (!c.client) return fail(BN_EUNSUPPORTED, "block scoring needs the client state (attach_client was not called)");
    if (!c.rows) return fail(BN_EINVAL, "empty corpus");
    if (c.n1 % 16) return fail(BN_EINVAL, "n1 = %u is not a multiple of 16", c.n1);
    CU(cudaSetDevice(e.ctx->device));
    const uint64_t rows = c.rows;
    c.k_alh = (uint32_t)align_up(2ull * c.n1, 128);
    // padded rows: list l's rows at list_p16[l] + i (16-row tiles of the
    // planes) and list_p128[l] + i (128-row tiles of [M | S])
    const std::vector<uint64_t> whole{0, rows};
    const std::vector<uint64_t>& off = offsets ? *offsets : whole;
    const size_t nl = off.size() - 1;
    c.list_p16.assign(nl, 0);
    c.list_p128.assign(nl, 0);
    std::vector<uint32_t> prow16, prow128;
    if (nl > 1) {
        prow16.resize(rows);
        prow128.resize(rows);
    }
    uint64_t p16 = 0, p128 = 0;
    for (size_t l = 0; l < nl; ++l) {
        const uint64_t r0 = off[l], m = off[l + 1] - r0;
        c.list_p16[l] = p16;
        c.list_p128[l] = p128;
        if (nl > 1)
            for (uint64_t i = 0; i < m; ++i) {
                prow16[r0 + i] = (uint32_t)(p16 + i);
                prow128[r0 + i] = (uint32_t)(p128 + i);
            }
        p16 += align_up(m, 16);
        p128 += align_up(m, 128);
    }
    if (p128 >= (1ull << 31) / 16) return fail(BN_EUNSUPPORTED, "corpus too large for block scoring");
    c.rows16 = p16;
    c.rows128 = p128;
    TRY(c.mp8.alloc(e.ctx, c.rows16 * 8 * N));
    TRY(c.alh8.alloc(e.ctx, c.rows16 * 8 * c.k_alh));
    TRY(c.ms8.alloc(e.ctx, c.rows128 * 2 * N));
    TRY(c.corr.alloc(e.ctx, rows * 8));
    DevMem bad, d_p16, d_p128;
    TRY(bad.alloc(e.ctx, 4));
    cudaStream_t s = e.stream;
    const uint32_t* pr16 = nullptr;
    const uint32_t* pr128 = nullptr;
    if (nl > 1) {
        TRY(d_p16.alloc(e.ctx, rows * 4));
        TRY(d_p128.alloc(e.ctx, rows * 4));
        CU(cudaMemcpyAsync(d_p16.p, prow16.data(), rows * 4, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(d_p128.p, prow128.data(), rows * 4, cudaMemcpyHostToDevice, s));
        pr16 = d_p16.at<uint32_t>();
        pr128 = d_p128.at<uint32_t>();
    }
    CU(cudaMemsetAsync(bad.p, 0, 4, s));
    // pad rows (and pad columns of [AL | H]) stay zero
    CU(cudaMemsetAsync(c.mp8.p, 0, c.mp8.bytes, s));
    CU(cudaMemsetAsync(c.alh8.p, 0, c.alh8.bytes, s));
    CU(cudaMemsetAsync(c.ms8.p, 0, c.ms8.bytes, s));
    launch_planar_rows(c.m_enc.at<uint64_t>(), rows, N, N, 0, c.mp8.at<uint8_t>(), 0, 0, s, pr16, N / BG_KSTEP);
    launch_planar_cm(c.al_cm.at<uint64_t>(), rows, c.n1, c.alh8.at<uint8_t>(), 0, 0, s, pr16, c.k_alh / BG_KSTEP);
    launch_planar_cm(c.h_cm.at<uint64_t>(), rows, c.n1, c.alh8.at<uint8_t>(), 0, c.n1, s, pr16, c.k_alh / BG_KSTEP);
    launch_ms8(c.mp_cm.at<uint64_t>(), c.s_ell.at<uint16_t>(), c.s_off.at<uint32_t>(), c.s_w.at<uint16_t>(), rows,
               c.ms8.at<int8_t>(), c.corr.at<uint64_t>(), bad.at<uint32_t>(), s, pr128);
    CU(cudaGetLastError());
    uint32_t hb = 0;
    CU(cudaMemcpyAsync(&hb, bad.p, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (hb) {
        c.mp8.release();
        c.alh8.release();
        c.ms8.release();
        c.corr.release();
        return fail(BN_EUNSUPPORTED,
                    "block scoring needs m_plain entries and S row entries in [-128, 127] (int8-quantised corpus)");
    }
    // K-blocked: rows of 128 bytes, one (tile, K step) box = 128 consecutive rows
    TRY(tmap(&c.tmap_mp, c.mp8.p, BG_KSTEP, c.mp8.bytes / BG_KSTEP, 128, "m_enc planes"));
    TRY(tmap(&c.tmap_alh, c.alh8.p, BG_KSTEP, c.alh8.bytes / BG_KSTEP, 128, "[AL | H] planes"));
    TRY(tmap(&c.tmap_ms, c.ms8.p, BG_KSTEP, c.ms8.bytes / BG_KSTEP, 128, "[M | S] bytes"));
    TRY(tmap(&c.tmap_mp2, c.mp8.p, BG_KSTEP, c.mp8.bytes / BG_KSTEP, 256, "m_enc planes"));
    TRY(tmap(&c.tmap_alh2, c.alh8.p, BG_KSTEP, c.alh8.bytes / BG_KSTEP, 256, "[AL | H] planes"));
    TRY(tmap(&c.tmap_ms2, c.ms8.p, BG_KSTEP, c.ms8.bytes / BG_KSTEP, 256, "[M | S] bytes"));
    c.block_ready = true;
    return BN_OK;
}

BgParams g1_params(const BlockPlan& b, const Corpus& c) {
    BgParams p{};
    p.mode = BG_PLANAR;
    p.a_tiles = (uint32_t)((c.rows * 8 + BG_AROWS - 1) / BG_AROWS);
    p.w_tiles = (8 * b.B + b.w_tile - 1) / b.w_tile;
    p.w_tile = b.w_tile;
    p.k_bytes = N;
    p.k_panel = N;
    p.x_count = (uint32_t)c.rows;
    p.y_count = b.B;
    p.out_ld = b.nld;
    p.order_a_fast = (int)b.order;
    p.a_resident = (int)b.a_res;
    p.a_blocked = 1;
    p.ksteps2 = (int)b.ks2;  // two K steps per stage: half the producer / MMA handoffs per item
    p.planar_ld = b.npad;
    return p;
}

int relayout(BlockPlan& b) {
    // W-operand tensor maps depend on the tuned w_tile
    char* d = b.ws.at<char>();
    TRY(tmap(&b.tm_vp, d + b.o_vp, N, 8ull * b.B, b.w_tile, "v planes"));
    TRY(tmap(&b.tm_gx, d + b.o_gx, b.h->e.c.k_alh, 8ull * b.B, b.w_tile, "[g | x] planes"));
    TRY(tmap(&b.tm_tv, d + b.o_tv, 2 * N, 8ull * b.B, b.w_tile, "[T | v] bytes"));
    const struct {
        CUtensorMap* m;
        uint64_t off, row_bytes;
    } w2[3] = {{&b.tm_vp2, b.o_vp, N}, {&b.tm_gx2, b.o_gx, b.h->e.c.k_alh}, {&b.tm_tv2, b.o_tv, 2 * N}};
    for (const auto& x : w2) {
        const cudaError_t e = make_tmap_u8_ksteps2(x.m, d + x.off, x.row_bytes, 8ull * b.B, b.w_tile);
        if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map of the W operands: %s", cudaGetErrorString(e));
    }
    return BN_OK;
}

// Times G1 for each candidate (w_tile, stages, order) and G4 for each K
// panel size on this corpus; keeps the fastest.
int autotune(BlockPlan& b, cudaStream_t s) {
    Corpus& c = b.h->e.c;
    char* d = b.ws.at<char>();
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    const uint32_t wmax = (uint32_t)std::min<uint64_t>(256, align_up(8ull * b.B, 16));
    float best = 1e30f;
    uint32_t bw = b.w_tile, bs = b.stages, bo = b.order, ba = b.a_res, bk = b.ks2;
    int rc = BN_OK;
    for (uint32_t w : {64u, 128u, 256u}) {
        if (w > wmax && w != 64u) continue;
        for (uint32_t combo = 0; combo < 4 && rc == BN_OK; ++combo) {  // (A resident, two K steps per stage)
            const uint32_t ares = combo >> 1;
            b.w_tile = w;
            b.a_res = ares;
            b.ks2 = combo & 1;
            const uint32_t smax = stages_for(g1_params(b, c));
            if (!smax) continue;
            for (uint32_t st : {std::min(3u, smax), smax}) {
                for (uint32_t order : {0u, 1u}) {
                    if (ares && order) continue;  // A-resident work order is fixed
                    if (st == smax && smax == 3u && st != std::min(3u, smax)) continue;
                    b.stages = st;
                    b.order = order;
                    if ((rc = relayout(b)) != BN_OK) break;
                    BgParams p = g1_params(b, c);
                    p.out = reinterpret_cast<uint64_t*>(d + b.o_r);
                    p.planar_out = reinterpret_cast<uint8_t*>(d + b.o_rp);
                    float ms = 0;
                    for (int rep = 0; rep < 3; ++rep) {
                        if (rep == 1) cudaEventRecord(e0, s);
                        launch_bgemm(c.tmap_mp, b.tm_vp, p, b.stages, b.h->e.ctx->num_sms,
                                     reinterpret_cast<uint32_t*>(d + b.o_err), s, &c.tmap_mp2, &b.tm_vp2);
                    }
                    cudaEventRecord(e1, s);
                    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                        rc = fail(BN_ECUDA, "autotune timing failed");
                        break;
                    }
                    if (ms < best) { best = ms; bw = w; bs = st; bo = order; ba = ares; bk = b.ks2; }
                }
                if (rc != BN_OK || smax <= 3u) break;
            }
            if (rc != BN_OK) break;
        }
        if (rc != BN_OK) break;
    }
    b.w_tile = bw;
    b.stages = bs;
    b.order = bo;
    b.a_res = ba;
    b.ks2 = bk;
    b.tuned_ms[0] = best / 2;  // two timed launches per candidate
    if (rc == BN_OK && b.trials) {  // K panel of the u . r GEMM
        float bestk = 1e30f;
        uint32_t bk = b.k_panel4;
        for (uint32_t kp : {4096u, 8192u, 16384u}) {
            b.k_panel4 = kp;
            BgParams p{};
            p.mode = BG_PLANAR;
            p.a_tiles = (8 * b.B + BG_AROWS - 1) / BG_AROWS;
            p.w_tiles = 1;
            p.w_tile = b.n_rows;
            p.k_bytes = (uint32_t)b.npad;
            p.k_panel = kp;
            p.x_count = b.B;
            p.y_count = b.t_pass;
            p.out = reinterpret_cast<uint64_t*>(d + b.o_urpart);
            p.out_ld = b.B;
            p.out_pstride = (uint64_t)b.trials * b.B;
            p.order_a_fast = 1;
            if ((uint64_t)kpanels_of(b) * b.trials * b.B * 8 > (b.o_ur - b.o_urpart)) continue;  // scratch sized for 4096
            float ms = 0;
            for (int rep = 0; rep < 3; ++rep) {
                if (rep == 1) cudaEventRecord(e0, s);
                launch_bgemm(b.tm_rp, b.tm_ub, p, stages_u(b.n_rows), b.h->e.ctx->num_sms,
                             reinterpret_cast<uint32_t*>(d + b.o_err), s);
            }
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = fail(BN_ECUDA, "autotune timing failed");
                break;
            }
            if (ms < bestk) { bestk = ms; bk = kp; }
        }
        b.k_panel4 = bk;
        b.tuned_ms[1] = bestk / 2;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == BN_OK) rc = relayout(b);
    if (rc == BN_OK) CU(cudaMemsetAsync(d + b.o_err, 0, 4, s));
    return rc;
}

}  // namespace

// Offsets of every buffer of a block plan's workspace; returns its size.
uint64_t block_layout(BlockPlan& b, uint32_t n1, uint32_t k_alh, bool verify_only) {
    const uint32_t B = b.B, k = b.k, trials = b.trials;
    const uint32_t ks = std::max<uint32_t>(k, 1);
    const uint32_t tt = std::max<uint32_t>(trials, 1);
    Layout L;
    b.o_err = L.take<uint32_t>(2);  // [0] pipeline flags, [1] operand range flags
    b.o_bad = b.o_err + 4;
    b.o_vseg = L.take<VerifySeg>(1);
    b.o_blocks = L.take<TcBlock>(b.nblocks);
    b.o_panels = L.take<TcPanel>(b.npanels);
    const uint64_t qb = verify_only ? 0 : B;  // per-query operand buffers of the scoring GEMMs
    b.o_vp = L.take<uint8_t>(8ull * qb * N);
    b.o_gx = L.take<uint8_t>(8ull * qb * k_alh);
    b.o_tv = L.take<uint8_t>(8ull * qb * 2 * N);
    b.o_x = L.take<uint64_t>(qb * n1);
    b.o_r = L.take<uint64_t>((uint64_t)B * b.nld);    // r = M_enc v
    b.o_f2 = L.take<uint64_t>(qb * b.nld);             // -(AL g + H x)
    b.o_f3 = L.take<uint64_t>(qb * b.nld);             // M T + S v   (Mv = r + f2 - f3)
    b.o_rp = L.take<uint8_t>(8ull * B * b.npad);
    b.o_ub = L.take<uint8_t>(trials ? (uint64_t)b.n_rows * b.npad : 0);
    b.o_zpart = L.take<uint64_t>(trials ? (uint64_t)b.npanels * tt * N : 0);
    b.o_z = L.take<uint64_t>((uint64_t)tt * N);
    b.o_zv = L.take<uint64_t>((uint64_t)tt * B);
    b.o_urpart = L.take<uint64_t>(trials ? (uint64_t)((b.npad + 4095) / 4096) * tt * B : 0);
    b.o_ur = L.take<uint64_t>((uint64_t)tt * B);
    b.o_fail = L.take<int32_t>(B);
    b.o_cs = L.take<int64_t>((uint64_t)B * b.topk_ctas * ks);
    b.o_ci = L.take<uint32_t>((uint64_t)B * b.topk_ctas * ks);
    b.o_cn = L.take<uint32_t>((uint64_t)B * b.topk_ctas);
    // host-buffer staging: inputs then outputs, contiguous
    b.o_in = L.take<uint8_t>(0);
    b.o_in_v = L.take<uint64_t>((uint64_t)B * N);
    b.o_in_g = L.take<uint64_t>((uint64_t)B * n1);
    b.o_in_t = L.take<uint32_t>((uint64_t)B * N);
    b.o_in_tn = L.take<uint32_t>(B);
    b.o_in_seed = L.take<uint8_t>(32);
    b.o_out_ids = L.take<uint32_t>((uint64_t)B * ks);
    b.o_out_sc = L.take<int64_t>((uint64_t)B * ks);
    b.o_out_n = L.take<uint32_t>(B);
    b.o_out_end = L.take<uint8_t>(0);
    return L.off + 1024;
}

int block_prepare_engine(Engine& e, const std::vector<uint64_t>* offsets) { return block_prepare_locked(e, offsets); }

int block_prepare(bn_flat* f) {
    std::lock_guard<std::mutex> g(f->e.mu);
    return block_prepare_locked(f->e, nullptr);
}

int block_plan_create(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k, uint32_t flags, BlockPlan** out) {
    *out = nullptr;
    if (!B || B > 8192) return fail(BN_EINVAL, "B = %u is outside 1..=8192 queries per block", B);
    if (k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX = %d", k, BN_TOPK_MAX);
    if (trials > BN_MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %d", trials, BN_MAX_TRIALS);
    if (!f->m) return fail(BN_EINVAL, "empty corpus");
    const bool verify_only = (flags & BLOCK_VERIFY_ONLY) != 0;  // Protocol 2 over claimed r: no planar corpus needed
    std::lock_guard<std::mutex> g(f->e.mu);
    if (!verify_only) TRY(block_prepare_locked(f->e, nullptr));
    Corpus& c = f->e.c;
    auto* b = new BlockPlan();
    b->h = f;
    b->verify_only = verify_only;
    b->B = B;
    b->trials = trials;
    b->k = k;
    b->rows = c.rows;
    b->nld = align_up(c.rows, 16);
    b->npad = align_up(c.rows, 128);
    b->t_pass = std::min<uint32_t>(std::max<uint32_t>(trials, 1), TC_MAX_TRIALS);
    b->n_rows = 8 * ((b->t_pass + 1) & ~1u);
    b->nblocks = (uint32_t)((c.rows + TC_ROWS - 1) / TC_ROWS);
    b->npanels = (uint32_t)((c.rows + TC_PANEL_ROWS - 1) / TC_PANEL_ROWS);
    b->w_tile = (uint32_t)std::min<uint64_t>(256, align_up(8ull * B, 16));
    b->a_res = 8ull * B > b->w_tile ? 1u : 0u;  // A tiles reused across several W tiles
    if (!c.block_ready) b->a_res = 0;
    b->k_panel4 = 4096;
    if (!verify_only) {
        // the first configuration with a pipeline of at least 3 stages, else of 2:
        // (A resident if useful, two K steps per stage) before (.., one K step)
        // before streaming A
        const uint32_t pref_ares = b->a_res;
        bool found = false;
        for (uint32_t min_st : {3u, 2u}) {
            for (uint32_t combo = 0; combo < 4 && !found; ++combo) {
                b->a_res = combo < 2 ? pref_ares : 0u;
                b->ks2 = (combo & 1) ? 0u : 1u;
                b->stages = stages_for(g1_params(*b, c));
                found = b->stages >= min_st;
            }
            if (found) break;
        }
    }
    const int sms = f->e.ctx->num_sms;
    b->topk_ctas = (int)std::max<uint64_t>(1, std::min<uint64_t>((c.rows + 511) / 512, (uint64_t)sms * 4 / B));
    const uint64_t total = block_layout(*b, c.n1, c.k_alh, verify_only);
    int rc = b->ws.alloc(f->e.ctx, total);
    cudaStream_t s = f->e.stream;
    if (rc == BN_OK) {
        // metadata: the whole corpus is one verification segment
        std::vector<char> hm(b->o_vp - b->o_vseg, 0);
        VerifySeg vs{0, 0, (uint32_t)c.rows, 0};
        memcpy(hm.data(), &vs, sizeof vs);
        auto* blocks = reinterpret_cast<TcBlock*>(hm.data() + (b->o_blocks - b->o_vseg));
        for (uint32_t i = 0; i < b->nblocks; ++i) blocks[i] = TcBlock{0, i * (uint32_t)TC_ROWS};
        auto* panels = reinterpret_cast<TcPanel*>(hm.data() + (b->o_panels - b->o_vseg));
        for (uint32_t p = 0; p < b->npanels; ++p) {
            const uint64_t r0 = (uint64_t)p * TC_PANEL_ROWS;
            panels[p] = TcPanel{r0, (uint32_t)std::min<uint64_t>(TC_PANEL_ROWS, c.rows - r0),
                                (uint32_t)(r0 / TC_ROWS), 0, 0};
        }
        if (cudaMemsetAsync(b->ws.p, 0, b->o_vseg, s) != cudaSuccess ||
            cudaMemcpyAsync(b->ws.at<char>() + b->o_vseg, hm.data(), hm.size(), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemsetAsync(b->ws.at<char>() + b->o_gx, 0, verify_only ? 0 : 8ull * B * c.k_alh, s) != cudaSuccess ||
            cudaMemsetAsync(b->ws.at<char>() + b->o_rp, 0, 8ull * B * b->npad, s) != cudaSuccess ||
            cudaMemsetAsync(b->ws.at<char>() + b->o_vp, 0, verify_only ? 0 : 8ull * B * N, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            rc = fail(BN_ECUDA, "block plan set-up failed");
    }
    if (rc == BN_OK) {
        char* d = b->ws.at<char>();
        rc = tmap(&b->tm_rp, d + b->o_rp, b->npad, 8ull * B, 128, "r planes");
        if (rc == BN_OK && trials) rc = tmap(&b->tm_ub, d + b->o_ub, b->npad, b->n_rows, b->n_rows, "u planes");
        if (rc == BN_OK && !verify_only) rc = relayout(*b);
        if (rc == BN_OK && !verify_only && (flags & BN_BLOCK_AUTOTUNE)) rc = autotune(*b, s);
        if (rc == BN_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(BN_ECUDA, "block plan set-up failed");
    }
    if (rc != BN_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return BN_OK;
}

// Workspace bytes a block plan of B queries would allocate (the corpus's
// byte-planar copies, made once per handle, are not included).
uint64_t block_plan_estimate(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k) {
    const Corpus& c = f->e.c;
    BlockPlan b;
    b.B = B;
    b.trials = trials;
    b.k = k;
    b.rows = c.rows;
    b.nld = align_up(c.rows, 16);
    b.npad = align_up(c.rows, 128);
    b.t_pass = std::min<uint32_t>(std::max<uint32_t>(trials, 1), TC_MAX_TRIALS);
    b.n_rows = 8 * ((b.t_pass + 1) & ~1u);
    b.nblocks = (uint32_t)((c.rows + TC_ROWS - 1) / TC_ROWS);
    b.npanels = (uint32_t)((c.rows + TC_PANEL_ROWS - 1) / TC_PANEL_ROWS);
    b.topk_ctas = (int)std::max<uint64_t>(1, std::min<uint64_t>((c.rows + 511) / 512, (uint64_t)f->e.ctx->num_sms * 4 / B));
    return block_layout(b, c.n1, (uint32_t)align_up(2ull * c.n1, 128), false);
}

void block_plan_config(const BlockPlan* b, uint32_t cfg[6], float tuned_ms[2]) {
    cfg[0] = b->w_tile;
    cfg[1] = b->stages;
    cfg[2] = b->order;
    cfg[3] = b->a_res;
    cfg[4] = b->k_panel4;
    cfg[5] = b->ks2;
    if (tuned_ms) {
        tuned_ms[0] = b->tuned_ms[0];
        tuned_ms[1] = b->tuned_ms[1];
    }
}

int block_plan_status(BlockPlan* b, uint32_t* flags) {
    CU(cudaMemcpy(flags, b->ws.at<char>() + b->o_err, 4, cudaMemcpyDeviceToHost));
    uint32_t bad = 0;
    CU(cudaMemcpy(&bad, b->ws.at<char>() + b->o_bad, 4, cudaMemcpyDeviceToHost));
    if (bad) *flags |= 0x100u;  // a T column sum left [-128, 127]
    return BN_OK;
}

// Protocol 2 for the block: rp holds the byte planes of r (G1 output or an
// uploaded claim); failed / ur / zv per query.
static void enqueue_verify(BlockPlan& b, const uint64_t* d_v, const uint8_t* d_seed, int32_t* d_failed, cudaStream_t s) {
    Corpus& c = b.h->e.c;
    char* d = b.ws.at<char>();
    uint32_t* err = reinterpret_cast<uint32_t*>(d + b.o_err);
    const auto* vseg = reinterpret_cast<const VerifySeg*>(d + b.o_vseg);
    const auto* blocks = reinterpret_cast<const TcBlock*>(d + b.o_blocks);
    const auto* panels = reinterpret_cast<const TcPanel*>(d + b.o_panels);
    uint8_t* ub = reinterpret_cast<uint8_t*>(d + b.o_ub);
    uint64_t* zpart = reinterpret_cast<uint64_t*>(d + b.o_zpart);
    uint64_t* z = reinterpret_cast<uint64_t*>(d + b.o_z);
    uint64_t* urpart = reinterpret_cast<uint64_t*>(d + b.o_urpart);
    const int sms = b.h->e.ctx->num_sms;
    if (b.trials && b.h->e.ctx->debug_draw_hit) launch_or_flag(err, DRAW_HIT_P, s);
    for (uint32_t t0 = 0; t0 < b.trials; t0 += TC_MAX_TRIALS) {
        const uint32_t tc = std::min<uint32_t>(TC_MAX_TRIALS, b.trials - t0);
        launch_tc_ugen(vseg, blocks, b.nblocks, reinterpret_cast<const ChaChaKey*>(d_seed), nullptr, t0, tc, b.n_rows,
                       ub, nullptr, b.trials, err, s, b.npad);
        launch_tc_freivalds(c.tmap_m, b.tm_ub, panels, b.npanels, t0, tc, b.n_rows, b.trials, zpart, err, sms, s, 1,
                            b.h->e.ctx->debug_wait_cycles);
        launch_zsum(zpart, b.npanels, t0, tc, b.trials, z, s);
        BgParams p{};
        p.mode = BG_PLANAR;
        p.a_tiles = (8 * b.B + BG_AROWS - 1) / BG_AROWS;
        p.w_tiles = 1;
        p.w_tile = b.n_rows;
        p.k_bytes = (uint32_t)b.npad;
        p.k_panel = b.k_panel4;
        p.x_count = b.B;
        p.y_count = tc;
        p.out = urpart + (uint64_t)t0 * b.B;
        p.out_ld = b.B;
        p.out_pstride = (uint64_t)b.trials * b.B;
        p.order_a_fast = 1;
        p.wait_cycles = b.h->e.ctx->debug_wait_cycles;
        launch_bgemm(b.tm_rp, b.tm_ub, p, stages_u(b.n_rows), sms, err, s);
    }
    uint64_t* zv = reinterpret_cast<uint64_t*>(d + b.o_zv);
    launch_zv(z, d_v, b.trials, b.B, zv, s);
    launch_ur_decide(urpart, kpanels_of(b), b.trials, b.B, zv, reinterpret_cast<uint64_t*>(d + b.o_ur), d_failed, s);
}

int block_enqueue(BlockPlan& b, const uint64_t* d_v, const uint64_t* d_g, const uint32_t* d_t, const uint32_t* d_tn,
                  const uint8_t* d_seed, uint32_t* d_ids, int64_t* d_scores, uint32_t* d_n, int32_t* d_failed,
                  cudaStream_t s, bool want_mv) {
    if (b.verify_only) return fail(BN_EINVAL, "verification-only block plan");
    if (!d_v || !d_g || !d_t || !d_tn || !d_failed || (b.trials && !d_seed) || (b.k && (!d_ids || !d_scores || !d_n)))
        return fail(BN_EINVAL, "null device pointer");
    Corpus& c = b.h->e.c;
    char* d = b.ws.at<char>();
    uint32_t* err = reinterpret_cast<uint32_t*>(d + b.o_err);
    const int sms = b.h->e.ctx->num_sms;
    CU(cudaMemsetAsync(err, 0, 8, s));  // pipeline + operand flags
    uint8_t* vp = reinterpret_cast<uint8_t*>(d + b.o_vp);
    uint8_t* gx = reinterpret_cast<uint8_t*>(d + b.o_gx);
    int8_t* tv = reinterpret_cast<int8_t*>(d + b.o_tv);
    uint64_t* x = reinterpret_cast<uint64_t*>(d + b.o_x);
    uint64_t* r = reinterpret_cast<uint64_t*>(d + b.o_r);
    uint8_t* rp = reinterpret_cast<uint8_t*>(d + b.o_rp);
    if (b.k == 0 && !d_ids) d_ids = reinterpret_cast<uint32_t*>(d + b.o_out_ids);  // unused when k = 0
    // operands of this block
    launch_planar_rows(d_v, b.B, N, N, 0, vp, N, 0, s);
    launch_lt_times_v(c.L.at<uint64_t>(), c.n1, d_v, b.B, x, s);
    launch_planar_rows(d_g, b.B, c.n1, c.n1, 1, gx, c.k_alh, 0, s);
    launch_planar_rows(x, b.B, c.n1, c.n1, 1, gx, c.k_alh, c.n1, s);
    launch_w_tv(d_v, d_t, d_tn, b.B, tv, reinterpret_cast<uint32_t*>(d + b.o_bad), s);
    // G1: r = M_enc v (and its byte planes for Protocol 2)
    BgParams p = g1_params(b, c);
    p.out = r;
    p.planar_out = rp;
    p.wait_cycles = b.h->e.ctx->debug_wait_cycles;
    launch_bgemm(c.tmap_mp, b.tm_vp, p, b.stages, sms, err, s, &c.tmap_mp2, &b.tm_vp2);
    // G2: f2 = -(AL g + H x)   (K = 2 n1 bytes per plane row: A tiles stay resident)
    p.k_bytes = c.k_alh;
    p.k_panel = c.k_alh;
    p.out = reinterpret_cast<uint64_t*>(d + b.o_f2);
    p.planar_out = nullptr;
    p.a_resident = (p.w_tiles > 1 && c.k_alh <= BG_MAX_ASLOTS * BG_KSTEP) ? 1 : 0;
    p.order_a_fast = p.a_resident ? 0 : (int)b.order;
    launch_bgemm(c.tmap_alh, b.tm_gx, p, stages_for(p), sms, err, s, &c.tmap_alh2, &b.tm_gx2);
    // G3: f3 = M T + S v
    BgParams q{};
    q.mode = BG_S8;
    q.a_tiles = (uint32_t)((c.rows + BG_AROWS - 1) / BG_AROWS);
    q.w_tiles = p.w_tiles;
    q.w_tile = b.w_tile;
    q.k_bytes = 2 * N;
    q.k_panel = 2 * N;
    q.x_count = (uint32_t)c.rows;
    q.y_count = b.B;
    q.out = reinterpret_cast<uint64_t*>(d + b.o_f3);
    q.out_ld = b.nld;
    q.corr = c.corr.at<uint64_t>();
    q.order_a_fast = (int)b.order;
    q.a_blocked = 1;
    q.ksteps2 = (int)b.ks2;
    q.wait_cycles = p.wait_cycles;
    launch_bgemm(c.tmap_ms, b.tm_tv, q, stages_for(q), sms, err, s, &c.tmap_ms2, &b.tm_tv2);
    // Mv = r + f2 - f3 (written over f3 when asked for), fp_to_signed, top-k
    if (b.k || want_mv) {
        TopkScratch ts{reinterpret_cast<int64_t*>(d + b.o_cs), reinterpret_cast<uint32_t*>(d + b.o_ci),
                       reinterpret_cast<uint32_t*>(d + b.o_cn)};
        const bool own = b.k == 0;  // only the residues wanted: ranks go to the plan's own buffers
        launch_topk_rows(r, reinterpret_cast<uint64_t*>(d + b.o_f2), reinterpret_cast<uint64_t*>(d + b.o_f3), b.nld,
                         c.rows, b.B, nullptr, own ? 1u : b.k, b.topk_ctas, ts,
                         own ? reinterpret_cast<uint32_t*>(d + b.o_out_ids) : d_ids,
                         own ? reinterpret_cast<int64_t*>(d + b.o_out_sc) : d_scores,
                         own ? reinterpret_cast<uint32_t*>(d + b.o_out_n) : d_n,
                         want_mv ? reinterpret_cast<uint64_t*>(d + b.o_f3) : nullptr, s);
    }
    if (b.trials) enqueue_verify(b, d_v, d_seed, d_failed, s);
    else CU(cudaMemsetAsync(d_failed, 0xff, (uint64_t)b.B * 4, s));
    CU(cudaGetLastError());
    return BN_OK;
}

// Host-buffer block query in two steps (so that a caller can keep several in
// flight): launch packs the first nq <= B queries (the rest of the block is
// padded with zero queries whose results are dropped), enqueues one H2D, the
// block pipeline and one D2H on s; finish reads the outputs after s drained.
int block_query_launch(BlockPlan& b, uint32_t nq, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                       const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* seed, cudaStream_t s, bool want_mv) {
    Corpus& c = b.h->e.c;
    const uint32_t B = b.B;
    if (nq > B) return fail(BN_EINVAL, "%u queries for a block plan of %u", nq, B);
    TRY(b.host.reserve(b.o_out_end - b.o_in + (uint64_t)B * 4 + 8));
    char* h = b.host.at<char>();
    auto at = [&](uint64_t off) { return h + (off - b.o_in); };
    memset(at(b.o_in_v), 0, (uint64_t)B * N * 8);
    memset(at(b.o_in_g), 0, (uint64_t)B * c.n1 * 8);
    memset(at(b.o_in_tn), 0, (uint64_t)B * 4);
    memcpy(at(b.o_in_v), v_enc, (uint64_t)nq * N * 8);
    memcpy(at(b.o_in_g), g, (uint64_t)nq * c.n1 * 8);
    uint32_t* ht = reinterpret_cast<uint32_t*>(at(b.o_in_t));
    uint64_t tp = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        if (t_nnz[q] > N) return fail(BN_EINVAL, "t_nnz[%u] = %u exceeds n", q, t_nnz[q]);
        for (uint32_t i = 0; i < t_nnz[q]; ++i, ++tp) {
            if (t_idx[tp] >= N || (t_sign[tp] != 1 && t_sign[tp] != -1))
                return fail(BN_EINVAL, "T entry %llu is not (col < n, sign +-1)", (unsigned long long)tp);
            ht[(uint64_t)q * N + i] = t_idx[tp] | (t_sign[tp] < 0 ? 0x80000000u : 0u);
        }
    }
    memcpy(at(b.o_in_tn), t_nnz, (uint64_t)nq * 4);
    if (seed) memcpy(at(b.o_in_seed), seed, 32);
    else memset(at(b.o_in_seed), 0, 32);
    char* d = b.ws.at<char>();
    CU(cudaSetDevice(b.h->e.ctx->device));
    CU(cudaMemcpyAsync(d + b.o_in, h, b.o_out_ids - b.o_in, cudaMemcpyHostToDevice, s));
    TRY(block_enqueue(b, reinterpret_cast<uint64_t*>(d + b.o_in_v), reinterpret_cast<uint64_t*>(d + b.o_in_g),
                      reinterpret_cast<uint32_t*>(d + b.o_in_t), reinterpret_cast<uint32_t*>(d + b.o_in_tn),
                      reinterpret_cast<uint8_t*>(d + b.o_in_seed), reinterpret_cast<uint32_t*>(d + b.o_out_ids),
                      reinterpret_cast<int64_t*>(d + b.o_out_sc), reinterpret_cast<uint32_t*>(d + b.o_out_n),
                      reinterpret_cast<int32_t*>(d + b.o_fail), s, want_mv));
    char* hf = h + (b.o_out_end - b.o_in);
    CU(cudaMemcpyAsync(at(b.o_out_ids), d + b.o_out_ids, b.o_out_end - b.o_out_ids, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hf, d + b.o_fail, (uint64_t)B * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hf + (uint64_t)B * 4, d + b.o_err, 8, cudaMemcpyDeviceToHost, s));
    return BN_OK;
}

int block_query_finish(BlockPlan& b, uint32_t nq, uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed) {
    const uint32_t B = b.B, ks = std::max<uint32_t>(b.k, 1);
    char* h = b.host.at<char>();
    auto at = [&](uint64_t off) { return h + (off - b.o_in); };
    const int32_t* hf = reinterpret_cast<const int32_t*>(h + (b.o_out_end - b.o_in));
    const uint32_t* flags = reinterpret_cast<const uint32_t*>(hf + B);
    TRY(device_flags_status(flags[0]));
    if (flags[1]) return fail(BN_EINVAL, "a T column sum leaves [-128, 127]");
    const uint32_t* hid = reinterpret_cast<const uint32_t*>(at(b.o_out_ids));
    const int64_t* hsc = reinterpret_cast<const int64_t*>(at(b.o_out_sc));
    const uint32_t* hn = reinterpret_cast<const uint32_t*>(at(b.o_out_n));
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t nh = b.k ? hn[q] : 0;
        if (n_hits) n_hits[q] = nh;
        for (uint32_t i = 0; i < nh; ++i) {
            if (ids) ids[(uint64_t)q * b.k + i] = hid[(uint64_t)q * ks + i];
            if (scores) scores[(uint64_t)q * b.k + i] = hsc[(uint64_t)q * ks + i];
        }
        if (failed) failed[q] = hf[q];
    }
    return BN_OK;
}

// Host-buffer block query: one H2D of the packed inputs, the block pipeline,
// one D2H of the ranked hits.
int block_query_host(BlockPlan& b, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                     const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* seed, uint32_t* ids, int64_t* scores,
                     uint32_t* n_hits, int32_t* failed, uint64_t* mv_out) {
    Corpus& c = b.h->e.c;
    cudaStream_t s = b.h->e.stream;
    TRY(block_query_launch(b, b.B, v_enc, g, t_idx, t_sign, t_nnz, seed, s, mv_out != nullptr));
    if (mv_out)
        for (uint32_t q = 0; q < b.B; ++q)
            CU(cudaMemcpyAsync(mv_out + (uint64_t)q * c.rows, b.ws.at<char>() + b.o_f3 + (uint64_t)q * b.nld * 8,
                               c.rows * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return block_query_finish(b, b.B, ids, scores, n_hits, failed);
}

uint64_t block_plan_bytes(const BlockPlan* b) { return b->ws.bytes; }

// Protocol 2 over claimed responses r (B x m, host) with the block seed.
int block_verify_host(BlockPlan& b, const uint64_t* r, const uint64_t* v_enc, const uint8_t* seed, int32_t* failed,
                      uint64_t* ur, uint64_t* zv) {
    Corpus& c = b.h->e.c;
    const uint32_t B = b.B;
    char* d = b.ws.at<char>();
    cudaStream_t s = b.h->e.stream;
    CU(cudaSetDevice(b.h->e.ctx->device));
    uint64_t* dr = reinterpret_cast<uint64_t*>(d + b.o_r);
    CU(cudaMemsetAsync(d + b.o_err, 0, 8, s));
    CU(cudaMemsetAsync(dr, 0, (uint64_t)B * b.nld * 8, s));
    for (uint32_t q = 0; q < B; ++q)
        CU(cudaMemcpyAsync(dr + (uint64_t)q * b.nld, r + (uint64_t)q * c.rows, c.rows * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(d + b.o_in_v, v_enc, (uint64_t)B * N * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(d + b.o_in_seed, seed, 32, cudaMemcpyHostToDevice, s));
    launch_planar_rows(dr, B, (uint32_t)b.nld, b.nld, 0, reinterpret_cast<uint8_t*>(d + b.o_rp), b.npad, 0, s);
    enqueue_verify(b, reinterpret_cast<uint64_t*>(d + b.o_in_v), reinterpret_cast<uint8_t*>(d + b.o_in_seed),
                   reinterpret_cast<int32_t*>(d + b.o_fail), s);
    CU(cudaGetLastError());
    std::vector<int32_t> hf(B);
    CU(cudaMemcpyAsync(hf.data(), d + b.o_fail, (uint64_t)B * 4, cudaMemcpyDeviceToHost, s));
    if (ur) CU(cudaMemcpyAsync(ur, d + b.o_ur, (uint64_t)b.trials * B * 8, cudaMemcpyDeviceToHost, s));
    if (zv) CU(cudaMemcpyAsync(zv, d + b.o_zv, (uint64_t)b.trials * B * 8, cudaMemcpyDeviceToHost, s));
    uint32_t flags = 0;
    CU(cudaMemcpyAsync(&flags, d + b.o_err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(device_flags_status(flags));
    if (failed) memcpy(failed, hf.data(), (uint64_t)B * 4);
    return BN_OK;
}

}  // namespace api
}  // namespace bn
