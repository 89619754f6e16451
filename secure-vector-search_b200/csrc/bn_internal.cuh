// bn_internal.cuh -- library-internal types shared by the translation units
// behind the C ABI (bn_capi.cu, bn_block.cu): the context, budget-accounted
// device memory, the resident corpus and the flat / IVF handles.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "bn_b200.h"
#include "bn_kernels.cuh"
#include "bn_tc.cuh"

// ------------------------------------------------------------------ context
struct bn_ctx {
    int device = 0;
    int num_sms = 148;
    int engine = BN_ENGINE_TENSOR;  // Protocol 2 engine
    int debug_draw_hit = 0;         // bn_debug_plant_draw_hit
    long long debug_wait_cycles = 0;  // bn_debug_set_wait_limit (0 = the kernels' ~1 s default)
    uint64_t budget = 0, used = 0, peak = 0;
    std::mutex mu;
};

namespace bn {
namespace api {

// Records the message for bn_last_error() (thread-local) and returns code.
int fail(int code, const char* fmt, ...);

#define CU(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return ::bn::api::fail(BN_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define TRY(call)                    \
    do {                             \
        int rc_ = (call);            \
        if (rc_ != BN_OK) return rc_; \
    } while (0)

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Status of a pipeline's device flag word once its stream has drained: a
// timed-out wait (any bit but DRAW_HIT_P) is BN_ECUDA, a draw that equalled
// p (and nothing else) BN_EDRAW.
inline int device_flags_status(uint32_t f) {
    if (f & ~DRAW_HIT_P) return fail(BN_ECUDA, "a device pipeline wait timed out (flags 0x%x); results discarded", f);
    if (f & DRAW_HIT_P)
        return fail(BN_EDRAW, "a Protocol 2 draw equalled p (the reference redraws there, crypto.rs:155-162, shifting "
                              "every later draw); results discarded");
    return BN_OK;
}


// Device allocation accounted against the context budget.  With `stream`
// set the buffer is allocated and freed in that stream's order
// (cudaMallocAsync / cudaFreeAsync): growing it then synchronises nothing,
// where cudaFree waits for the whole device (the serving loop's slot
// workspaces, which grow while other slots' batches are in flight).
struct DevMem {
    bn_ctx* ctx = nullptr;
    void* p = nullptr;
    uint64_t bytes = 0;
    cudaStream_t stream = nullptr;

    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }

    void release() {
        if (p) {
            if (stream) cudaFreeAsync(p, stream);
            else cudaFree(p);
            std::lock_guard<std::mutex> g(ctx->mu);
            ctx->used -= bytes;
        }
        p = nullptr;
        bytes = 0;
    }
    int alloc(bn_ctx* c, uint64_t b) {
        release();
        ctx = c;
        if (b == 0) return BN_OK;
        {
            std::lock_guard<std::mutex> g(c->mu);
            if (c->used + b > c->budget)
                return fail(BN_EBUDGET, "cluster payload %llu bytes exceeds budget %llu bytes (%llu bytes in use)",
                            (unsigned long long)b, (unsigned long long)c->budget, (unsigned long long)c->used);
            c->used += b;
            c->peak = std::max(c->peak, c->used);
        }
        cudaError_t e = stream ? cudaMallocAsync(&p, b, stream) : cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            std::lock_guard<std::mutex> g(c->mu);
            c->used -= b;
            p = nullptr;
            return fail(BN_ECUDA, "cudaMalloc(%llu): %s", (unsigned long long)b, cudaGetErrorString(e));
        }
        bytes = b;
        return BN_OK;
    }
    // Grow-only reallocation (contents not kept).
    int reserve(bn_ctx* c, uint64_t b) { return (p && bytes >= b) ? BN_OK : alloc(c, b); }
    // The size reserve_grow makes room for: at least `need`, and half again
    // the current size when it grows at all, so a stream of slowly growing
    // requests reallocates (and so synchronises the device) a few times, not
    // every time.
    static uint64_t grown(uint64_t have, uint64_t need) {
        return have >= need ? have : (need > have + have / 2 ? need : have + have / 2);
    }
    int reserve_grow(bn_ctx* c, uint64_t b) {
        if (p && bytes >= b) return BN_OK;
        const uint64_t g = grown(bytes, b);
        const int rc = alloc(c, g);
        return rc == BN_EBUDGET && g > b ? alloc(c, b) : rc;  // the headroom is optional
    }
    template <class T>
    T* at(uint64_t off = 0) const {
        return reinterpret_cast<T*>(static_cast<char*>(p) + off);
    }
};

struct PinnedMem {
    void* p = nullptr;
    uint64_t bytes = 0;
    // cudaFreeHost synchronises the whole device: a buffer that other streams
    // keep busy (a serving slot's) sets keep_retired, and the buffers it grows
    // out of are freed with it instead of at each growth.
    bool keep_retired = false;
    std::vector<void*> retired;
    ~PinnedMem() {
        if (p) cudaFreeHost(p);
        for (void* x : retired) cudaFreeHost(x);
    }
    // Grows by half again at least.
    int reserve(uint64_t b) {
        if (p && bytes >= b) return BN_OK;
        const uint64_t g = b > bytes + bytes / 2 ? b : bytes + bytes / 2;
        if (p) {
            if (keep_retired) retired.push_back(p);
            else cudaFreeHost(p);
        }
        p = nullptr;
        bytes = 0;
        CU(cudaMallocHost(&p, g));
        bytes = g;
        return BN_OK;
    }
    template <class T>
    T* at(uint64_t off = 0) const {
        return reinterpret_cast<T*>(static_cast<char*>(p) + off);
    }
};

// Bump allocator computing sub-buffer offsets (256-byte aligned).
struct Layout {
    uint64_t off = 0;
    template <class T>
    uint64_t take(uint64_t count) {
        off = align_up(off, 256);
        uint64_t o = off;
        off += count * sizeof(T);
        return o;
    }
};

// Resident corpus: a flat cluster, or all IVF lists concatenated.
struct Corpus {
    uint64_t rows = 0;
    uint32_t n = N, n1 = 128;
    DevMem m_enc, al_cm, h_cm;
    bool client = false;
    DevMem L, mp_cm, s_ell, s_off, s_w, ids;
    DevMem alh_b, m8_cm;  // decode copies (bn_kernels.cuh): [AL | H] in 32-row blocks, int8 M column-major
    CUtensorMap tmap_m;  // m_enc as bytes {8192, rows}, 128x128 boxes, 128-byte swizzle

    // Byte-planar operands of block scoring (built on first use, see
    // bn_block.cu), K-blocked for the GEMMs' A operand: m_enc planes
    // (rows16 * 8 plane rows x 1024 bytes), [AL | H] planes (rows16 * 8 x
    // k_alh), [M | S] as signed bytes (rows128 x 2048), corr[rows].  Each
    // list starts on a tile boundary: list c's rows sit at padded rows
    // list_p16[c] (16-row plane tiles) and list_p128[c] (128-row tiles).
    bool block_ready = false;
    DevMem mp8, alh8, ms8, corr;
    uint32_t k_alh = 0;
    uint64_t rows16 = 0, rows128 = 0;
    std::vector<uint64_t> list_p16, list_p128;
    CUtensorMap tmap_mp, tmap_alh, tmap_ms;
    CUtensorMap tmap_mp2, tmap_alh2, tmap_ms2;  // the same with 256-row boxes (two K steps of a tile)

    uint64_t bytes() const {
        return m_enc.bytes + al_cm.bytes + h_cm.bytes + L.bytes + mp_cm.bytes + s_ell.bytes + s_off.bytes + s_w.bytes +
               ids.bytes + alh_b.bytes + m8_cm.bytes + mp8.bytes + alh8.bytes + ms8.bytes + corr.bytes;
    }
};

// Handle-side state shared by flat and IVF.
struct Engine {
    bn_ctx* ctx = nullptr;
    Corpus c;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    DevMem ws;
    PinnedMem host;
};

// ---------------------------------------------------------------- one pipeline run
constexpr uint32_t MAX_TRIALS = 64;  // Protocol 2 trials per call

struct TcMaps {  // host-side tensor maps of the U buffer, one per pass of <= 20 trials
    CUtensorMap u[(MAX_TRIALS + TC_MAX_TRIALS - 1) / TC_MAX_TRIALS];
    CUtensorMap w;  // the queries' diagonal byte images (fused scan)
};
inline uint32_t pass_rows(uint32_t t_cnt) { return 8 * ((t_cnt + 1) & ~1u); }

struct Meta {  // device pointers (+ host tensor maps)
    const ScanSeg* segs;
    const uint64_t* seg_blk;
    const uint64_t* seg_unit;  // decode units (32-row corpus blocks) per segment, prefix sums
    uint32_t nseg;
    uint64_t total_blocks;
    const VerifySeg* vsegs;
    uint32_t nvseg;
    const DecodeQuery* dq;
    const TcBlock* tc_blocks;
    uint32_t nblocks;
    const TcPanel* tc_panels;
    uint32_t npanels;
    const uint32_t* seg_panel0;
    const uint32_t* seg_block0;
    const TcMaps* maps;
};
struct Scratch {  // device pointers
    QLimb* limbs;
    uint64_t* x;
    uint64_t* r;
    uint64_t* z_part;
    uint64_t* ur_part;
    uint32_t* flags;
    uint64_t* ur;
    uint64_t* zv;
    TopkScratch topk;
    uint32_t* err;  // device pipeline timeout flags
    uint8_t* u_buf;
    uint64_t* r_part;  // fused pass: per strip-group partial dots
    uint64_t* zv_chunks;
    uint8_t* wimg;     // fused pass: diagonal byte images of the queries
};
struct Inputs {
    const uint64_t* v;
    const uint64_t* g;
    const uint32_t* t;
    const uint32_t* t_nnz;
    const uint8_t* seeds;
};
struct Outputs {
    uint32_t* ids;
    int64_t* scores;
    uint32_t* n;
    int32_t* vfailed;  // per verify segment
    uint64_t* mv;      // nullable
};

struct HostMeta {
    std::vector<ScanSeg> segs;
    std::vector<uint64_t> seg_blk;
    std::vector<uint64_t> seg_unit;     // prefix sums of the 32-row corpus blocks each segment touches
    std::vector<VerifySeg> vsegs;
    std::vector<DecodeQuery> dq;
    std::vector<uint32_t> seg_cluster;  // IVF: list id of each segment
    std::vector<TcBlock> blocks;        // 128-row blocks of every verify segment
    std::vector<TcPanel> panels;        // 4096-row panels of every verify segment
    std::vector<uint32_t> seg_block0, seg_panel0;
    uint64_t total_out = 0, max_rows = 0;
};

struct Sizes {
    uint32_t B, n1, trials, k, ctas;  // ctas: decode CTAs of all queries together
    uint64_t total_out, nseg, nvseg, nblocks, npanels;
    FreivaldsPlan fp;  // CUDA-core engine
    int engine;        // BN_ENGINE_*
};


// Offsets of every device buffer of one pipeline run.
struct RunLayout {
    // inputs (contiguous from 0 -> one H2D)
    uint64_t v, g, t, t_nnz, seeds, segs, seg_blk, seg_unit, vsegs, dq, tc_blocks, tc_panels, seg_panel0, seg_block0,
        in_end;
    // outputs (contiguous -> one D2H)
    uint64_t ids, scores, n, vfailed, ur, zv, err, out_begin, out_end;
    // internal
    uint64_t limbs, x, r, mv, z_part, ur_part, flags, cand_s, cand_i, cand_n, cand_done, u_buf, r_part, zv_chunks, wimg,
        total;
};

// One run of the query pipeline over host inputs (bn_capi.cu): hm is the
// segment metadata of the B queries, kept alive by the caller.
struct QueryJob {
    HostMeta* hm = nullptr;  // job_prepare assigns the decode CTAs into it
    uint32_t B = 0, trials = 0, k = 0;
    bool want_mv = false;
    Sizes z{};
    RunLayout o{};
    TcMaps maps;
};
void finish_meta(HostMeta& hm);
void flat_meta(uint64_t m, uint32_t B, HostMeta& hm);
Sizes sizes_for(const Engine& e, HostMeta& hm, uint32_t B, uint32_t trials, uint32_t k);
RunLayout make_layout(const Sizes& z, bool want_mv);
// Validates and packs the inputs into host (pinned, grown as needed) and
// sizes ws (grown as needed, budget-accounted).
int job_prepare(Engine& e, QueryJob& j, DevMem& ws, PinnedMem& host, const uint64_t* v_enc, const uint64_t* g,
                const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds);
// Enqueues H2D, the pipeline and the D2H of the outputs on s; waits for nothing.
int job_launch(Engine& e, QueryJob& j, DevMem& ws, PinnedMem& host, cudaStream_t s, uint64_t* r_out, uint64_t* mv_out);
// After s has drained: device flags, hits (k per query) and per-segment verdicts.
int job_finish(const QueryJob& j, const PinnedMem& host, uint32_t* ids, int64_t* scores, uint32_t* n_hits,
               std::vector<int32_t>& vfailed);

// Block scoring (bn_block.cu).
struct BlockPlan;
void block_plan_free(BlockPlan* b);

// IVF block scoring (bn_ivf_block.cu): plan (host), pack (pinned staging +
// workspace sizing), launch (H2D, pipeline, D2H on s), finish (after s drained).
struct IvfBlockJob;
IvfBlockJob* ivf_block_job_new();
void ivf_block_job_free(IvfBlockJob* j);
uint64_t ivf_block_job_bytes(const IvfBlockJob* j);
int ivf_block_plan(const bn_ivf& v, IvfBlockJob& j, uint32_t B, const uint32_t* probe_off, const uint32_t* probes,
                   uint32_t trials, uint32_t k, bool verify_only, int sms);
int ivf_block_pack(Engine& e, IvfBlockJob& j, DevMem& ws, PinnedMem& host, const uint64_t* v_enc, const uint64_t* g,
                   const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* seed);
// ev (nullable): 9 events recorded on s at the stage boundaries (start; operand
// images; G1; G2; G3; top-k; Protocol 2 passes; z . v and verdicts; D2H).
int ivf_block_launch(Engine& e, IvfBlockJob& j, DevMem& ws, PinnedMem& host, cudaStream_t s,
                     cudaEvent_t* ev = nullptr);
int ivf_block_finish(const IvfBlockJob& j, const PinnedMem& host, uint32_t* ids, int64_t* scores, uint32_t* n_hits,
                     int32_t* failed_cluster, int32_t* failed_trial);
int ivf_block_prepare(bn_ivf* v);

}  // namespace api
}  // namespace bn

// ------------------------------------------------------------------ handles
struct bn_flat {
    bn::api::Engine e;
    uint64_t m = 0;
    // segment metadata of the last bn_flat_query batch size (rebuilding it
    // walks every 128-row block of the corpus: tens of us per call at 1M rows)
    bn::api::HostMeta query_meta;
    uint32_t query_meta_B = 0;
    // block plan cached by the host-buffer block entry points
    bn::api::BlockPlan* block_cache = nullptr;
    uint32_t cache_B = 0, cache_trials = 0, cache_k = 0, cache_flags = 0;
    std::mutex block_mu;
    ~bn_flat() {
        if (block_cache) bn::api::block_plan_free(block_cache);
    }
};

struct bn_ivf {
    bn::api::Engine e;
    uint32_t nlist = 0;
    std::vector<uint64_t> offsets;
    // routing (bn_ivf_set_centroids): centroids dimension-major, [cent_d][nlist] f32
    bn::api::DevMem cent_t;
    uint32_t cent_d = 0;
    // block GEMM tiling chosen by the caller (bn_ivf_block_tune; 0 = automatic)
    uint32_t blk_w = 0, blk_stages = 0;
    // stage timing of the host-buffer IVF block entry point (bn_ivf_block_profile)
    static constexpr int PROF_EVENTS = 11;
    bool prof = false, prof_have = false;
    cudaEvent_t prof_ev[PROF_EVENTS] = {};
    float prof_host_ms = 0.f;
    ~bn_ivf() {
        for (cudaEvent_t ev : prof_ev)
            if (ev) cudaEventDestroy(ev);
    }
};


namespace bn {
namespace api {
int block_prepare(bn_flat* f);
constexpr uint32_t BLOCK_VERIFY_ONLY = 1u << 31;  // internal block_plan_create flag
int block_plan_create(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k, uint32_t flags, BlockPlan** out);
void block_plan_config(const BlockPlan* b, uint32_t cfg[6], float tuned_ms[2]);
int block_plan_status(BlockPlan* b, uint32_t* flags);
int block_enqueue(BlockPlan& b, const uint64_t* d_v, const uint64_t* d_g, const uint32_t* d_t, const uint32_t* d_tn,
                  const uint8_t* d_seed, uint32_t* d_ids, int64_t* d_scores, uint32_t* d_n, int32_t* d_failed,
                  cudaStream_t s, bool want_mv);
int block_query_host(BlockPlan& b, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                     const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* seed, uint32_t* ids, int64_t* scores,
                     uint32_t* n_hits, int32_t* failed, uint64_t* mv_out);
int block_query_launch(BlockPlan& b, uint32_t nq, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                       const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* seed, cudaStream_t s, bool want_mv);
int block_query_finish(BlockPlan& b, uint32_t nq, uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed);
uint64_t block_plan_bytes(const BlockPlan* b);
uint64_t block_plan_estimate(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k);
// Byte-planar corpus copies of block scoring (once per handle; caller holds
// e.mu); offsets (nullable): the IVF list boundaries.
int block_prepare_engine(Engine& e, const std::vector<uint64_t>* offsets);
int pick_ctas(uint64_t max_rows_per_query, uint32_t B, int sms);
int validate_residues(const uint64_t* a, uint64_t count, const char* what);
// bn_ivf_build_keygen over lists whose global indices start at list0 (the
// keys of list c are drawn from derive_h_seed(upload_seed, list0 + c)).
int ivf_build_keygen_from(bn_ctx* ctx, uint32_t nlist, const uint64_t* off, const uint32_t* ids, const uint64_t* m_q,
                          uint32_t n, uint32_t n1, const uint64_t* L, uint64_t upload_seed, uint32_t list0,
                          bn_ivf** out);
int engine_init(Engine& e, bn_ctx* ctx);
void engine_free(Engine& e);
int corpus_tmap(Corpus& c);
int check_shape(uint32_t n, uint32_t n1);
int block_verify_host(BlockPlan& b, const uint64_t* r, const uint64_t* v_enc, const uint8_t* seed, int32_t* failed,
                      uint64_t* ur, uint64_t* zv);
}  // namespace api
}  // namespace bn
