// bn_server.cu -- the serving loop: continuous batching of flat and IVF
// queries over device-resident corpora.
//
// The reference serves each request by calling the scorer once per query
// (BnTmScorer::score, lib.rs:326-475; BnTmIvfScorer::score, ivf.rs:746-927)
// with every GPU call synchronous on one stream (gpu/mod.rs:169-200).  Here
// requests are queued on submit and a scheduler thread keeps up to `slots`
// batches in flight, one CUDA stream and one workspace per slot:
//   - a slot that frees up takes the next batch at once: up to max_batch
//     queued requests of one corpus (IVF requests with different nprobe share
//     a batch: every probed list of every query is its own segment), after
//     waiting at most max_wait_us for the batch to fill;
//   - flat block plans are pooled across slots, one per block size and
//     concurrent use, and kept, so a small batch runs a small block (or
//     pads into an idle larger one rather than creating a plan while
//     batches are in flight);
//   - admission is by device memory: a batch's workspace (the pipeline's
//     layout for exactly those requests, or a new block plan) must fit in
//     mem_budget together with what the slots and the plan pool hold;
//     otherwise it is cut shorter or waits for a slot to drain (idle slots and
//     plans give their memory back);
//   - admission is also by queue: a submit is refused with BN_EAGAIN when
//     max_queue requests wait, or when the expected wait (waiting requests
//     over the completion rate of the recent batches) exceeds queue_wait_us;
//   - each query's hits depend only on its own inputs (its own segments,
//     decode and top-k), so they are the same alone and in any mix; a
//     per-query batch verifies each query with its own seed, a block batch
//     with one seed derived from all its members' seeds.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "bn_host.h"
#include "bn_internal.cuh"

using namespace bn;
using namespace bn::api;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    int kind = 0;  // BN_SERVER_FLAT / BN_SERVER_IVF
    std::vector<uint64_t> v, g;
    std::vector<uint32_t> t_idx, probes;
    std::vector<int8_t> t_sign;
    uint8_t seed[32];
    Clock::time_point t_submit;
};

struct Result {
    int status = BN_OK;
    std::string error;
    std::vector<uint32_t> ids;
    std::vector<int64_t> scores;
    int32_t failed_trial = -1, failed_cluster = -1;
    double latency_us = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    DevMem ws;
    PinnedMem host;
    bool busy = false;
    int kind = 0;
    std::vector<Request> reqs;
    HostMeta hm;
    QueryJob job;
    // block scoring of flat batches: the index of the pooled plan in use
    int plan = -1;
    bool block_run = false;
    // block scoring of IVF batches (pairs grouped by list), in ws / host
    IvfBlockJob* ivj = nullptr;
    bool ivf_block_run = false;
    // ivj holds the host plan of these requests (the first one's ticket and
    // the count): planned while sizing the batch, reused by its launch
    uint64_t ivj_ticket0 = 0;
    size_t ivj_count = 0;
    ~Slot() {
        if (ivj) ivf_block_job_free(ivj);
    }
};

// A block plan of the server's pool: one per block size (8, 16, 32, ...)
// and concurrent use, lent to a slot for one batch.
struct PooledPlan {
    BlockPlan* bp = nullptr;
    uint32_t B = 0;
    bool busy = false;
};

}  // namespace

struct bn_server {
    bn_flat* flat = nullptr;
    bn_ivf* ivf = nullptr;
    bn_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> pending[2];
    std::unordered_map<uint64_t, Result> results;
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<PooledPlan> plans;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread sched;
    // statistics
    uint64_t submitted = 0, completed = 0, batches = 0, batched_queries = 0, block_batches = 0, peak_mem = 0;
    bool block_off = false;      // block scoring refused by the flat corpus: per-query path only
    bool ivf_block_off = false;  // the same for the IVF corpus
    std::vector<double> lat_us;
    Clock::time_point t_first{}, t_last{};
    uint64_t rejected = 0;
    // completion times and sizes of the recent batches (queue admission)
    std::deque<std::pair<Clock::time_point, uint32_t>> recent;
    ~bn_server() {
        for (PooledPlan& pp : plans) block_plan_free(pp.bp);
    }
};

namespace {

Engine& engine_of(bn_server* s, int kind) { return kind == BN_SERVER_FLAT ? s->flat->e : s->ivf->e; }

// Segment metadata of a batch (flat: one segment per query over the whole
// corpus; IVF: one per non-empty probed list, in probe order).
template <class It>
void batch_meta(bn_server* s, int kind, It first, It last, HostMeta& hm) {
    const uint32_t B = (uint32_t)(last - first);
    if (kind == BN_SERVER_FLAT) {
        flat_meta(s->flat->m, B, hm);
        return;
    }
    hm = HostMeta();
    uint64_t out = 0;
    const bn_ivf* v = s->ivf;
    for (uint32_t b = 0; b < B; ++b) {
        const uint32_t seg0 = (uint32_t)hm.segs.size();
        for (uint32_t ci : first[b].probes) {
            const uint64_t row0 = v->offsets[ci], m = v->offsets[ci + 1] - row0;
            if (!m) continue;  // ivf.rs:787-789 skips empty clusters
            hm.segs.push_back(ScanSeg{row0, out, (uint32_t)m, b});
            hm.vsegs.push_back(VerifySeg{row0, out, (uint32_t)m, b});
            hm.seg_cluster.push_back(ci);
            hm.max_rows = std::max(hm.max_rows, m);
            out += m;
        }
        hm.dq.push_back(DecodeQuery{seg0, (uint32_t)hm.segs.size() - seg0});
    }
    hm.total_out = out;
    finish_meta(hm);
}

uint32_t block_bucket(bn_server* s, size_t count);
uint64_t held_bytes(bn_server* s);
int pool_find(const bn_server* s, uint32_t bucket, bool exact);

// IVF batches of at least block_min requests run as IVF block scoring.
bool ivf_block(const bn_server* s, size_t count) {
    return s->cfg.block_min && count >= s->cfg.block_min && !s->ivf_block_off;
}

// Host plan of an IVF block over requests [first, first + count).
template <class It>
int ivf_block_plan_reqs(bn_server* s, It first, size_t count, IvfBlockJob& j) {
    std::vector<uint32_t> off(count + 1, 0), probes;
    for (size_t b = 0; b < count; ++b) {
        probes.insert(probes.end(), first[b].probes.begin(), first[b].probes.end());
        off[b + 1] = (uint32_t)probes.size();
    }
    return ivf_block_plan(*s->ivf, j, (uint32_t)count, off.data(), probes.data(), s->cfg.trials, s->cfg.k, false,
                          s->ivf->e.ctx->num_sms);
}

// Device workspace of a batch made of the first `count` requests of q (a
// block plan's workspace when the batch runs as a block).  An IVF block's
// host plan is made in `me`'s job and kept for the launch.
uint64_t batch_bytes(bn_server* s, int kind, const std::deque<Request>& q, size_t count, Slot* me) {
    if (kind == BN_SERVER_FLAT)
        if (const uint32_t bucket = block_bucket(s, count))
            return block_plan_estimate(s->flat, bucket, s->cfg.trials, s->cfg.k);
    if (kind == BN_SERVER_IVF && ivf_block(s, count)) {
        if (me) {
            if (!me->ivj) me->ivj = ivf_block_job_new();
            me->ivj_count = 0;
            if (ivf_block_plan_reqs(s, q.begin(), count, *me->ivj) == BN_OK) {
                me->ivj_ticket0 = q.front().ticket;
                me->ivj_count = count;
                return ivf_block_job_bytes(me->ivj);
            }
        } else {
            std::unique_ptr<IvfBlockJob, void (*)(IvfBlockJob*)> j(ivf_block_job_new(), ivf_block_job_free);
            if (ivf_block_plan_reqs(s, q.begin(), count, *j) == BN_OK) return ivf_block_job_bytes(j.get());
        }
    }
    HostMeta hm;
    batch_meta(s, kind, q.begin(), q.begin() + count, hm);
    const Sizes z = sizes_for(engine_of(s, kind), hm, (uint32_t)count, s->cfg.trials, s->cfg.k);
    return make_layout(z, false).total;
}

void complete(bn_server* s, std::vector<Request>& reqs, const std::vector<Result>& res) {
    const auto now = Clock::now();
    for (size_t i = 0; i < reqs.size(); ++i) {
        Result r = res[i];
        r.latency_us = std::chrono::duration<double, std::micro>(now - reqs[i].t_submit).count();
        s->lat_us.push_back(r.latency_us);
        s->results[reqs[i].ticket] = std::move(r);
    }
    s->completed += reqs.size();
    s->t_last = now;
    s->recent.emplace_back(now, (uint32_t)reqs.size());
    while (s->recent.size() > 32) s->recent.pop_front();
}

// Completion rate of the recent batches (queries per second; 0 = unknown).
double recent_rate(const bn_server* s) {
    if (s->recent.size() < 4) return 0.0;
    uint64_t n = 0;
    for (size_t i = 1; i < s->recent.size(); ++i) n += s->recent[i].second;
    const double span = std::chrono::duration<double>(s->recent.back().first - s->recent.front().first).count();
    return span > 0 ? (double)n / span : 0.0;
}

// The Protocol 2 seed of a block batch: domain_separate of the XOR of its
// members' seeds, so every member's seed takes part and the seed of the batch
// is a function of its members alone.
void block_seed(const std::vector<uint8_t>& seeds, uint32_t B, uint8_t out[32]) {
    uint8_t x[32] = {0};
    for (uint32_t b = 0; b < B; ++b)
        for (int i = 0; i < 32; ++i) x[i] ^= seeds[(uint64_t)b * 32 + i];
    bn_host_domain_separate(x, "serve-block", out);
}

// Reads a finished slot's outputs (called with s->mu held).
void harvest(bn_server* s, Slot& sl) {
    const uint32_t B = (uint32_t)sl.reqs.size(), k = s->cfg.k, ks = std::max<uint32_t>(k, 1);
    std::vector<uint32_t> ids((uint64_t)B * ks), nh(B);
    std::vector<int64_t> sc((uint64_t)B * ks);
    std::vector<int32_t> vf;
    std::vector<Result> res(B);
    int rc = cudaEventSynchronize(sl.done) == cudaSuccess ? BN_OK : fail(BN_ECUDA, "batch failed on the device");
    std::vector<int32_t> bf(B, -1), bc(B, -1);
    if (rc == BN_OK)
        rc = sl.block_run       ? block_query_finish(*s->plans[sl.plan].bp, B, ids.data(), sc.data(), nh.data(), bf.data())
             : sl.ivf_block_run ? ivf_block_finish(*sl.ivj, sl.host, ids.data(), sc.data(), nh.data(), bc.data(),
                                                   bf.data())
                                : job_finish(sl.job, sl.host, ids.data(), sc.data(), nh.data(), vf);
    for (uint32_t b = 0; b < B; ++b) {
        Result& r = res[b];
        r.status = rc;
        if (rc != BN_OK) {
            r.error = bn_last_error();
            continue;
        }
        r.ids.assign(ids.begin() + (uint64_t)b * k, ids.begin() + (uint64_t)b * k + nh[b]);
        r.scores.assign(sc.begin() + (uint64_t)b * k, sc.begin() + (uint64_t)b * k + nh[b]);
        if (sl.block_run || sl.ivf_block_run) {
            r.failed_trial = bf[b];
            r.failed_cluster = bc[b];
            continue;
        }
        const DecodeQuery& dq = sl.hm.dq[b];
        for (uint32_t g = dq.seg0; g < dq.seg0 + dq.nseg; ++g)
            if (vf[g] >= 0) {
                r.failed_trial = vf[g];
                r.failed_cluster = sl.kind == BN_SERVER_IVF ? (int32_t)sl.hm.seg_cluster[g] : -1;
                break;
            }
    }
    complete(s, sl.reqs, res);
    sl.reqs.clear();
    sl.busy = false;
    if (sl.plan >= 0) s->plans[sl.plan].busy = false;
    sl.plan = -1;
}

// Packs and launches one batch on a free slot (called with s->mu held; the
// launch itself only enqueues work).
int launch(bn_server* s, Slot& sl, int kind, std::vector<Request>&& reqs) {
    const uint32_t B = (uint32_t)reqs.size();
    sl.reqs = std::move(reqs);
    sl.kind = kind;
    batch_meta(s, kind, sl.reqs.begin(), sl.reqs.end(), sl.hm);
    const uint32_t n1 = engine_of(s, kind).c.n1;
    std::vector<uint64_t> v((uint64_t)B * N), g((uint64_t)B * n1);
    std::vector<uint32_t> tn(B), ti;
    std::vector<int8_t> ts;
    std::vector<uint8_t> seeds((uint64_t)B * 32);
    for (uint32_t b = 0; b < B; ++b) {
        const Request& r = sl.reqs[b];
        memcpy(&v[(uint64_t)b * N], r.v.data(), N * 8);
        memcpy(&g[(uint64_t)b * n1], r.g.data(), (uint64_t)n1 * 8);
        tn[b] = (uint32_t)r.t_idx.size();
        ti.insert(ti.end(), r.t_idx.begin(), r.t_idx.end());
        ts.insert(ts.end(), r.t_sign.begin(), r.t_sign.end());
        memcpy(&seeds[(uint64_t)b * 32], r.seed, 32);
    }
    int rc = BN_OK;
    const uint32_t bucket = kind == BN_SERVER_FLAT ? block_bucket(s, B) : 0;
    sl.block_run = false;
    sl.ivf_block_run = false;
    uint8_t bseed[32];
    block_seed(seeds, B, bseed);
    if (kind == BN_SERVER_IVF && ivf_block(s, B)) {
        // IVF block scoring: the batch's (query, list) pairs grouped by list,
        // every probed list read once; Protocol 2 per block and list with the
        // batch seed
        if (!sl.ivj) sl.ivj = ivf_block_job_new();
        Engine& e = s->ivf->e;
        if (!(sl.ivj_count == B && sl.ivj_ticket0 == sl.reqs.front().ticket))  // not planned while sizing
            rc = ivf_block_plan_reqs(s, sl.reqs.begin(), B, *sl.ivj);
        sl.ivj_count = 0;
        if (rc == BN_OK)
            rc = ivf_block_pack(e, *sl.ivj, sl.ws, sl.host, v.data(), g.data(), ti.empty() ? nullptr : ti.data(),
                                ts.empty() ? nullptr : ts.data(), tn.data(), bseed);
        if (rc == BN_OK) rc = ivf_block_launch(e, *sl.ivj, sl.ws, sl.host, sl.stream);
        if (rc == BN_OK) {
            sl.ivf_block_run = true;
            s->block_batches += 1;
        }
    }
    if (bucket) {
        // block scoring: the batch's queries share one pass over the corpus;
        // Protocol 2 runs per block with the batch seed.  Plans are pooled
        // and kept (creating plans or freeing device memory mid-stream
        // synchronises the device and stalls every slot): an idle plan of
        // the batch's own size, else an idle larger one padded with zero
        // queries, else a new one.
        int pi = pool_find(s, bucket, true);
        if (pi < 0) pi = pool_find(s, bucket, false);
        if (pi < 0) {
            BlockPlan* bp = nullptr;
            rc = block_plan_create(s->flat, bucket, s->cfg.trials, s->cfg.k, 0, &bp);
            if (rc == BN_OK) {
                s->plans.push_back(PooledPlan{bp, bucket, false});
                pi = (int)s->plans.size() - 1;
            }
        }
        if (rc == BN_OK) {
            sl.block_run = true;
            sl.plan = pi;
            s->plans[pi].busy = true;
            rc = block_query_launch(*s->plans[pi].bp, B, v.data(), g.data(), ti.empty() ? nullptr : ti.data(),
                                    ts.empty() ? nullptr : ts.data(), tn.data(), bseed, sl.stream, false);
            if (rc == BN_OK) s->block_batches += 1;
        } else if (rc == BN_EUNSUPPORTED) {
            s->block_off = true;  // e.g. plaintext outside int8: serve flat queries per query from now on
            rc = BN_OK;
        }
    }
    if (!sl.block_run && !sl.ivf_block_run && rc == BN_OK) {
        sl.job = QueryJob();
        sl.job.hm = &sl.hm;
        sl.job.B = B;
        sl.job.trials = s->cfg.trials;
        sl.job.k = s->cfg.k;
        Engine& e = engine_of(s, kind);
        rc = job_prepare(e, sl.job, sl.ws, sl.host, v.data(), g.data(), ti.empty() ? nullptr : ti.data(),
                         ts.empty() ? nullptr : ts.data(), tn.data(), seeds.data());
        if (rc == BN_OK) rc = job_launch(e, sl.job, sl.ws, sl.host, sl.stream, nullptr, nullptr);
    }
    if (rc == BN_OK && cudaEventRecord(sl.done, sl.stream) != cudaSuccess) rc = fail(BN_ECUDA, "cudaEventRecord failed");
    if (rc != BN_OK) {
        std::vector<Result> res(B);
        for (auto& r : res) {
            r.status = rc;
            r.error = bn_last_error();
        }
        complete(s, sl.reqs, res);
        sl.reqs.clear();
        return rc;
    }
    sl.busy = true;
    s->batches += 1;
    s->batched_queries += B;
    return BN_OK;
}

uint64_t held_bytes(bn_server* s) {
    uint64_t t = 0;
    for (auto& sl : s->slots) t += sl->ws.bytes;
    for (const PooledPlan& pp : s->plans) t += block_plan_bytes(pp.bp);
    return t;
}

// An idle pooled plan for blocks of `bucket` queries (exact) or of the
// fewest queries at least `bucket` (not exact); -1 if none.
int pool_find(const bn_server* s, uint32_t bucket, bool exact) {
    int best = -1;
    for (size_t i = 0; i < s->plans.size(); ++i) {
        const PooledPlan& pp = s->plans[i];
        if (pp.busy || pp.B < bucket || (exact && pp.B != bucket)) continue;
        if (best < 0 || pp.B < s->plans[best].B) best = (int)i;
    }
    return best;
}

// Block size a flat batch of `count` requests runs as (0: per-query path).
uint32_t block_bucket(bn_server* s, size_t count) {
    if (!s->cfg.block_min || count < s->cfg.block_min || s->block_off) return 0;
    uint32_t b = 8;
    while (b < count) b <<= 1;
    return b;
}

// One scheduling decision for a free slot: the batch to launch (empty: none now).
std::vector<Request> take_batch(bn_server* s, Slot& me, int& kind_out, bool& reject_front, int& reject_kind) {
    reject_front = false;
    // the corpus whose oldest request waited longest goes first
    int kind = -1;
    for (int k = 0; k < 2; ++k)
        if (!s->pending[k].empty() && (kind < 0 || s->pending[k].front().t_submit < s->pending[kind].front().t_submit))
            kind = k;
    if (kind < 0) return {};
    std::deque<Request>& q = s->pending[kind];
    // batching window: wait for more arrivals unless the batch is full or old enough
    const double age_us = std::chrono::duration<double, std::micro>(Clock::now() - q.front().t_submit).count();
    if (q.size() < s->cfg.max_batch && age_us < s->cfg.max_wait_us) return {};
    // memory admission: the largest prefix whose workspace fits beside the
    // memory held by the other slots and the plan pool.  A flat block reuses
    // an idle pooled plan of its size, else needs a new one (or, when that
    // does not fit, pads into an idle larger one) and keeps this slot's
    // workspace; a per-query or IVF batch grows this slot's workspace.
    const uint64_t others = held_bytes(s) - me.ws.bytes;
    const uint64_t budget = s->cfg.mem_budget;
    auto need = [&](size_t cnt) -> uint64_t {
        const uint32_t bucket = kind == BN_SERVER_FLAT ? block_bucket(s, cnt) : 0;
        if (bucket) {
            if (pool_find(s, bucket, false) >= 0) return me.ws.bytes;  // an idle plan of this size or larger
            return me.ws.bytes + batch_bytes(s, kind, q, cnt, &me);
        }
        return DevMem::grown(me.ws.bytes, batch_bytes(s, kind, q, cnt, &me));  // reserve_grow's size
    };
    size_t count = std::min<size_t>(q.size(), s->cfg.max_batch);
    while (count > 0 && budget && others + need(count) > budget) count = count > 8 ? count / 2 : count - 1;
    if (count == 0) {
        bool any_busy = false;
        for (auto& sl : s->slots) any_busy |= sl->busy;
        if (!any_busy) {
            // idle slots and plans keep their memory: give it back, then retry once
            for (auto& sl : s->slots) sl->ws.release();
            for (PooledPlan& pp : s->plans) block_plan_free(pp.bp);
            s->plans.clear();
            if (batch_bytes(s, kind, q, 1, nullptr) + held_bytes(s) > budget) {
                reject_front = true;  // this request alone exceeds the budget
                reject_kind = kind;
            } else {
                count = 1;
            }
        }
        if (count == 0) return {};
    }
    std::vector<Request> reqs;
    for (size_t i = 0; i < count; ++i) {
        reqs.push_back(std::move(q.front()));
        q.pop_front();
    }
    kind_out = kind;
    return reqs;
}

void scheduler(bn_server* s) {
    cudaSetDevice((s->flat ? s->flat->e : s->ivf->e).ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        // completions
        for (auto& sp : s->slots)
            if (sp->busy && cudaEventQuery(sp->done) != cudaErrorNotReady) {
                harvest(s, *sp);
                progressed = true;
            }
        if (progressed) s->cv_done.notify_all();
        // launches on free slots
        for (auto& sp : s->slots) {
            Slot& sl = *sp;
            if (sl.busy) continue;
            int kind = 0, rkind = 0;
            bool reject = false;
            std::vector<Request> reqs = take_batch(s, sl, kind, reject, rkind);
            if (reject) {
                Request r = std::move(s->pending[rkind].front());
                s->pending[rkind].pop_front();
                std::vector<Request> one;
                one.push_back(std::move(r));
                Result res;
                res.status = fail(BN_EBUDGET, "request needs more device memory than the server budget");
                res.error = bn_last_error();
                complete(s, one, {res});
                s->cv_done.notify_all();
                progressed = true;
                continue;
            }
            if (reqs.empty()) break;
            launch(s, sl, kind, std::move(reqs));
            if (!sl.busy) s->cv_done.notify_all();  // the batch failed to launch: its requests are answered
            progressed = true;
        }
        s->peak_mem = std::max(s->peak_mem, held_bytes(s));
        bool any_busy = false;
        for (auto& sl : s->slots) any_busy |= sl->busy;
        const bool any_pending = !s->pending[0].empty() || !s->pending[1].empty();
        if (s->stop && !any_busy && !any_pending) break;
        if (progressed) continue;
        // nothing to do right now: poll in-flight batches often, idle otherwise
        s->cv_work.wait_for(lk, any_busy || any_pending ? std::chrono::microseconds(20) : std::chrono::milliseconds(5));
    }
}

int validate_request(const bn_server* s, const Engine& e, const uint64_t* v_enc, const uint64_t* g,
                     const uint32_t* t_idx, const int8_t* t_sign, uint32_t t_nnz, const uint8_t* seed) {
    if (!v_enc || !g || (t_nnz && (!t_idx || !t_sign)) || (s->cfg.trials && !seed))
        return fail(BN_EINVAL, "null request input");
    if (t_nnz > N) return fail(BN_EINVAL, "t_nnz = %u exceeds n", t_nnz);
    for (uint32_t i = 0; i < N; ++i)
        if (v_enc[i] >= P) return fail(BN_EINVAL, "v_enc[%u] is not a canonical residue", i);
    for (uint32_t i = 0; i < e.c.n1; ++i)
        if (g[i] >= P) return fail(BN_EINVAL, "g[%u] is not a canonical residue", i);
    for (uint32_t i = 0; i < t_nnz; ++i)
        if (t_idx[i] >= N || (t_sign[i] != 1 && t_sign[i] != -1)) return fail(BN_EINVAL, "T entry %u is invalid", i);
    return BN_OK;
}

int submit(bn_server* s, int kind, Request&& r, uint64_t* ticket) {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return fail(BN_EINVAL, "server is stopping");
    const size_t waiting = s->pending[0].size() + s->pending[1].size();
    if (s->cfg.max_queue && waiting >= s->cfg.max_queue) {
        s->rejected += 1;
        return fail(BN_EAGAIN, "queue full (%zu requests waiting)", waiting);
    }
    if (s->cfg.queue_wait_us) {
        const double rate = recent_rate(s);
        if (rate > 0 && (double)waiting / rate * 1e6 > (double)s->cfg.queue_wait_us) {
            s->rejected += 1;
            return fail(BN_EAGAIN, "expected queue wait %.0f us exceeds %u us", (double)waiting / rate * 1e6,
                        s->cfg.queue_wait_us);
        }
    }
    r.ticket = s->next_ticket++;
    r.t_submit = Clock::now();
    if (s->submitted == 0) s->t_first = r.t_submit;
    s->submitted += 1;
    *ticket = r.ticket;
    s->pending[kind].push_back(std::move(r));
    s->cv_work.notify_one();
    return BN_OK;
}

void fill_request(Request& r, int kind, const Engine& e, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                  const int8_t* t_sign, uint32_t t_nnz, const uint8_t* seed) {
    r.kind = kind;
    r.v.assign(v_enc, v_enc + N);
    r.g.assign(g, g + e.c.n1);
    r.t_idx.assign(t_idx, t_idx + t_nnz);
    r.t_sign.assign(t_sign, t_sign + t_nnz);
    if (seed) memcpy(r.seed, seed, 32);
    else memset(r.seed, 0, 32);
}

}  // namespace

extern "C" {

int bn_server_create(bn_flat* flat, bn_ivf* ivf, const bn_server_config* cfg, bn_server** out) {
    if (!out || !cfg) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    if (!flat && !ivf) return fail(BN_EINVAL, "a server needs a flat or an IVF corpus");
    if (flat && !flat->e.c.client) return fail(BN_EUNSUPPORTED, "the flat handle has no client state");
    if (ivf && !ivf->e.c.client) return fail(BN_EUNSUPPORTED, "the IVF handle has no client state");
    if (flat && ivf && flat->e.ctx != ivf->e.ctx) return fail(BN_EINVAL, "both corpora must live in one context");
    if (!cfg->max_batch || cfg->max_batch > 4096) return fail(BN_EINVAL, "max_batch must be in 1..=4096");
    if (!cfg->slots || cfg->slots > 16) return fail(BN_EINVAL, "slots must be in 1..=16");
    if (cfg->k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX", cfg->k);
    if (cfg->trials > BN_MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %d", cfg->trials, BN_MAX_TRIALS);
    auto* s = new bn_server();
    s->flat = flat;
    s->ivf = ivf;
    s->cfg = *cfg;
    for (uint32_t i = 0; i < cfg->slots; ++i) s->slots.push_back(std::make_unique<Slot>());
    bn_ctx* ctx = (flat ? flat->e : ivf->e).ctx;
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        delete s;
        return fail(BN_ECUDA, "cudaSetDevice failed");
    }
    for (auto& sl : s->slots) {
        if (cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming) != cudaSuccess) {
            for (auto& x : s->slots) {
                if (x->stream) cudaStreamDestroy(x->stream);
                if (x->done) cudaEventDestroy(x->done);
            }
            delete s;
            return fail(BN_ECUDA, "stream / event creation failed");
        }
        sl->ws.ctx = ctx;
        sl->ws.stream = sl->stream;  // grows in the slot's stream order, with no device-wide sync
        sl->host.keep_retired = true;  // and its staging buffer without a cudaFreeHost while batches run
    }
    if (cfg->block_min) {
        // byte-planar corpus copies of block scoring, built now rather than
        // inside the first block batch; a corpus that cannot take them
        // (plaintext outside int8) is served per query
        if (flat && block_prepare(flat) == BN_EUNSUPPORTED) s->block_off = true;
        if (ivf && ivf_block_prepare(ivf) == BN_EUNSUPPORTED) s->ivf_block_off = true;
        // pooled plans now: one per block size, smallest first, then more
        // of the largest size until every slot could run one, while they fit
        // in half the budget; creating one later stalls the device while
        // batches are in flight
        if (flat && !s->block_off) {
            uint64_t held = 0;
            const uint32_t top = block_bucket(s, cfg->max_batch);
            auto add = [&](uint32_t b) {
                const uint64_t need = block_plan_estimate(flat, b, cfg->trials, cfg->k);
                if (cfg->mem_budget && 2 * (held + need) > cfg->mem_budget) return false;
                BlockPlan* bp = nullptr;
                if (block_plan_create(flat, b, cfg->trials, cfg->k, 0, &bp) != BN_OK) return false;
                s->plans.push_back(PooledPlan{bp, b, false});
                held += block_plan_bytes(bp);
                return true;
            };
            bool ok = true;
            for (uint32_t b = block_bucket(s, cfg->block_min); ok && b && b <= top; b <<= 1) ok = add(b);
            for (uint32_t i = 1; ok && top && i < cfg->slots; ++i) ok = add(top);
        }
    }
    s->sched = std::thread(scheduler, s);
    *out = s;
    return BN_OK;
}

int bn_server_submit_flat(bn_server* s, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                          const int8_t* t_sign, uint32_t t_nnz, const uint8_t* v_seed, uint64_t* ticket) {
    if (!s || !ticket) return fail(BN_EINVAL, "null argument");
    if (!s->flat) return fail(BN_EUNSUPPORTED, "this server has no flat corpus");
    TRY(validate_request(s, s->flat->e, v_enc, g, t_idx, t_sign, t_nnz, v_seed));
    Request r;
    fill_request(r, BN_SERVER_FLAT, s->flat->e, v_enc, g, t_idx, t_sign, t_nnz, v_seed);
    return submit(s, BN_SERVER_FLAT, std::move(r), ticket);
}

int bn_server_submit_ivf(bn_server* s, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc, const uint64_t* g,
                         const uint32_t* t_idx, const int8_t* t_sign, uint32_t t_nnz, const uint8_t* v_seed,
                         uint64_t* ticket) {
    if (!s || !ticket || (nprobe && !probes)) return fail(BN_EINVAL, "null argument");
    if (!s->ivf) return fail(BN_EUNSUPPORTED, "this server has no IVF corpus");
    TRY(validate_request(s, s->ivf->e, v_enc, g, t_idx, t_sign, t_nnz, v_seed));
    for (uint32_t p = 0; p < nprobe; ++p)
        if (probes[p] >= s->ivf->nlist) return fail(BN_EINVAL, "probe %u names list %u of %u", p, probes[p], s->ivf->nlist);
    Request r;
    fill_request(r, BN_SERVER_IVF, s->ivf->e, v_enc, g, t_idx, t_sign, t_nnz, v_seed);
    r.probes.assign(probes, probes + nprobe);
    return submit(s, BN_SERVER_IVF, std::move(r), ticket);
}

int bn_server_wait(bn_server* s, uint64_t ticket, uint32_t timeout_ms, uint32_t* ids, int64_t* scores, uint32_t* n_hits,
                   int32_t* failed_trial, int32_t* failed_cluster, double* latency_us) {
    if (!s) return fail(BN_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket == 0 || ticket >= s->next_ticket) return fail(BN_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
    const bool ready = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                           [&] { return s->results.count(ticket) != 0; });
    if (!ready) return fail(BN_EAGAIN, "ticket %llu is not complete", (unsigned long long)ticket);
    Result r = std::move(s->results[ticket]);
    s->results.erase(ticket);
    if (r.status != BN_OK) return fail(r.status, "%s", r.error.c_str());
    if (n_hits) *n_hits = (uint32_t)r.ids.size();
    if (ids) memcpy(ids, r.ids.data(), r.ids.size() * 4);
    if (scores) memcpy(scores, r.scores.data(), r.scores.size() * 8);
    if (failed_trial) *failed_trial = r.failed_trial;
    if (failed_cluster) *failed_cluster = r.failed_cluster;
    if (latency_us) *latency_us = r.latency_us;
    return BN_OK;
}

int bn_server_stats(bn_server* s, int reset, bn_server_stats_t* out) {
    if (!s || !out) return fail(BN_EINVAL, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    memset(out, 0, sizeof *out);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->batches = s->batches;
    out->mean_batch = s->batches ? (double)s->batched_queries / (double)s->batches : 0.0;
    out->peak_workspace_bytes = s->peak_mem;
    out->block_batches = s->block_batches;
    out->rejected = s->rejected;
    std::vector<double> l = s->lat_us;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (double)(l.size() - 1) + 0.5))]; };
        out->p50_us = pct(0.50);
        out->p99_us = pct(0.99);
        out->max_us = l.back();
        const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
        out->throughput_qps = span > 0 ? (double)l.size() / span : 0.0;
    }
    if (reset) {
        s->lat_us.clear();
        s->batches = s->batched_queries = s->block_batches = s->rejected = 0;
        s->submitted = s->completed = 0;
    }
    return BN_OK;
}

int bn_server_destroy(bn_server* s) {
    if (!s) return BN_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->sched.joinable()) s->sched.join();  // drains queued and in-flight batches
    for (auto& sl : s->slots) {
        sl->ws.release();  // freed in its stream's order, before the stream goes
        if (sl->stream) cudaStreamSynchronize(sl->stream);
        if (sl->stream) cudaStreamDestroy(sl->stream);
        if (sl->done) cudaEventDestroy(sl->done);
    }
    delete s;
    return BN_OK;
}

}  // extern "C"
