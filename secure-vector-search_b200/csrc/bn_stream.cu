// bn_stream.cu -- corpora larger than device memory, flat and IVF.
//
// The reference keeps a corpus that does not fit in VRAM in host memory and
// uploads it on demand through an LRU of device-resident entries bounded by
// a byte budget (ClusterStore::get_or_upload, scorer-gpu-common/src/
// store.rs:247-395; the flat scorer's lazy upload and the IVF scorer's
// per-cluster uploads, scorer-bntm/src/gpu/mod.rs:279-577).  Here the corpus
// is cut into chunks: runs of chunk_rows rows (flat) or of whole lists up to
// chunk_rows rows (IVF; a longer list is a chunk of its own).  Each chunk is
// built once on the device (encryption, the decode layouts) and its device
// image -- exactly the bytes the query kernels read: m_enc, the [AL | H]
// 32-row blocks, the int8 (or residue) column-major plaintext, the
// sliced-ELL S and the IVF row ids -- is kept in pinned host memory.  Device
// memory holds budget_bytes / slot_bytes chunk slots, each a complete corpus
// of the largest chunk's size with its own stream and workspace.
//
// A call visits each chunk it needs once (flat: all of them; IVF: those
// holding a probed list): the resident ones first, least recently used
// first, then the others, each uploaded on the upload stream into the slot
// of the least recently used chunk -- one this call has already scored, so
// for a flat corpus scanned in full the slots keep the chunks the next call
// meets first.  Events order each slot's upload after its last scoring and
// its scoring after the upload, so uploads overlap the scoring of the
// resident chunks.  Flat chunks are scored as row shards of the whole
// corpus: Protocol 2 draws at the rows' positions in the whole corpus (draw
// t of row i at t * rows + i, crypto.rs:1013-1059), so the per-trial sums
// u.r and z.v add up over the chunks to the whole corpus's values.  IVF
// lists are verified one by one (ivf.rs:746-927), so a chunk's verdicts are
// the lists' own, and a query reports the first failing list in probe
// order.  Top-k lists merge by (score desc, id asc) (lib.rs:452-469).
// Results equal the resident bn_flat_query / bn_ivf_query bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "bn_internal.cuh"

using namespace bn;
using namespace bn::api;

namespace {

// LRU + budget bookkeeping (the reference's LruInner, store.rs:133-245):
// entries with their bytes, a recency queue (front = next evicted), the
// resident total and the telemetry counters of store.rs:36-80.
struct Lru {
    struct Entry {
        uint64_t bytes;
    };
    std::unordered_map<uint64_t, Entry> entries;
    std::deque<uint64_t> order;
    uint64_t resident = 0, budget = 0;
    bn_store_stats st{};

    bool touch(uint64_t id) {
        if (!entries.count(id)) return false;
        auto it = std::find(order.begin(), order.end(), id);
        if (it != order.end()) order.erase(it);
        order.push_back(id);
        return true;
    }
    // Evicts from the front until `bytes` fits on top of what stays
    // resident; BN_EBUDGET (nothing evicted) when it cannot fit at all.
    int pre_evict(uint64_t bytes, std::vector<uint64_t>& evicted) {
        if (bytes > budget)
            return fail(BN_EBUDGET, "entry of %llu bytes exceeds the store budget of %llu bytes",
                        (unsigned long long)bytes, (unsigned long long)budget);
        while (resident + bytes > budget) {
            if (order.empty())  // bookkeeping out of step with the entries: cannot happen
                return fail(BN_EBUDGET, "store budget of %llu bytes cannot hold %llu more bytes",
                            (unsigned long long)budget, (unsigned long long)bytes);
            const uint64_t id = order.front();
            order.pop_front();
            auto it = entries.find(id);
            if (it != entries.end()) {
                resident -= it->second.bytes;
                entries.erase(it);
                st.evictions += 1;
                evicted.push_back(id);
            }
        }
        return BN_OK;
    }
    // False when the id is already resident (the store keeps that entry).
    bool insert(uint64_t id, uint64_t bytes) {
        if (entries.count(id)) return false;
        entries[id] = Entry{bytes};
        order.push_back(id);
        resident += bytes;
        return true;
    }
    void erase(uint64_t id) {
        auto it = std::find(order.begin(), order.end(), id);
        if (it != order.end()) order.erase(it);
        auto e = entries.find(id);
        if (e != entries.end()) {
            resident -= e->second.bytes;
            entries.erase(e);
        }
    }
    void stats(bn_store_stats* out) const {
        *out = st;
        out->resident_bytes = resident;
        out->budget_bytes = budget;
    }
};

// Corpus arrays a chunk image holds (A_*), and the image's seven slots:
// m_enc, [AL | H] blocks, the plaintext (int8 copy when every value is
// int8-valued, else the residues), the ELL values, slice offsets and slice
// widths, and the row ids (IVF).
enum { A_MENC = 0, A_ALH, A_M8, A_MP, A_SELL, A_SOFF, A_SW, A_IDS, A_COUNT_MAX };
constexpr int A_COUNT = 7;

DevMem& corpus_array(Corpus& c, int a) {
    switch (a) {
        case A_MENC: return c.m_enc;
        case A_ALH: return c.alh_b;
        case A_M8: return c.m8_cm;
        case A_MP: return c.mp_cm;
        case A_SELL: return c.s_ell;
        case A_SOFF: return c.s_off;
        case A_SW: return c.s_w;
        default: return c.ids;
    }
}

// One chunk's device image in pinned host memory.
struct ChunkImage {
    uint64_t row0 = 0, rows = 0;
    uint32_t list0 = 0, list1 = 0;  // IVF: the chunk's lists [list0, list1)
    void* host = nullptr;           // cudaMallocHost: the arrays below back to back
    uint64_t off[A_COUNT] = {0}, bytes[A_COUNT] = {0};
    uint64_t total = 0;
};

// A chunk slot: a corpus of the largest chunk's size on the device, with its
// stream, workspace, the events that order it against the upload stream,
// and the job in flight on it.
struct Slot {
    Engine e;  // runs the pipeline
    cudaEvent_t uploaded = nullptr, scored = nullptr;
    int64_t chunk = -1;    // resident chunk (-1: none)
    bool pending = false;  // a job of the current call awaits its results
    HostMeta hm;
    QueryJob job;
    uint32_t job_chunk = 0;           // the chunk the job in flight scores (the slot may be reassigned first)
    std::vector<uint32_t> seg_probe;  // IVF: each segment's probe position
};

// The chunk images, the slots and the LRU shared by the flat and IVF stores.
struct Store {
    bn_ctx* ctx = nullptr;
    uint32_t n1 = 128;
    bool use_m8 = true, has_ids = false;
    uint64_t slot_bytes = 0;
    std::vector<ChunkImage> chunks;
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<uint64_t> cap;  // per image array: slot capacity in bytes
    std::vector<uint64_t> L;    // the client's subspace (same for every chunk)
    cudaStream_t upload = nullptr;
    Lru lru;

    ~Store() {
        for (auto& sl : slots) {
            if (sl->e.stream) cudaStreamSynchronize(sl->e.stream);
            if (sl->uploaded) cudaEventDestroy(sl->uploaded);
            if (sl->scored) cudaEventDestroy(sl->scored);
            engine_free(sl->e);
        }
        if (upload) {
            cudaStreamSynchronize(upload);
            cudaStreamDestroy(upload);
        }
        for (ChunkImage& ci : chunks)
            if (ci.host) cudaFreeHost(ci.host);
    }

    int array_index(int a) const {  // image slot of corpus array a, -1 if unused
        if (a == A_M8 && !use_m8) return -1;
        if (a == A_MP && use_m8) return -1;
        if (a == A_IDS && !has_ids) return -1;
        return a < A_MP ? a : (a == A_MP ? A_M8 : a - 1);  // A_M8 and A_MP share image slot 2
    }
};

// True when every plaintext residue is int8-valued (the test of the decode
// layout kernel: fp_to_signed in [-128, 127]); then every chunk carries the
// int8 copy, else every chunk carries the residues.
bool all_int8(const uint64_t* mp, uint64_t count) {
    for (uint64_t i = 0; i < count; ++i)
        if (mp[i] > 127 && mp[i] < P - 128) return false;
    return true;
}

// Snapshots the query arrays of a freshly built chunk corpus into pinned host memory.
int snapshot(Store& st, Corpus& c, ChunkImage& ci, cudaStream_t s) {
    uint64_t total = 0;
    for (int a = 0; a < A_COUNT_MAX; ++a) {
        const int x = st.array_index(a);
        if (x < 0) continue;
        ci.off[x] = total;
        ci.bytes[x] = corpus_array(c, a).bytes;
        total += (ci.bytes[x] + 255) / 256 * 256;
    }
    ci.total = total;
    CU(cudaMallocHost(&ci.host, std::max<uint64_t>(total, 256)));
    for (int a = 0; a < A_COUNT_MAX; ++a) {
        const int x = st.array_index(a);
        if (x < 0 || !ci.bytes[x]) continue;
        CU(cudaMemcpyAsync(static_cast<char*>(ci.host) + ci.off[x], corpus_array(c, a).p, ci.bytes[x],
                           cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

// Builds every chunk's corpus in turn (build_one makes a temporary corpus
// for chunk ci and returns its Engine, freed by done()) and keeps its image.
int build_chunks(Store& st, const std::function<int(ChunkImage&, Engine*&)>& build_one,
                 const std::function<void()>& done) {
    for (ChunkImage& ci : st.chunks) {
        Engine* e = nullptr;
        TRY(build_one(ci, e));
        int rc = BN_OK;
        if (st.use_m8 && ci.rows && !e->c.m8_cm.p)
            rc = fail(BN_ECUDA, "store: chunk at row %llu has no int8 copy", (unsigned long long)ci.row0);
        if (rc == BN_OK) rc = snapshot(st, e->c, ci, e->stream);
        done();
        TRY(rc);
    }
    return BN_OK;
}

// Slot capacity per image array, the slots the budget holds, and their
// device memory (allocated once; loads only copy).
int make_slots(Store& st, uint64_t budget) {
    st.cap.assign(A_COUNT, 0);
    for (const ChunkImage& ci : st.chunks)
        for (int x = 0; x < A_COUNT; ++x) st.cap[x] = std::max(st.cap[x], ci.bytes[x]);
    uint64_t slot = 0;
    for (int x = 0; x < A_COUNT; ++x) slot += st.cap[x];
    slot += (uint64_t)N * st.n1 * 8;  // L
    st.slot_bytes = slot;
    st.lru.budget = budget;
    const uint64_t nslots = std::min<uint64_t>(budget / slot, st.chunks.size());
    if (!nslots)
        return fail(BN_EBUDGET, "store budget of %llu bytes holds no chunk slot of %llu bytes",
                    (unsigned long long)budget, (unsigned long long)slot);
    CU(cudaStreamCreateWithFlags(&st.upload, cudaStreamNonBlocking));
    for (uint64_t i = 0; i < nslots; ++i) {
        auto sl = std::make_unique<Slot>();
        TRY(engine_init(sl->e, st.ctx));
        CU(cudaEventCreateWithFlags(&sl->uploaded, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&sl->scored, cudaEventDisableTiming));
        Corpus& c = sl->e.c;
        c.n1 = st.n1;
        c.client = true;
        for (int a = 0; a < A_COUNT_MAX; ++a) {
            const int x = st.array_index(a);
            if (x >= 0) TRY(corpus_array(c, a).alloc(st.ctx, std::max<uint64_t>(st.cap[x], 1)));
        }
        TRY(c.L.alloc(st.ctx, (uint64_t)N * st.n1 * 8));
        CU(cudaMemcpy(c.L.p, st.L.data(), (uint64_t)N * st.n1 * 8, cudaMemcpyHostToDevice));
        st.slots.push_back(std::move(sl));
    }
    return BN_OK;
}

// Copies chunk c's image into slot sl on the upload stream, after the
// slot's last scoring; the slot's corpus then describes chunk c.
int load_chunk(Store& st, Slot& sl, uint32_t c) {
    const ChunkImage& ci = st.chunks[c];
    Corpus& cp = sl.e.c;
    CU(cudaStreamWaitEvent(st.upload, sl.scored, 0));
    for (int a = 0; a < A_COUNT_MAX; ++a) {
        const int x = st.array_index(a);
        if (x < 0 || !ci.bytes[x]) continue;
        CU(cudaMemcpyAsync(corpus_array(cp, a).p, static_cast<const char*>(ci.host) + ci.off[x], ci.bytes[x],
                           cudaMemcpyHostToDevice, st.upload));
    }
    CU(cudaEventRecord(sl.uploaded, st.upload));
    CU(cudaStreamWaitEvent(sl.e.stream, sl.uploaded, 0));
    cp.rows = ci.rows;
    TRY(corpus_tmap(cp));
    sl.chunk = c;
    st.lru.st.uploads += 1;
    st.lru.st.bytes_uploaded += ci.total;
    return BN_OK;
}

// Visits the chunks `needed` (resident ones first, least recently used
// first, then the rest in the given order): launch(slot, chunk) enqueues a
// job on a slot that holds the chunk, finish(slot) reads a finished job's
// results (called before the slot is reused and at the end; the job's chunk
// is slot.job_chunk, since the slot may already be assigned elsewhere).
int visit(Store& st, const std::vector<uint32_t>& needed, const std::function<int(Slot&, uint32_t)>& launch,
          const std::function<int(Slot&)>& finish) {
    std::vector<char> want(st.chunks.size(), 0);
    for (uint32_t c : needed) want[c] = 1;
    std::vector<uint32_t> order;
    for (uint64_t id : st.lru.order)
        if (want[id]) {
            order.push_back((uint32_t)id);
            want[id] = 0;
        }
    for (uint32_t c : needed)
        if (want[c]) order.push_back(c);
    std::vector<int> slot_of(st.chunks.size(), -1);
    for (size_t i = 0; i < st.slots.size(); ++i)
        if (st.slots[i]->chunk >= 0) slot_of[st.slots[i]->chunk] = (int)i;
    auto finish_slot = [&](Slot& sl) -> int {
        if (!sl.pending) return BN_OK;
        sl.pending = false;
        CU(cudaEventSynchronize(sl.scored));
        return finish(sl);
    };

    int rc = BN_OK;
    for (uint32_t c : order) {
        st.lru.st.gets += 1;
        int si = slot_of[c];
        if (si >= 0) {
            st.lru.touch(c);
        } else {
            std::vector<uint64_t> evicted;
            if ((rc = st.lru.pre_evict(st.slot_bytes, evicted)) != BN_OK) break;
            for (uint64_t e : evicted) {
                const int es = slot_of[e];
                slot_of[e] = -1;
                if (es >= 0) {
                    st.slots[es]->chunk = -1;
                    if (si < 0) si = es;
                }
            }
            for (size_t i = 0; i < st.slots.size() && si < 0; ++i)  // a free slot (fewer chunks than slots resident)
                if (st.slots[i]->chunk < 0) si = (int)i;
            if (si < 0) {
                rc = fail(BN_EBUDGET, "store: no slot for chunk %u", c);
                break;
            }
            Slot& sl = *st.slots[si];
            if ((rc = finish_slot(sl)) != BN_OK) break;  // the slot's previous chunk of this call first
            if ((rc = load_chunk(st, sl, c)) != BN_OK) break;
            st.lru.insert(c, st.slot_bytes);
            slot_of[c] = si;
        }
        Slot& sl = *st.slots[si];
        if ((rc = finish_slot(sl)) != BN_OK) break;
        sl.job_chunk = c;
        if ((rc = launch(sl, c)) != BN_OK) break;
        if (cudaEventRecord(sl.scored, sl.e.stream) != cudaSuccess) {
            rc = fail(BN_ECUDA, "cudaEventRecord failed");
            break;
        }
        sl.pending = true;
    }
    for (auto& sl : st.slots) {  // every job in flight ends before the store moves on
        const int r2 = finish_slot(*sl);
        if (rc == BN_OK) rc = r2;
    }
    if (rc != BN_OK)  // a failed load or launch may leave a slot's contents undefined: drop them
        for (auto& sl : st.slots) {
            if (sl->chunk >= 0) st.lru.erase((uint64_t)sl->chunk);
            sl->chunk = -1;
        }
    return rc;
}

// Per-query accumulators of a call: candidates (score, id), Protocol 2 sums
// (flat) and the first failing list by probe position (IVF).
struct Acc {
    std::vector<std::vector<std::pair<int64_t, uint32_t>>> cand;
    std::vector<uint64_t> ur, zv;  // flat: [B][trials]
    std::vector<uint32_t> fail_pos;
    std::vector<int32_t> fail_cluster, fail_trial;
};

// Reads a finished job's hits (and per-segment verdicts) into acc; id0 is
// added to the ids (a flat chunk's first row).
int read_job(Slot& sl, uint32_t id0, Acc& acc, std::vector<int32_t>& vf) {
    const QueryJob& j = sl.job;
    const uint32_t B = j.B, k = j.k, ks = std::max<uint32_t>(k, 1);
    std::vector<uint32_t> ids((uint64_t)B * ks), nh(B, 0);
    std::vector<int64_t> sc((uint64_t)B * ks);
    TRY(job_finish(j, sl.e.host, ids.data(), sc.data(), nh.data(), vf));
    for (uint32_t b = 0; b < B; ++b)
        for (uint32_t i = 0; i < nh[b]; ++i)
            acc.cand[b].emplace_back(sc[(uint64_t)b * k + i], ids[(uint64_t)b * k + i] + id0);
    return BN_OK;
}

void write_hits(Acc& acc, uint32_t B, uint32_t k, uint32_t* ids, int64_t* scores, uint32_t* n_hits) {
    for (uint32_t b = 0; b < B; ++b) {
        auto& v = acc.cand[b];
        std::sort(v.begin(), v.end(), [](const std::pair<int64_t, uint32_t>& x, const std::pair<int64_t, uint32_t>& y) {
            return x.first != y.first ? x.first > y.first : x.second < y.second;
        });
        const uint32_t n = (uint32_t)std::min<uint64_t>(k, v.size());
        for (uint32_t i = 0; i < n; ++i) {
            if (ids) ids[(uint64_t)b * k + i] = v[i].second;
            if (scores) scores[(uint64_t)b * k + i] = v[i].first;
        }
        if (n_hits) n_hits[b] = n;
    }
}

std::vector<uint64_t> rebased_rowptr(const uint64_t* rowptr, uint64_t row0, uint64_t rows) {
    std::vector<uint64_t> rp(rows + 1);
    for (uint64_t i = 0; i <= rows; ++i) rp[i] = rowptr[row0 + i] - rowptr[row0];
    return rp;
}

int check_query_args(uint32_t trials, uint32_t k, const void* ids, const void* scores, const void* n_hits) {
    if (k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX = %d", k, BN_TOPK_MAX);
    if (trials > MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %u", trials, MAX_TRIALS);
    if (k && (!ids || !scores || !n_hits)) return fail(BN_EINVAL, "ids, scores and n_hits are required when k > 0");
    return BN_OK;
}

}  // namespace

struct bn_stream {
    Store st;
    uint64_t rows = 0;
    std::mutex mu;
};

struct bn_ivf_stream {
    Store st;
    uint32_t nlist = 0;
    std::vector<uint64_t> offsets;
    std::vector<uint32_t> chunk_of;  // list -> chunk
    std::mutex mu;
};

namespace {

int flat_new(bn_ctx* ctx, uint64_t m, uint32_t n, uint32_t n1, const uint64_t* L, uint64_t chunk_rows,
             bn_stream** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    if (!m) return fail(BN_EINVAL, "empty corpus");
    if (m > 0xffffffffull) return fail(BN_EINVAL, "corpus rows must fit in u32");
    if (!L) return fail(BN_EINVAL, "l_subspace is required");
    if (chunk_rows < 32 || chunk_rows % 32)
        return fail(BN_EINVAL, "chunk_rows = %llu is not a positive multiple of 32", (unsigned long long)chunk_rows);
    TRY(validate_residues(L, (uint64_t)N * n1, "l_subspace"));
    auto* s = new bn_stream();
    s->st.ctx = ctx;
    s->st.n1 = n1;
    s->st.L.assign(L, L + (uint64_t)N * n1);
    s->rows = m;
    for (uint64_t row0 = 0; row0 < m; row0 += chunk_rows) {
        ChunkImage ci;
        ci.row0 = row0;
        ci.rows = std::min<uint64_t>(chunk_rows, m - row0);
        s->st.chunks.push_back(ci);
    }
    *out = s;
    return BN_OK;
}

int flat_finish_build(bn_stream* s, uint64_t budget, const std::function<int(ChunkImage&, bn_flat**)>& one) {
    bn_flat* tmp = nullptr;
    int rc = cudaSetDevice(s->st.ctx->device) == cudaSuccess ? BN_OK : fail(BN_ECUDA, "cudaSetDevice failed");
    if (rc == BN_OK)
        rc = build_chunks(
            s->st,
            [&](ChunkImage& ci, Engine*& e) -> int {
                TRY(one(ci, &tmp));
                e = &tmp->e;
                return BN_OK;
            },
            [&]() {
                bn_flat_destroy(tmp);
                tmp = nullptr;
            });
    if (rc == BN_OK) rc = make_slots(s->st, budget);
    return rc;
}

int ivf_new(bn_ctx* ctx, uint32_t nlist, const uint64_t* off, uint32_t n, uint32_t n1, const uint64_t* L,
            uint64_t chunk_rows, bn_ivf_stream** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    if (!nlist || !off) return fail(BN_EINVAL, "an IVF store needs lists");
    if (!L) return fail(BN_EINVAL, "l_subspace is required");
    if (!chunk_rows) return fail(BN_EINVAL, "chunk_rows must be positive");
    if (off[0] != 0) return fail(BN_EINVAL, "list_offsets[0] must be 0");
    for (uint32_t c = 0; c < nlist; ++c)
        if (off[c + 1] < off[c]) return fail(BN_EINVAL, "list_offsets are not monotone at list %u", c);
    if (!off[nlist]) return fail(BN_EINVAL, "empty corpus");
    if (off[nlist] > 0xffffffffull) return fail(BN_EINVAL, "corpus rows must fit in u32");
    TRY(validate_residues(L, (uint64_t)N * n1, "l_subspace"));
    auto* s = new bn_ivf_stream();
    s->st.ctx = ctx;
    s->st.n1 = n1;
    s->st.has_ids = true;
    s->st.L.assign(L, L + (uint64_t)N * n1);
    s->nlist = nlist;
    s->offsets.assign(off, off + nlist + 1);
    s->chunk_of.assign(nlist, 0);
    // whole lists, up to chunk_rows rows per chunk (a longer list alone); a
    // chunk takes lists while it is empty, and trailing empty lists join the
    // last chunk, so no chunk is empty
    uint32_t l0 = 0;
    while (l0 < nlist) {
        uint32_t l1 = l0 + 1;
        while (l1 < nlist && (off[l1] == off[l0] || off[l1 + 1] - off[l0] <= chunk_rows)) ++l1;
        if (off[l1] == off[l0] && !s->st.chunks.empty()) {
            s->st.chunks.back().list1 = l1;
        } else {
            ChunkImage ci;
            ci.list0 = l0;
            ci.list1 = l1;
            ci.row0 = off[l0];
            ci.rows = off[l1] - off[l0];
            s->st.chunks.push_back(ci);
        }
        for (uint32_t c = l0; c < l1; ++c) s->chunk_of[c] = (uint32_t)s->st.chunks.size() - 1;
        l0 = l1;
    }
    *out = s;
    return BN_OK;
}

int ivf_finish_build(bn_ivf_stream* s, uint64_t budget, const std::function<int(ChunkImage&, bn_ivf**)>& one) {
    bn_ivf* tmp = nullptr;
    int rc = cudaSetDevice(s->st.ctx->device) == cudaSuccess ? BN_OK : fail(BN_ECUDA, "cudaSetDevice failed");
    if (rc == BN_OK)
        rc = build_chunks(
            s->st,
            [&](ChunkImage& ci, Engine*& e) -> int {
                TRY(one(ci, &tmp));
                e = &tmp->e;
                return BN_OK;
            },
            [&]() {
                bn_ivf_destroy(tmp);
                tmp = nullptr;
            });
    if (rc == BN_OK) rc = make_slots(s->st, budget);
    return rc;
}

// List offsets of chunk ci relative to its first row.
std::vector<uint64_t> local_offsets(const bn_ivf_stream* s, const ChunkImage& ci) {
    std::vector<uint64_t> o(ci.list1 - ci.list0 + 1);
    for (uint32_t c = ci.list0; c <= ci.list1; ++c) o[c - ci.list0] = s->offsets[c] - ci.row0;
    return o;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- flat

int bn_stream_build(bn_ctx* ctx, const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint64_t m,
                    uint32_t n, uint32_t n1, const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat,
                    uint64_t chunk_rows, uint64_t budget_bytes, bn_stream** out) {
    bn_stream* s = nullptr;
    TRY(flat_new(ctx, m, n, n1, l_subspace, chunk_rows, &s));
    int rc = BN_OK;
    if (!m_enc || !a_l || !h || !m_plain || !s_mat.rowptr) rc = fail(BN_EINVAL, "null corpus array");
    if (rc == BN_OK) rc = validate_residues(m_plain, m * N, "m_plain");
    if (rc == BN_OK) {
        s->st.use_m8 = all_int8(m_plain, m * N);
        rc = flat_finish_build(s, budget_bytes, [&](ChunkImage& ci, bn_flat** f) -> int {
            TRY(bn_flat_build(ctx, m_enc + ci.row0 * N, a_l + ci.row0 * n1, h + ci.row0 * n1, ci.rows, n, n1, f));
            const std::vector<uint64_t> rp = rebased_rowptr(s_mat.rowptr, ci.row0, ci.rows);
            const uint64_t nz0 = s_mat.rowptr[ci.row0];
            bn_sparse_csr sc{rp.data(), s_mat.idx ? s_mat.idx + nz0 : nullptr, s_mat.sign ? s_mat.sign + nz0 : nullptr};
            const int r = bn_flat_attach_client(*f, l_subspace, m_plain + ci.row0 * N, sc);
            if (r != BN_OK) {
                bn_flat_destroy(*f);
                *f = nullptr;
            }
            return r;
        });
    }
    if (rc != BN_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return BN_OK;
}

int bn_stream_build_from_plain(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1,
                               const uint64_t* l_subspace, const uint64_t* h, bn_sparse_csr s_mat, uint64_t chunk_rows,
                               uint64_t budget_bytes, bn_stream** out) {
    bn_stream* s = nullptr;
    TRY(flat_new(ctx, m, n, n1, l_subspace, chunk_rows, &s));
    int rc = BN_OK;
    if (!m_q || !h || !s_mat.rowptr) rc = fail(BN_EINVAL, "null input array");
    if (rc == BN_OK) rc = validate_residues(m_q, m * N, "m_q");
    if (rc == BN_OK) {
        s->st.use_m8 = all_int8(m_q, m * N);
        rc = flat_finish_build(s, budget_bytes, [&](ChunkImage& ci, bn_flat** f) -> int {
            const std::vector<uint64_t> rp = rebased_rowptr(s_mat.rowptr, ci.row0, ci.rows);
            const uint64_t nz0 = s_mat.rowptr[ci.row0];
            bn_sparse_csr sc{rp.data(), s_mat.idx ? s_mat.idx + nz0 : nullptr, s_mat.sign ? s_mat.sign + nz0 : nullptr};
            return bn_flat_build_from_plain(ctx, m_q + ci.row0 * N, ci.rows, n, n1, l_subspace, h + ci.row0 * n1, sc, f);
        });
    }
    if (rc != BN_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return BN_OK;
}

int bn_stream_info(const bn_stream* s, uint64_t* rows, uint32_t* chunks, uint32_t* slots, uint64_t* slot_bytes,
                   uint64_t* host_bytes) {
    if (!s) return fail(BN_EINVAL, "null handle");
    if (rows) *rows = s->rows;
    if (chunks) *chunks = (uint32_t)s->st.chunks.size();
    if (slots) *slots = (uint32_t)s->st.slots.size();
    if (slot_bytes) *slot_bytes = s->st.slot_bytes;
    if (host_bytes) {
        uint64_t t = 0;
        for (const ChunkImage& ci : s->st.chunks) t += ci.total;
        *host_bytes = t;
    }
    return BN_OK;
}

int bn_stream_query(bn_stream* s, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                    const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
                    uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial) {
    if (!s) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    TRY(check_query_args(trials, k, ids, scores, n_hits));
    if (!failed_trial) return fail(BN_EINVAL, "failed_trial is required");
    std::lock_guard<std::mutex> g_(s->mu);
    CU(cudaSetDevice(s->st.ctx->device));
    Acc acc;
    acc.cand.resize(B);
    acc.ur.assign((uint64_t)B * trials, 0);
    acc.zv.assign((uint64_t)B * trials, 0);
    std::vector<uint32_t> all(s->st.chunks.size());
    for (uint32_t c = 0; c < all.size(); ++c) all[c] = c;
    TRY(visit(
        s->st, all,
        [&](Slot& sl, uint32_t c) -> int {
            const ChunkImage& ci = s->st.chunks[c];
            flat_meta(ci.rows, B, sl.hm);
            for (VerifySeg& vs : sl.hm.vsegs) {  // draw positions within the whole corpus
                vs.draw_stride = s->rows;
                vs.draw_base = ci.row0;
            }
            sl.job = QueryJob();
            sl.job.hm = &sl.hm;
            sl.job.B = B;
            sl.job.trials = trials;
            sl.job.k = k;
            TRY(job_prepare(sl.e, sl.job, sl.e.ws, sl.e.host, v_enc, g, t_idx, t_sign, t_nnz, v_seeds));
            return job_launch(sl.e, sl.job, sl.e.ws, sl.e.host, sl.e.stream, nullptr, nullptr);
        },
        [&](Slot& sl) -> int {
            std::vector<int32_t> vf;  // per-shard verdicts mean nothing: decided on the sums
            TRY(read_job(sl, (uint32_t)s->st.chunks[sl.job_chunk].row0, acc, vf));
            if (sl.job.trials) {
                const char* h = sl.e.host.at<char>();
                const uint64_t* ur = reinterpret_cast<const uint64_t*>(h + sl.job.o.ur);
                const uint64_t* zv = reinterpret_cast<const uint64_t*>(h + sl.job.o.zv);
                for (uint64_t i = 0; i < (uint64_t)B * trials; ++i) {
                    acc.ur[i] = add_mod(acc.ur[i], ur[i]);
                    acc.zv[i] = add_mod(acc.zv[i], zv[i]);
                }
            }
            return BN_OK;
        }));
    write_hits(acc, B, k, ids, scores, n_hits);
    for (uint32_t b = 0; b < B; ++b) {
        failed_trial[b] = -1;
        for (uint32_t t = 0; t < trials; ++t)
            if (acc.ur[(uint64_t)b * trials + t] != acc.zv[(uint64_t)b * trials + t]) {
                failed_trial[b] = (int32_t)t;
                break;
            }
    }
    return BN_OK;
}

int bn_stream_stats(bn_stream* s, int reset, bn_store_stats* out) {
    if (!s || !out) return fail(BN_EINVAL, "null argument");
    std::lock_guard<std::mutex> g_(s->mu);
    s->st.lru.stats(out);
    if (reset) s->st.lru.st = bn_store_stats{};
    return BN_OK;
}

int bn_stream_destroy(bn_stream* s) {
    delete s;
    return BN_OK;
}

// ---------------------------------------------------------------- IVF

int bn_ivf_stream_build(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids,
                        const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint32_t n, uint32_t n1,
                        const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat, uint64_t chunk_rows,
                        uint64_t budget_bytes, bn_ivf_stream** out) {
    bn_ivf_stream* s = nullptr;
    TRY(ivf_new(ctx, nlist, list_offsets, n, n1, l_subspace, chunk_rows, &s));
    const uint64_t rows = list_offsets[nlist];
    int rc = BN_OK;
    if (!ids || !m_enc || !a_l || !h || !m_plain || !s_mat.rowptr) rc = fail(BN_EINVAL, "null corpus array");
    if (rc == BN_OK) rc = validate_residues(m_plain, rows * N, "m_plain");
    if (rc == BN_OK) {
        s->st.use_m8 = all_int8(m_plain, rows * N);
        rc = ivf_finish_build(s, budget_bytes, [&](ChunkImage& ci, bn_ivf** v) -> int {
            const std::vector<uint64_t> lo = local_offsets(s, ci);
            TRY(bn_ivf_build(ctx, ci.list1 - ci.list0, lo.data(), ids + ci.row0, m_enc + ci.row0 * N,
                             a_l + ci.row0 * n1, h + ci.row0 * n1, n, n1, v));
            const std::vector<uint64_t> rp = rebased_rowptr(s_mat.rowptr, ci.row0, ci.rows);
            const uint64_t nz0 = s_mat.rowptr[ci.row0];
            bn_sparse_csr sc{rp.data(), s_mat.idx ? s_mat.idx + nz0 : nullptr, s_mat.sign ? s_mat.sign + nz0 : nullptr};
            const int r = bn_ivf_attach_client(*v, l_subspace, m_plain + ci.row0 * N, sc);
            if (r != BN_OK) {
                bn_ivf_destroy(*v);
                *v = nullptr;
            }
            return r;
        });
    }
    if (rc != BN_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return BN_OK;
}

int bn_ivf_stream_build_keygen(bn_ctx* ctx, uint32_t nlist, const uint64_t* list_offsets, const uint32_t* ids,
                               const uint64_t* m_q, uint32_t n, uint32_t n1, const uint64_t* l_subspace,
                               uint64_t upload_seed, uint64_t chunk_rows, uint64_t budget_bytes, bn_ivf_stream** out) {
    bn_ivf_stream* s = nullptr;
    TRY(ivf_new(ctx, nlist, list_offsets, n, n1, l_subspace, chunk_rows, &s));
    const uint64_t rows = list_offsets[nlist];
    int rc = BN_OK;
    if (!ids || !m_q) rc = fail(BN_EINVAL, "null corpus array");
    if (rc == BN_OK) rc = validate_residues(m_q, rows * N, "m_q");
    if (rc == BN_OK) {
        s->st.use_m8 = all_int8(m_q, rows * N);
        rc = ivf_finish_build(s, budget_bytes, [&](ChunkImage& ci, bn_ivf** v) -> int {
            const std::vector<uint64_t> lo = local_offsets(s, ci);
            return ivf_build_keygen_from(ctx, ci.list1 - ci.list0, lo.data(), ids + ci.row0, m_q + ci.row0 * N, n, n1,
                                         l_subspace, upload_seed, ci.list0, v);
        });
    }
    if (rc != BN_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return BN_OK;
}

int bn_ivf_stream_info(const bn_ivf_stream* s, uint64_t* rows, uint32_t* chunks, uint32_t* slots,
                       uint64_t* slot_bytes, uint64_t* host_bytes) {
    if (!s) return fail(BN_EINVAL, "null handle");
    if (rows) *rows = s->offsets[s->nlist];
    if (chunks) *chunks = (uint32_t)s->st.chunks.size();
    if (slots) *slots = (uint32_t)s->st.slots.size();
    if (slot_bytes) *slot_bytes = s->st.slot_bytes;
    if (host_bytes) {
        uint64_t t = 0;
        for (const ChunkImage& ci : s->st.chunks) t += ci.total;
        *host_bytes = t;
    }
    return BN_OK;
}

int bn_ivf_stream_query(bn_ivf_stream* s, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc,
                        const uint64_t* g, const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz,
                        const uint8_t* v_seeds, uint32_t trials, uint32_t k, uint32_t* ids, int64_t* scores,
                        uint32_t* n_hits, int32_t* failed_cluster, int32_t* failed_trial) {
    if (!s) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (nprobe && !probes) return fail(BN_EINVAL, "null probes");
    TRY(check_query_args(trials, k, ids, scores, n_hits));
    for (uint64_t i = 0; i < (uint64_t)B * nprobe; ++i)
        if (probes[i] >= s->nlist)
            return fail(BN_EINVAL, "probe %llu names list %u of %u", (unsigned long long)i, probes[i], s->nlist);
    std::lock_guard<std::mutex> g_(s->mu);
    CU(cudaSetDevice(s->st.ctx->device));
    Acc acc;
    acc.cand.resize(B);
    acc.fail_pos.assign(B, 0xffffffffu);
    acc.fail_cluster.assign(B, -1);
    acc.fail_trial.assign(B, -1);
    // the chunks holding a non-empty probed list, in order of first probe
    std::vector<uint32_t> needed;
    std::vector<char> seen(s->st.chunks.size(), 0);
    for (uint64_t i = 0; i < (uint64_t)B * nprobe; ++i) {
        const uint32_t ci = probes[i];
        if (s->offsets[ci + 1] == s->offsets[ci]) continue;  // ivf.rs:787-789 skips empty clusters
        const uint32_t c = s->chunk_of[ci];
        if (!seen[c]) {
            seen[c] = 1;
            needed.push_back(c);
        }
    }
    TRY(visit(
        s->st, needed,
        [&](Slot& sl, uint32_t c) -> int {
            const ChunkImage& ch = s->st.chunks[c];
            HostMeta& hm = sl.hm;
            hm = HostMeta();
            sl.seg_probe.clear();
            uint64_t out = 0;
            for (uint32_t b = 0; b < B; ++b) {
                const uint32_t seg0 = (uint32_t)hm.segs.size();
                for (uint32_t p = 0; p < nprobe; ++p) {
                    const uint32_t ci = probes[(uint64_t)b * nprobe + p];
                    if (s->chunk_of[ci] != c) continue;
                    const uint64_t row0 = s->offsets[ci] - ch.row0, m = s->offsets[ci + 1] - s->offsets[ci];
                    if (!m) continue;
                    hm.segs.push_back(ScanSeg{row0, out, (uint32_t)m, b});
                    hm.vsegs.push_back(VerifySeg{row0, out, (uint32_t)m, b});
                    hm.seg_cluster.push_back(ci);
                    sl.seg_probe.push_back(p);
                    hm.max_rows = std::max(hm.max_rows, m);
                    out += m;
                }
                hm.dq.push_back(DecodeQuery{seg0, (uint32_t)hm.segs.size() - seg0});
            }
            hm.total_out = out;
            finish_meta(hm);
            sl.job = QueryJob();
            sl.job.hm = &sl.hm;
            sl.job.B = B;
            sl.job.trials = trials;
            sl.job.k = k;
            TRY(job_prepare(sl.e, sl.job, sl.e.ws, sl.e.host, v_enc, g, t_idx, t_sign, t_nnz, v_seeds));
            return job_launch(sl.e, sl.job, sl.e.ws, sl.e.host, sl.e.stream, nullptr, nullptr);
        },
        [&](Slot& sl) -> int {
            std::vector<int32_t> vf;
            TRY(read_job(sl, 0, acc, vf));  // IVF ids are the corpus's own (the ids array)
            const HostMeta& hm = sl.hm;
            for (uint32_t b = 0; b < B; ++b)
                for (uint32_t sg = hm.dq[b].seg0; sg < hm.dq[b].seg0 + hm.dq[b].nseg; ++sg)
                    if (vf[sg] >= 0 && sl.seg_probe[sg] < acc.fail_pos[b]) {
                        acc.fail_pos[b] = sl.seg_probe[sg];
                        acc.fail_cluster[b] = (int32_t)hm.seg_cluster[sg];
                        acc.fail_trial[b] = vf[sg];
                    }
            return BN_OK;
        }));
    write_hits(acc, B, k, ids, scores, n_hits);
    for (uint32_t b = 0; b < B; ++b) {
        if (failed_cluster) failed_cluster[b] = acc.fail_cluster[b];
        if (failed_trial) failed_trial[b] = acc.fail_trial[b];
    }
    return BN_OK;
}

int bn_ivf_stream_stats(bn_ivf_stream* s, int reset, bn_store_stats* out) {
    if (!s || !out) return fail(BN_EINVAL, "null argument");
    std::lock_guard<std::mutex> g_(s->mu);
    s->st.lru.stats(out);
    if (reset) s->st.lru.st = bn_store_stats{};
    return BN_OK;
}

int bn_ivf_stream_destroy(bn_ivf_stream* s) {
    delete s;
    return BN_OK;
}

// ---------------------------------------------------------------- LRU bookkeeping alone

struct bn_lru {
    Lru l;
};

int bn_lru_create(uint64_t budget_bytes, bn_lru** out) {
    if (!out) return fail(BN_EINVAL, "null argument");
    *out = new bn_lru();
    (*out)->l.budget = budget_bytes;
    return BN_OK;
}

int bn_lru_touch(bn_lru* l, uint64_t id, int* hit) {
    if (!l || !hit) return fail(BN_EINVAL, "null argument");
    l->l.st.gets += 1;
    *hit = l->l.touch(id) ? 1 : 0;
    return BN_OK;
}

int bn_lru_pre_evict(bn_lru* l, uint64_t bytes, uint64_t* evicted, uint32_t cap, uint32_t* n_evicted) {
    if (!l || !n_evicted || (cap && !evicted)) return fail(BN_EINVAL, "null argument");
    std::vector<uint64_t> ev;
    const int rc = l->l.pre_evict(bytes, ev);
    *n_evicted = (uint32_t)ev.size();
    for (uint32_t i = 0; i < std::min<uint32_t>(cap, (uint32_t)ev.size()); ++i) evicted[i] = ev[i];
    return rc;
}

int bn_lru_insert(bn_lru* l, uint64_t id, uint64_t bytes, int* inserted) {
    if (!l || !inserted) return fail(BN_EINVAL, "null argument");
    *inserted = l->l.insert(id, bytes) ? 1 : 0;
    if (*inserted) {
        l->l.st.uploads += 1;
        l->l.st.bytes_uploaded += bytes;
    }
    return BN_OK;
}

int bn_lru_stats(const bn_lru* l, bn_store_stats* out) {
    if (!l || !out) return fail(BN_EINVAL, "null argument");
    l->l.stats(out);
    return BN_OK;
}

int bn_lru_destroy(bn_lru* l) {
    delete l;
    return BN_OK;
}

}  // extern "C"
