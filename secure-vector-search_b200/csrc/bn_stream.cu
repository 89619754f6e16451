// bn_stream.cu -- flat corpora larger than device memory.
//
// The reference keeps a corpus that does not fit in VRAM in host memory and
// uploads it on demand through an LRU of device-resident entries bounded by
// a byte budget (ClusterStore::get_or_upload, scorer-gpu-common/src/
// store.rs:247-395; the flat scorer's lazy upload, scorer-bntm/src/gpu/
// mod.rs:279-376).  Here the corpus is cut into chunks of chunk_rows rows.
// Each chunk is built once on the device (encryption, the decode layouts) and
// its device image -- exactly the bytes the query kernels read: m_enc, the
// [AL | H] 32-row blocks, the int8 (or residue) column-major plaintext and
// the sliced-ELL S -- is kept in pinned host memory.  Device memory holds
// budget_bytes / slot_bytes chunk slots, each a complete corpus of up to
// chunk_rows rows with its own stream and workspace.
//
// A query of B requests visits every chunk once: the resident chunks first
// (least recently used first), then the others, each uploaded on the upload
// stream into the slot of the least recently used chunk -- one this query
// has already scored, so for a corpus scanned in full the slots keep the
// chunks the next query meets first.  The upload of one chunk overlaps the
// scoring of the chunks already resident (events order the two streams).
// Every chunk runs the query pipeline as a row shard of the whole corpus:
// Protocol 2 draws at the rows' positions in the whole corpus (draw t of row
// i at position t * rows + i, crypto.rs:1013-1059), so the per-trial sums
// u.r and z.v add up over the chunks to the whole corpus's values, and the
// top-k lists merge by (score desc, id asc) (lib.rs:452-469).  Results are
// bit-identical to the resident bn_flat_query on the same corpus.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
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
    void stats(bn_store_stats* out) const {
        *out = st;
        out->resident_bytes = resident;
        out->budget_bytes = budget;
    }
};

// One chunk's device image in pinned host memory.
struct ChunkImage {
    uint64_t row0 = 0, rows = 0;
    void* host = nullptr;  // cudaMallocHost: the arrays below back to back
    uint64_t off[6] = {0}, bytes[6] = {0};
    uint64_t total = 0;
};
// Corpus arrays a chunk image holds (A_*), and the image's six slots: m_enc,
// [AL | H] blocks, the plaintext (int8 copy when every value is int8-valued,
// else the residues), the ELL values, slice offsets and slice widths.
enum { A_MENC = 0, A_ALH, A_M8, A_MP, A_SELL, A_SOFF, A_SW, A_COUNT_MAX };
constexpr int A_COUNT = 6;

DevMem& corpus_array(Corpus& c, int a) {
    switch (a) {
        case 0: return c.m_enc;
        case 1: return c.alh_b;
        case 2: return c.m8_cm;
        case 3: return c.mp_cm;
        case 4: return c.s_ell;
        case 5: return c.s_off;
        default: return c.s_w;
    }
}

// A chunk slot: a corpus of capacity rows on the device, with its stream,
// workspace, the events that order it against the upload stream, and the
// query job in flight on it.
struct Slot {
    bn_flat f;               // its Engine runs the pipeline
    cudaEvent_t uploaded = nullptr, scored = nullptr;
    int64_t chunk = -1;      // resident chunk (-1: none)
    bool pending = false;    // a job of the current query awaits its results
    HostMeta hm;
    QueryJob job;
    uint64_t job_row0 = 0;
};

}  // namespace

struct bn_stream {
    bn_ctx* ctx = nullptr;
    uint64_t rows = 0, chunk_rows = 0, slot_bytes = 0;
    uint32_t n1 = 128;
    bool use_m8 = true;
    std::vector<ChunkImage> chunks;
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<uint64_t> cap;  // per array: slot capacity in bytes
    std::vector<uint64_t> L;    // the client's subspace (same for every chunk)
    cudaStream_t upload = nullptr;
    Lru lru;
    std::mutex mu;

    ~bn_stream() {
        for (auto& sl : slots) {
            if (sl->f.e.stream) cudaStreamSynchronize(sl->f.e.stream);
            if (sl->uploaded) cudaEventDestroy(sl->uploaded);
            if (sl->scored) cudaEventDestroy(sl->scored);
            engine_free(sl->f.e);
        }
        if (upload) {
            cudaStreamSynchronize(upload);
            cudaStreamDestroy(upload);
        }
        for (ChunkImage& ci : chunks)
            if (ci.host) cudaFreeHost(ci.host);
    }
};

namespace {

int array_index(const bn_stream* st, int a) {  // image slot of corpus array a, -1 if unused
    if (a == A_M8 && !st->use_m8) return -1;
    if (a == A_MP && st->use_m8) return -1;
    return a < A_MP ? a : (a == A_MP ? A_M8 : a - 1);  // A_M8 and A_MP share image index 2
}

// Snapshots the query arrays of a freshly built chunk corpus into pinned host memory.
int snapshot(bn_stream* st, Corpus& c, ChunkImage& ci, cudaStream_t s) {
    uint64_t total = 0;
    for (int a = 0; a < A_COUNT_MAX; ++a) {
        const int x = array_index(st, a);
        if (x < 0) continue;
        ci.off[x] = total;
        ci.bytes[x] = corpus_array(c, a).bytes;
        total += (ci.bytes[x] + 255) / 256 * 256;
    }
    ci.total = total;
    CU(cudaMallocHost(&ci.host, std::max<uint64_t>(total, 256)));
    for (int a = 0; a < A_COUNT_MAX; ++a) {
        const int x = array_index(st, a);
        if (x < 0 || !ci.bytes[x]) continue;
        CU(cudaMemcpyAsync(static_cast<char*>(ci.host) + ci.off[x], corpus_array(c, a).p, ci.bytes[x],
                           cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

// True when every plaintext residue is int8-valued (the test of the decode
// layout kernel: fp_to_signed in [-128, 127]); then every chunk carries the
// int8 copy, else every chunk carries the residues.
bool all_int8(const uint64_t* mp, uint64_t count) {
    for (uint64_t i = 0; i < count; ++i)
        if (mp[i] > 127 && mp[i] < P - 128) return false;
    return true;
}

// Builds the chunk corpora one at a time (build_one makes a temporary flat
// handle of rows [row0, row0 + rows)) and keeps their images.
template <class BuildOne>
int build_chunks(bn_stream* st, BuildOne build_one) {
    for (uint64_t row0 = 0; row0 < st->rows; row0 += st->chunk_rows) {
        ChunkImage ci;
        ci.row0 = row0;
        ci.rows = std::min<uint64_t>(st->chunk_rows, st->rows - row0);
        bn_flat* tmp = nullptr;
        TRY(build_one(row0, ci.rows, &tmp));
        int rc = BN_OK;
        if (st->use_m8 && !tmp->e.c.m8_cm.p) rc = fail(BN_ECUDA, "store: chunk at row %llu has no int8 copy",
                                                        (unsigned long long)row0);
        if (rc == BN_OK) rc = snapshot(st, tmp->e.c, ci, tmp->e.stream);
        bn_flat_destroy(tmp);
        st->chunks.push_back(ci);  // owns ci.host from here on
        TRY(rc);
    }
    return BN_OK;
}

// Slot capacity per image array, the slots the budget holds, and their
// device memory (allocated once; loads only copy).
int make_slots(bn_stream* st, uint64_t budget) {
    st->cap.assign(A_COUNT, 0);
    for (const ChunkImage& ci : st->chunks)
        for (int x = 0; x < A_COUNT; ++x) st->cap[x] = std::max(st->cap[x], ci.bytes[x]);
    uint64_t slot = 0;
    for (int x = 0; x < A_COUNT; ++x) slot += st->cap[x];
    slot += (uint64_t)N * st->n1 * 8;  // L
    st->slot_bytes = slot;
    st->lru.budget = budget;
    const uint64_t nslots = std::min<uint64_t>(budget / slot, st->chunks.size());
    if (!nslots)
        return fail(BN_EBUDGET, "store budget of %llu bytes holds no chunk slot of %llu bytes",
                    (unsigned long long)budget, (unsigned long long)slot);
    CU(cudaStreamCreateWithFlags(&st->upload, cudaStreamNonBlocking));
    for (uint64_t i = 0; i < nslots; ++i) {
        auto sl = std::make_unique<Slot>();
        TRY(engine_init(sl->f.e, st->ctx));
        CU(cudaEventCreateWithFlags(&sl->uploaded, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&sl->scored, cudaEventDisableTiming));
        Corpus& c = sl->f.e.c;
        c.n1 = st->n1;
        c.client = true;
        for (int a = 0; a < A_COUNT_MAX; ++a) {
            const int x = array_index(st, a);
            if (x >= 0) TRY(corpus_array(c, a).alloc(st->ctx, st->cap[x]));
        }
        TRY(c.L.alloc(st->ctx, (uint64_t)N * st->n1 * 8));
        CU(cudaMemcpy(c.L.p, st->L.data(), (uint64_t)N * st->n1 * 8, cudaMemcpyHostToDevice));
        st->slots.push_back(std::move(sl));
    }
    return BN_OK;
}

// Reads a finished job's hits and per-trial sums into the query's accumulators.
struct Acc {
    std::vector<std::vector<std::pair<int64_t, uint32_t>>> cand;  // per query: (score, id)
    std::vector<uint64_t> ur, zv;                                  // [B][trials]
};

int finish_slot(bn_stream* st, Slot& sl, Acc& acc) {
    if (!sl.pending) return BN_OK;
    sl.pending = false;
    CU(cudaEventSynchronize(sl.scored));
    const QueryJob& j = sl.job;
    const uint32_t B = j.B, k = j.k, ks = std::max<uint32_t>(k, 1);
    std::vector<uint32_t> ids((uint64_t)B * ks), nh(B, 0);
    std::vector<int64_t> sc((uint64_t)B * ks);
    std::vector<int32_t> vf;
    TRY(job_finish(j, sl.f.e.host, ids.data(), sc.data(), nh.data(), vf));
    for (uint32_t b = 0; b < B; ++b)
        for (uint32_t i = 0; i < nh[b]; ++i)
            acc.cand[b].emplace_back(sc[(uint64_t)b * k + i], ids[(uint64_t)b * k + i] + (uint32_t)sl.job_row0);
    if (j.trials) {
        const char* h = sl.f.e.host.at<char>();
        const uint64_t* ur = reinterpret_cast<const uint64_t*>(h + j.o.ur);
        const uint64_t* zv = reinterpret_cast<const uint64_t*>(h + j.o.zv);
        for (uint64_t i = 0; i < (uint64_t)B * j.trials; ++i) {
            acc.ur[i] = add_mod(acc.ur[i], ur[i]);
            acc.zv[i] = add_mod(acc.zv[i], zv[i]);
        }
    }
    (void)st;
    return BN_OK;
}

// Copies chunk c's image into slot sl on the upload stream, after the
// slot's last scoring; the slot's corpus then describes chunk c.
int load_chunk(bn_stream* st, Slot& sl, uint32_t c) {
    const ChunkImage& ci = st->chunks[c];
    Corpus& cp = sl.f.e.c;
    CU(cudaStreamWaitEvent(st->upload, sl.scored, 0));
    for (int a = 0; a < A_COUNT_MAX; ++a) {
        const int x = array_index(st, a);
        if (x < 0 || !ci.bytes[x]) continue;
        CU(cudaMemcpyAsync(corpus_array(cp, a).p, static_cast<const char*>(ci.host) + ci.off[x], ci.bytes[x],
                           cudaMemcpyHostToDevice, st->upload));
    }
    CU(cudaEventRecord(sl.uploaded, st->upload));
    CU(cudaStreamWaitEvent(sl.f.e.stream, sl.uploaded, 0));
    cp.rows = ci.rows;
    sl.f.m = ci.rows;
    TRY(corpus_tmap(cp));
    sl.chunk = c;
    st->lru.st.uploads += 1;
    st->lru.st.bytes_uploaded += ci.total;
    return BN_OK;
}

int query_locked(bn_stream* st, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                 const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
                 uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed) {
    Acc acc;
    acc.cand.resize(B);
    acc.ur.assign((uint64_t)B * trials, 0);
    acc.zv.assign((uint64_t)B * trials, 0);
    // visiting order: resident chunks from the least recently used, then the rest
    std::vector<uint32_t> order;
    std::vector<char> seen(st->chunks.size(), 0);
    for (uint64_t id : st->lru.order) {
        order.push_back((uint32_t)id);
        seen[id] = 1;
    }
    for (uint32_t c = 0; c < st->chunks.size(); ++c)
        if (!seen[c]) order.push_back(c);
    std::vector<int> slot_of(st->chunks.size(), -1);
    for (size_t i = 0; i < st->slots.size(); ++i)
        if (st->slots[i]->chunk >= 0) slot_of[st->slots[i]->chunk] = (int)i;

    int rc = BN_OK;
    for (uint32_t c : order) {
        st->lru.st.gets += 1;
        int si = slot_of[c];
        if (si >= 0) {
            st->lru.touch(c);
        } else {
            std::vector<uint64_t> evicted;
            rc = st->lru.pre_evict(st->slot_bytes, evicted);
            if (rc != BN_OK) break;
            for (uint64_t e : evicted) {
                const int es = slot_of[e];
                slot_of[e] = -1;
                if (es >= 0) {
                    st->slots[es]->chunk = -1;
                    if (si < 0) si = es;
                }
            }
            if (si < 0)  // a free slot (fewer chunks resident than slots)
                for (size_t i = 0; i < st->slots.size() && si < 0; ++i)
                    if (st->slots[i]->chunk < 0) si = (int)i;
            if (si < 0) {
                rc = fail(BN_EBUDGET, "store: no slot for chunk %u", c);
                break;
            }
            Slot& sl = *st->slots[si];
            // the slot's previous chunk of this query: its results first
            if ((rc = finish_slot(st, sl, acc)) != BN_OK) break;
            if ((rc = load_chunk(st, sl, c)) != BN_OK) break;
            st->lru.insert(c, st->slot_bytes);
            slot_of[c] = si;
        }
        Slot& sl = *st->slots[si];
        if ((rc = finish_slot(st, sl, acc)) != BN_OK) break;
        const ChunkImage& ci = st->chunks[c];
        flat_meta(ci.rows, B, sl.hm);
        for (VerifySeg& vs : sl.hm.vsegs) {  // draw positions within the whole corpus
            vs.draw_stride = st->rows;
            vs.draw_base = ci.row0;
        }
        sl.job = QueryJob();
        sl.job.hm = &sl.hm;
        sl.job.B = B;
        sl.job.trials = trials;
        sl.job.k = k;
        sl.job_row0 = ci.row0;
        Engine& e = sl.f.e;
        if ((rc = job_prepare(e, sl.job, e.ws, e.host, v_enc, g, t_idx, t_sign, t_nnz, v_seeds)) != BN_OK) break;
        if ((rc = job_launch(e, sl.job, e.ws, e.host, e.stream, nullptr, nullptr)) != BN_OK) break;
        if (cudaEventRecord(sl.scored, e.stream) != cudaSuccess) {
            rc = fail(BN_ECUDA, "cudaEventRecord failed");
            break;
        }
        sl.pending = true;
    }
    for (auto& sl : st->slots) {  // every job in flight ends before the store moves on
        const int r2 = finish_slot(st, *sl, acc);
        if (rc == BN_OK) rc = r2;
    }
    if (rc != BN_OK) {
        // a failed load or launch may leave a slot's contents undefined: drop them
        for (auto& sl : st->slots) {
            if (sl->chunk >= 0) {
                auto it = std::find(st->lru.order.begin(), st->lru.order.end(), (uint64_t)sl->chunk);
                if (it != st->lru.order.end()) st->lru.order.erase(it);
                if (st->lru.entries.erase((uint64_t)sl->chunk)) st->lru.resident -= st->slot_bytes;
            }
            sl->chunk = -1;
        }
        return rc;
    }
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
        if (failed) {
            failed[b] = -1;
            for (uint32_t t = 0; t < trials; ++t)
                if (acc.ur[(uint64_t)b * trials + t] != acc.zv[(uint64_t)b * trials + t]) {
                    failed[b] = (int32_t)t;
                    break;
                }
        }
    }
    return BN_OK;
}

int stream_new(bn_ctx* ctx, uint64_t m, uint32_t n, uint32_t n1, const uint64_t* L, uint64_t chunk_rows,
               bn_stream** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    if (!m) return fail(BN_EINVAL, "empty corpus");
    if (m > 0xffffffffull) return fail(BN_EINVAL, "corpus rows must fit in u32");
    if (!L) return fail(BN_EINVAL, "l_subspace is required");
    if (chunk_rows < 32 || chunk_rows % 32) return fail(BN_EINVAL, "chunk_rows = %llu is not a positive multiple of 32",
                                                       (unsigned long long)chunk_rows);
    TRY(validate_residues(L, (uint64_t)N * n1, "l_subspace"));
    auto* st = new bn_stream();
    st->ctx = ctx;
    st->rows = m;
    st->chunk_rows = chunk_rows;
    st->n1 = n1;
    st->L.assign(L, L + (uint64_t)N * n1);
    *out = st;
    return BN_OK;
}

std::vector<uint64_t> rebased_rowptr(const uint64_t* rowptr, uint64_t row0, uint64_t rows) {
    std::vector<uint64_t> rp(rows + 1);
    for (uint64_t i = 0; i <= rows; ++i) rp[i] = rowptr[row0 + i] - rowptr[row0];
    return rp;
}

}  // namespace

extern "C" {

int bn_stream_build(bn_ctx* ctx, const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint64_t m,
                    uint32_t n, uint32_t n1, const uint64_t* l_subspace, const uint64_t* m_plain, bn_sparse_csr s_mat,
                    uint64_t chunk_rows, uint64_t budget_bytes, bn_stream** out) {
    bn_stream* st = nullptr;
    TRY(stream_new(ctx, m, n, n1, l_subspace, chunk_rows, &st));
    *out = nullptr;
    int rc = BN_OK;
    if (!m_enc || !a_l || !h || !m_plain || !s_mat.rowptr) rc = fail(BN_EINVAL, "null corpus array");
    if (rc == BN_OK) rc = validate_residues(m_plain, m * N, "m_plain");
    if (rc == BN_OK) {
        st->use_m8 = all_int8(m_plain, m * N);
        if (cudaSetDevice(ctx->device) != cudaSuccess) rc = fail(BN_ECUDA, "cudaSetDevice failed");
    }
    if (rc == BN_OK) {
        rc = build_chunks(st, [&](uint64_t row0, uint64_t rows, bn_flat** f) -> int {
            TRY(bn_flat_build(ctx, m_enc + row0 * N, a_l + row0 * n1, h + row0 * n1, rows, n, n1, f));
            const std::vector<uint64_t> rp = rebased_rowptr(s_mat.rowptr, row0, rows);
            const uint64_t nz0 = s_mat.rowptr[row0];
            bn_sparse_csr sc{rp.data(), s_mat.idx ? s_mat.idx + nz0 : nullptr, s_mat.sign ? s_mat.sign + nz0 : nullptr};
            const int r = bn_flat_attach_client(*f, l_subspace, m_plain + row0 * N, sc);
            if (r != BN_OK) {
                bn_flat_destroy(*f);
                *f = nullptr;
            }
            return r;
        });
    }
    if (rc == BN_OK) rc = make_slots(st, budget_bytes);
    if (rc != BN_OK) {
        delete st;
        return rc;
    }
    *out = st;
    return BN_OK;
}

int bn_stream_build_from_plain(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1,
                               const uint64_t* l_subspace, const uint64_t* h, bn_sparse_csr s_mat, uint64_t chunk_rows,
                               uint64_t budget_bytes, bn_stream** out) {
    bn_stream* st = nullptr;
    TRY(stream_new(ctx, m, n, n1, l_subspace, chunk_rows, &st));
    *out = nullptr;
    int rc = BN_OK;
    if (!m_q || !h || !s_mat.rowptr) rc = fail(BN_EINVAL, "null input array");
    if (rc == BN_OK) rc = validate_residues(m_q, m * N, "m_q");
    if (rc == BN_OK) {
        st->use_m8 = all_int8(m_q, m * N);
        if (cudaSetDevice(ctx->device) != cudaSuccess) rc = fail(BN_ECUDA, "cudaSetDevice failed");
    }
    if (rc == BN_OK) {
        rc = build_chunks(st, [&](uint64_t row0, uint64_t rows, bn_flat** f) -> int {
            const std::vector<uint64_t> rp = rebased_rowptr(s_mat.rowptr, row0, rows);
            const uint64_t nz0 = s_mat.rowptr[row0];
            bn_sparse_csr sc{rp.data(), s_mat.idx ? s_mat.idx + nz0 : nullptr, s_mat.sign ? s_mat.sign + nz0 : nullptr};
            return bn_flat_build_from_plain(ctx, m_q + row0 * N, rows, n, n1, l_subspace, h + row0 * n1, sc, f);
        });
    }
    if (rc == BN_OK) rc = make_slots(st, budget_bytes);
    if (rc != BN_OK) {
        delete st;
        return rc;
    }
    *out = st;
    return BN_OK;
}

int bn_stream_info(const bn_stream* st, uint64_t* rows, uint32_t* chunks, uint32_t* slots, uint64_t* slot_bytes,
                   uint64_t* host_bytes) {
    if (!st) return fail(BN_EINVAL, "null handle");
    if (rows) *rows = st->rows;
    if (chunks) *chunks = (uint32_t)st->chunks.size();
    if (slots) *slots = (uint32_t)st->slots.size();
    if (slot_bytes) *slot_bytes = st->slot_bytes;
    if (host_bytes) {
        uint64_t t = 0;
        for (const ChunkImage& ci : st->chunks) t += ci.total;
        *host_bytes = t;
    }
    return BN_OK;
}

int bn_stream_query(bn_stream* st, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                    const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
                    uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial) {
    if (!st) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX = %d", k, BN_TOPK_MAX);
    if (trials > MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %u", trials, MAX_TRIALS);
    if (k && (!ids || !scores || !n_hits)) return fail(BN_EINVAL, "ids, scores and n_hits are required when k > 0");
    if (!failed_trial) return fail(BN_EINVAL, "failed_trial is required");
    std::lock_guard<std::mutex> g_(st->mu);
    CU(cudaSetDevice(st->ctx->device));
    return query_locked(st, B, v_enc, g, t_idx, t_sign, t_nnz, v_seeds, trials, k, ids, scores, n_hits, failed_trial);
}

int bn_stream_stats(bn_stream* st, int reset, bn_store_stats* out) {
    if (!st || !out) return fail(BN_EINVAL, "null argument");
    std::lock_guard<std::mutex> g_(st->mu);
    st->lru.stats(out);
    if (reset) st->lru.st = bn_store_stats{};
    return BN_OK;
}

int bn_stream_destroy(bn_stream* st) {
    delete st;
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
