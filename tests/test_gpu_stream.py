"""Corpora streamed through device memory (bn_stream, csrc/bn_stream.cu):
the chunked, LRU-resident corpus must answer exactly like the resident flat
corpus and the oracle (hits, Protocol 2 verdicts) at every budget, and its
counters must follow the reference store's (scorer-gpu-common/src/
store.rs:36-80, 327-392)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, cluster, query

pytestmark = pytest.mark.gpu


def capi():
    from bn_b200 import capi as c

    return c


@pytest.fixture(scope="module")
def corpus():
    m = 3000
    M, L, cl = cluster(m, 8800)
    qs = [query(L, 8810 + i) for i in range(3)]
    return M, L, cl, qs


def build_stream(ctx, M, L, cl, chunk_rows, slots):
    c = capi()
    probe = c.Stream.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m, L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx,
                           cl.s_mat.sign, chunk_rows, 1 << 40)
    slot = probe.info()["slot_bytes"]
    probe.close()
    return c.Stream.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m, L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx,
                          cl.s_mat.sign, chunk_rows, slots * slot)


def args(qs, trials, k):
    encs = [q[2] for q in qs]
    seeds = [O.domain_separate(q[1], b"protocol2") for q in qs]
    return (np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]), [(e.t_idx, e.t_sign) for e in encs],
            seeds, trials, k)


@pytest.mark.parametrize("chunk_rows,slots", [(1024, 1), (1024, 2), (1024, 3), (992, 2), (4096, 1)])
def test_stream_equals_resident_and_oracle(ctx, corpus, chunk_rows, slots):
    c = capi()
    M, L, cl, qs = corpus
    flat = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    flat.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    st = build_stream(ctx, M, L, cl, chunk_rows, slots)
    info = st.info()
    assert info["chunks"] == -(-cl.m // chunk_rows) and info["slots"] == min(slots, info["chunks"])
    a = args(qs, 20, 10)
    want, wf, _, _ = flat.query(*a)
    for _ in range(3):  # repeated queries: resident chunks first, then the uploads
        got, gf = st.query(*a)
        for b in range(len(qs)):
            assert np.array_equal(got[b][0], want[b][0]) and np.array_equal(got[b][1], want[b][1])
        assert np.array_equal(gf, wf) and np.all(gf == -1)
    for b, (v, q_seed, _) in enumerate(qs):  # and the oracle
        fo, ids, sc, _, _ = O.score_flat(cl, L, v, q_seed, 20, 10)
        assert fo == -1 and np.array_equal(got[b][0], ids) and np.array_equal(got[b][1], sc)
    s = st.stats()
    ch, sl = info["chunks"], info["slots"]
    assert s["gets"] == 3 * ch
    assert s["uploads"] == ch + 2 * (ch - sl)  # every chunk once, then the ones that do not fit
    assert s["evictions"] == s["uploads"] - sl
    assert s["resident_bytes"] == sl * info["slot_bytes"] and s["bytes_uploaded"] > 0
    st.close()
    flat.close()


def test_stream_other_trials_and_k(ctx, corpus):
    """k = 0, k = 1024 and no Protocol 2, trials 3 (the reference's default):
    the same as the resident corpus."""
    c = capi()
    M, L, cl, qs = corpus
    st = build_stream(ctx, M, L, cl, 1024, 2)
    flat = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    flat.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    for trials, k in [(3, 0), (3, 1024), (0, 5)]:
        a = args(qs, trials, k)
        got, gf = st.query(*a)
        want, wf, _, _ = flat.query(*a)
        assert np.array_equal(gf, wf)
        for b in range(len(qs)):
            assert np.array_equal(got[b][0], want[b][0]) and np.array_equal(got[b][1], want[b][1])
    st.close()
    flat.close()


def test_stream_from_plain_and_budget_errors(ctx, corpus):
    c = capi()
    M, L, cl, qs = corpus
    st = c.Stream.build_from_plain(ctx, M.reshape(-1), cl.m, L, cl.h_mat, cl.s_mat.rowptr, cl.s_mat.idx,
                                   cl.s_mat.sign, 2048, 1 << 40)
    got, gf = st.query(*args(qs, 20, 10))
    for b, (v, q_seed, _) in enumerate(qs):
        fo, ids, sc, _, _ = O.score_flat(cl, L, v, q_seed, 20, 10)
        assert gf[b] == fo == -1 and np.array_equal(got[b][0], ids) and np.array_equal(got[b][1], sc)
    st.close()
    with pytest.raises(c.BnError) as e:  # the reference's BudgetTooSmall
        c.Stream.build_from_plain(ctx, M.reshape(-1), cl.m, L, cl.h_mat, cl.s_mat.rowptr, cl.s_mat.idx,
                                  cl.s_mat.sign, 1024, 1 << 20)
    assert e.value.code == c.BN_EBUDGET
    with pytest.raises(c.BnError) as e:
        c.Stream.build_from_plain(ctx, M.reshape(-1), cl.m, L, cl.h_mat, cl.s_mat.rowptr, cl.s_mat.idx,
                                  cl.s_mat.sign, 1000, 1 << 40)  # not a multiple of 32
    assert e.value.code == c.BN_EINVAL


def test_stream_non_int8_plaintext(ctx):
    """Plaintext outside int8: every chunk keeps the residues (M . T from them)."""
    c = capi()
    m = 700
    M, L, cl = cluster(m, 8850, uniform=True)
    st = build_stream(ctx, M, L, cl, 256, 1)
    v, q_seed, enc = query(L, 8851)
    got, gf = st.query(*args([(v, q_seed, enc)], 20, 10))
    fo, ids, sc, _, _ = O.score_flat(cl, L, v, q_seed, 20, 10)
    assert gf[0] == fo and np.array_equal(got[0][0], ids) and np.array_equal(got[0][1], sc)
    st.close()


# ---------------------------------------------------------------- IVF

def ivf_args(case, B, nprobe, trials, k, seed):
    rng = np.random.default_rng(seed)
    probes = np.stack([rng.choice(case.nlist, nprobe, replace=False) for _ in range(B)]).astype(np.uint32)
    encs = [O.encode_query(case.M[(7 * b) % case.M.shape[0]], case.L, bytes([90 + b]) * 32) for b in range(B)]
    seeds = [O.domain_separate(bytes([90 + b]) * 32, b"protocol2") for b in range(B)]
    return probes, encs, seeds, (probes, np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                                 [(e.t_idx, e.t_sign) for e in encs], seeds, trials, k)


@pytest.mark.parametrize("chunk_rows,slots", [(256, 1), (256, 2), (700, 2), (100000, 1)])
def test_ivf_stream_equals_resident_and_oracle(ctx, chunk_rows, slots):
    """Lists larger than a chunk (400 rows at chunk 256), empty lists, chunks
    that hold several lists; repeated calls go through the LRU."""
    from ivfutil import IvfCase

    c = capi()
    case = IvfCase([50, 0, 3, 200, 1, 0, 97, 400, 33, 120, 64, 9])
    m_enc, a_l, h, rp, ix, sg = case.concat()
    res = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    res.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    probe = c.IvfStream.build(ctx, case.offsets, case.ids, m_enc, a_l, h, case.L, case.M.reshape(-1), rp, ix, sg,
                              chunk_rows, 1 << 40)
    slot = probe.info()["slot_bytes"]
    probe.close()
    st = c.IvfStream.build(ctx, case.offsets, case.ids, m_enc, a_l, h, case.L, case.M.reshape(-1), rp, ix, sg,
                           chunk_rows, slots * slot)
    info = st.info()
    assert info["rows"] == int(case.offsets[-1]) and info["slots"] == min(slots, info["chunks"])
    for call in range(3):
        probes, encs, seeds, a = ivf_args(case, 5, 4, 20, 10, 70 + call)
        want, wc, wt = res.query(*a)
        got, gc, gt = st.query(*a)
        assert np.array_equal(gc, wc) and np.array_equal(gt, wt) and np.all(gt == -1)
        for b in range(5):
            assert np.array_equal(got[b][0], want[b][0]) and np.array_equal(got[b][1], want[b][1])
            o = case.oracle_score(probes[b], encs[b], seeds[b], 20, 10)
            assert np.array_equal(got[b][0], o[0]) and np.array_equal(got[b][1], o[1])
    s = st.stats()
    assert s["gets"] >= s["uploads"] >= 1 and s["resident_bytes"] <= slots * slot
    st.close()
    res.close()


def test_ivf_stream_keygen_equals_resident_keygen(ctx):
    """Chunks built by device keygen draw each list's keys from its global
    list index (derive_h_seed(upload_seed, list), ivf.rs:258-264)."""
    from ivfutil import IvfCase

    c = capi()
    case = IvfCase([50, 0, 3, 200, 1, 0, 97, 400, 33], upload_seed=7)
    res = c.Ivf.build_keygen(ctx, case.offsets, case.ids, case.M.reshape(-1), case.L, 7)
    st = c.IvfStream.build_keygen(ctx, case.offsets, case.ids, case.M.reshape(-1), case.L, 7, 256, 1 << 40)
    assert st.info()["chunks"] >= 3
    probes, encs, seeds, a = ivf_args(case, 4, 5, 3, 20, 81)
    want, wc, wt = res.query(*a)
    got, gc, gt = st.query(*a)
    assert np.array_equal(gc, wc) and np.array_equal(gt, wt)
    for b in range(4):
        assert np.array_equal(got[b][0], want[b][0]) and np.array_equal(got[b][1], want[b][1])
        o = case.oracle_score(probes[b], encs[b], seeds[b], 3, 20)
        assert np.array_equal(got[b][0], o[0]) and np.array_equal(got[b][1], o[1])
    st.close()
    res.close()
