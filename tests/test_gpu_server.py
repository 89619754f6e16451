"""The serving loop (bn_server): continuous batching over a flat and an IVF
corpus.  Every result must be bit-identical to the per-query entry points
(bn_flat_query / bn_ivf_query, themselves pinned to the oracle) whether the
request ran alone or in a mix of concurrent flat and IVF requests with
different nprobe; memory admission must bound the workspace and refuse a
request that cannot fit."""
from __future__ import annotations

import threading

import numpy as np
import pytest

import oracle as O
from bnutil import cluster, int8_matrix, query
from ivfutil import IvfCase

pytestmark = pytest.mark.gpu

SIZES = [50, 0, 3, 200, 1, 0, 97, 400, 33, 120, 7, 260]
TRIALS, K = 5, 10


def capi():
    from bn_b200 import capi as c

    return c


@pytest.fixture(scope="module")
def corpora(ctx):
    c = capi()
    M, L, cl = cluster(3000, 4100)
    flat = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    flat.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    case = IvfCase(SIZES, seed=4200)
    m_enc, a_l, h, rp, ix, sg = case.concat()
    ivf = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    ivf.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    return flat, L, ivf, case


def requests(L, case, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = "flat" if i % 2 == 0 else "ivf"
        lk = L if kind == "flat" else case.L
        v, q_seed, enc = query(lk, seed + i)
        vs = O.domain_separate(q_seed, b"protocol2")
        probes = rng.choice(case.nlist, size=int(rng.choice([1, 4, 12])), replace=False).astype(np.uint32)
        out.append((kind, enc, vs, probes))
    return out


def direct(flat, ivf, req):
    kind, enc, vs, probes = req
    if kind == "flat":
        hits, failed, _, _ = flat.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [vs], TRIALS, K)
        return hits[0][0], hits[0][1], int(failed[0]), -1
    hits, fc, ft = ivf.query(probes[None], enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [vs], TRIALS, K)
    return hits[0][0], hits[0][1], int(ft[0]), int(fc[0])


def submit(srv, req):
    kind, enc, vs, probes = req
    if kind == "flat":
        return srv.submit_flat(enc.v_enc, enc.g, enc.t_idx, enc.t_sign, vs)
    return srv.submit_ivf(probes, enc.v_enc, enc.g, enc.t_idx, enc.t_sign, vs)


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2] and a[3] == b[3]


def test_alone_and_mixed_results_are_identical(corpora):
    c = capi()
    flat, L, ivf, case = corpora
    reqs = requests(L, case, 24, 5000)
    want = [direct(flat, ivf, r) for r in reqs]
    # the per-query IVF path is pinned to the oracle (flat: test_gpu_flat); spot-check two requests
    for i in (1, 3):
        kind, enc, vs, probes = reqs[i]
        ids, sc = case.oracle_score(probes, enc, vs, TRIALS, K)
        assert np.array_equal(want[i][0], ids) and np.array_equal(want[i][1], sc)
    srv = c.Server(flat, ivf, max_batch=8, slots=3, max_wait_us=300, trials=TRIALS, k=K)
    alone = []
    for r in reqs:  # one at a time: every batch holds a single request
        t = submit(srv, r)
        ids, sc, ft, fc, lat = srv.wait(t)
        alone.append((ids, sc, ft, fc))
    for a, w in zip(alone, want):
        assert same(a, w)
    # all at once from two threads: mixed flat / IVF batches, several in flight
    tickets = [None] * len(reqs)

    def worker(lo):
        for i in range(lo, len(reqs), 2):
            tickets[i] = submit(srv, reqs[i])

    th = [threading.Thread(target=worker, args=(lo,)) for lo in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    mixed = []
    for t in tickets:
        ids, sc, ft, fc, lat = srv.wait(t)
        mixed.append((ids, sc, ft, fc))
    for m, w in zip(mixed, want):
        assert same(m, w)
    st = srv.stats()
    assert st["completed"] == st["submitted"] == 2 * len(reqs)
    assert st["mean_batch"] > 1.0  # the mix really was batched
    assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
    srv.close()


def test_memory_admission_bounds_workspace(corpora):
    c = capi()
    flat, L, ivf, case = corpora
    reqs = requests(L, case, 16, 6100)
    want = [direct(flat, ivf, r) for r in reqs]
    # a budget that holds a batch of a few queries but not of all 16: the
    # largest single-request workspace, times three
    probe = c.Server(flat, ivf, max_batch=1, slots=1, max_wait_us=0, trials=TRIALS, k=K)
    for r in reqs:
        probe.wait(submit(probe, r))
    one = probe.stats()["peak_workspace_bytes"]
    probe.close()
    budget = 3 * one
    srv = c.Server(flat, ivf, max_batch=16, slots=2, mem_budget=budget, max_wait_us=2000, trials=TRIALS, k=K)
    tickets = [submit(srv, r) for r in reqs]
    got = [srv.wait(t)[:4] for t in tickets]
    for g, w in zip(got, want):
        assert same(g, w)
    st = srv.stats()
    assert st["peak_workspace_bytes"] <= budget
    srv.close()
    # a request that cannot fit alone is refused with BN_EBUDGET
    tiny = c.Server(flat, ivf, max_batch=4, slots=1, mem_budget=1024, max_wait_us=0, trials=TRIALS, k=K)
    t = submit(tiny, reqs[0])
    with pytest.raises(c.BnError) as e:
        tiny.wait(t)
    assert e.value.code == c.BN_EBUDGET
    tiny.close()


def test_wait_timeout_and_bad_requests(corpora):
    c = capi()
    flat, L, ivf, case = corpora
    srv = c.Server(flat, ivf, max_batch=4, slots=1, max_wait_us=0, trials=TRIALS, k=K)
    with pytest.raises(c.BnError) as e:
        srv.wait(12345, timeout_ms=1)
    assert e.value.code == c.BN_EINVAL  # unknown ticket
    v, q_seed, enc = query(case.L, 77)
    with pytest.raises(c.BnError) as e:
        srv.submit_ivf(np.array([case.nlist], np.uint32), enc.v_enc, enc.g, enc.t_idx, enc.t_sign, bytes(32))
    assert e.value.code == c.BN_EINVAL  # list out of range
    bad = enc.v_enc.copy()
    bad[3] = O.P
    with pytest.raises(c.BnError) as e:
        srv.submit_flat(bad, enc.g, enc.t_idx, enc.t_sign, bytes(32))
    assert e.value.code == c.BN_EINVAL  # not a canonical residue
    srv.close()


def test_flat_block_batches_match_per_query(corpora):
    """Flat batches of >= block_min requests run as block scoring (one pass
    over the corpus for the batch): hits identical to the per-query path,
    honest responses accepted."""
    c = capi()
    flat, L, ivf, case = corpora
    reqs = [r for r in requests(L, case, 40, 7300) if r[0] == "flat"]
    want = [direct(flat, ivf, r) for r in reqs]
    srv = c.Server(flat, ivf, max_batch=16, slots=2, max_wait_us=20000, trials=TRIALS, k=K, block_min=4)
    tickets = [submit(srv, r) for r in reqs]
    got = [srv.wait(t)[:4] for t in tickets]
    for g, w in zip(got, want):
        assert same(g, w)
    st = srv.stats()
    assert st["block_batches"] > 0 and st["completed"] == len(reqs)
    srv.close()


@pytest.fixture(scope="module")
def big_flat(ctx):
    """100k rows: every top-k CTA compacts its candidate buffer several times."""
    c = capi()
    rows = 100_000
    M = int8_matrix(rows, 768, 9100)
    L = O.generate_subspace(bytes([9]) * 32)
    H, rp, ix, sg = c.host_regenerate_h_s(O.derive_h_seed(91, 0), rows)
    f = c.Flat.build_from_plain(ctx, M.reshape(-1), rows, L, H, rp, ix, sg)
    return f, L


def test_concurrent_block_and_per_query_batches(big_flat):
    """Block batches and per-query batches in flight together on several
    slots (the timing under which warps of one CTA drift apart): every result
    equals the per-query path."""
    c = capi()
    flat, L = big_flat
    pool = [query(L, 9200 + i) for i in range(64)]
    want = []
    for v, qs, enc in pool:
        hits, failed, _, _ = flat.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)],
                                        [O.domain_separate(qs, b"protocol2")], TRIALS, K)
        want.append((hits[0][0], hits[0][1]))
    srv = c.Server(flat, None, max_batch=64, slots=4, max_wait_us=0, trials=TRIALS, k=K, block_min=8)
    rng = np.random.default_rng(93)
    bad = 0
    for burst in range(12):
        picks = rng.integers(0, len(pool), size=40)
        ts = []
        for i in picks:
            v, qs, enc = pool[i]
            ts.append(srv.submit_flat(enc.v_enc, enc.g, enc.t_idx, enc.t_sign, O.domain_separate(qs, b"protocol2")))
        for t, i in zip(ts, picks):
            ids, sc, ft, fc, lat = srv.wait(t)
            bad += not (np.array_equal(ids, want[i][0]) and np.array_equal(sc, want[i][1]) and ft == -1)
    st = srv.stats()
    srv.close()
    assert bad == 0
    assert st["block_batches"] > 0 and st["batches"] > st["block_batches"]  # both paths were exercised


def test_ivf_block_batches_match_per_query(corpora):
    """IVF batches of >= block_min requests (mixed nprobe) run as IVF block
    scoring (pairs grouped by list, every probed list read once): hits
    identical to the per-query path, honest responses accepted."""
    c = capi()
    flat, L, ivf, case = corpora
    reqs = [r for r in requests(L, case, 48, 7700) if r[0] == "ivf"]
    want = [direct(flat, ivf, r) for r in reqs]
    srv = c.Server(flat, ivf, max_batch=16, slots=2, max_wait_us=20000, trials=TRIALS, k=K, block_min=4)
    tickets = [submit(srv, r) for r in reqs]
    got = [srv.wait(t)[:4] for t in tickets]
    for g, w in zip(got, want):
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1]) and g[2] == -1 and g[3] == -1
    st = srv.stats()
    assert st["block_batches"] > 0 and st["completed"] == len(reqs)
    srv.close()


def test_queue_admission_refuses_with_eagain(corpora):
    """A bounded queue: with max_queue waiting requests a submit is refused
    with BN_EAGAIN (nothing queued); every admitted request is served and
    equals the per-query path."""
    c = capi()
    flat, L, ivf, case = corpora
    reqs = requests(L, case, 24, 8100)
    want = [direct(flat, ivf, r) for r in reqs]
    srv = c.Server(flat, ivf, max_batch=4, slots=1, max_wait_us=200000, trials=TRIALS, k=K, max_queue=6)
    tickets, refused = [], 0
    for i, r in enumerate(reqs):
        try:
            tickets.append((submit(srv, r), i))
        except c.BnError as e:
            assert e.code == c.BN_EAGAIN and "queue full" in str(e)
            refused += 1
    for t, i in tickets:
        assert same(srv.wait(t)[:4], want[i])
    st = srv.stats()
    srv.close()
    assert refused > 0 and st["rejected"] == refused and st["completed"] == len(tickets)


def test_queue_wait_admission(corpora):
    """Latency-aware admission: once completions give a service rate, a
    submit whose expected queue wait exceeds queue_wait_us is refused."""
    c = capi()
    flat, L, ivf, case = corpora
    reqs = [r for r in requests(L, case, 80, 8300) if r[0] == "flat"]
    srv = c.Server(flat, ivf, max_batch=2, slots=1, max_wait_us=0, trials=TRIALS, k=K, queue_wait_us=1)
    for r in reqs[:10]:  # completions give the server its service rate
        srv.wait(submit(srv, r))
    refused, tickets = 0, []
    for r in reqs[10:]:
        try:
            tickets.append(submit(srv, r))
        except c.BnError as e:
            assert e.code == c.BN_EAGAIN and "expected queue wait" in str(e)
            refused += 1
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    srv.close()
    assert refused > 0 and st["rejected"] == refused
