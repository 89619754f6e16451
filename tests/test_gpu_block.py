"""GPU parity of block scoring (B queries per launch on the tensor cores).

Every query of a block must give exactly what the oracle's per-query path
gives for r, the decoded Mv, the top-k ids and scores; the Freivalds verdict
and every trial's (u.r, (u^T M).v) pair must equal the oracle's
verify_response (crypto.rs:1013-1059) run with the block's one seed.  All
comparisons are bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, cluster, query, uniform_fp

pytestmark = pytest.mark.gpu


def capi():
    from bn_b200 import capi as c

    return c


def flat_from_cluster(ctx, M, L, cl):
    c = capi()
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    return f


def block_inputs(L, B, seed0):
    encs, vs = [], []
    for b in range(B):
        v, q_seed, enc = query(L, seed0 + b)
        encs.append(enc)
        vs.append(v)
    return vs, encs


def oracle_block(cl, L, vs, encs, block_seed, trials, k):
    out = []
    for v, enc in zip(vs, encs):
        r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
        mv = O.decode_scores(r, cl, L, enc)
        ids, sc = O.topk(O.to_signed(mv), k)
        f = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, trials, block_seed)[0] if trials else -1
        out.append((r, mv, ids, sc, f))
    return out


@pytest.mark.parametrize("m,B,trials,k", [(2000, 8, 3, 10), (777, 3, 20, 16), (4097, 20, 23, 10), (1, 1, 2, 5),
                                          (300, 33, 0, 1024), (130, 64, 1, 7)])
def test_block_query_matches_oracle(ctx, m, B, trials, k):
    M, L, cl = cluster(m, 700 + m)
    f = flat_from_cluster(ctx, M, L, cl)
    vs, encs = block_inputs(L, B, 1300 + m)
    seed = bytes([m % 251, 3]) * 16
    want = oracle_block(cl, L, vs, encs, seed, trials, k)
    hits, failed, mv = f.query_block(np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                                     [(e.t_idx, e.t_sign) for e in encs], seed if trials else None, trials, k,
                                     want_mv=True)
    for b in range(B):
        r, mvo, ids, sc, fo = want[b]
        assert np.array_equal(mv[b], mvo), b
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc), b
        assert failed[b] == fo == -1
        assert len(hits[b][0]) == min(k, m)


@pytest.mark.parametrize("n1", [64, 512])
def test_block_query_matches_oracle_across_n1(ctx, n1):
    """Block scoring at the smallest and largest n1 of the reference's delta
    sweep: [AL | H] planes of 2 n1 bytes per plane row (one or eight K steps)."""
    from bnutil import int8_matrix

    c = capi()
    m, B, trials, k = 900, 6, 3, 12
    M = int8_matrix(m, 768, 90 + n1)
    L = O.generate_subspace(bytes([5]) * 32, n1=n1)
    cl = O.encrypt_cluster(M.reshape(-1), m, L, O.derive_h_seed(9, 0), n1=n1)
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m, n1=n1)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    encs = [O.encode_query(int8_matrix(1, 768, 91 + n1 + b)[0], L, O.derive_h_seed(92, b), n1=n1) for b in range(B)]
    seed = bytes([n1 % 251, 7]) * 16
    hits, failed, mv = f.query_block(np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                                     [(e.t_idx, e.t_sign) for e in encs], seed, trials, k, want_mv=True)
    for b, enc in enumerate(encs):
        r = O.matvec(cl.m_enc, m, N, enc.v_enc)
        mvo = O.decode_scores(r, cl, L, enc)
        ids, sc = O.topk(O.to_signed(mvo), k)
        assert np.array_equal(mv[b], mvo), b
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc), b
        assert failed[b] == O.verify_response(r, cl.m_enc, m, N, enc.v_enc, trials, seed)[0] == -1


@pytest.mark.parametrize("m,B,trials", [(777, 5, 20), (4097, 17, 3), (10000, 2, 29), (1, 1, 1)])
def test_block_verify_matches_oracle(ctx, m, B, trials):
    """Uniform F_p corpus (no client state needed): every trial's pair per query."""
    c = capi()
    m_enc = uniform_fp((m, N), 810 + m)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    v = uniform_fp((B, N), 811 + m)
    r = O.matvec_batch(m_enc, m, N, v)
    seed = bytes([9]) * 32
    fl, ur, zv = f.verify_block(r, v, seed, trials)
    for b in range(B):
        fo, uro, zvo = O.verify_response(r[b], m_enc, m, N, v[b], trials, seed)
        assert fl[b] == fo == -1
        assert np.array_equal(ur[:, b], uro) and np.array_equal(zv[:, b], zvo)


def test_block_verify_extreme_residues(ctx):
    """All-(p-1) corpus and queries: the largest byte limbs everywhere."""
    c = capi()
    m, B = 4500, 4
    m_enc = np.full((m, N), P - 1, np.uint64)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    v = np.full((B, N), P - 1, np.uint64)
    v[1, ::2] = 0
    r = O.matvec_batch(m_enc, m, N, v)
    seed = bytes([77]) * 32
    fl, ur, zv = f.verify_block(r, v, seed, 20)
    for b in range(B):
        fo, uro, zvo = O.verify_response(r[b], m_enc, m, N, v[b], 20, seed)
        assert fl[b] == fo == -1 and np.array_equal(ur[:, b], uro) and np.array_equal(zv[:, b], zvo)


@pytest.mark.parametrize("pos", [0, 400, 776])
def test_block_verify_detects_tampered_response(ctx, pos):
    """crypto.rs:1445-1474 per query: only the tampered query is rejected, at trial 0."""
    c = capi()
    m, B = 777, 6
    m_enc = uniform_fp((m, N), 820)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    v = uniform_fp((B, N), 821)
    r = O.matvec_batch(m_enc, m, N, v)
    bad = 4
    r[bad, pos] = (int(r[bad, pos]) + 1) % P
    seed = bytes([35]) * 32
    fl, ur, zv = f.verify_block(r, v, seed, 20)
    for b in range(B):
        fo, uro, zvo = O.verify_response(r[b], m_enc, m, N, v[b], 20, seed)
        assert fl[b] == fo == (0 if b == bad else -1)
        ran = 20 if fo < 0 else fo + 1
        assert np.array_equal(ur[:ran, b], uro) and np.array_equal(zv[:ran, b], zvo)


def test_block_plan_autotune_and_graph_capture(ctx):
    """Plan enqueue (autotuned tiling), and its CUDA-graph replay, equal query_block."""
    torch = pytest.importorskip("torch")
    M, L, cl = cluster(5000, 61)
    f = flat_from_cluster(ctx, M, L, cl)
    B, trials, k = 32, 20, 10
    vs, encs = block_inputs(L, B, 3100)
    seed = bytes([5]) * 32
    want, wf, _ = f.query_block(np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                                [(e.t_idx, e.t_sign) for e in encs], seed, trials, k)
    dev = torch.device("cuda:0")
    t = np.zeros((B, N), np.uint32)
    tn = np.zeros(B, np.uint32)
    for b, e in enumerate(encs):
        tn[b] = e.t_idx.size
        t[b, : e.t_idx.size] = e.t_idx | np.where(e.t_sign < 0, np.uint32(0x80000000), np.uint32(0))
    d_v = torch.from_numpy(np.stack([e.v_enc for e in encs]).view(np.int64)).to(dev)
    d_g = torch.from_numpy(np.stack([e.g for e in encs]).view(np.int64)).to(dev)
    d_t = torch.from_numpy(t.view(np.int32)).to(dev)
    d_tn = torch.from_numpy(tn.view(np.int32)).to(dev)
    d_s = torch.from_numpy(np.frombuffer(seed, np.uint8).copy()).to(dev)
    d_ids = torch.zeros((B, k), dtype=torch.int32, device=dev)
    d_sc = torch.zeros((B, k), dtype=torch.int64, device=dev)
    d_n = torch.zeros(B, dtype=torch.int32, device=dev)
    d_f = torch.zeros(B, dtype=torch.int32, device=dev)
    plan = f.block_plan(B, trials, k, autotune=True)
    cfg = plan.block_config()
    assert cfg["w_tile"] in (64, 128, 256) and 2 <= cfg["stages"] <= 12 and cfg["two_ksteps_per_stage"] in (0, 1) and cfg["k_panel"] in (4096, 8192, 16384)
    stream = torch.cuda.Stream()
    args = [x.data_ptr() for x in (d_v, d_g, d_t, d_tn, d_s, d_ids, d_sc, d_n, d_f)]

    def check():
        ids, sc, n, fl = (d_ids.cpu().numpy().view(np.uint32), d_sc.cpu().numpy(), d_n.cpu().numpy(),
                          d_f.cpu().numpy())
        for b in range(B):
            assert n[b] == len(want[b][0])
            assert np.array_equal(ids[b, : n[b]], want[b][0]) and np.array_equal(sc[b, : n[b]], want[b][1])
            assert fl[b] == wf[b] == -1

    with torch.cuda.stream(stream):
        plan.enqueue(*args, stream.cuda_stream)
    stream.synchronize()
    assert plan.status() == 0
    check()
    for x in (d_ids, d_sc, d_n):
        x.zero_()
    d_f.fill_(7)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        plan.enqueue(*args, torch.cuda.current_stream().cuda_stream)
    graph.replay()
    torch.cuda.synchronize()
    assert plan.status() == 0
    check()
    del graph


def test_block_needs_int8_client_state(ctx):
    """A corpus whose plaintext is not int8-valued is refused (per-query paths still serve it)."""
    c = capi()
    M, L, cl = cluster(300, 71, uniform=True)
    f = flat_from_cluster(ctx, M, L, cl)
    v, q_seed, enc = query(L, 72)
    with pytest.raises(c.BnError) as e:
        f.query_block(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], bytes(32), 3, 10)
    assert e.value.code == c.BN_EUNSUPPORTED
    hits, failed, _, _ = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)],
                                 [O.domain_separate(q_seed, b"protocol2")], 3, 10)
    assert failed[0] == -1 and len(hits[0][0]) == 10
