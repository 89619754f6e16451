"""Bit-exact parity with the oracle at the full size of the flat workloads.

The corpus is the one bench.py measures: N = 1,000,000 rows, d = 768
(n = 1024, n1 = 128), seeded Gaussian -> L2-normalise -> int8 -> F_p, BN
keygen on the host and encryption on the device (seed 1).  At this size the
fused scan runs 245 panels x 22 strip groups = 5390 work items (36 rounds of
148 CTAs), the Protocol 2 draws of 20 trials reach index 2 * 10^7, and the
decode spans 31,250 32-row units; none of that is reached by the small-case
tests.

Checked, each against the oracle's restatement of the reference
(scorer-bntm/src/crypto.rs, lib.rs), bit for bit:
  - keygen: L, H and S from the product's host code (crypto.rs:235-270);
  - encryption M_enc = M + H L^T + S and AL = M L on sampled rows
    (crypto.rs:405-478);
  - the single-query path of the bench (BnTmScorer::score, lib.rs:326-475):
    every r residue, every decoded residue, the top-10, the accept bit and
    every trial's u.r and z.v (verify_response, crypto.rs:1013-1059), on both
    Protocol 2 engines and through the device-buffer plan;
  - blocks of 8 queries (compute_products_batch + decode, crypto.rs:782-989):
    every decoded residue, the top-10 and the Protocol 2 verdict and sums
    under the block seed, on the host-buffer path and on an autotuned plan;
  - the decoded scores equal the exact integer dot products of the int8
    plaintexts (an order-free fact that needs no oracle)."""
from __future__ import annotations

import gc
import os
import sys
import types

import numpy as np
import pytest

import oracle as O
from bnutil import N, P

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ROWS, D, SEED, TRIALS, K = 1_000_000, 768, 1, 20, 10


def capi():
    from bn_b200 import capi as c

    return c


@pytest.fixture(scope="module")
def corpus(ctx):
    import bench

    c = capi()
    gc.collect()
    x8 = bench.synth_int8(ROWS, D, SEED)
    Mu = bench.to_residues(x8)
    key_seed = bytes([SEED & 0xFF]) * 32
    L = c.host_generate_subspace(key_seed)
    h_seed = c.host_derive_h_seed(SEED, 0)
    H, rp, ix, sg = c.host_regenerate_h_s(h_seed, ROWS)
    # full-size keygen parity: the product's host keygen against the oracle's
    assert h_seed == O.derive_h_seed(SEED, 0)
    assert np.array_equal(L, O.generate_subspace(key_seed))
    H_o, S_o = O.regenerate_h_s(h_seed, ROWS)
    assert np.array_equal(H, H_o) and np.array_equal(rp, S_o.rowptr)
    assert np.array_equal(ix, S_o.idx) and np.array_equal(sg, S_o.sign)
    del H_o, S_o
    flat = c.Flat.build_from_plain(ctx, Mu.reshape(-1), ROWS, L, H, rp, ix, sg)
    # host copies of the device encryption (the same kernels as the build)
    m_enc, a_l = c.encrypt_cluster(ctx, Mu.reshape(-1), ROWS, L, H, rp, ix, sg)
    m_enc = m_enc.reshape(ROWS, N)
    a_l = a_l.reshape(ROWS, 128)
    Hm = H.reshape(ROWS, 128)
    rng = np.random.default_rng(99)
    for i in [0, 1, 2**19 - 1, 2**19, ROWS - 1] + rng.choice(ROWS, 200, replace=False).tolist():
        hl = O.matvec(L, N, 128, Hm[i])  # row i of H L^T
        want = (Mu[i].astype(object) + hl.astype(object)) % P
        for e in range(int(rp[i]), int(rp[i + 1])):
            want[ix[e]] = (want[ix[e]] + int(sg[e])) % P
        assert np.array_equal(m_enc[i], want.astype(np.uint64)), f"M_enc row {i}"
        assert np.array_equal(a_l[i], O.matvec_transpose(L, N, 128, Mu[i])), f"AL row {i}"
    cl = O.Cluster(ROWS, N, 128, m_enc.reshape(-1), a_l.reshape(-1), Mu.reshape(-1), H, O.Sparse(rp, ix, sg))
    yield types.SimpleNamespace(flat=flat, cl=cl, L=L, x8=x8)
    flat.close()
    del cl, m_enc, a_l, Mu
    gc.collect()


def bench_queries(L, count, qseed_base, xseed):
    """The bench's encoded queries: int8 vectors of synth_int8(.., xseed) and
    q_seed i = derive_h_seed(qseed_base, i); the product's host encode is
    checked against the oracle's."""
    import bench

    c = capi()
    q8 = bench.synth_int8(count, D, xseed)
    qv = bench.to_residues(q8)
    out = []
    for i in range(count):
        q_seed = c.host_derive_h_seed(qseed_base, i)
        v_enc, g, ti, ts = c.host_encode_query(qv[i], L, q_seed)
        enc = O.encode_query(qv[i], L, q_seed)
        assert np.array_equal(v_enc, enc.v_enc) and np.array_equal(g, enc.g)
        assert np.array_equal(ti, enc.t_idx) and np.array_equal(ts, enc.t_sign)
        assert c.host_domain_separate(q_seed) == O.domain_separate(q_seed, b"protocol2")
        out.append((q8[i], qv[i], q_seed, enc))
    return out


def oracle_query(cl, L, enc, v_seed):
    r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
    f, ur, zv = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, TRIALS, v_seed)
    mv = O.decode_scores(r, cl, L, enc)
    ids, sc = O.topk(O.to_signed(mv), K)
    return r, f, ur, zv, mv, ids, sc


def test_single_query_path_at_one_million_rows(ctx, corpus):
    c = capi()
    qs = bench_queries(corpus.L, 2, SEED ^ 0x5155455259, SEED + 1000)
    for q8, qv, q_seed, enc in qs:
        vs = O.domain_separate(q_seed, b"protocol2")
        r_o, f_o, ur_o, zv_o, mv_o, ids_o, sc_o = oracle_query(corpus.cl, corpus.L, enc, vs)
        # the decoded residues are the plaintext dot products (int8 inputs, exact)
        # (f32 is exact here: products <= 127^2, |sums| <= 768 * 127^2 < 2^24)
        exact = corpus.x8.astype(np.float32) @ q8.astype(np.float32)
        assert np.array_equal(O.to_signed(mv_o), exact.astype(np.int64))
        args = (enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [vs])
        for engine in (c.ENGINE_TENSOR, c.ENGINE_CUDA_CORE):
            ctx.set_engine(engine)
            try:
                hits, failed, r, mv = corpus.flat.query(*args, TRIALS, K, want_r=True, want_mv=True)
                f_g, ur_g, zv_g = corpus.flat.verify(r_o, enc.v_enc, vs, TRIALS)
            finally:
                ctx.set_engine(c.ENGINE_TENSOR)
            assert np.array_equal(r[0], r_o), "scan residues differ"
            assert np.array_equal(mv[0], mv_o), "decoded residues differ"
            assert failed[0] == f_o == f_g == -1
            assert np.array_equal(ur_g, ur_o) and np.array_equal(zv_g, zv_o) and ur_o.size == TRIALS
            assert np.array_equal(hits[0][0], ids_o) and np.array_equal(hits[0][1], sc_o)


def test_device_buffer_plan_at_one_million_rows(corpus):
    """The bench's headline path: bn_plan_enqueue with device-resident inputs."""
    torch = pytest.importorskip("torch")
    qs = bench_queries(corpus.L, 3, SEED ^ 0x5155455259, SEED + 1000)[2:]
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    plan = corpus.flat.plan(1, TRIALS, K)
    for q8, qv, q_seed, enc in qs:
        vs = O.domain_separate(q_seed, b"protocol2")
        _, f_o, _, _, _, ids_o, sc_o = oracle_query(corpus.cl, corpus.L, enc, vs)
        t = np.zeros(N, np.uint32)
        t[: enc.t_idx.size] = enc.t_idx | np.where(enc.t_sign < 0, np.uint32(0x80000000), np.uint32(0))
        bufs = [torch.from_numpy(enc.v_enc.view(np.int64).copy()).to(dev),
                torch.from_numpy(enc.g.view(np.int64).copy()).to(dev),
                torch.from_numpy(t.view(np.int32)).to(dev),
                torch.tensor([enc.t_idx.size], dtype=torch.int32, device=dev),
                torch.from_numpy(np.frombuffer(vs, np.uint8).copy()).to(dev),
                torch.zeros(K, dtype=torch.int32, device=dev), torch.zeros(K, dtype=torch.int64, device=dev),
                torch.zeros(1, dtype=torch.int32, device=dev), torch.full((1,), 7, dtype=torch.int32, device=dev)]
        plan.enqueue(*[b.data_ptr() for b in bufs], stream)
        torch.cuda.synchronize(dev)
        assert plan.status() == 0
        n = int(bufs[7].item())
        assert n == K and int(bufs[8].item()) == f_o == -1
        assert np.array_equal(bufs[5].cpu().numpy().view(np.uint32)[:n], ids_o)
        assert np.array_equal(bufs[6].cpu().numpy()[:n], sc_o)
    plan.close()


def test_blocks_of_eight_at_one_million_rows(corpus):
    """Config 3's smallest block: 8 queries, one seed per block."""
    torch = pytest.importorskip("torch")
    B = 8
    qs = bench_queries(corpus.L, B, SEED ^ 0x424C4B, SEED + 2000)
    block_seed = bytes([1]) * 32
    encs = [q[3] for q in qs]
    vb = np.stack([e.v_enc for e in encs])
    gb = np.stack([e.g for e in encs])
    tb = [(e.t_idx, e.t_sign) for e in encs]
    R = O.matvec_batch(corpus.cl.m_enc, ROWS, N, vb)
    want = []
    for q in range(B):
        f, ur, zv = O.verify_response(R[q], corpus.cl.m_enc, ROWS, N, vb[q], TRIALS, block_seed)
        mv = O.decode_scores(R[q], corpus.cl, corpus.L, encs[q])
        ids, sc = O.topk(O.to_signed(mv), K)
        want.append((f, ur, zv, mv, ids, sc))
    hits, failed, mv = corpus.flat.query_block(vb, gb, tb, block_seed, TRIALS, K, want_mv=True)
    fl, ur, zv = corpus.flat.verify_block(R, vb, block_seed, TRIALS)
    for q in range(B):
        f_o, ur_o, zv_o, mv_o, ids_o, sc_o = want[q]
        assert np.array_equal(mv[q], mv_o), f"decoded residues of query {q}"
        assert failed[q] == fl[q] == f_o == -1
        assert np.array_equal(ur[:, q], ur_o) and np.array_equal(zv[:, q], zv_o)
        assert np.array_equal(hits[q][0], ids_o) and np.array_equal(hits[q][1], sc_o)
    # the autotuned device-buffer plan the bench replays in CUDA graphs
    dev = torch.device("cuda:0")
    t = np.zeros((B, N), np.uint32)
    for q, e in enumerate(encs):
        t[q, : e.t_idx.size] = e.t_idx | np.where(e.t_sign < 0, np.uint32(0x80000000), np.uint32(0))
    bufs = [torch.from_numpy(vb.view(np.int64).copy()).to(dev), torch.from_numpy(gb.view(np.int64).copy()).to(dev),
            torch.from_numpy(t.view(np.int32)).to(dev),
            torch.tensor([e.t_idx.size for e in encs], dtype=torch.int32, device=dev),
            torch.from_numpy(np.frombuffer(block_seed, np.uint8).copy()).to(dev),
            torch.zeros((B, K), dtype=torch.int32, device=dev), torch.zeros((B, K), dtype=torch.int64, device=dev),
            torch.zeros(B, dtype=torch.int32, device=dev), torch.full((B,), 7, dtype=torch.int32, device=dev)]
    plan = corpus.flat.block_plan(B, TRIALS, K, autotune=True)
    plan.enqueue(*[b.data_ptr() for b in bufs], torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    assert plan.status() == 0
    ids = bufs[5].cpu().numpy().view(np.uint32)
    sc = bufs[6].cpu().numpy()
    for q in range(B):
        assert int(bufs[8][q].item()) == -1 and int(bufs[7][q].item()) == K
        assert np.array_equal(ids[q], want[q][4]) and np.array_equal(sc[q], want[q][5])
    plan.close()
