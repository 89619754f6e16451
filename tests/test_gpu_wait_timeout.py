"""Failure detection on the device without a GPU fault.

Every pipeline wait of the scan, fused Protocol 2 and block GEMM kernels
(mbarrier waits between their copy, MMA and drain roles) is bounded: after
the limit the kernel records the event in its status word, waits (with the
full limit) for the copies and MMAs its CTA already issued, frees its tensor
memory and returns, so the context stays usable.  Here the limit is cut to a
few hundred cycles, far below a copy's latency, so the waits run out on
purpose: each call must fail with BN_ECUDA, the plan status must carry the
timeout bits, and the next call with the default limit must again equal the
oracle."""
from __future__ import annotations

import contextlib

import numpy as np
import pytest

import oracle as O
from bnutil import N, cluster, query

pytestmark = pytest.mark.gpu

TINY = 200  # cycles: any copy or MMA takes longer


def capi():
    from bn_b200 import capi as c

    return c


@contextlib.contextmanager
def short_waits(ctx):
    ctx.set_wait_limit(TINY)
    try:
        yield
    finally:
        ctx.set_wait_limit(0)


@pytest.fixture(scope="module")
def corpus(ctx):
    c = capi()
    M, L, cl = cluster(6000, 515)
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    yield M, L, cl, f
    f.close()


def expect_timeout(fn):
    c = capi()
    with pytest.raises(c.BnError) as ei:
        fn()
    assert ei.value.code == c.BN_ECUDA and "timed out" in str(ei.value), str(ei.value)


@pytest.mark.parametrize("engine", ["tensor", "cuda_core"])
def test_query_reports_timeout_then_recovers(ctx, corpus, engine):
    c = capi()
    M, L, cl, f = corpus
    v, q_seed, enc = query(L, 808)
    vs = O.domain_separate(q_seed, b"protocol2")
    args = (enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [vs])
    ctx.set_engine(c.ENGINE_TENSOR if engine == "tensor" else c.ENGINE_CUDA_CORE)
    try:
        with short_waits(ctx):
            expect_timeout(lambda: f.query(*args, 20, 10))
            expect_timeout(lambda: f.compute_products(enc.v_enc))
        hits, failed, r, _ = f.query(*args, 20, 10, want_r=True)
    finally:
        ctx.set_engine(c.ENGINE_TENSOR)
    want_f, ids, sc, r_o, _ = O.score_flat(cl, L, v, q_seed, 20, 10, want_r=True)
    assert failed[0] == want_f == -1
    assert np.array_equal(r[0], r_o)
    assert np.array_equal(hits[0][0], ids) and np.array_equal(hits[0][1], sc)


def test_plan_status_carries_timeout_bits(ctx, corpus):
    torch = pytest.importorskip("torch")
    M, L, cl, f = corpus
    v, q_seed, enc = query(L, 809)
    dev = torch.device("cuda:0")
    t = np.zeros(N, np.uint32)
    t[: enc.t_idx.size] = enc.t_idx | np.where(enc.t_sign < 0, np.uint32(0x80000000), np.uint32(0))
    bufs = [torch.from_numpy(enc.v_enc.view(np.int64).copy()).to(dev),
            torch.from_numpy(enc.g.view(np.int64).copy()).to(dev), torch.from_numpy(t.view(np.int32)).to(dev),
            torch.tensor([enc.t_idx.size], dtype=torch.int32, device=dev),
            torch.from_numpy(np.frombuffer(O.domain_separate(q_seed, b"protocol2"), np.uint8).copy()).to(dev),
            torch.zeros(10, dtype=torch.int32, device=dev), torch.zeros(10, dtype=torch.int64, device=dev),
            torch.zeros(1, dtype=torch.int32, device=dev), torch.zeros(1, dtype=torch.int32, device=dev)]
    stream = torch.cuda.current_stream(dev).cuda_stream
    plan = f.plan(1, 20, 10)
    with short_waits(ctx):
        plan.enqueue(*[b.data_ptr() for b in bufs], stream)
        torch.cuda.synchronize(dev)
    st = plan.status()
    assert st & 0x3f and not st & 0x40, hex(st)  # a pipeline wait ran out; the wind-down completed
    plan.enqueue(*[b.data_ptr() for b in bufs], stream)
    torch.cuda.synchronize(dev)
    assert plan.status() == 0 and int(bufs[8].item()) == -1
    plan.close()


def test_block_query_reports_timeout_then_recovers(ctx, corpus):
    M, L, cl, f = corpus
    encs = [query(L, 900 + b)[2] for b in range(8)]
    vb = np.stack([e.v_enc for e in encs])
    gb = np.stack([e.g for e in encs])
    tb = [(e.t_idx, e.t_sign) for e in encs]
    seed = bytes([4]) * 32
    with short_waits(ctx):
        expect_timeout(lambda: f.query_block(vb, gb, tb, seed, 20, 10))
    hits, failed, _ = f.query_block(vb, gb, tb, seed, 20, 10)
    assert np.all(failed == -1)
    for q in range(8):
        r = O.matvec(cl.m_enc, cl.m, N, encs[q].v_enc)
        ids, sc = O.topk(O.to_signed(O.decode_scores(r, cl, L, encs[q])), 10)
        assert np.array_equal(hits[q][0], ids) and np.array_equal(hits[q][1], sc)
