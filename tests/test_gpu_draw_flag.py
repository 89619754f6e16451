"""A Protocol 2 draw equal to p is reported, never silently replaced.

The reference's sample_fp (scorer-bntm/src/crypto.rs:155-162) rejects a
draw equal to p and takes the next one, which shifts every later draw of the
stream.  The kernels draw by stream position, so on that event (odds 2^-61
per draw) every call that verifies fails with BN_EDRAW instead of returning a
verdict that could differ from the reference's.  No seed that produces the
event can be found, so these tests plant it with bn_debug_plant_draw_hit and
check that each path reports it, and that calls without Protocol 2 or with
the plant removed give their normal, oracle-equal results."""
from __future__ import annotations

import contextlib

import numpy as np
import pytest

import oracle as O
from bnutil import N, cluster, query
from ivfutil import IvfCase

pytestmark = pytest.mark.gpu


def capi():
    from bn_b200 import capi as c

    return c


@contextlib.contextmanager
def planted(ctx):
    ctx.plant_draw_hit(True)
    try:
        yield
    finally:
        ctx.plant_draw_hit(False)


@pytest.fixture(scope="module")
def flat_case(ctx):
    c = capi()
    M, L, cl = cluster(700, 4242)
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    yield M, L, cl, f
    f.close()


def expect_edraw(fn):
    c = capi()
    with pytest.raises(c.BnError) as ei:
        fn()
    assert ei.value.code == c.BN_EDRAW, str(ei.value)


@pytest.mark.parametrize("engine", ["tensor", "cuda_core"])
def test_flat_query_and_verify_report_the_draw(ctx, flat_case, engine):
    c = capi()
    M, L, cl, f = flat_case
    ctx.set_engine(c.ENGINE_TENSOR if engine == "tensor" else c.ENGINE_CUDA_CORE)
    try:
        v, q_seed, enc = query(L, 77)
        vs = O.domain_separate(q_seed, b"protocol2")
        args = (enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [vs])
        r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
        with planted(ctx):
            expect_edraw(lambda: f.query(*args, 20, 10))
            expect_edraw(lambda: f.verify(r, enc.v_enc, vs, 5))
            hits0, failed0, _, _ = f.query(*args, 0, 10)  # no Protocol 2: unaffected
        hits, failed, _, _ = f.query(*args, 20, 10)
        want_f, want_ids, want_sc, _, _ = O.score_flat(cl, L, v, q_seed, 20, 10)
        assert failed[0] == want_f == -1 and failed0[0] == -1
        assert np.array_equal(hits[0][0], want_ids) and np.array_equal(hits[0][1], want_sc)
        assert np.array_equal(hits0[0][0], want_ids) and np.array_equal(hits0[0][1], want_sc)
    finally:
        ctx.set_engine(c.ENGINE_TENSOR)


def test_plan_status_carries_the_draw_bit(ctx, flat_case):
    torch = pytest.importorskip("torch")
    c = capi()
    M, L, cl, f = flat_case
    v, q_seed, enc = query(L, 78)
    dev = torch.device("cuda:0")
    t = np.zeros(N, np.uint32)
    t[: enc.t_idx.size] = enc.t_idx | np.where(enc.t_sign < 0, np.uint32(0x80000000), np.uint32(0))
    d_v = torch.from_numpy(enc.v_enc.view(np.int64).copy()).to(dev)
    d_g = torch.from_numpy(enc.g.view(np.int64).copy()).to(dev)
    d_t = torch.from_numpy(t.view(np.int32)).to(dev)
    d_tn = torch.tensor([enc.t_idx.size], dtype=torch.int32, device=dev)
    d_s = torch.from_numpy(np.frombuffer(O.domain_separate(q_seed, b"protocol2"), np.uint8).copy()).to(dev)
    d_ids = torch.zeros(10, dtype=torch.int32, device=dev)
    d_sc = torch.zeros(10, dtype=torch.int64, device=dev)
    d_n = torch.zeros(1, dtype=torch.int32, device=dev)
    d_f = torch.zeros(1, dtype=torch.int32, device=dev)
    plan = f.plan(1, 20, 10)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ptrs = [x.data_ptr() for x in (d_v, d_g, d_t, d_tn, d_s, d_ids, d_sc, d_n, d_f)]
    with planted(ctx):
        plan.enqueue(*ptrs, stream)
        torch.cuda.synchronize(dev)
        assert plan.status() & c.STATUS_DRAW_HIT_P
    plan.enqueue(*ptrs, stream)
    torch.cuda.synchronize(dev)
    assert plan.status() == 0 and int(d_f.item()) == -1
    plan.close()


def test_block_paths_report_the_draw(ctx, flat_case):
    M, L, cl, f = flat_case
    encs = [query(L, 90 + b)[2] for b in range(4)]
    vb = np.stack([e.v_enc for e in encs])
    gb = np.stack([e.g for e in encs])
    tb = [(e.t_idx, e.t_sign) for e in encs]
    r = np.stack([O.matvec(cl.m_enc, cl.m, N, e.v_enc) for e in encs])
    seed = bytes([9]) * 32
    with planted(ctx):
        expect_edraw(lambda: f.query_block(vb, gb, tb, seed, 20, 10))
        expect_edraw(lambda: f.verify_block(r, vb, seed, 3))
    hits, failed, _ = f.query_block(vb, gb, tb, seed, 20, 10)
    assert np.all(failed == -1)


def test_ivf_paths_report_the_draw(ctx):
    c = capi()
    case = IvfCase([40, 0, 130, 7, 300])
    m_enc, a_l, h, rp, ix, sg = case.concat()
    v = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    v.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    encs = [O.encode_query(case.M[3 + b], case.L, bytes([50 + b]) * 32) for b in range(3)]
    seeds = [O.domain_separate(bytes([50 + b]) * 32, b"protocol2") for b in range(3)]
    probes = np.array([[0, 2, 4], [2, 3, 1], [4, 0, 3]], np.uint32)
    vb = np.stack([e.v_enc for e in encs])
    gb = np.stack([e.g for e in encs])
    tb = [(e.t_idx, e.t_sign) for e in encs]
    with planted(ctx):
        expect_edraw(lambda: v.query(probes, vb, gb, tb, seeds, 20, 10))
        expect_edraw(lambda: v.query_block(probes, vb, gb, tb, bytes([3]) * 32, 20, 10))
    hits, fc, ft = v.query(probes, vb, gb, tb, seeds, 20, 10)
    assert np.all(fc == -1)
    v.close()
