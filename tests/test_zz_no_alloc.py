"""bn_flat_verify_noalloc: Protocol 2 verification whose scratch is a fixed
array inside the library instead of memory allocated per call.  It serves
callers that cannot allocate device memory while scoring (a service that has
reserved its whole budget up front, or a latency-critical thread that must
not block on the allocator).  Its results must equal those of the existing
bn_flat_verify entry point and of the oracle's verify_response exactly, call
after call, even though every call reuses the same array, and a call must
leave the device's free memory unchanged.  This file is collected last on
purpose: a run that stops at the first failure has run every other test."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, cluster, uniform_fp

pytestmark = pytest.mark.gpu


def _dev_tensors(torch, dev, r, v_enc, v_seed, trials):
    d_r = torch.from_numpy(np.ascontiguousarray(r).view(np.int64).copy()).to(dev)
    d_v = torch.from_numpy(v_enc.view(np.int64).copy()).to(dev)
    d_s = torch.from_numpy(np.frombuffer(v_seed, np.uint8).copy()).to(dev)
    d_f = torch.full((1,), 7, dtype=torch.int32, device=dev)
    d_ur = torch.full((trials,), 5, dtype=torch.int64, device=dev)
    d_zv = torch.full((trials,), 5, dtype=torch.int64, device=dev)
    return d_r, d_v, d_s, d_f, d_ur, d_zv


def _noalloc(capi, f, tensors, trials, stream):
    d_r, d_v, d_s, d_f, d_ur, d_zv = tensors
    return capi.lib.bn_flat_verify_noalloc(f.h, d_r.data_ptr(), d_v.data_ptr(), d_s.data_ptr(), trials,
                                           d_f.data_ptr(), d_ur.data_ptr(), d_zv.data_ptr(), stream)


@pytest.mark.parametrize("trials", [20, 24])
def test_noalloc_verify_matches_existing_entry_point_on_two_calls(ctx, trials):
    torch = pytest.importorskip("torch")
    from bn_b200 import capi

    m = 3000
    M, L, cl = cluster(m, 5, uniform=True)
    f = capi.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    # call 1: honest response; call 2: a response with one tampered residue
    for call, tamper in enumerate([None, 1234]):
        q_seed = bytes([40 + call]) * 32
        enc = O.encode_query(uniform_fp(N, 60 + call), L, q_seed)
        r = O.matvec(cl.m_enc, m, N, enc.v_enc)
        if tamper is not None:
            r[tamper] = (int(r[tamper]) + 1) % P
        v_seed = O.domain_separate(q_seed, b"protocol2")
        want_f, want_ur, want_zv = O.verify_response(r, cl.m_enc, m, N, enc.v_enc, trials, v_seed)
        ex_f, ex_ur, ex_zv = f.verify(r, enc.v_enc, v_seed, trials)

        tensors = _dev_tensors(torch, dev, r, enc.v_enc, v_seed, trials)
        torch.cuda.synchronize(dev)
        free0 = torch.cuda.mem_get_info(dev)[0]
        capi.check(_noalloc(capi, f, tensors, trials, stream.cuda_stream))
        torch.cuda.synchronize(dev)
        assert torch.cuda.mem_get_info(dev)[0] == free0, "the call changed the device's free memory"
        d_f, d_ur, d_zv = tensors[3:]
        got_f = int(d_f.item())
        ran = trials if want_f < 0 else want_f + 1
        ur = d_ur.cpu().numpy().view(np.uint64)[:ran]
        zv = d_zv.cpu().numpy().view(np.uint64)[:ran]
        assert got_f == want_f == ex_f == (-1 if tamper is None else 0)
        assert np.array_equal(ur, want_ur) and np.array_equal(zv, want_zv)
        assert np.array_equal(ur, ex_ur) and np.array_equal(zv, ex_zv)
    f.close()


def test_noalloc_empty_corpus_and_planted_draw(ctx):
    torch = pytest.importorskip("torch")
    from bn_b200 import capi

    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    trials = 3
    v = uniform_fp(N, 3)
    seed = bytes([8]) * 32
    # empty corpus: -1 and zero sums, as bn_flat_verify gives
    f0 = capi.Flat.build(ctx, np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0, np.uint64), 0)
    assert f0.verify(np.zeros(0, np.uint64), v, seed, trials)[0] == -1
    t0 = _dev_tensors(torch, dev, np.zeros(1, np.uint64), v, seed, trials)
    capi.check(_noalloc(capi, f0, t0, trials, stream))
    torch.cuda.synchronize(dev)
    assert int(t0[3].item()) == -1 and not t0[4].any().item() and not t0[5].any().item()
    f0.close()
    # a draw equal to p (planted): -2 instead of a verdict; then normal again
    m = 500
    M, L, cl = cluster(m, 6, uniform=True)
    f = capi.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m)
    r = O.matvec(cl.m_enc, m, N, v)
    t1 = _dev_tensors(torch, dev, r, v, seed, trials)
    ctx.plant_draw_hit(True)
    try:
        capi.check(_noalloc(capi, f, t1, trials, stream))
        torch.cuda.synchronize(dev)
        assert int(t1[3].item()) == -2
    finally:
        ctx.plant_draw_hit(False)
    capi.check(_noalloc(capi, f, t1, trials, stream))
    torch.cuda.synchronize(dev)
    assert int(t1[3].item()) == O.verify_response(r, cl.m_enc, m, N, v, trials, seed)[0] == -1
    f.close()


def test_noalloc_rejects_sizes_beyond_its_limit(ctx):
    from bn_b200 import capi

    m = 64
    M, L, cl = cluster(m, 6, uniform=True)
    f = capi.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m)
    rc = capi.lib.bn_flat_verify_noalloc(f.h, 1, 1, 1, 25, 1, 1, 1, None)  # 25 > BN_NOALLOC_MAX_TRIALS
    assert rc == capi.BN_EINVAL and "static scratch limit" in capi.last_error()
    f.close()
