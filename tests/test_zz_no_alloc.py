"""bn_flat_verify_noalloc: Protocol 2 verification whose scratch is a fixed
array inside the library instead of memory allocated per call.  It serves
callers that cannot allocate device memory while scoring (a service that has
reserved its whole budget up front, or a latency-critical thread that must
not block on the allocator).  Its results must equal those of the existing
bn_flat_verify entry point exactly, call after call, even though every call
reuses the same array.  This file is collected last on purpose."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, cluster, uniform_fp

pytestmark = pytest.mark.gpu


def test_noalloc_verify_matches_existing_entry_point_on_two_calls(ctx):
    torch = pytest.importorskip("torch")
    from bn_b200 import capi

    m, trials = 3000, 20
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
        want_f, want_ur, want_zv = f.verify(r, enc.v_enc, v_seed, trials)

        d_r = torch.from_numpy(r.view(np.int64).copy()).to(dev)
        d_v = torch.from_numpy(enc.v_enc.view(np.int64).copy()).to(dev)
        d_s = torch.from_numpy(np.frombuffer(v_seed, np.uint8).copy()).to(dev)
        d_f = torch.full((1,), 7, dtype=torch.int32, device=dev)
        d_ur = torch.zeros(trials, dtype=torch.int64, device=dev)
        d_zv = torch.zeros(trials, dtype=torch.int64, device=dev)
        capi.check(capi.lib.bn_flat_verify_noalloc(f.h, d_r.data_ptr(), d_v.data_ptr(), d_s.data_ptr(), trials,
                                                   d_f.data_ptr(), d_ur.data_ptr(), d_zv.data_ptr(),
                                                   stream.cuda_stream))
        torch.cuda.synchronize(dev)
        got_f = int(d_f.item())
        ran = trials if want_f < 0 else want_f + 1
        ur = d_ur.cpu().numpy().view(np.uint64)[:ran]
        zv = d_zv.cpu().numpy().view(np.uint64)[:ran]
        assert got_f == want_f == (-1 if tamper is None else 0)
        assert np.array_equal(ur, want_ur) and np.array_equal(zv, want_zv)


def test_noalloc_rejects_sizes_beyond_its_limit(ctx):
    from bn_b200 import capi

    m = 64
    M, L, cl = cluster(m, 6, uniform=True)
    f = capi.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m)
    rc = capi.lib.bn_flat_verify_noalloc(f.h, 1, 1, 1, 25, 1, 1, 1, None)  # 25 > BN_NOALLOC_MAX_TRIALS
    assert rc == capi.BN_EINVAL and "static scratch limit" in capi.last_error()
