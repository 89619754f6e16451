"""bn_flat_query_shard on the device: a corpus split by rows over several
handles (here on one GPU, standing in for one handle per GPU: the shards do
not wait on one another) gives, after the host-side merge and exact sums of
bn_b200/shard.py, exactly the oracle's answer for the whole corpus: the
top-k, the verdict and every trial's u.r and z.v (verify_response,
crypto.rs:1013-1059, with the draws at the rows' global positions)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, cluster, query
from test_shard import shard_cluster

pytestmark = pytest.mark.gpu

TRIALS, K = 20, 10


@pytest.mark.parametrize("engine,world", [("tensor", 2), ("tensor", 3), ("cuda_core", 2)])
def test_shards_equal_the_whole_corpus(ctx, engine, world):
    from bn_b200 import capi, shard

    m = 3001
    M, L, cl = cluster(m, 4400)
    flats = []
    for g in range(world):
        a, n = shard.split_rows(m, world, g)
        sub = shard_cluster(cl, a, a + n)
        f = capi.Flat.build(ctx, sub.m_enc, sub.a_l, sub.h_mat, n)
        f.attach_client(L, sub.m_plain, sub.s_mat.rowptr, sub.s_mat.idx, sub.s_mat.sign)
        flats.append((f, a))
    encs, seeds, qseeds = [], [], []
    for i in range(3):
        v, q_seed, enc = query(L, 4401 + i)
        encs.append(enc)
        qseeds.append(q_seed)
        seeds.append(O.domain_separate(q_seed, b"protocol2"))
    args = (np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]), [(e.t_idx, e.t_sign) for e in encs],
            seeds)
    ctx.set_engine(capi.ENGINE_TENSOR if engine == "tensor" else capi.ENGINE_CUDA_CORE)
    try:
        parts = [f.query_shard(*args, TRIALS, K, a, m) for f, a in flats]
    finally:
        ctx.set_engine(capi.ENGINE_TENSOR)
    for b in range(3):
        ids, sc = shard.merge_topk([p[0][b] for p in parts], K)
        failed, ur, zv = shard.combine_protocol2([p[1][b] for p in parts], [p[2][b] for p in parts])
        r = O.matvec(cl.m_enc, m, N, encs[b].v_enc)
        f_o, ur_o, zv_o = O.verify_response(r, cl.m_enc, m, N, encs[b].v_enc, TRIALS, seeds[b])
        ids_o, sc_o = O.topk(O.to_signed(O.decode_scores(r, cl, L, encs[b])), K)
        assert failed == f_o == -1
        assert np.array_equal(ur, ur_o) and np.array_equal(zv, zv_o)
        assert np.array_equal(ids, ids_o) and np.array_equal(sc, sc_o)
        # each shard's sums are its own rows' share: no shard alone verifies
        assert all(not np.array_equal(p[1][b], ur_o) for p in parts)
    for f, _ in flats:
        f.close()


def test_shard_rows_out_of_range(ctx):
    from bn_b200 import capi

    m = 64
    M, L, cl = cluster(m, 4500)
    f = capi.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    v, q_seed, enc = query(L, 4501)
    with pytest.raises(capi.BnError) as e:
        f.query_shard(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [bytes(32)], 3, 5, 100, 120)
    assert e.value.code == capi.BN_EINVAL
    f.close()


@pytest.mark.parametrize("world", [2, 3])
def test_ivf_list_shards_equal_one_handle(ctx, world):
    """An IVF corpus split by whole lists (shard.split_lists) into one handle
    per rank (here all on one GPU): each rank's bn_ivf_query over the probes
    that name its lists, merged on the host (top-k by score and id, the
    earliest failing probe), equals one handle holding every list and the
    oracle's BnTmIvfScorer::score (ivf.rs:778-823)."""
    from bn_b200 import capi, shard
    from ivfutil import IvfCase
    from test_shard import IVF_SIZES, ivf_batch

    case = IvfCase(IVF_SIZES, seed=81)
    m_enc, a_l, h, rp, ix, sg = case.concat()
    client = (case.L, case.M.reshape(-1), rp, ix, sg)
    one = capi.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    one.attach_client(*client)
    owner = shard.split_lists(case.sizes, world)
    ranks = []
    for g in range(world):
        v, lists = shard.build_ivf_shard(capi, ctx, case.offsets, case.ids, m_enc, a_l, h, owner, g, client)
        ranks.append(shard.ShardedIvf(v, lists, owner, g, dist=None))
    probes, encs, seeds = ivf_batch(case, 5, 6, 82)
    args = (np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]), [(e.t_idx, e.t_sign) for e in encs],
            seeds, TRIALS, K)
    want, wc, wt = one.query(probes.astype(np.uint32), *args)
    parts = [r.local(probes, *args) for r in ranks]
    fc, ft = shard.merge_verdicts([p[1] for p in parts])
    assert np.array_equal(fc, wc) and np.array_equal(ft, wt) and np.all(fc == -1)
    for b in range(len(probes)):
        ids, sc = shard.merge_topk([p[0][b] for p in parts], K)
        assert np.array_equal(ids, want[b][0]) and np.array_equal(sc, want[b][1])
        o = case.oracle_score(probes[b], encs[b], seeds[b], TRIALS, K)
        assert np.array_equal(ids, o[0]) and np.array_equal(sc, o[1])
    for r in ranks:
        r.ivf.close()
    one.close()
