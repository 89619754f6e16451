"""Bit-exact parity with the oracle at the full size of the IVF workload.

The corpus is the one bench.py measures: N = 2,000,000 rows, d = 768, a
Zipf(1.1)-weighted Gaussian mixture partitioned into nlist = 4096 k-means
lists (seed 3), every list BN-encrypted on the device with its own h_seed
(ivf.rs:258-264, 627-653).  One batch of 64 queries at nprobe = 8 goes
through the per-query form (BnTmIvfScorer::score, ivf.rs:746-927: every
probed list scanned, verified with the query's seed, decoded, merged) and
the block form; the oracle scores the same (query, list) pairs from host
copies of the probed lists.  Checked bit for bit: routing (probe_route,
ivf-index/src/ivf.rs:150-164), per-list keygen, per-list r, every trial's
u.r / z.v on sampled pairs for both seed conventions, the global top-10 and
the accept verdicts."""
from __future__ import annotations

import gc
import os
import sys
import types

import numpy as np
import pytest

import oracle as O
from bnutil import N

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ROWS, D, NLIST, SEED, TRIALS, K, BQ, NPROBE = 2_000_000, 768, 4096, 3, 20, 10, 64, 8


def capi():
    from bn_b200 import capi as c

    return c


@pytest.fixture(scope="module")
def ivf2m(ctx):
    import bench

    c = capi()
    gc.collect()
    data = bench.synth_ivf(ROWS, D, NLIST, SEED)
    off = data["offsets"]
    assert int(off[-1]) == ROWS
    L = c.host_generate_subspace(bytes([SEED & 0xFF, 0x1F]) * 16)
    H, rp, ix, sg = c.host_regenerate_h_s_lists(SEED, off)
    mq = np.zeros((ROWS, N), np.uint64)
    for r0 in range(0, ROWS, 1 << 18):
        mq[r0 : r0 + (1 << 18)] = bench.to_residues(data["m8"][r0 : r0 + (1 << 18)])
    ivf = c.Ivf.build_from_plain(ctx, off, data["ids"], mq.reshape(-1), L, H, rp, ix, sg)
    yield types.SimpleNamespace(data=data, ivf=ivf, L=L, H=H.reshape(ROWS, 128), rp=rp, ix=ix, sg=sg, mq=mq)
    ivf.close()
    gc.collect()


def list_clusters(ctx, t, lists):
    """Oracle clusters of the given lists: the plaintext rows, the list's H
    and S (checked against the oracle's per-list keygen) and host copies of
    the device encryption of exactly those rows."""
    c = capi()
    off = t.data["offsets"]
    lists = sorted(set(int(x) for x in lists if off[x + 1] > off[x]))
    rows = np.concatenate([np.arange(int(off[x]), int(off[x + 1])) for x in lists])
    sub_rp = [np.zeros(1, np.uint64)]
    sub_ix, sub_sg, base = [], [], 0
    for x in lists:
        o, e = int(off[x]), int(off[x + 1])
        a, b = int(t.rp[o]), int(t.rp[e])
        sub_rp.append(t.rp[o + 1 : e + 1] - np.uint64(a) + np.uint64(base))
        sub_ix.append(t.ix[a:b])
        sub_sg.append(t.sg[a:b])
        base += b - a
    rp, ix, sg = np.concatenate(sub_rp), np.concatenate(sub_ix), np.concatenate(sub_sg)
    Hs = t.H[rows]
    m_enc, a_l = c.encrypt_cluster(ctx, t.mq[rows].reshape(-1), rows.size, t.L, Hs.reshape(-1), rp, ix, sg)
    m_enc = m_enc.reshape(-1, N)
    a_l = a_l.reshape(-1, 128)
    out, r0 = {}, 0
    for x in lists:
        m = int(off[x + 1] - off[x])
        s0, s1 = int(rp[r0]), int(rp[r0 + m])
        h_l, s_l = O.regenerate_h_s(O.derive_h_seed(SEED, x), m)  # ivf.rs:258-264 per-list h_seed
        assert np.array_equal(h_l, Hs[r0 : r0 + m].reshape(-1)), f"H of list {x}"
        assert np.array_equal(s_l.rowptr, rp[r0 : r0 + m + 1] - np.uint64(s0)), f"S of list {x}"
        assert np.array_equal(s_l.idx, ix[s0:s1]) and np.array_equal(s_l.sign, sg[s0:s1])
        out[x] = O.Cluster(m, N, 128, m_enc[r0 : r0 + m].reshape(-1).copy(), a_l[r0 : r0 + m].reshape(-1).copy(),
                           t.mq[rows[r0 : r0 + m]].reshape(-1).copy(), h_l, s_l)
        r0 += m
    return out


def test_ivf_batch_at_two_million_rows(ctx, ivf2m):
    import bench

    c = capi()
    t = ivf2m
    data, ivf = t.data, t.ivf
    qx, q8 = bench.synth_ivf_queries(data, BQ, SEED)
    encs, seeds = bench.encode_pool(t.L, BQ, q8, SEED)
    probes = c.host_probe_route(data["centres"], qx, NPROBE)
    for q in range(BQ):
        assert np.array_equal(probes[q], O.probe_route(data["centres"], qx[q], NPROBE)), f"routing of query {q}"
    vb = np.stack([e[0] for e in encs])
    gb = np.stack([e[1] for e in encs])
    tb = [(e[2], e[3]) for e in encs]
    hits, fc, ft = ivf.query(probes, vb, gb, tb, seeds, TRIALS, K)
    bhits, bfc, bft = ivf.query_block(probes, vb, gb, tb, bytes([SEED, NPROBE]) * 16, TRIALS, K)
    cls = list_clusters(ctx, t, np.unique(probes))
    ids_all = data["ids"]
    off = data["offsets"]
    for q in range(BQ):
        enc = O.Encoded(*encs[q])
        allid, allsc = [], []
        for x in probes[q]:
            x = int(x)
            if x not in cls:
                continue  # an empty list is skipped (ivf.rs:787-789)
            cl = cls[x]
            r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
            f, _, _ = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, TRIALS, seeds[q])
            assert f == -1
            allid.append(ids_all[int(off[x]) : int(off[x + 1])])
            allsc.append(O.to_signed(O.decode_scores(r, cl, t.L, enc)))
        ids_o, sc_o = O.topk(np.concatenate(allsc), K, ids=np.concatenate(allid))
        assert fc[q] == ft[q] == bfc[q] == bft[q] == -1
        assert np.array_equal(hits[q][0], ids_o) and np.array_equal(hits[q][1], sc_o), f"query {q}"
        assert np.array_equal(bhits[q][0], ids_o) and np.array_equal(bhits[q][1], sc_o), f"block query {q}"
    # per-list r, and every trial's sums on sampled (query, list) pairs under
    # the query's own seed (per-query form) and the block seed (block form)
    rng = np.random.default_rng(5)
    pairs = ivf.pairs(probes)
    rall = []
    for q, x, m in pairs:
        r = O.matvec(cls[x].m_enc, m, N, vb[q])
        rall.append(r)
    for i in rng.choice(len(pairs), 4, replace=False):
        q, x, m = pairs[i]
        assert np.array_equal(ivf.compute_products(x, vb[q]), rall[i])
        f_g, ur_g, zv_g = ivf.verify(x, rall[i], vb[q], seeds[q], TRIALS)
        f_o, ur_o, zv_o = O.verify_response(rall[i], cls[x].m_enc, m, N, vb[q], TRIALS, seeds[q])
        assert f_g == f_o == -1 and np.array_equal(ur_g, ur_o) and np.array_equal(zv_g, zv_o)
    bseed = bytes([SEED, NPROBE]) * 16
    vfc, vft, ur_b, zv_b = ivf.verify_block(probes, np.concatenate(rall), vb, bseed, TRIALS)
    assert np.all(vfc == -1) and np.all(vft == -1)
    for i in rng.choice(len(pairs), 4, replace=False):
        q, x, m = pairs[i]
        f_o, ur_o, zv_o = O.verify_response(rall[i], cls[x].m_enc, m, N, vb[q], TRIALS, bseed)
        assert f_o == -1 and np.array_equal(ur_b[i], ur_o) and np.array_equal(zv_b[i], zv_o)
