"""GPU parity of IVF block scoring (a batch's (query, list) pairs grouped by
list, one grouped GEMM per operand) against the oracle.

Scores and ranking must equal the oracle's BnTmIvfScorer::score
(ivf.rs:778-823: every probed list, empty ones skipped, global top-k) bit
for bit; Protocol 2 must equal verify_response (crypto.rs:1013-1059) run per
(query, list) with the block seed, trial by trial.  Lists are ragged (empty,
1 row, below and above the 16- and 128-row GEMM tiles, above the 4096-row
Freivalds panel) and shared by several queries of the batch."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, int8_matrix
from ivfutil import IvfCase

pytestmark = pytest.mark.gpu

SIZES = [50, 0, 3, 200, 1, 0, 97, 4500, 33, 129, 16, 17, 700, 128, 2]


def capi():
    from bn_b200 import capi as c

    return c


@pytest.fixture(scope="module")
def case():
    return IvfCase(SIZES, seed=31)


@pytest.fixture(scope="module")
def ivf(ctx, case):
    c = capi()
    m_enc, a_l, h, rp, ix, sg = case.concat()
    v = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    v.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    v.block_prepare()
    return v


def batch(case, B, nprobe, seed):
    rng = np.random.default_rng(seed)
    # a few popular lists, so that most lists are shared by several queries
    w = np.array([5.0 if s > 100 else 1.0 for s in case.sizes])
    probes = np.stack([rng.choice(case.nlist, size=nprobe, replace=False, p=w / w.sum()) for _ in range(B)])
    encs = []
    for b in range(B):
        enc = O.encode_query(int8_matrix(1, 768, seed * 100 + b)[0], case.L, O.derive_h_seed(seed, b))
        encs.append(enc)
    return probes.astype(np.uint32), encs


def run_block(ivf, probes, encs, seed, trials, k):
    return ivf.query_block(probes, np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                           [(e.t_idx, e.t_sign) for e in encs], seed, trials, k)


@pytest.mark.parametrize("B,nprobe,trials,k", [(12, 5, 20, 10), (7, 3, 3, 25), (20, 8, 0, 10), (5, 4, 23, 1024),
                                               (1, 1, 2, 5), (33, 2, 1, 7)])
def test_query_block_matches_oracle(case, ivf, B, nprobe, trials, k):
    probes, encs = batch(case, B, nprobe, 11 + B)
    if B > 1:
        probes[1, 0] = 1  # an empty list first in probe order
    seed = bytes([B, nprobe, trials]) * 10 + b"ab"
    hits, fc, ft = run_block(ivf, probes, encs, seed, trials, k)
    for b in range(B):
        ids, sc = case.oracle_score(list(probes[b]), encs[b], seed, trials, k)
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc), b
        assert fc[b] == -1 and ft[b] == -1


def test_query_block_edge_batches(case, ivf):
    """All-empty probes, a duplicated probe (the list is scored twice, as the
    per-query path does), and k above every query's row count."""
    probes, encs = batch(case, 4, 3, 77)
    probes[0] = [1, 5, 1]       # nothing to score
    probes[2] = [7, 7, 4]       # a list probed twice by one query
    hits, fc, ft = run_block(ivf, probes, encs, bytes([3]) * 32, 4, 1024)
    for b in range(4):
        ids, sc = case.oracle_score(list(probes[b]), encs[b], bytes([3]) * 32, 4, 1024)
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc), b
    assert len(hits[0][0]) == 0
    assert fc.tolist() == [-1] * 4 and ft.tolist() == [-1] * 4


def test_query_block_equals_per_query_hits(case, ivf):
    """The block path ranks exactly like bn_ivf_query (the seeds differ only in Protocol 2)."""
    probes, encs = batch(case, 16, 6, 5)
    seeds = [O.domain_separate(O.derive_h_seed(5, b), b"protocol2") for b in range(16)]
    want, wfc, _ = ivf.query(probes, np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                             [(e.t_idx, e.t_sign) for e in encs], seeds, 20, 10)
    hits, fc, _ = run_block(ivf, probes, encs, bytes([8]) * 32, 20, 10)
    for b in range(16):
        assert np.array_equal(hits[b][0], want[b][0]) and np.array_equal(hits[b][1], want[b][1])
    assert np.all(fc == -1) and np.all(wfc == -1)


def pair_responses(case, ivf, probes, encs):
    r = []
    for q, c, m in ivf.pairs(probes):
        cl = case.clusters[c]
        r.append(O.matvec(cl.m_enc, cl.m, N, encs[q].v_enc))
    return r


@pytest.mark.parametrize("trials", [1, 20, 29])
def test_verify_block_matches_oracle(case, ivf, trials):
    probes, encs = batch(case, 9, 4, 40 + trials)
    rs = pair_responses(case, ivf, probes, encs)
    seed = bytes([trials, 1]) * 16
    fc, ft, ur, zv = ivf.verify_block(probes, np.concatenate(rs), np.stack([e.v_enc for e in encs]), seed, trials)
    assert np.all(fc == -1) and np.all(ft == -1)
    for i, (q, c, m) in enumerate(ivf.pairs(probes)):
        cl = case.clusters[c]
        fo, uro, zvo = O.verify_response(rs[i], cl.m_enc, m, N, encs[q].v_enc, trials, seed)
        assert fo == -1
        assert np.array_equal(ur[i], uro) and np.array_equal(zv[i], zvo), i


@pytest.mark.parametrize("where", ["first", "later", "big_list_end"])
def test_verify_block_detects_tampered_response(case, ivf, where):
    """crypto.rs:1445-1474 per (query, list): only the tampered query is
    rejected, at the tampered list and trial 0."""
    probes, encs = batch(case, 6, 3, 90)
    probes[3] = [7, 12, 0]  # 4500, 700 and 50 rows
    pairs = ivf.pairs(probes)
    rs = pair_responses(case, ivf, probes, encs)
    idx = [i for i, (q, c, m) in enumerate(pairs) if q == 3]
    target = {"first": idx[0], "later": idx[2], "big_list_end": idx[0]}[where]
    pos = {"first": 17, "later": 49, "big_list_end": 4499}[where]
    rs[target] = rs[target].copy()
    rs[target][pos] = (int(rs[target][pos]) + 5) % P
    fc, ft, ur, zv = ivf.verify_block(probes, np.concatenate(rs), np.stack([e.v_enc for e in encs]),
                                      bytes([66]) * 32, 20)
    for b in range(6):
        if b == 3:
            assert fc[b] == pairs[target][1] and ft[b] == 0
        else:
            assert fc[b] == -1 and ft[b] == -1
    assert ur[target][0] != zv[target][0]


@pytest.mark.parametrize("n1", [64, 512])
def test_query_block_across_n1(ctx, n1):
    """IVF block scoring at the smallest and largest n1 of the reference's
    delta sweep ([AL | H] pair images of 2 n1 bytes per plane row)."""
    c = capi()
    case = IvfCase([40, 0, 300, 7, 129], seed=n1, n1=n1)
    m_enc, a_l, h, rp, ix, sg = case.concat()
    v = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h, n1=n1)
    v.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    v.block_prepare()
    rng = np.random.default_rng(n1)
    B, nprobe, trials, k = 5, 3, 4, 12
    probes = np.stack([rng.choice(case.nlist, nprobe, replace=False) for _ in range(B)]).astype(np.uint32)
    encs = [O.encode_query(int8_matrix(1, 768, 500 + n1 + b)[0], case.L, O.derive_h_seed(n1, b), n1=n1)
            for b in range(B)]
    seed = bytes([n1 % 251, 9]) * 16
    hits, fc, ft = run_block(v, probes, encs, seed, trials, k)
    for b in range(B):
        ids, sc = case.oracle_score(list(probes[b]), encs[b], seed, trials, k)
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc), b
        assert fc[b] == -1 and ft[b] == -1


def test_query_block_rejects_bad_input(case, ivf):
    c = capi()
    probes, encs = batch(case, 2, 2, 3)
    probes[1, 1] = case.nlist
    with pytest.raises(c.BnError) as e:
        run_block(ivf, probes, encs, bytes(32), 2, 10)
    assert e.value.code == c.BN_EINVAL
    probes[1, 1] = 0
    bad = [e for e in encs]
    v = np.stack([e.v_enc for e in bad])
    v[0, 5] = P
    with pytest.raises(c.BnError) as e:
        ivf.query_block(probes, v, np.stack([e.g for e in encs]), [(e.t_idx, e.t_sign) for e in encs], bytes(32), 2, 10)
    assert e.value.code == c.BN_EINVAL


def test_block_profile_stages(case, ivf):
    """Stage timing of a profiled block call: one non-negative time per named
    stage (host plan, H2D, G1-G3, top-k, the three Protocol 2 steps, verdicts,
    D2H), and the same hits as an unprofiled call."""
    probes, encs = batch(case, 6, 4, 61)
    want = run_block(ivf, probes, encs, bytes([6]) * 32, 20, 10)
    ivf.block_profile(True)
    got = run_block(ivf, probes, encs, bytes([6]) * 32, 20, 10)
    st = ivf.block_profile_read()
    ivf.block_profile(False)
    assert list(st) == list(capi().Ivf.IVF_BLOCK_STAGES) and len(st) == 11
    assert all(x >= 0 for x in st.values()) and st["protocol2_z_passes"] > 0 and st["g1_r"] > 0
    for a, b in zip(want[0], got[0]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(want[1], got[1])


def test_verify_block_many_short_lists(ctx):
    """More short lists (1 to 384 rows: panels of 1, 2 and 3 row blocks, in
    random order) than SMs, so that CTAs of the short-list Protocol 2 kernel
    take several panels in turn: every pair's u_t . r and z_t . v equal
    verify_response's, trial by trial."""
    c = capi()
    rng = np.random.default_rng(77)
    sizes = rng.integers(1, 385, 320).tolist()
    big = IvfCase(sizes, seed=77)
    m_enc, a_l, h, _, _, _ = big.concat()
    v = c.Ivf.build(ctx, big.offsets, big.ids, m_enc, a_l, h)
    probes = np.stack([rng.choice(big.nlist, size=64, replace=False) for _ in range(6)]).astype(np.uint32)
    assert len(np.unique(probes)) > 200
    encs = [O.encode_query(int8_matrix(1, 768, 7700 + b)[0], big.L, O.derive_h_seed(77, b)) for b in range(6)]
    rs = pair_responses(big, v, probes, encs)
    seed = bytes([77]) * 32
    fc, ft, ur, zv = v.verify_block(probes, np.concatenate(rs), np.stack([e.v_enc for e in encs]), seed, 20)
    assert np.all(fc == -1) and np.all(ft == -1)
    for i, (q, ci, m) in enumerate(v.pairs(probes)):
        cl = big.clusters[ci]
        fo, uro, zvo = O.verify_response(rs[i], cl.m_enc, m, N, encs[q].v_enc, 20, seed)
        assert fo == -1 and np.array_equal(ur[i], uro) and np.array_equal(zv[i], zvo), i
    v.close()
