"""Row-sharded flat scoring (bn_b200/shard.py) on the host: the merge of the
shards' top-k lists and the exact sums of their Protocol 2 partials must
give exactly what the oracle gives for the whole corpus (BnTmScorer::score,
lib.rs:326-475; verify_response, crypto.rs:1013-1059), in one process and
over a gloo process group of two ranks."""
from __future__ import annotations

import json
import os
import socket
import sys

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, cluster, query

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

TRIALS, K = 6, 12


def shard_cluster(cl, a: int, b: int):
    """Rows [a, b) of an oracle cluster."""
    n, n1, s = cl.n, cl.n1, cl.s_mat
    e0, e1 = int(s.rowptr[a]), int(s.rowptr[b])
    return O.Cluster(b - a, n, n1, cl.m_enc[a * n : b * n].copy(), cl.a_l[a * n1 : b * n1].copy(),
                     cl.m_plain[a * n : b * n].copy(), cl.h_mat[a * n1 : b * n1].copy(),
                     O.Sparse(s.rowptr[a : b + 1] - s.rowptr[a], s.idx[e0:e1].copy(), s.sign[e0:e1].copy()))


def local_part(cl, L, enc, v_seed, a, b, total, tamper=None):
    """What one rank computes for rows [a, b) (the oracle standing in for
    bn_flat_query_shard): its top-k with global ids and its partial sums."""
    sub = shard_cluster(cl, a, b)
    r = O.matvec(sub.m_enc, sub.m, N, enc.v_enc)
    if tamper is not None and a <= tamper < b:
        r[tamper - a] = (int(r[tamper - a]) + 1) % P
    ur, zv = O.verify_shard_partials(r, sub.m_enc, sub.m, N, enc.v_enc, TRIALS, v_seed, a, total)
    ids, sc = O.topk(O.to_signed(O.decode_scores(r, sub, L, enc)), K, ids=np.arange(a, b, dtype=np.uint32))
    return (ids, sc), ur, zv


def whole(cl, L, enc, v_seed, tamper=None):
    r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
    if tamper is not None:
        r[tamper] = (int(r[tamper]) + 1) % P
    f, ur, zv = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, TRIALS, v_seed)
    ids, sc = O.topk(O.to_signed(O.decode_scores(r, cl, L, enc)), K)
    return f, ur, zv, ids, sc


def test_split_rows_covers_the_corpus():
    from bn_b200 import shard

    for total in (1, 7, 1000, 1_000_003):
        for world in (1, 2, 3, 8):
            parts = [shard.split_rows(total, world, g) for g in range(world)]
            assert parts[0][0] == 0 and sum(p[1] for p in parts) == total
            assert all(parts[g][0] + parts[g][1] == parts[g + 1][0] for g in range(world - 1))
            assert max(p[1] for p in parts) - min(p[1] for p in parts) <= 1


@pytest.mark.parametrize("tamper", [None, 1777])
def test_three_shards_equal_the_whole_corpus(tamper):
    from bn_b200 import shard

    m = 2500
    M, L, cl = cluster(m, 4100)
    v, q_seed, enc = query(L, 4101)
    v_seed = O.domain_separate(q_seed, b"protocol2")
    f, ur_w, zv_w, ids_w, sc_w = whole(cl, L, enc, v_seed, tamper)
    parts = [shard.split_rows(m, 3, g) for g in range(3)]
    locs = [local_part(cl, L, enc, v_seed, a, a + n, m, tamper) for a, n in parts]
    ids, sc = shard.merge_topk([x[0] for x in locs], K)
    failed, ur, zv = shard.combine_protocol2([x[1] for x in locs], [x[2] for x in locs])
    assert np.array_equal(ids, ids_w) and np.array_equal(sc, sc_w)
    assert failed == f == (-1 if tamper is None else 0)
    ran = TRIALS if f < 0 else f + 1
    assert np.array_equal(ur[:ran], ur_w) and np.array_equal(zv[:ran], zv_w)


def test_merge_keeps_ties_in_id_order():
    from bn_b200 import shard

    a = (np.array([5, 9], np.uint32), np.array([10, 7], np.int64))
    b = (np.array([2, 3], np.uint32), np.array([10, 7], np.int64))
    ids, sc = shard.merge_topk([a, b], 3)
    assert ids.tolist() == [2, 5, 3] and sc.tolist() == [10, 10, 7]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank: int, world: int, port: int, out_dir: str, tamper):
    for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "secure-vector-search_b200"), os.path.join(ROOT, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist

    from bn_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    m = 1900
    M, L, cl = cluster(m, 4200)
    encs, seeds = [], []
    for i in range(3):  # a batch of three queries
        v, q_seed, enc = query(L, 4201 + i)
        encs.append(enc)
        seeds.append(O.domain_separate(q_seed, b"protocol2"))
    a, n = shard.split_rows(m, world, rank)
    hits, urs, zvs = [], [], []
    for enc, s in zip(encs, seeds):
        h, ur, zv = local_part(cl, L, enc, s, a, a + n, m, tamper)
        hits.append(h)
        urs.append(ur)
        zvs.append(zv)
    got, failed = shard.exchange(dist, None, "cpu", hits, np.stack(urs), np.stack(zvs), K)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump({"ids": [g[0].tolist() for g in got], "scores": [g[1].tolist() for g in got],
                   "failed": failed.tolist()}, fh)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("tamper", [None, 1200])
def test_gloo_two_ranks_equal_the_whole_corpus(tmp_path, tamper):
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(worker, args=(2, free_port(), str(tmp_path), tamper), nprocs=2, join=True)
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert got[0] == got[1]  # every rank ends with the same answer
    m = 1900
    M, L, cl = cluster(m, 4200)
    for i in range(3):
        v, q_seed, enc = query(L, 4201 + i)
        f, _, _, ids, sc = whole(cl, L, enc, O.domain_separate(q_seed, b"protocol2"), tamper)
        assert got[0]["ids"][i] == ids.tolist() and got[0]["scores"][i] == sc.tolist()
        assert got[0]["failed"][i] == f == (-1 if tamper is None else 0)


# ---------------------------------------------------------------- IVF: whole lists per rank

IVF_SIZES = [50, 0, 3, 200, 1, 0, 97, 400, 33, 120, 64, 9, 260, 5]


def ivf_local(case, probes_row, enc, v_seed, trials, k, owned, tamper_list=None):
    """One query over the probes that name `owned` lists, in probe order (the
    oracle standing in for one rank's bn_ivf_query): top-k with global ids
    over their rows, and the first failing (probe position, list, trial)."""
    allid, allsc = [], []
    verdict = (-1, -1, -1)
    for j, ci in enumerate(probes_row):
        ci = int(ci)
        cl = case.clusters[ci]
        if ci not in owned or cl is None:
            continue
        r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
        if tamper_list == ci:
            r[0] = (int(r[0]) + 1) % P
        if trials and verdict[0] < 0:
            f, _, _ = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, trials, v_seed)
            if f >= 0:
                verdict = (j, ci, f)
        o = int(case.offsets[ci])
        allid.append(case.ids[o : o + cl.m])
        allsc.append(O.to_signed(O.decode_scores(r, cl, case.L, enc)))
    if not allid:
        return (np.zeros(0, np.uint32), np.zeros(0, np.int64)), verdict
    return O.topk(np.concatenate(allsc), k, ids=np.concatenate(allid)), verdict


def ivf_batch(case, B, nprobe, seed):
    rng = np.random.default_rng(seed)
    probes = np.stack([rng.choice(case.nlist, nprobe, replace=False) for _ in range(B)])
    encs = [O.encode_query(case.M[(5 * b + seed) % case.M.shape[0]], case.L, bytes([seed, b]) * 16) for b in range(B)]
    seeds = [O.domain_separate(bytes([seed, b]) * 16, b"protocol2") for b in range(B)]
    return probes, encs, seeds


def test_split_lists_balances_rows():
    from bn_b200 import shard

    sizes = [50, 0, 3, 200, 1, 0, 97, 400, 33, 120]
    for world in (1, 2, 3, 4):
        owner = shard.split_lists(sizes, world)
        assert owner.shape == (len(sizes),) and set(owner.tolist()) == set(range(world))
        load = [sum(s for s, o in zip(sizes, owner) if o == g) for g in range(world)]
        assert max(load) - min(load) <= max(sizes)
        offs = np.concatenate([[0], np.cumsum(sizes)])
        rows = np.concatenate([shard.shard_rows(offs, shard.shard_lists(owner, g)) for g in range(world)])
        assert sorted(rows.tolist()) == list(range(sum(sizes)))  # every row on exactly one rank


def test_local_probes_keep_probe_order_and_pad():
    from bn_b200 import shard

    owner = np.array([0, 1, 1, 0, 1])
    lp, pos = shard.local_probes(np.array([[4, 0, 2], [3, 0, 1]]), owner, 1)
    # rank 1 owns lists 1, 2, 4 (local 0, 1, 2); its empty list is local 3
    assert lp.tolist() == [[2, 1], [0, 3]] and pos.tolist() == [[0, 2], [2, -1]]
    v = shard.local_verdicts(lp, pos, shard.shard_lists(owner, 1), np.array([1, -1]), np.array([4, -1]))
    assert v.tolist() == [[2, 2, 4], [-1, -1, -1]]
    fc, ft = shard.merge_verdicts([v, np.array([[1, 0, 0], [-1, -1, -1]])])
    assert fc.tolist() == [0, -1] and ft.tolist() == [0, -1]  # the earlier probe position wins


@pytest.mark.parametrize("tamper", [None, "late", "two"])
def test_ivf_three_shards_equal_the_whole_corpus(tamper):
    """Lists split over three ranks by split_lists: the merged top-k and the
    first failing (list, trial) in probe order equal one rank holding every
    list, and (honest) the oracle's BnTmIvfScorer::score (ivf.rs:778-823)."""
    from bn_b200 import shard
    from ivfutil import IvfCase

    case = IvfCase(IVF_SIZES, seed=61)
    owner = shard.split_lists(case.sizes, 3)
    probes, encs, seeds = ivf_batch(case, 4, 6, 62)
    for b in range(len(probes)):
        live = [int(c) for c in probes[b] if case.clusters[int(c)] is not None]
        tl = None if tamper is None else (live[-1] if tamper == "late" else live[min(1, len(live) - 1)])
        whole_hits, whole_v = ivf_local(case, probes[b], encs[b], seeds[b], 20, K, set(range(case.nlist)), tl)
        parts = [ivf_local(case, probes[b], encs[b], seeds[b], 20, K, set(shard.shard_lists(owner, g).tolist()), tl)
                 for g in range(3)]
        ids, sc = shard.merge_topk([p[0] for p in parts], K)
        fc, ft = shard.merge_verdicts([np.array([p[1]]) for p in parts])
        assert np.array_equal(ids, whole_hits[0]) and np.array_equal(sc, whole_hits[1])
        assert (fc[0], ft[0]) == (whole_v[1], whole_v[2])
        if tamper is None:
            o = case.oracle_score(probes[b], encs[b], seeds[b], 20, K)
            assert fc[0] == -1 and np.array_equal(ids, o[0]) and np.array_equal(sc, o[1])
        else:
            assert fc[0] == tl and ft[0] == 0


def ivf_worker(rank: int, world: int, port: int, out_dir: str):
    for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "secure-vector-search_b200"), os.path.join(ROOT, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist

    from bn_b200 import shard
    from ivfutil import IvfCase

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    case = IvfCase(IVF_SIZES, seed=71)
    owner = shard.split_lists(case.sizes, world)
    owned = set(shard.shard_lists(owner, rank).tolist())
    probes, encs, seeds = ivf_batch(case, 3, 5, 72)
    tl = int(probes[2][0]) if case.clusters[int(probes[2][0])] is not None else None  # query 2: a tampered first probe
    hits, ver = [], []
    for b in range(3):
        h, v = ivf_local(case, probes[b], encs[b], seeds[b], 20, K, owned, tl if b == 2 else None)
        hits.append(h)
        ver.append(v)
    got, fc, ft = shard.exchange_ivf(dist, None, "cpu", hits, np.array(ver, np.int64), K)
    with open(os.path.join(out_dir, f"ivf_rank{rank}.json"), "w") as fh:
        json.dump({"ids": [g[0].tolist() for g in got], "scores": [g[1].tolist() for g in got],
                   "fc": fc.tolist(), "ft": ft.tolist(), "tampered": tl}, fh)
    dist.barrier()
    dist.destroy_process_group()


def test_ivf_gloo_two_ranks_equal_the_whole_corpus(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    from ivfutil import IvfCase

    mp.spawn(ivf_worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    got = [json.loads((tmp_path / f"ivf_rank{r}.json").read_text()) for r in range(2)]
    assert got[0] == got[1]
    case = IvfCase(IVF_SIZES, seed=71)
    probes, encs, seeds = ivf_batch(case, 3, 5, 72)
    tl = got[0]["tampered"]
    for b in range(3):
        h, v = ivf_local(case, probes[b], encs[b], seeds[b], 20, K, set(range(case.nlist)), tl if b == 2 else None)
        assert got[0]["ids"][b] == h[0].tolist() and got[0]["scores"][b] == h[1].tolist()
        assert (got[0]["fc"][b], got[0]["ft"][b]) == (v[1], v[2])


def test_ivf_shard_edge_cases():
    """More ranks than lists (a rank owns nothing and pads every query with
    its empty list), a batch whose probes miss a rank, k = 0, and a verdict
    from the only shard that failed."""
    from bn_b200 import shard

    owner = shard.split_lists([5, 3], 3)
    assert sorted(owner.tolist()) == [0, 1] and shard.shard_lists(owner, 2).size == 0
    lp, pos = shard.local_probes(np.array([[0, 1], [1, 0]]), owner, 2)
    assert lp.tolist() == [[0], [0]] and pos.tolist() == [[-1], [-1]]  # the empty list only
    assert shard.shard_offsets([0, 5, 8], shard.shard_lists(owner, 2)).tolist() == [0, 0]
    ids, sc = shard.merge_topk([(np.zeros(0, np.uint32), np.zeros(0, np.int64))] * 3, 0)
    assert ids.size == 0 and sc.size == 0
    fc, ft = shard.merge_verdicts([np.array([[-1, -1, -1]]), np.array([[3, 17, 2]])])
    assert fc.tolist() == [17] and ft.tolist() == [2]
