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
