"""Row-sharded flat scoring over several GPUs, one process per GPU.

The reference serves a corpus from one card per process (scorer-bntm/src/
gpu/mod.rs); a corpus split by rows over G GPUs needs one exchange per query
batch, which this module does over torch.distributed (NCCL between GPUs, gloo
on the host for tests):

  - rank g holds rows [row0_g, row0_g + rows_g) (split_rows) and runs
    bn_flat_query_shard on them: its top-k with global row ids, and its
    partial Protocol 2 sums u_t . r and z_t . v_enc for every trial, drawn at
    its rows' positions in the whole corpus (verify_response,
    crypto.rs:1013-1059);
  - the top-k lists are all-gathered and merged (score desc, id asc): the
    global top-k is the top-k of the union of the shards' lists;
  - the partial sums are all-reduced exactly: each canonical residue is split
    into its low 32 and high 29 bits, summed as int64 (no overflow below 2^31
    ranks) and recombined mod p = 2^61 - 1; trial t passes iff both sides
    agree, the first failing trial is the verdict (-1 when all pass).

The pure functions (merge_topk, combine_protocol2) are shared by the
collective path and by single-process emulation of the ranks."""
from __future__ import annotations

import numpy as np

P = (1 << 61) - 1


def split_rows(total: int, world: int, rank: int) -> tuple[int, int]:
    """(row0, rows) of rank's shard: contiguous, sizes differing by at most one."""
    base, extra = divmod(total, world)
    row0 = rank * base + min(rank, extra)
    return row0, base + (1 if rank < extra else 0)


def merge_topk(lists, k: int):
    """lists: per shard (ids u32, scores i64), each ranked.  The global top-k
    ranked by (score desc, id asc), the order of lib.rs:452-469 with the
    tie-break of this backend."""
    ids = np.concatenate([np.asarray(a, np.int64) for a, _ in lists]) if lists else np.zeros(0, np.int64)
    sc = np.concatenate([np.asarray(b, np.int64) for _, b in lists]) if lists else np.zeros(0, np.int64)
    order = np.lexsort((ids, -sc))[:k]
    return ids[order].astype(np.uint32), sc[order]


def _mod_p_sum(lo: int, hi: int) -> int:
    return (int(lo) + (int(hi) << 32)) % P


def combine_protocol2(ur_parts, zv_parts) -> tuple[int, np.ndarray, np.ndarray]:
    """ur_parts / zv_parts: per shard, the canonical partial sums of every
    trial.  Returns (first failing trial or -1, ur, zv) with the sums mod p."""
    ur = [sum(int(x[t]) for x in ur_parts) % P for t in range(len(ur_parts[0]))] if ur_parts else []
    zv = [sum(int(x[t]) for x in zv_parts) % P for t in range(len(zv_parts[0]))] if zv_parts else []
    failed = next((t for t, (a, b) in enumerate(zip(ur, zv)) if a != b), -1)
    return failed, np.array(ur, np.uint64), np.array(zv, np.uint64)


def _split_words(a: np.ndarray) -> np.ndarray:
    """Canonical residues -> int64 [..., 2] (low 32 bits, high 29 bits)."""
    a = np.asarray(a, np.uint64)
    return np.stack([(a & np.uint64(0xFFFFFFFF)).astype(np.int64), (a >> np.uint64(32)).astype(np.int64)], axis=-1)


def exchange(dist, group, device, hits, ur, zv, k: int):
    """The collective step of one batch on every rank (same order on all):
    all-gather of the shards' top-k lists, exact all-reduce of the Protocol 2
    partial sums.  hits: per query (ids, scores) of this shard; ur / zv:
    (B, trials).  Returns (hits, failed_trial per query) of the whole corpus."""
    import torch

    B = len(hits)
    world = dist.get_world_size(group)
    lst = torch.full((B, k, 2), -1, dtype=torch.int64)
    cnt = torch.zeros(B, dtype=torch.int64)
    for b, (ids, sc) in enumerate(hits):
        cnt[b] = len(ids)
        lst[b, : len(ids), 0] = torch.from_numpy(np.asarray(ids, np.int64))
        lst[b, : len(ids), 1] = torch.from_numpy(np.asarray(sc, np.int64))
    lst, cnt = lst.to(device), cnt.to(device)
    all_lst = [torch.empty_like(lst) for _ in range(world)]
    all_cnt = [torch.empty_like(cnt) for _ in range(world)]
    dist.all_gather(all_lst, lst, group=group)
    dist.all_gather(all_cnt, cnt, group=group)
    words = torch.from_numpy(np.stack([_split_words(ur), _split_words(zv)])).to(device)  # [2, B, trials, 2]
    dist.all_reduce(words, op=dist.ReduceOp.SUM, group=group)
    words = words.cpu().numpy()
    all_lst = [x.cpu().numpy() for x in all_lst]
    all_cnt = [x.cpu().numpy() for x in all_cnt]
    out_hits, failed = [], []
    for b in range(B):
        lists = [(L[b, : C[b], 0], L[b, : C[b], 1]) for L, C in zip(all_lst, all_cnt)]
        out_hits.append(merge_topk(lists, k))
        sums = [[_mod_p_sum(*words[side, b, t]) for t in range(words.shape[2])] for side in range(2)]
        failed.append(next((t for t, (a, c) in enumerate(zip(*sums)) if a != c), -1))
    return out_hits, np.array(failed, np.int32)


class ShardedFlat:
    """One rank's shard of a flat corpus: query() runs the shard's pipeline on
    its GPU and the exchange with the other ranks; every rank calls it with
    the same queries, in the same order."""

    def __init__(self, flat, row0: int, total_rows: int, dist, group=None, device=None):
        self.flat, self.row0, self.total, self.dist, self.group = flat, row0, total_rows, dist, group
        self.device = device if device is not None else "cpu"

    def query(self, v_enc, g, t_list, v_seeds, trials: int, k: int):
        hits, ur, zv = self.flat.query_shard(v_enc, g, t_list, v_seeds, trials, k, self.row0, self.total)
        return exchange(self.dist, self.group, self.device, hits, ur, zv, k)
