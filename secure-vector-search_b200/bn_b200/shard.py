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

An IVF corpus is split by whole lists instead (split_lists: longest lists
first, each to the rank holding the fewest rows so far).  A (query, list)
pair is scanned, verified with the query's own seed and decoded exactly as
on one GPU (ivf.rs:778-823), so a rank answers for the probes that name its
lists (local_probes; padding with one empty list of its own, skipped as every
empty list is, ivf.rs:787-789), and one exchange per batch all-gathers the
ranks' top-k lists and their first failing (probe position, list, trial); the
query's verdict is the failure at the earliest probe position.

The pure functions (merge_topk, combine_protocol2, split_lists,
local_probes, merge_verdicts) are shared by the collective path and by
single-process emulation of the ranks."""
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


# ---------------------------------------------------------------- IVF: lists per rank

def split_lists(sizes, world: int) -> np.ndarray:
    """owner[c] for every list: longest-processing-time assignment by rows
    (lists by size descending, ties by id; each to the rank holding the fewest
    rows so far, ties to the lower rank).  Needs world <= number of lists for
    every rank to own one."""
    sizes = np.asarray(sizes, np.int64)
    owner = np.zeros(len(sizes), np.int32)
    load = [0] * world
    count = [0] * world
    for c in sorted(range(len(sizes)), key=lambda c: (-int(sizes[c]), c)):
        g = min(range(world), key=lambda r: (load[r], count[r], r))
        owner[c] = g
        load[g] += int(sizes[c])
        count[g] += 1
    return owner


def shard_lists(owner, rank: int) -> np.ndarray:
    """The global ids of rank's lists, ascending (local list i = global list out[i])."""
    return np.flatnonzero(np.asarray(owner) == rank).astype(np.uint32)


def shard_rows(offsets, lists) -> np.ndarray:
    """Corpus rows of the given lists, list by list (the rows of a shard's
    corpus, whose list offsets are shard_offsets)."""
    off = np.asarray(offsets, np.int64)
    parts = [np.arange(off[c], off[c + 1], dtype=np.int64) for c in lists]
    return np.concatenate(parts) if parts else np.zeros(0, np.int64)


def shard_offsets(offsets, lists) -> np.ndarray:
    """List offsets of a shard's corpus: its lists in order, then one empty
    list (local id len(lists)) that pads the probes of a query."""
    off = np.asarray(offsets, np.int64)
    sizes = np.array([off[c + 1] - off[c] for c in lists], np.int64)
    return np.concatenate([[0], np.cumsum(sizes), [sizes.sum()]]).astype(np.uint64)


def local_probes(probes, owner, rank: int):
    """The part of a batch's probes (B x nprobe global list ids) that names
    rank's lists: (local probes B x width, their positions in the query's
    probe order, -1 for padding).  Padding names the shard's empty list."""
    probes = np.asarray(probes, np.int64)
    owner = np.asarray(owner)
    lists = shard_lists(owner, rank)
    local_id = {int(c): i for i, c in enumerate(lists)}
    pad = len(lists)
    rows = [[(j, local_id[int(c)]) for j, c in enumerate(q) if owner[c] == rank] for q in probes]
    width = max(1, max((len(r) for r in rows), default=0))
    lp = np.full((len(rows), width), pad, np.uint32)
    pos = np.full((len(rows), width), -1, np.int64)
    for b, r in enumerate(rows):
        for i, (j, c) in enumerate(r):
            lp[b, i], pos[b, i] = c, j
    return lp, pos


def local_verdicts(lp, pos, lists, failed_local, failed_trial) -> np.ndarray:
    """A shard's verdicts as (probe position, global list, trial) per query,
    (-1, -1, -1) when every pair of the shard passed."""
    out = np.full((len(lp), 3), -1, np.int64)
    for b in range(len(lp)):
        c = int(failed_local[b])
        if c >= 0:
            i = int(np.flatnonzero(lp[b] == c)[0])  # a list appears once among a query's probes
            out[b] = (pos[b, i], int(lists[c]), int(failed_trial[b]))
    return out


def merge_verdicts(verdicts) -> tuple[np.ndarray, np.ndarray]:
    """verdicts: per shard (B x 3: position, list, trial).  The query's first
    failing pair in probe order: (failed list, failed trial), -1 when none."""
    v = np.stack(verdicts)  # [shards, B, 3]
    fc = np.full(v.shape[1], -1, np.int32)
    ft = np.full(v.shape[1], -1, np.int32)
    for b in range(v.shape[1]):
        hit = [x for x in v[:, b] if x[0] >= 0]
        if hit:
            first = min(hit, key=lambda x: x[0])
            fc[b], ft[b] = int(first[1]), int(first[2])
    return fc, ft


def exchange_ivf(dist, group, device, hits, verdicts, k: int):
    """The collective step of one IVF batch on every rank (same order on all):
    all-gather of the shards' top-k lists and of their verdicts.  Returns
    (hits, failed list, failed trial) per query of the whole corpus."""
    import torch

    B = len(hits)
    world = dist.get_world_size(group)
    lst = torch.full((B, max(k, 1), 2), -1, dtype=torch.int64)
    cnt = torch.zeros(B, dtype=torch.int64)
    for b, (ids, sc) in enumerate(hits):
        cnt[b] = len(ids)
        lst[b, : len(ids), 0] = torch.from_numpy(np.asarray(ids, np.int64))
        lst[b, : len(ids), 1] = torch.from_numpy(np.asarray(sc, np.int64))
    ver = torch.from_numpy(np.asarray(verdicts, np.int64).reshape(B, 3))
    lst, cnt, ver = lst.to(device), cnt.to(device), ver.to(device)
    all_lst = [torch.empty_like(lst) for _ in range(world)]
    all_cnt = [torch.empty_like(cnt) for _ in range(world)]
    all_ver = [torch.empty_like(ver) for _ in range(world)]
    dist.all_gather(all_lst, lst, group=group)
    dist.all_gather(all_cnt, cnt, group=group)
    dist.all_gather(all_ver, ver, group=group)
    all_lst = [x.cpu().numpy() for x in all_lst]
    all_cnt = [x.cpu().numpy() for x in all_cnt]
    out_hits = [merge_topk([(L[b, : C[b], 0], L[b, : C[b], 1]) for L, C in zip(all_lst, all_cnt)], k)
                for b in range(B)]
    fc, ft = merge_verdicts([x.cpu().numpy() for x in all_ver])
    return out_hits, fc, ft


def build_ivf_shard(capi, ctx, offsets, ids, m_enc, a_l, h, owner, rank: int, client=None, n1: int = 128):
    """rank's shard of an IVF corpus as an Ivf handle: its lists' rows (ids
    kept global) and one trailing empty list.  m_enc / a_l / h are the whole
    corpus's rows (rows x 1024, rows x n1, rows x n1); client (nullable) is
    (L, m_plain rows x 1024, S rowptr, S idx, S sign) of the whole corpus,
    attached for the rows of the shard."""
    lists = shard_lists(owner, rank)
    rows = shard_rows(offsets, lists)
    n = 1024
    m_enc = np.asarray(m_enc, np.uint64).reshape(-1, n)[rows]
    a_l = np.asarray(a_l, np.uint64).reshape(-1, n1)[rows]
    h = np.asarray(h, np.uint64).reshape(-1, n1)[rows]
    v = capi.Ivf.build(ctx, shard_offsets(offsets, lists), np.asarray(ids, np.uint32)[rows], m_enc, a_l, h, n1=n1)
    if client is not None:
        L, m_plain, rp, ix, sg = client
        rp = np.asarray(rp, np.int64)
        m_plain = np.asarray(m_plain, np.uint64).reshape(-1, n)[rows]
        starts, ends = rp[rows], rp[rows + 1]
        sub_rp = np.concatenate([[0], np.cumsum(ends - starts)]).astype(np.uint64)
        take = np.concatenate([np.arange(a, b) for a, b in zip(starts, ends)]) if len(rows) else np.zeros(0, np.int64)
        v.attach_client(L, m_plain, sub_rp, np.asarray(ix)[take], np.asarray(sg)[take])
    return v, lists


class ShardedIvf:
    """One rank's lists of an IVF corpus: query() runs the per-query IVF
    pipeline on the probes that name its lists and the exchange with the
    other ranks; every rank calls it with the same batch, in the same order."""

    def __init__(self, ivf, lists, owner, rank: int, dist, group=None, device=None):
        self.ivf, self.lists, self.owner, self.rank = ivf, lists, np.asarray(owner), rank
        self.dist, self.group = dist, group
        self.device = device if device is not None else "cpu"

    def local(self, probes, v_enc, g, t_list, v_seeds, trials: int, k: int):
        """This rank's part: (hits with global ids, verdicts B x 3)."""
        lp, pos = local_probes(probes, self.owner, self.rank)
        hits, fc, ft = self.ivf.query(lp, v_enc, g, t_list, v_seeds, trials, k)
        return hits, local_verdicts(lp, pos, self.lists, fc, ft)

    def query(self, probes, v_enc, g, t_list, v_seeds, trials: int, k: int):
        hits, ver = self.local(probes, v_enc, g, t_list, v_seeds, trials, k)
        return exchange_ivf(self.dist, self.group, self.device, hits, ver, k)
