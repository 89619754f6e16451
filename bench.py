"""Benchmark of the BN F_p scan path on B200.

Default workload (one GPU): flat corpus N = 1,000,000, d = 768 (padded to
n = 1024), int8 data mapped into F_p and BN-encrypted, one query per step
with Protocol 2 (Freivalds, 20 trials) fused into the same launch sequence,
then on-device decode and top-10.  A step = one query through the whole
server + client path.  After it, block scoring (B = 8, 32, 128, 512 queries per
launch as tensor-core GEMMs with Protocol 2 per block) is timed on the same
corpus and reported under "block" in the same JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--block-sizes 8,32,128,512]

Also in the line: a sustained run of 1,000 queries, the reference's default
3 trials, the reference's own GPU scan kernel timed on the same corpus,
the CPU baseline (the oracle over the full corpus, compared bit for bit),
IVF (2M rows, 4096 k-means lists), the serving loop and the N = 100k,
d = 384 workload.

--impl reference times the reference's CPU path (the CPU restatement under
oracle/) on the host cores, one full-size query per timed step.
Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "secure-vector-search_b200"))

N_DIM = 1024
P = (1 << 61) - 1
# DRAM bytes (read + write) per corpus row of one tc_fused_kernel launch:
# dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the
# kernel on a 262,144-row corpus, divided by its rows (the traffic grows in
# proportion to the rows, so it is scaled to the bench's N).
FUSED_DRAM_BYTES_PER_ROW = 8670
METRIC = "BN F_p scan queries/s (flat N=1M, d=768, Freivalds k=20 fused, decode + top-10)"


def synth_int8(rows: int, d: int, seed: int, offset: int = 0) -> np.ndarray:
    """Gaussian -> L2-normalise -> int8 rows (per-row max-abs scaling), as
    int8.  Rows are generated in fixed 65536-row blocks so any prefix is
    identical however many rows are asked for."""
    out = np.empty((rows, d), np.int8)
    blk = 65536
    for b0 in range(0, rows, blk):
        rng = np.random.default_rng([seed, (offset + b0) // blk])
        x = rng.standard_normal((min(blk, rows - b0), d), dtype=np.float32)
        x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
        s = 127.0 / np.maximum(np.abs(x).max(axis=1, keepdims=True), 1e-12)
        out[b0 : b0 + x.shape[0]] = np.clip(np.rint(x * s), -127, 127).astype(np.int8)
    return out


def to_residues(x8: np.ndarray) -> np.ndarray:
    """int8 rows -> F_p residues (u64), zero-padded to n (quantise_vector with Q = 1)."""
    out = np.zeros((x8.shape[0], N_DIM), np.uint64)
    v = x8.astype(np.int64)
    out[:, : x8.shape[1]] = np.where(v < 0, v + P, v).astype(np.uint64)
    return out


def _int8_rows(x: np.ndarray) -> np.ndarray:
    """L2-normalise rows in place, then per-row max-abs int8 quantisation."""
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    s = 127.0 / np.maximum(np.abs(x).max(axis=1, keepdims=True), 1e-12)
    return np.clip(np.rint(x * s), -127, 127).astype(np.int8)


def kmeans_lists(x8: np.ndarray, nlist: int, seed: int, iters: int = 25, device=None):
    """Lloyd k-means (ivf-index/src/kmeans.rs:15-132: k-means++ seeding, then
    assign / recompute until stable or `iters` rounds; an empty cluster's
    centroid becomes 0) over the int8-valued f32 vectors, run with torch on
    the GPU as data preparation: 2M x 4096 x 768 distances per round are
    hours for the host restatement.  Distances are GEMM-form f32 and seeding
    runs on a 65,536-point sample, so the partition is not the reference's
    bit for bit (nor could it be: the reference sums in rayon order); it is
    a real k-means partition of the corpus, fed identically to the GPU path
    and to the oracle.  Centroid sums are exact (integer data, f64 sums), so
    the result is reproducible.  Returns (centroids f32 [nlist][d],
    assignment u32 [rows])."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    X = torch.from_numpy(x8).to(dev).to(torch.float32)
    n = X.shape[0]
    xn = (X * X).sum(1)  # exact: integers below 2^24
    g = torch.Generator(device=dev)
    g.manual_seed(seed)

    def assign(C):
        cn = (C * C).sum(1)
        out = torch.empty(n, dtype=torch.int64, device=dev)
        for r0 in range(0, n, 131072):
            r1 = min(n, r0 + 131072)
            dist = xn[r0:r1, None] - 2.0 * (X[r0:r1] @ C.T) + cn[None, :]
            out[r0:r1] = dist.argmin(1)
        return out

    # k-means++ seeding on a sample: first centre uniform, then each next one
    # with probability proportional to the squared distance to the nearest
    # centre chosen so far (kmeans.rs:93-132)
    samp = X[torch.randperm(n, generator=g, device=dev)[: min(n, 65536)]]
    sn = (samp * samp).sum(1)
    first = int(torch.randint(samp.shape[0], (1,), generator=g, device=dev).item())
    C = torch.empty((nlist, X.shape[1]), dtype=torch.float32, device=dev)
    C[0] = samp[first]
    mind = (sn - 2.0 * (samp @ C[0]) + (C[0] * C[0]).sum()).clamp_min(0)
    for ci in range(1, nlist):
        pick = torch.multinomial(mind + 1e-12, 1, generator=g)
        C[ci] = samp[pick[0]]
        mind = torch.minimum(mind, (sn - 2.0 * (samp @ C[ci]) + (C[ci] * C[ci]).sum()).clamp_min(0))
    for _ in range(iters):
        a = assign(C)
        sums = torch.zeros((nlist, X.shape[1]), dtype=torch.float64, device=dev)
        for r0 in range(0, n, 262144):
            sums.index_add_(0, a[r0 : r0 + 262144], X[r0 : r0 + 262144].to(torch.float64))
        cnt = torch.bincount(a, minlength=nlist).to(torch.float64)
        newC = torch.where(cnt[:, None] > 0, sums / cnt.clamp_min(1)[:, None], 0.0).to(torch.float32)
        if torch.equal(newC, C):
            break
        C = newC
    a = assign(C)
    out = C.cpu().numpy(), a.to(torch.int32).cpu().numpy().astype(np.uint32)
    del X, C, a
    torch.cuda.empty_cache()
    return out


def synth_ivf(rows: int, d: int, nlist: int, seed: int, device=None):
    """Gaussian mixture with nlist unit-norm centres and Zipf(1.1) component
    weights; points = centre + 0.3 * N(0, I) / sqrt(d), L2-normalised,
    int8-quantised per row (data order: ids are row numbers).  The inverted
    lists are a k-means partition of those vectors (kmeans_lists, nlist
    centroids, 25 rounds); rows are stored list by list, members of a list
    in data order (ivf-index/src/ivf.rs build_index)."""
    rng = np.random.default_rng([seed, 0x1FF])
    mix = rng.standard_normal((nlist, d), dtype=np.float32)
    mix /= np.linalg.norm(mix, axis=1, keepdims=True)
    w = 1.0 / np.arange(1, nlist + 1, dtype=np.float64) ** 1.1
    w /= w.sum()
    w = w[rng.permutation(nlist)]
    sigma = np.float32(0.3 / np.sqrt(d))
    x8 = np.empty((rows, d), np.int8)
    for r0 in range(0, rows, 262144):
        r1 = min(rows, r0 + 262144)
        comp = rng.choice(nlist, size=r1 - r0, p=w)
        x8[r0:r1] = _int8_rows(mix[comp] + sigma * rng.standard_normal((r1 - r0, d), dtype=np.float32))
    centroids, assign = kmeans_lists(x8, nlist, seed, device=device)
    order = np.argsort(assign, kind="stable")
    sizes = np.bincount(assign, minlength=nlist).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    return {"centres": centroids, "mix_centres": mix, "weights": w, "sizes": sizes, "offsets": offsets,
            "m8": x8[order], "ids": order.astype(np.uint32), "sigma": sigma, "seed": seed}


def synth_ivf_queries(data, nq: int, seed: int):
    """Queries drawn like the corpus points (mixture component by weight):
    the int8 vector, and the same values as f32 for routing (the scorer sees
    integer-valued f32 vectors, quantisation_q = 1)."""
    rng = np.random.default_rng([seed, 0x9E])
    nlist, d = data["mix_centres"].shape
    comp = rng.choice(nlist, size=nq, p=data["weights"])
    x8 = _int8_rows(data["mix_centres"][comp] + data["sigma"] * rng.standard_normal((nq, d), dtype=np.float32))
    return x8.astype(np.float32), x8


def build_ivf(ctx, data, seed: int):
    """Keys (per-list h_seed, ivf.rs:258-264) and encryption of every list on
    the device (bn_ivf_build_keygen)."""
    from bn_b200 import capi

    rows = int(data["offsets"][-1])
    L = capi.host_generate_subspace(bytes([seed & 0xFF, 0x1F]) * 16)
    data["L"] = L
    mq = np.zeros((rows, N_DIM), np.uint64)
    blk = 1 << 18
    for r0 in range(0, rows, blk):
        mq[r0 : r0 + blk] = to_residues(data["m8"][r0 : r0 + blk])
    ivf = capi.Ivf.build_keygen(ctx, data["offsets"], data["ids"], mq.reshape(-1), L, seed)
    del mq
    return ivf


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int, interval_ms: int = 100):
        self.index, self.samples, self.proc, self.t = index, [], None, None
        self.interval_ms = interval_ms

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", str(self.interval_ms),
                                          "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) >= 9 for i in range(4) if s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU legs
def oracle_module():
    """The CPU restatement of the reference path (oracle/): only the
    cpu_baseline leg and the --impl reference arm run it."""
    p = os.path.join(ROOT, "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)
    import oracle as O

    return O


def prefix_cluster(O, cl, rows: int):
    """The first `rows` rows of an oracle cluster (views, no copies)."""
    n, n1, s = cl.n, cl.n1, cl.s_mat
    e = int(s.rowptr[rows])
    return O.Cluster(rows, n, n1, cl.m_enc[: rows * n], cl.a_l[: rows * n1], cl.m_plain[: rows * n],
                     cl.h_mat[: rows * n1], O.Sparse(s.rowptr[: rows + 1], s.idx[:e], s.sign[:e]))


def cpu_reference_arm(args):
    """--impl reference: the reference's CPU path restated in C (oracle/;
    the Rust reference cannot be built here) on the box's host cores, on the
    bench's own workload: keygen and encryption of the whole corpus on the
    host (crypto.rs:235-270, 405-478), then every timed step one query over
    all N rows (BnTmScorer::score, lib.rs:326-475: scan, Protocol 2, decode,
    top-k).  Warm-up steps query the first 65,536 rows only (they page the
    code and the corpus in; a CPU has no other warm-up)."""
    O = oracle_module()
    n, d, seed = args.rows, 768, 1
    t0 = time.perf_counter()
    Mu = to_residues(synth_int8(n, d, seed))
    L = O.generate_subspace(bytes([seed & 0xFF]) * 32)
    cl = O.encrypt_cluster(Mu.reshape(-1), n, L, O.derive_h_seed(seed, 0))
    del Mu
    setup_s = time.perf_counter() - t0
    qs = to_residues(synth_int8(args.warmup + args.steps, d, seed + 1000))
    warm = prefix_cluster(O, cl, min(n, 65536))
    times = []
    for i in range(args.warmup + args.steps):
        q_seed = O.derive_h_seed(seed ^ 0x5155455259, i)
        ta = time.perf_counter()
        f, _, _, _, _ = O.score_flat(warm if i < args.warmup else cl, L, qs[i], q_seed, args.trials, 10)
        if i >= args.warmup:
            times.append(time.perf_counter() - ta)
        assert f == -1
    return len(times) / sum(times), setup_s, O.NTHREADS, O.lib.bno_have_avx512() != 0


def cpu_baseline_leg(ctx, flat, Mu, L, H, rp, ix, sg, encs, seeds, q_seeds, qv, trials, k, nq=2):
    """cpu_baseline of the GPU arm: the oracle on the host cores over the
    GPU's own corpus (host copies of the device encryption), nq queries of
    all N rows each, timed; the same queries through bn_flat_query are
    compared with it bit for bit (every r residue, the top-k, the verdict)."""
    from bn_b200 import capi

    O = oracle_module()
    n = flat.m
    m_enc, a_l = capi.encrypt_cluster(ctx, Mu.reshape(-1), n, L, H, rp, ix, sg)
    cl = O.Cluster(n, N_DIM, 128, m_enc, a_l, Mu.reshape(-1), H, O.Sparse(rp, ix, sg))
    times, same = [], []
    for i in range(nq):
        ta = time.perf_counter()
        f, ids, sc, r, _ = O.score_flat(cl, L, qv[i], q_seeds[i], trials, k, want_r=True)
        times.append(time.perf_counter() - ta)
        hits, gf, gr, _ = flat.query(encs[i][0][None], encs[i][1][None], [(encs[i][2], encs[i][3])], [seeds[i]],
                                     trials, k, want_r=True)
        same.append(bool(np.array_equal(gr[0], r) and np.array_equal(hits[0][0], ids)
                         and np.array_equal(hits[0][1], sc) and int(gf[0]) == f == -1))
    del m_enc, a_l, cl
    return {"value": nq / sum(times), "unit": "queries/s", "cores": O.NTHREADS, "kind": "port",
            "sample": f"{nq} queries over all {n} rows of the bench corpus (the GPU arm's own encryption, copied "
                      f"to the host); AVX-512 row dot {'on' if O.lib.bno_have_avx512() else 'off'}",
            "parity_vs_gpu": {"queries": nq, "r_topk_verdict_bit_exact": all(same)}}


# ------------------------------------------------------------------ GPU leg
def progress(msg: str):
    """Leg boundaries on stderr (stdout carries only the JSON line)."""
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def max_over_ranks(x: float, dist, device) -> float:
    """The slowest rank's value of x (a time): every rank calls it at the same
    point; on one process (dist None) it is x itself."""
    if not dist:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, slowest_s: float) -> float:
    """Units all ranks processed (each rank the same count) per second of the slowest rank."""
    return world * units_per_rank / slowest_s


class QueryBuffers:
    """Device-resident per-step inputs and outputs of the single-query path
    (one query per step, B = 1)."""

    def __init__(self, torch, dev, encs, seeds, k):
        nq = len(encs)
        t_arr = np.zeros((nq, N_DIM), np.uint32)
        self.tn = tn = np.zeros(nq, np.uint32)
        for i, (ve, g, ti, ts) in enumerate(encs):
            tn[i] = ti.size
            t_arr[i, : ti.size] = ti | np.where(ts < 0, np.uint32(0x80000000), np.uint32(0))
        self.v = torch.from_numpy(np.stack([e[0] for e in encs]).view(np.int64)).to(dev)
        self.g = torch.from_numpy(np.stack([e[1] for e in encs]).view(np.int64)).to(dev)
        self.t = torch.from_numpy(t_arr.view(np.int32)).to(dev)
        self.t_nnz = torch.from_numpy(tn.view(np.int32)).to(dev)
        self.s = torch.from_numpy(np.frombuffer(b"".join(seeds), np.uint8).copy()).to(dev)
        self.ids = torch.zeros((nq, k), dtype=torch.int32, device=dev)
        self.sc = torch.zeros((nq, k), dtype=torch.int64, device=dev)
        self.n = torch.zeros(nq, dtype=torch.int32, device=dev)
        self.f = torch.full((nq,), 7, dtype=torch.int32, device=dev)
        self.nq = nq

    def ptrs(self, i):
        i %= self.nq
        return (self.v[i].data_ptr(), self.g[i].data_ptr(), self.t[i].data_ptr(), self.t_nnz[i : i + 1].data_ptr(),
                self.s[32 * i : 32 * (i + 1)].data_ptr(), self.ids[i].data_ptr(), self.sc[i].data_ptr(),
                self.n[i : i + 1].data_ptr(), self.f[i : i + 1].data_ptr())


def make_timer(torch, stream, dist, dev):
    """timed(fn, warmup, reps): warm-up calls, then reps calls bracketed by a
    barrier + synchronize and CUDA events on the launch stream; returns the
    slowest rank's ms."""

    def timed(fn, warmup, reps, arm=None):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for i in range(warmup):
            fn(i)
        if arm:
            arm()
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(reps):
            fn(warmup + i)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1), dist, dev)

    return timed


def run_gpu(args, rank: int, world: int, local_rank: int):
    import torch

    from bn_b200 import capi

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n_rows, d, trials, k = args.rows, 768, args.trials, 10
    seed = 1 + rank
    t_setup = time.perf_counter()
    Mu = to_residues(synth_int8(n_rows, d, seed))
    key_seed = bytes([seed & 0xFF]) * 32
    L = capi.host_generate_subspace(key_seed)
    H, rp, ix, sg = capi.host_regenerate_h_s(capi.host_derive_h_seed(seed, 0), n_rows)
    ctx = capi.Context(local_rank)
    flat = capi.Flat.build_from_plain(ctx, Mu.reshape(-1), n_rows, L, H, rp, ix, sg)
    if not (rank == 0 and world == 1 and not args.no_cpu_baseline):
        del Mu, H, rp, ix, sg  # kept only for the CPU baseline leg

    nq = max(args.warmup + args.steps, args.sustained)
    qv = to_residues(synth_int8(nq, d, seed + 1000))
    encs, seeds, q_seeds = [], [], []
    for i in range(nq):
        q_seed = capi.host_derive_h_seed(seed ^ 0x5155455259, i)
        encs.append(capi.host_encode_query(qv[i], L, q_seed))
        seeds.append(capi.host_domain_separate(q_seed))
        q_seeds.append(q_seed)
    setup_s = time.perf_counter() - t_setup

    qb = QueryBuffers(torch, dev, encs, seeds, k)
    d_r = torch.zeros(n_rows, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    plans = {"full": flat.plan(1, trials, k), "noverify": flat.plan(1, 0, k), "trials3": flat.plan(1, 3, k)}
    dist = torch.distributed if world > 1 else None
    timed = make_timer(torch, stream, dist, dev)

    # The K timed steps, with the clocks sampled every 25 ms during them; the
    # dominant kernel (the one pass over M_enc: fused scan + Protocol 2) is
    # timed inside every step with CUDA events on its launch stream.  Then the
    # sustained run (config 2's 1,000 queries one at a time, seconds of load
    # under the 1 kW power cap) with its own clock record.
    with ClockSampler(local_rank, interval_ms=25) as clk:
        full_ms = timed(lambda i: plans["full"].enqueue(*qb.ptrs(i), sp), args.warmup, args.steps,
                        arm=lambda: plans["full"].profile(args.steps))
    fused_ms = plans["full"].profile_read()
    with ClockSampler(local_rank) as clk_sus:
        sus_ms = timed(lambda i: plans["full"].enqueue(*qb.ptrs(i), sp), 0, args.sustained) if args.sustained else 0.0
    assert plans["full"].status() == 0
    assert np.all(qb.f.cpu().numpy() == -1), "honest-server verification failed"
    nov_ms = timed(lambda i: plans["noverify"].enqueue(*qb.ptrs(i), sp), args.warmup, args.steps)
    t3_ms = timed(lambda i: plans["trials3"].enqueue(*qb.ptrs(i), sp), args.warmup, args.steps)
    scan_ms = timed(lambda i: plans["full"].enqueue_scan(qb.v[i % qb.nq].data_ptr(), d_r.data_ptr(), sp),
                    args.warmup, args.steps)
    assert np.all(qb.f.cpu().numpy() == -1), "honest-server verification failed"

    # e2e through the C ABI with host buffers (H2D of the encoded query, D2H of hits)
    for i in range(min(args.warmup, nq)):
        flat.query(encs[i][0][None], encs[i][1][None], [(encs[i][2], encs[i][3])], [seeds[i]], trials, k)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        j = args.warmup + i
        flat.query(encs[j][0][None], encs[j][1][None], [(encs[j][2], encs[j][3])], [seeds[j]], trials, k)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)

    per_step_full = full_ms / args.steps / 1e3
    scan_s = scan_ms / args.steps / 1e3
    verify_s = max((full_ms - nov_ms) / args.steps / 1e3, 0.0)
    decode_s = max((nov_ms - scan_ms) / args.steps / 1e3, 0.0)
    bytes_scan = n_rows * N_DIM * 8
    peak, peak_kind = load_peaks()
    stages = {"scan_only_step": scan_s, "protocol2_extra": verify_s, "decode_topk": decode_s}
    fused_s = float(np.mean(fused_ms)) / 1e3
    achieved = bytes_scan / fused_s / 1e9
    h2d = 1024 * 8 + 128 * 8 + 4 * int(np.mean(qb.tn)) + 4 + 32
    d2h = k * 12 + 8
    res = {
        "metric": METRIC,
        "value": whole_job_rate(args.steps, world, full_ms / 1e3),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": full_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64 (exact F_p, p=2^61-1)",
        "data": "synthetic (seeded Gaussian -> L2-normalised -> int8 -> F_p, BN-encrypted on device)",
        "config": {"workload": "bn_flat_single_query", "N": n_rows, "d": 768, "n": N_DIM, "n1": 128,
                   "freivalds_trials": trials, "k": k, "B": 1, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2: every step streams the 8.19 GB M_enc"},
        "stages_ms": dict({s: v * 1e3 for s, v in stages.items()}, fused_kernel=fused_s * 1e3),
        "roofline": {"kernel": "tc_fused_kernel (one pass over M_enc: r = M_enc v and z_t = u_t^T M_enc, 20 trials)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "frac_of_spec_8tbs": achieved / 8000.0,  # B200 HBM3e data-sheet figure, for context
                     "traffic": FUSED_DRAM_BYTES_PER_ROW * n_rows if FUSED_DRAM_BYTES_PER_ROW else None,
                     "algorithmic_bytes_per_launch": bytes_scan, "launches_timed": int(len(fused_ms)),
                     "scan_only_kernel_step": {"achieved": bytes_scan / scan_s / 1e9,
                                               "frac": bytes_scan / scan_s / 1e9 / peak}},
        "e2e": {"value": whole_job_rate(args.steps, world, e2e_s), "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": 9 * args.steps,  # limbs, ugen, query image, fused, rreduce, finish, decide, L^T v, decode + top-k
        "clocks": dict(clk.summary(), window="the K timed steps (sampled every 25 ms)"),
        "sustained": {"queries": args.sustained, "qps": whole_job_rate(args.sustained, world, sus_ms / 1e3)
                      if args.sustained else None, "ms_per_query": sus_ms / max(args.sustained, 1),
                      "clocks": clk_sus.summary(),
                      "note": "config 2's 1,000 queries one at a time right after the K steps, device-resident "
                              "inputs, same plan"},
        "trials3": {"qps": whole_job_rate(args.steps, world, t3_ms / 1e3), "ms_per_step": t3_ms / args.steps,
                    "note": "the reference's default lambda' = 3 trials (params.rs:198-205), same workload"},
        "setup_s": setup_s,
    }
    for p in plans.values():
        p.close()
    progress("single-query leg done")
    if args.ref_kernel:
        res["reference_gpu_kernel"] = run_ref_kernel(args, flat, qb, d_r, stream, timed, peak, scan_s, fused_s,
                                                      nov_ms)
        progress("reference GPU kernel leg done")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res["cpu_baseline"] = cpu_baseline_leg(ctx, flat, Mu, L, H, rp, ix, sg, encs, seeds, q_seeds, qv, trials, k)
        del Mu, H, rp, ix, sg
        progress("CPU baseline leg done")
    del qb, d_r
    if args.block_sizes:
        res["block"] = run_block(args, flat, L, seed, dev, stream, res["value"], dist)
        res["block_qps"] = {B: round(v["qps"], 1) for B, v in res["block"]["per_B"].items()}
        progress("block leg done")
    if args.ivf_rows:
        res["ivf"], ivf, data = run_ivf(args, ctx, dist)
        progress("IVF leg done")
        if args.serve_rates:
            res["serving"] = run_serving(args, flat, ivf, L, data, dist)
            progress("serving leg done")
        ivf.close()
    flat.close()
    if args.config1:
        res["config1"] = run_config1(args, ctx, dev, stream, timed, rank, world)
        progress("config-1 leg done")
    if args.stream_rows:
        res["stream"] = run_stream(args, ctx)
        progress("streaming leg done")
    ctx.close()
    return res


def run_ref_kernel(args, flat, qb, d_r, stream, timed, peak, scan_s, fused_s, nov_ms):
    """The reference's own GPU scan kernel (bntm_compute_products,
    scorer-bntm/src/gpu/kernels.cu:100-178, compiled from the reference
    source for sm_100a; one 256-thread CTA per row) timed on the same corpus,
    stream and queries as the product's kernels, its r checked bit for bit
    against the product's scan."""
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu

    lib = ref_gpu.load()
    if lib is None:
        return {"unavailable": "oracle/_ref/libbnref_gpu.so was not built (no reference checkout at build time)"}
    m_enc = flat.device_m_enc()
    r_ref = torch.zeros_like(d_r)
    sp = stream.cuda_stream

    def ref(i):
        assert lib.bnref_compute_products(m_enc, qb.v[i % qb.nq].data_ptr(), r_ref.data_ptr(), flat.m, sp) == 0

    ms = timed(ref, args.warmup, args.steps) / args.steps
    # bit-exact against the product's scan on one query
    plan = flat.plan(1, 0, 0)
    with torch.cuda.stream(stream):
        plan.enqueue_scan(qb.v[0].data_ptr(), d_r.data_ptr(), sp)
        ref(0)
    stream.synchronize()
    same = bool(torch.equal(d_r, r_ref))
    plan.close()
    gbs = flat.m * N_DIM * 8 / (ms / 1e3) / 1e9
    return {"kernel": "bntm_compute_products (reference kernels.cu:100-178, built for sm_100a)",
            "ms_per_launch": ms, "achieved_gbs": gbs, "frac_of_peak": gbs / peak,
            "r_equals_product_scan": same,
            "product_scan_only_ms": scan_s * 1e3, "product_fused_scan_protocol2_ms": fused_s * 1e3,
            "speedup_scan_only": ms / (scan_s * 1e3), "speedup_fused_incl_20_trials": ms / (fused_s * 1e3)}


def run_config1(args, ctx, dev, stream, timed, rank, world):
    """Config 1 (the reference's CPU case): N = 100,000, d = 384, seed 0,
    100 queries one at a time, top-10, trials 20 and the reference's default
    3: the GPU path timed, and the oracle on the host cores over the first 10
    queries of each, compared bit for bit."""
    import torch

    from bn_b200 import capi

    n, d, k, seed, nq = 100_000, 384, 10, 0, 100
    Mu = to_residues(synth_int8(n, d, seed))
    L = capi.host_generate_subspace(bytes([seed]) * 32)
    H, rp, ix, sg = capi.host_regenerate_h_s(capi.host_derive_h_seed(seed, 0), n)
    flat = capi.Flat.build_from_plain(ctx, Mu.reshape(-1), n, L, H, rp, ix, sg)
    qv = to_residues(synth_int8(nq, d, seed + 1000))
    encs, seeds, q_seeds = [], [], []
    for i in range(nq):
        q_seed = capi.host_derive_h_seed(seed ^ 0x5155455259, i)
        encs.append(capi.host_encode_query(qv[i], L, q_seed))
        seeds.append(capi.host_domain_separate(q_seed))
        q_seeds.append(q_seed)
    qb = QueryBuffers(torch, dev, encs, seeds, k)
    sp = stream.cuda_stream
    out = {"N": n, "d": d, "queries": nq, "k": k, "per_trials": {}}
    cl = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        O = oracle_module()
        m_enc, a_l = capi.encrypt_cluster(ctx, Mu.reshape(-1), n, L, H, rp, ix, sg)
        cl = O.Cluster(n, N_DIM, 128, m_enc, a_l, Mu.reshape(-1), H, O.Sparse(rp, ix, sg))
    for trials in (20, 3):
        plan = flat.plan(1, trials, k)
        ms = timed(lambda i: plan.enqueue(*qb.ptrs(i), sp), 3, nq)
        assert plan.status() == 0 and np.all(qb.f.cpu().numpy() == -1)
        rec = {"gpu_qps": whole_job_rate(nq, world, ms / 1e3), "gpu_ms_per_query": ms / nq}
        if cl is not None:
            O = oracle_module()
            ids_g = qb.ids.cpu().numpy().view(np.uint32)
            sc_g = qb.sc.cpu().numpy()
            times, same = [], []
            for i in range(10):
                ta = time.perf_counter()
                f, ids, sc, _, _ = O.score_flat(cl, L, qv[i], q_seeds[i], trials, k)
                times.append(time.perf_counter() - ta)
                same.append(bool(f == -1 and np.array_equal(ids_g[i], ids) and np.array_equal(sc_g[i], sc)))
            rec.update({"cpu_qps": 10 / sum(times), "cpu_cores": O.NTHREADS, "cpu_queries": 10,
                        "gpu_over_cpu": rec["gpu_qps"] / (10 / sum(times)), "topk_verdict_bit_exact": all(same)})
        out["per_trials"][str(trials)] = rec
        plan.close()
    flat.close()
    return out


def run_stream(args, ctx):
    """A flat corpus streamed through device memory (bn_stream): N rows in
    chunks of C rows with a budget of S chunk slots, B queries per call.  A
    call scores every chunk: the resident ones first while the others are
    uploaded from pinned host memory into the slots of chunks already scored.
    Timed end to end on the host clock (host inputs and outputs, every copy
    inside); the first call's hits and verdicts are compared with a resident
    flat corpus built from the same data."""
    from bn_b200 import capi

    n, d, seed, k, trials = args.stream_rows, 768, 11, 10, args.trials
    chunk, slots = args.stream_chunk_rows, args.stream_slots
    Mu = to_residues(synth_int8(n, d, seed))
    L = capi.host_generate_subspace(bytes([seed]) * 32)
    H, rp, ix, sg = capi.keygen_h_s(ctx, capi.host_derive_h_seed(seed, 0), n, 128)
    # slot size from a one-chunk probe (+4 % for chunks with wider ELL slices)
    probe = capi.Stream.build_from_plain(ctx, Mu[:chunk].reshape(-1), chunk, L, H[: chunk * 128], rp[: chunk + 1],
                                         ix, sg, chunk, 1 << 42)
    budget = int(slots * probe.info()["slot_bytes"] * 1.04)
    probe.close()
    t0 = time.perf_counter()
    st = capi.Stream.build_from_plain(ctx, Mu.reshape(-1), n, L, H, rp, ix, sg, chunk, budget)
    build_s = time.perf_counter() - t0
    info = st.info()
    nq = 64
    x8 = synth_int8(nq, d, seed + 500)
    encs, seeds = encode_pool(L, nq, x8, seed + 500)
    out = {"N": n, "chunk_rows": chunk, "chunks": info["chunks"], "slots": info["slots"],
           "slot_gib": info["slot_bytes"] / 2**30, "host_image_gib": info["host_bytes"] / 2**30,
           "corpus_over_budget": info["chunks"] / max(info["slots"], 1), "build_s": build_s, "per_B": {}}
    flat = capi.Flat.build_from_plain(ctx, Mu.reshape(-1), n, L, H, rp, ix, sg)
    for B in (1, 16, 64):
        a = (np.stack([e[0] for e in encs[:B]]), np.stack([e[1] for e in encs[:B]]),
             [(e[2], e[3]) for e in encs[:B]], seeds[:B], trials, k)
        got, gf = st.query(*a)  # warm-up call, checked against the resident corpus
        want, wf, _, _ = flat.query(*a)
        same = bool(np.array_equal(gf, wf) and np.all(gf == -1) and
                    all(np.array_equal(got[b][0], want[b][0]) and np.array_equal(got[b][1], want[b][1])
                        for b in range(B)))
        st.stats(reset=True)
        calls = 3
        t0 = time.perf_counter()
        for _ in range(calls):
            st.query(*a)
        dt = time.perf_counter() - t0
        s = st.stats()
        out["per_B"][str(B)] = {"qps": B * calls / dt, "ms_per_call": dt / calls * 1e3,
                                "uploads_per_call": s["uploads"] / calls,
                                "gib_uploaded_per_call": s["bytes_uploaded"] / calls / 2**30,
                                "h2d_gbs": s["bytes_uploaded"] / dt / 1e9, "hits_verdicts_equal_resident": same}
    flat.close()
    st.close()
    out["ivf"] = run_stream_ivf(args, ctx)
    return out


def run_stream_ivf(args, ctx):
    """The IVF form (bn_ivf_stream): a k-means-partitioned corpus of N rows
    and 512 lists in chunks of whole lists, a budget of S chunk slots,
    batches of 64 queries routed to nprobe lists; a call uploads only the
    chunks holding a probed list.  The first call's hits and verdicts are
    compared with a resident IVF corpus built from the same data."""
    from bn_b200 import capi

    n, nlist, seed, k, trials = args.stream_rows, 512, 12, 10, args.trials
    chunk, slots = args.stream_chunk_rows, args.stream_slots
    data = synth_ivf(n, 768, nlist, seed)
    L = capi.host_generate_subspace(bytes([seed & 0xFF, 0x1F]) * 16)
    mq = to_residues(data["m8"])
    probe = capi.IvfStream.build_keygen(ctx, data["offsets"], data["ids"], mq.reshape(-1), L, seed, chunk, 1 << 42)
    budget = slots * probe.info()["slot_bytes"]
    probe.close()
    t0 = time.perf_counter()
    st = capi.IvfStream.build_keygen(ctx, data["offsets"], data["ids"], mq.reshape(-1), L, seed, chunk, budget)
    build_s = time.perf_counter() - t0
    res = capi.Ivf.build_keygen(ctx, data["offsets"], data["ids"], mq.reshape(-1), L, seed)
    del mq
    info = st.info()
    B = 64
    qx, q8 = synth_ivf_queries(data, B, seed + 1)
    encs, seeds = encode_pool(L, B, q8, seed + 1)
    out = {"N": n, "nlist": nlist, "chunk_rows": chunk, "chunks": info["chunks"], "slots": info["slots"],
           "slot_gib": info["slot_bytes"] / 2**30, "host_image_gib": info["host_bytes"] / 2**30,
           "build_s": build_s, "B": B, "per_nprobe": {}}
    for nprobe in (8, 32):
        probes = np.stack([capi.host_probe_route(data["centres"], qx[i], nprobe)[0] for i in range(B)])
        a = (probes, np.stack([e[0] for e in encs]), np.stack([e[1] for e in encs]),
             [(e[2], e[3]) for e in encs], seeds, trials, k)
        got, gc, gt = st.query(*a)  # warm-up call, checked against the resident corpus
        want, wc, wt = res.query(*a)
        same = bool(np.array_equal(gc, wc) and np.array_equal(gt, wt) and np.all(gt == -1) and
                    all(np.array_equal(got[b][0], want[b][0]) and np.array_equal(got[b][1], want[b][1])
                        for b in range(B)))
        st.stats(reset=True)
        calls = 3
        t0 = time.perf_counter()
        for _ in range(calls):
            st.query(*a)
        dt = time.perf_counter() - t0
        s = st.stats()
        out["per_nprobe"][str(nprobe)] = {
            "qps": B * calls / dt, "ms_per_call": dt / calls * 1e3, "chunks_needed_per_call": s["gets"] / calls,
            "uploads_per_call": s["uploads"] / calls, "gib_uploaded_per_call": s["bytes_uploaded"] / calls / 2**30,
            "h2d_gbs": s["bytes_uploaded"] / dt / 1e9, "hits_verdicts_equal_resident": same}
    res.close()
    st.close()
    return out


def run_block(args, flat, L, seed, dev, stream, single_qps, dist):
    """Block scoring (B queries per launch, tensor-core GEMMs, Protocol 2 per
    block): each timed step is one CUDA-graph replay of G consecutive blocks
    with distinct inputs; ~10,240 queries per block size (bounded)."""
    import torch

    from bn_b200 import capi

    d, k, trials = 768, 10, args.trials
    sizes = [int(b) for b in args.block_sizes.split(",") if b]
    pool = max(sizes) * 4
    qv = to_residues(synth_int8(pool, d, seed + 2000))
    encs = [capi.host_encode_query(qv[i], L, capi.host_derive_h_seed(seed ^ 0x424C4B, i)) for i in range(pool)]
    t_arr = np.zeros((pool, N_DIM), np.uint32)
    tn = np.zeros(pool, np.uint32)
    for i, (ve, g, ti, ts) in enumerate(encs):
        tn[i] = ti.size
        t_arr[i, : ti.size] = ti | np.where(ts < 0, np.uint32(0x80000000), np.uint32(0))
    d_v = torch.from_numpy(np.stack([e[0] for e in encs]).view(np.int64)).to(dev)
    d_g = torch.from_numpy(np.stack([e[1] for e in encs]).view(np.int64)).to(dev)
    d_t = torch.from_numpy(t_arr.view(np.int32)).to(dev)
    d_tn = torch.from_numpy(tn.view(np.int32)).to(dev)
    seeds = torch.from_numpy(np.frombuffer(b"".join(bytes([j + 1]) * 32 for j in range(8)), np.uint8).copy()).to(dev)
    d_ids = torch.zeros((pool, k), dtype=torch.int32, device=dev)
    d_sc = torch.zeros((pool, k), dtype=torch.int64, device=dev)
    d_n = torch.zeros(pool, dtype=torch.int32, device=dev)
    d_f = torch.full((pool,), 7, dtype=torch.int32, device=dev)
    flat.block_prepare()
    out = {"trials": trials, "k": k, "freivalds": "one seed per block, every query checked", "per_B": {}}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_tops = 2.0 * float(json.load(f)["bf16_tflops"])  # dense int8 rate = 2x dense bf16 on sm_100
        peak_src = "2 x measured dense bf16 (int8 tensor rate on sm_100)"
    except (OSError, KeyError, ValueError):
        peak_tops = 2.0 * 1590.0
        peak_src = "2 x fallback dense bf16 1590 TFLOP/s (int8 tensor rate on sm_100)"
    best = None
    for B in sizes:
        plan = flat.block_plan(B, trials, k, autotune=args.block_autotune)
        cfg = plan.block_config()
        G = max(1, min(4, pool // B))
        reps = max(args.warmup + 1, min(10240 // B, 1280) // G)

        def ptrs(j):
            o = j * B
            return (d_v[o].data_ptr(), d_g[o].data_ptr(), d_t[o].data_ptr(), d_tn[o : o + 1].data_ptr(),
                    seeds[32 * j : 32 * (j + 1)].data_ptr(), d_ids[o].data_ptr(), d_sc[o].data_ptr(),
                    d_n[o : o + 1].data_ptr(), d_f[o : o + 1].data_ptr())

        with torch.cuda.stream(stream):
            for j in range(G):
                plan.enqueue(*ptrs(j), stream.cuda_stream)
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            for j in range(G):
                plan.enqueue(*ptrs(j), torch.cuda.current_stream().cuda_stream)
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(reps):
            graph.replay()
        ev1.record()
        ev1.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
        del graph
        status = plan.status()
        fl = d_f[: G * B].cpu().numpy()
        assert status == 0 and np.all(fl == -1), "block verification failed on honest responses"
        nq = reps * G * B
        qps = whole_job_rate(nq, dist.get_world_size() if dist else 1, ms / 1e3)
        macs = flat.m * 8 * 8 * B * N_DIM  # byte-planar r = M_enc v GEMM
        gemm_tops = 2 * macs / (cfg["tuned_scan_ms"] / 1e3) / 1e12 if cfg["tuned_scan_ms"] else None
        out["per_B"][str(B)] = {"qps": qps, "ms_per_block": ms / (reps * G), "queries_timed": nq, "graph_blocks": G,
                                "tiling": {kk: cfg[kk] for kk in ("w_tile", "stages", "order", "a_resident", "k_panel",
                                                                  "two_ksteps_per_stage")},
                                "scan_gemm_ms": cfg["tuned_scan_ms"], "scan_gemm_tops": gemm_tops}
        if best is None or qps > best[1]:
            best = (B, qps, gemm_tops)
        plan.close()
    out["best"] = {"B": best[0], "qps": best[1], "vs_single_query": best[1] / single_qps}
    if best[2]:
        out["roofline"] = {"kernel": f"bgemm r = M_enc v (B={best[0]})", "bound": "tensor", "achieved": best[2],
                           "peak": peak_tops, "unit": "TOP/s int8", "frac": best[2] / peak_tops,
                           "peak_source": peak_src}
    # e2e through the C ABI with host buffers (pack + H2D + block pipeline + D2H of hits)
    B = 32 if 32 in sizes else sizes[0]
    vb = np.stack([e[0] for e in encs[:B]])
    gb = np.stack([e[1] for e in encs[:B]])
    tb = [(e[2], e[3]) for e in encs[:B]]
    for _ in range(2):
        flat.query_block(vb, gb, tb, bytes([1]) * 32, trials, k)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        hits, fl, _ = flat.query_block(vb, gb, tb, bytes([1]) * 32, trials, k)
    e2e_s = (time.perf_counter() - t0) / reps
    assert np.all(fl == -1)
    h2d = B * (N_DIM * 8 + 128 * 8 + 4 * N_DIM + 4) + 32
    out["e2e"] = {"B": B, "value": B / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                  "d2h_bytes_per_step": B * (k * 12 + 8)}
    return out


def encode_pool(L, n: int, x8: np.ndarray, seed: int):
    """Encoded queries (v_enc, g, T) and their Protocol 2 seeds."""
    from bn_b200 import capi

    encs, seeds = [], []
    for i in range(n):
        q_seed = capi.host_derive_h_seed(seed ^ 0x5155455259, i)
        encs.append(capi.host_encode_query(to_residues(x8[i : i + 1])[0], L, q_seed))
        seeds.append(capi.host_domain_separate(q_seed))
    return encs, seeds


def run_ivf(args, ctx, dist):
    """BN-IVF with uneven lists (Zipf-weighted Gaussian mixture, nlist 4096):
    batches of 64 queries, nprobe 8 / 32 / 128, every probed list of every
    query scanned, verified (Protocol 2, per query and list), decoded and
    ranked in one launch per stage; through the C ABI with host buffers."""
    from bn_b200 import capi

    seed, nlist, bq = 3, 4096, 64
    t0 = time.perf_counter()
    data = synth_ivf(args.ivf_rows, 768, nlist, seed)
    ivf = build_ivf(ctx, data, seed)
    setup_s = time.perf_counter() - t0
    qx, q8 = synth_ivf_queries(data, bq, seed)
    encs, seeds = encode_pool(data["L"], bq, q8, seed)
    out = {"N": args.ivf_rows, "nlist": nlist, "batch": bq, "trials": args.trials, "k": 10,
           "lists": {"max": int(data["sizes"].max()), "median": float(np.median(data["sizes"])),
                     "min": int(data["sizes"].min())},
           "data": "synthetic Gaussian mixture, Zipf(1.1) weights; lists = k-means partition (4096 centroids, "
                   "k-means++ seeding, 25 Lloyd rounds)",
           "setup_s": setup_s, "per_nprobe": {}}
    vb = np.stack([e[0] for e in encs])
    gb = np.stack([e[1] for e in encs])
    tb = [(e[2], e[3]) for e in encs]
    for nprobe in (8, 32, 128):
        pr = capi.host_probe_route(data["centres"], qx, nprobe)
        rows_q = float(np.mean([data["sizes"][p].sum() for p in pr]))
        hits, fc, ft = ivf.query(pr, vb, gb, tb, seeds, args.trials, 10)
        assert np.all(fc == -1), "IVF verification failed on honest responses"
        ivf.query(pr, vb, gb, tb, seeds, args.trials, 10)  # a second warm-up call
        if dist:
            dist.barrier()
        reps, t = 5, []  # median of 5 calls
        for _ in range(reps):
            ta = time.perf_counter()
            ivf.query(pr, vb, gb, tb, seeds, args.trials, 10)
            t.append(time.perf_counter() - ta)
        dt = statistics.median(t)
        uniq = np.unique(pr)
        rows_u = float(data["sizes"][uniq].sum())
        res = {"qps": bq / dt, "ms_per_batch": dt * 1e3, "rows_per_query": rows_q,
               "effective_gbs": bq * rows_q * N_DIM * 8 / dt / 1e9, "distinct_lists": int(len(uniq)),
               "distinct_rows": rows_u}
        # block form: the batch's (query, list) pairs grouped by list, every
        # probed list read once; Protocol 2 per block and list
        progress(f"IVF nprobe {nprobe}: per-query path timed")
        bseed = bytes([seed, nprobe & 0xFF]) * 16
        bh, bfc, _ = ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)
        assert np.all(bfc == -1), "IVF block verification failed on honest responses"
        same = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(hits, bh))
        ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)  # a second warm-up call
        t = []
        for _ in range(reps):
            ta = time.perf_counter()
            ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)
            t.append(time.perf_counter() - ta)
        db = statistics.median(t)
        t_first = t
        ivf.block_profile(True)  # one more call with stage events (not part of the timing above)
        ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)
        stages = ivf.block_profile_read()
        # GEMM tilings (W rows per tile, pipeline stages; 0 = automatic): G1 time of each
        sweep = {}
        for w_tile, st in ((0, 0), (32, 0), (64, 0), (128, 0), (256, 0), (64, 6)):  # 0: the automatic choice
            ivf.block_tune(w_tile, st)
            ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)
            g1, wall = [], []
            for _ in range(3):
                ta = time.perf_counter()
                ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)
                wall.append(time.perf_counter() - ta)
                g1.append(ivf.block_profile_read())
            sweep[f"w{w_tile}_s{st}"] = dict({k: round(statistics.median(x[k] for x in g1), 3)
                                              for k in ("g1_r", "g2_al_h", "g3_m_t_s_v")},
                                             call_ms=round(statistics.median(wall) * 1e3, 3))
        ivf.block_tune(0, 0)
        ivf.block_profile(False)
        # the same five timed calls again after the sweep
        t_late = []
        for _ in range(reps):
            ta = time.perf_counter()
            ivf.query_block(pr, vb, gb, tb, bseed, args.trials, 10)
            t_late.append(time.perf_counter() - ta)
        res["block_repeat"] = {"calls_ms_first": [round(x * 1e3, 3) for x in t_first],
                               "calls_ms_after_sweep": [round(x * 1e3, 3) for x in t_late]}
        res["block"] = {"qps": bq / db, "ms_per_batch": db * 1e3, "hits_equal_per_query": bool(same),
                        "distinct_rows_gbs": rows_u * N_DIM * 8 / db / 1e9, "stages_ms": stages,
                        "tiling_sweep_ms": sweep}
        out["per_nprobe"][str(nprobe)] = res
    return out, ivf, data


def run_serving(args, flat, ivf, flat_L, data, dist):
    """Poisson arrivals, 50% flat / 50% IVF with nprobe uniform in {8, 32,
    128}, Protocol 2 on for all, through bn_server (continuous batching,
    memory admission); every served result compared with the per-query path
    on the same inputs."""
    from bn_b200 import capi

    seed, pool = 4, 256
    rng = np.random.default_rng(seed)
    fx8 = synth_int8(pool, 768, seed + 3000)
    fenc, fseeds = encode_pool(flat_L, pool, fx8, seed)
    qx, q8 = synth_ivf_queries(data, pool, seed + 1)
    ienc, iseeds = encode_pool(data["L"], pool, q8, seed + 1)
    nps = rng.choice([8, 32, 128], size=pool)
    probes = [capi.host_probe_route(data["centres"], qx[i], int(nps[i]))[0] for i in range(pool)]
    # per-query references (the plain per-query path on the same GPU)
    ref_f, ref_i = [], []
    for i in range(pool):
        h, f, _, _ = flat.query(fenc[i][0][None], fenc[i][1][None], [(fenc[i][2], fenc[i][3])], [fseeds[i]],
                                args.trials, 10)
        ref_f.append((h[0][0], h[0][1], int(f[0])))
        h, fc, ft = ivf.query(probes[i][None], ienc[i][0][None], ienc[i][1][None], [(ienc[i][2], ienc[i][3])],
                              [iseeds[i]], args.trials, 10)
        ref_i.append((h[0][0], h[0][1], int(ft[0])))
    qwait = args.serve_queue_wait_ms * 1000
    mb = args.serve_max_batch
    srv = capi.Server(flat, ivf, max_batch=mb, slots=4, mem_budget=24 << 30, max_wait_us=1000, trials=args.trials,
                      k=10, block_min=2, queue_wait_us=qwait)
    out = {"corpora": {"flat_N": flat.m, "ivf_N": int(data["offsets"][-1]), "nlist": int(len(data["sizes"]))},
           "config": {"max_batch": mb, "slots": 4, "mem_budget_gib": 24, "max_wait_us": 1000, "block_min": 2,
                      "queue_wait_us": qwait},
           "mix": "50% flat / 50% IVF, nprobe uniform in {8, 32, 128}",
           "warmup": "the server creates one flat block plan per block size at start-up; before the timed "
                     "rates, 256 flat requests, 256 IVF requests at nprobe 128 and 512 mixed ones submitted at "
                     "once (the slots grow their workspaces and staging buffers), not counted",
           "rates": {}}
    # warm-up: the slots grow their workspaces to the largest batches once,
    # as a service does at start-up: full flat batches, full IVF batches of
    # the widest probes (nprobe 128), then the mix
    heavy = [i for i in range(pool) if nps[i] == 128] or list(range(pool))
    order = ([(1, j % pool) for j in range(256)] + [(0, heavy[j % len(heavy)]) for j in range(256)] +
             [(j & 1, j % pool) for j in range(512)])
    warm = []
    for is_flat, i in order:
        while True:  # a refused submit (queue admission) waits for the oldest request, then retries
            try:
                if is_flat:
                    warm.append(srv.submit_flat(fenc[i][0], fenc[i][1], fenc[i][2], fenc[i][3], fseeds[i]))
                else:
                    warm.append(srv.submit_ivf(probes[i], ienc[i][0], ienc[i][1], ienc[i][2], ienc[i][3], iseeds[i]))
                break
            except capi.BnError as err:
                if err.code != capi.BN_EAGAIN or not warm:
                    raise
                srv.wait(warm.pop(0), 600000)
    for t in warm:
        srv.wait(t, 600000)
    for rate in [float(r) for r in args.serve_rates.split(",") if r]:
        n = int(min(max(rate * args.serve_seconds, 200), 16000))
        kinds = rng.random(n) < 0.5
        picks = rng.integers(0, pool, size=n)
        gaps = rng.exponential(1.0 / rate, size=n)
        srv.stats(reset=True)
        tickets = []
        t_start = time.perf_counter()
        due = t_start
        for j in range(n):
            due += gaps[j]
            while time.perf_counter() < due:
                pass
            i = int(picks[j])
            try:  # refused (BN_EAGAIN) when the queue's expected wait exceeds queue_wait_us
                if kinds[j]:
                    e = fenc[i]
                    tickets.append((j, srv.submit_flat(e[0], e[1], e[2], e[3], fseeds[i])))
                else:
                    e = ienc[i]
                    tickets.append((j, srv.submit_ivf(probes[i], e[0], e[1], e[2], e[3], iseeds[i])))
            except capi.BnError as err:
                if err.code != capi.BN_EAGAIN:
                    raise
        offered = n / (time.perf_counter() - t_start)
        bad = 0
        for j, t in tickets:
            ids, sc, ft, fc, lat = srv.wait(t, 600000)
            ref = ref_f[picks[j]] if kinds[j] else ref_i[picks[j]]
            if not (np.array_equal(ids, ref[0]) and np.array_equal(sc, ref[1]) and ft == ref[2]):
                bad += 1
        st = srv.stats()
        out["rates"][str(int(rate))] = {"offered_qps": offered, "requests": n, "admitted": len(tickets),
                                        "refused": int(st["rejected"]), "served_qps": st["throughput_qps"],
                                        "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3,
                                        "max_ms": st["max_us"] / 1e3, "mean_batch": st["mean_batch"],
                                        "block_batches": st["block_batches"],
                                        "peak_workspace_gib": st["peak_workspace_bytes"] / 2**30,
                                        "mismatches_vs_per_query": bad}
    srv.close()
    ok = [float(r) for r, v in out["rates"].items() if v["p99_ms"] <= 100.0 and v["refused"] == 0]
    out["max_offered_qps_all_admitted_p99_le_100ms"] = max(ok) if ok else None
    out["saturated_served_qps"] = max(v["served_qps"] for v in out["rates"].values())
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=1_000_000)
    ap.add_argument("--trials", type=int, default=20)
    ap.add_argument("--sustained", type=int, default=1000,
                    help="queries of the sustained single-query run (config 2's 1,000; 0 to skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-kernel", dest="ref_kernel", action="store_false",
                    help="skip timing the reference's own GPU scan kernel")
    ap.add_argument("--no-config1", dest="config1", action="store_false",
                    help="skip the N = 100k, d = 384 workload (the reference's CPU case)")
    ap.add_argument("--block-sizes", default="8,32,128,512",
                    help="block scoring sizes B to time after the single-query metric ('' to skip)")
    ap.add_argument("--no-block-autotune", dest="block_autotune", action="store_false",
                    help="block plans keep the default GEMM tiling (no autotuning launches)")
    ap.add_argument("--ivf-rows", type=int, default=2_000_000, help="IVF corpus rows (0 to skip the IVF legs)")
    ap.add_argument("--serve-rates", default="1000,2000,4000,6000,8000,50000",
                    help="Poisson arrival rates of the serving leg")
    ap.add_argument("--serve-seconds", type=float, default=1.5)
    ap.add_argument("--stream-rows", type=int, default=262_144,
                    help="rows of the streamed corpus (bn_stream, larger than its budget; 0 to skip)")
    ap.add_argument("--stream-chunk-rows", type=int, default=32_768)
    ap.add_argument("--stream-slots", type=int, default=3, help="chunk slots the streamed corpus's budget holds")
    ap.add_argument("--serve-max-batch", type=int, default=64, help="serving: most queries per launched batch")
    ap.add_argument("--serve-queue-wait-ms", type=int, default=40,
                    help="serving admission: refuse a request when the queue's expected wait exceeds this (0: off)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        qps, setup_s, cores, avx = cpu_reference_arm(args)
        line = {"metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u64 (exact F_p, p=2^61-1)", "data": "synthetic",
                "config": {"workload": "bn_flat_single_query", "N": args.rows, "d": 768, "n": N_DIM, "n1": 128,
                           "freivalds_trials": args.trials, "k": 10, "B": 1},
                "impl": "reference",
                "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": cores, "kind": "port",
                                 "sample": f"every timed step one query over all {args.rows} rows (warm-up steps: "
                                           f"the first 65,536 rows); corpus keygen + encryption on the host took "
                                           f"{setup_s:.0f} s; AVX-512 row dot {'on' if avx else 'off'}"},
                "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                             device_id=torch.device("cuda", local_rank))
    res = run_gpu(args, rank, world, local_rank)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
