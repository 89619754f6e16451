"""GPU parity of the flat path through the C ABI against the oracle.

Restates the reference's GPU tests (scorer-bntm/src/lib.rs:1189-1639) and its
crypto.rs tests on the device path.  Every comparison is bit-exact (integer
F_p work, no tolerance)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, cluster, int8_matrix, query, uniform_fp

pytestmark = pytest.mark.gpu


def capi():
    from bn_b200 import capi as c

    return c


def flat_from_cluster(ctx, M, L, cl):
    c = capi()
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    return f


@pytest.mark.parametrize("m", [1, 7, 256, 257, 300, 511, 1024, 1500])
def test_compute_products_varied_m(ctx, m):
    """lib.rs:1256-1312: uniform F_p inputs, bit-equal r."""
    c = capi()
    m_enc = uniform_fp((m, N), 2400 + m)
    v = uniform_fp(N, 9400 + m)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    assert np.array_equal(f.compute_products(v), O.matvec(m_enc, m, N, v))


def test_compute_products_extreme_residues(ctx):
    c = capi()
    m = 37
    m_enc = np.full((m, N), P - 1, np.uint64)
    m_enc[::3] = 0
    v = np.full(N, P - 1, np.uint64)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    assert np.array_equal(f.compute_products(v), O.matvec(m_enc, m, N, v))


@pytest.mark.parametrize("B", [1, 8, 64])
def test_compute_products_batch_matches_per_query(ctx, B):
    c = capi()
    m = 333
    m_enc = uniform_fp((m, N), 57)
    vs = uniform_fp((B, N), 58 + B)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    got = f.compute_products_batch(vs)
    assert np.array_equal(got, O.matvec_batch(m_enc, m, N, vs))


@pytest.mark.parametrize("m", [1, 7, 257, 1500])
def test_decode_dense_terms(ctx, m):
    """gpu_dense_terms_matches_cpu_exact (lib.rs:1324-1420) at n1 = 128."""
    c = capi()
    al = uniform_fp((m, 128), 11 + m)
    h = uniform_fp((m, 128), 12 + m)
    g = uniform_fp(128, 13)
    x = uniform_fp(128, 14)
    f = c.Flat.build(ctx, uniform_fp((m, N), 15), al, h, m)
    want = [(int(a) + int(b)) % P for a, b in zip(O.matvec(al, m, 128, g), O.matvec(h, m, 128, x))]
    assert [int(v) for v in f.decode_dense_terms(g, x)] == want


@pytest.fixture(params=["tensor", "cuda_core"])
def engine(request, ctx):
    c = capi()
    ctx.set_engine(c.ENGINE_TENSOR if request.param == "tensor" else c.ENGINE_CUDA_CORE)
    yield request.param
    ctx.set_engine(c.ENGINE_TENSOR)


@pytest.mark.parametrize("m,trials", [(777, 1), (777, 3), (777, 20), (777, 29), (4097, 16), (10000, 17), (1, 5)])
def test_verify_honest_matches_oracle(ctx, engine, m, trials):
    """Protocol 2 on both engines: every trial's (u.r, (u^T M).v) pair is
    bit-equal to the oracle's; panel and row-block boundaries, multi-pass
    trial counts and both strip widths are covered."""
    c = capi()
    M, L, cl = cluster(m, 21 + m, uniform=True)
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    enc = O.encode_query(uniform_fp(N, 22), L, bytes([23]) * 32)
    r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
    seed = O.domain_separate(bytes([23]) * 32, b"protocol2")
    fo, uro, zvo = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, trials, seed)
    fg, urg, zvg = f.verify(r, enc.v_enc, seed, trials)
    assert fo == -1 and fg == -1
    assert np.array_equal(urg, uro) and np.array_equal(zvg, zvo)


def test_verify_extreme_residues_tensor(ctx):
    """All-(p-1) matrix: the largest byte limbs in every position."""
    c = capi()
    m = 4500
    m_enc = np.full((m, N), P - 1, np.uint64)
    v = np.full(N, P - 1, np.uint64)
    f = c.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    r = O.matvec(m_enc, m, N, v)
    seed = bytes([77]) * 32
    fo, uro, zvo = O.verify_response(r, m_enc, m, N, v, 20, seed)
    fg, urg, zvg = f.verify(r, v, seed, 20)
    assert fo == fg == -1 and np.array_equal(urg, uro) and np.array_equal(zvg, zvo)


@pytest.mark.parametrize("pos", [0, 400, 776])
def test_verify_detects_tampered_response(ctx, engine, pos):
    """crypto.rs:1445-1474: r[pos] += 1 is rejected at trial 0."""
    c = capi()
    M, L, cl = cluster(777, 31, uniform=True)
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, cl.m)
    enc = O.encode_query(uniform_fp(N, 33), L, bytes([34]) * 32)
    r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
    r[pos] = (int(r[pos]) + 1) % P
    seed = bytes([35]) * 32
    fo, uro, zvo = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, 20, seed)
    fg, urg, zvg = f.verify(r, enc.v_enc, seed, 20)
    assert fg == fo == 0
    assert np.array_equal(urg, uro) and np.array_equal(zvg, zvo)


def test_encrypt_matches_oracle(ctx):
    c = capi()
    M, L, cl = cluster(211, 41)
    me, al = c.encrypt_cluster(ctx, M.reshape(-1), 211, L, cl.h_mat, cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    assert np.array_equal(me, cl.m_enc) and np.array_equal(al, cl.a_l)


def _oracle_query(M, L, cl, v, qs, trials, k):
    f, ids, sc, r, _ = O.score_flat(cl, L, v, qs, trials, k, want_r=True)
    enc = O.encode_query(v, L, qs)
    mv = O.decode_scores(r, cl, L, enc)
    return f, ids, sc, r, mv, enc


@pytest.mark.parametrize("m,trials,k", [(2000, 3, 10), (1, 0, 10), (513, 20, 100), (300, 3, 1024), (9000, 20, 10)])
def test_query_matches_oracle(ctx, engine, m, trials, k):
    """Whole BnTmScorer::score path (lib.rs:326-475): r, decoded Mv, top-k
    ids and scores, and the Freivalds bit, for several queries at once."""
    M, L, cl = cluster(m, 100 + m)
    f = flat_from_cluster(ctx, M, L, cl)
    qs, encs, want = [], [], []
    for b in range(3):
        v, q_seed, _ = query(L, 500 + b)
        want.append(_oracle_query(M, L, cl, v, q_seed, trials, k))
        encs.append(want[-1][5])
        qs.append(O.domain_separate(q_seed, b"protocol2"))
    hits, failed, r, mv = f.query(np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                                  [(e.t_idx, e.t_sign) for e in encs], qs if trials else None, trials, k,
                                  want_r=True, want_mv=True)
    for b in range(3):
        fo, ids, sc, ro, mvo, _ = want[b]
        assert np.array_equal(r[b], ro)
        assert np.array_equal(mv[b], mvo)
        assert failed[b] == fo == -1
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc)
        assert len(hits[b][0]) == min(k, m)


@pytest.mark.parametrize("mode", ["int8", "uniform", "row_of_128", "row_of_minus_129"])
def test_query_plaintext_ranges_match_oracle(ctx, mode):
    """The decode sums M T from an int8 copy of the plaintext when every entry
    is int8-valued, and from the u64 residues otherwise (uniform residues, or
    one row just outside [-128, 127]); both are bit-exact."""
    m = 1500
    if mode == "uniform":
        M, L, cl = cluster(m, 61, uniform=True)
    else:
        M = int8_matrix(m, 768, 62)
        if mode != "int8":
            M[777, :768] = 128 if mode == "row_of_128" else P - 129
        L = O.generate_subspace(bytes([1]) * 32)
        cl = O.encrypt_cluster(M.reshape(-1), m, L, O.derive_h_seed(7, 0))
    f = flat_from_cluster(ctx, M, L, cl)
    v, q_seed, _ = query(L, 63)
    fo, ids, sc, ro, mvo, enc = _oracle_query(M, L, cl, v, q_seed, 2, 20)
    hits, failed, r, mv = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)],
                                  [O.domain_separate(q_seed, b"protocol2")], 2, 20, want_r=True, want_mv=True)
    assert np.array_equal(r[0], ro) and np.array_equal(mv[0], mvo)
    assert np.array_equal(hits[0][0], ids) and np.array_equal(hits[0][1], sc)
    assert failed[0] == fo == -1


def test_decode_int8_copy_is_kept_only_for_int8_plaintext(ctx):
    """Device bytes of the client state: the int8 copy of M (1024 bytes per
    row, rows rounded up to 32) exists only for int8-valued plaintext."""
    m = 1000
    M = int8_matrix(m, 768, 64)
    L = O.generate_subspace(bytes([1]) * 32)
    cl = O.encrypt_cluster(M.reshape(-1), m, L, O.derive_h_seed(7, 0))
    a = flat_from_cluster(ctx, M, L, cl).info()[1]
    M2 = M.copy()
    M2[3, 0] = 128
    cl2 = O.encrypt_cluster(M2.reshape(-1), m, L, O.derive_h_seed(7, 0))
    b = flat_from_cluster(ctx, M2, L, cl2).info()[1]
    assert a - b == (m + 31) // 32 * 32 * N


@pytest.mark.parametrize("n1", [64, 256, 512])
def test_query_matches_oracle_across_n1(ctx, n1):
    """The delta sweep of the reference's parameter sets (n1 = 1024 >> k,
    params.rs:102-120): scan, Protocol 2, decode and top-k at every n1 the
    ABI accepts (128 is covered above)."""
    c = capi()
    m = 1500
    M = int8_matrix(m, 768, 70 + n1)
    L = O.generate_subspace(bytes([3]) * 32, n1=n1)
    cl = O.encrypt_cluster(M.reshape(-1), m, L, O.derive_h_seed(7, 0), n1=n1)
    f = c.Flat.build(ctx, cl.m_enc, cl.a_l, cl.h_mat, m, n1=n1)
    f.attach_client(L, M.reshape(-1), cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    v = int8_matrix(1, 768, 71 + n1)[0]
    q_seed = O.derive_h_seed(72, n1)
    enc = O.encode_query(v, L, q_seed, n1=n1)
    fo, ids, sc, ro, _ = O.score_flat(cl, L, v, q_seed, 4, 25, want_r=True)
    mvo = O.decode_scores(ro, cl, L, enc)
    hits, failed, r, mv = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)],
                                  [O.domain_separate(q_seed, b"protocol2")], 4, 25, want_r=True, want_mv=True)
    assert np.array_equal(r[0], ro) and np.array_equal(mv[0], mvo)
    assert np.array_equal(hits[0][0], ids) and np.array_equal(hits[0][1], sc)
    assert failed[0] == fo == -1


def test_device_encrypted_handle_matches_host_encrypted(ctx):
    c = capi()
    M, L, cl = cluster(1234, 77)
    fh = flat_from_cluster(ctx, M, L, cl)
    fd = c.Flat.build_from_plain(ctx, M.reshape(-1), cl.m, L, cl.h_mat, cl.s_mat.rowptr, cl.s_mat.idx, cl.s_mat.sign)
    v, q_seed, enc = query(L, 78)
    seed = [O.domain_separate(q_seed, b"protocol2")]
    a = fh.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], seed, 20, 50, want_r=True)
    b = fd.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], seed, 20, 50, want_r=True)
    assert np.array_equal(a[2], b[2])
    assert np.array_equal(a[0][0][0], b[0][0][0]) and np.array_equal(a[0][0][1], b[0][0][1])
    assert a[1][0] == b[1][0] == -1


def test_k_zero_and_capping(ctx):
    M, L, cl = cluster(5, 9)
    f = flat_from_cluster(ctx, M, L, cl)
    v, q_seed, enc = query(L, 10)
    hits, failed, _, _ = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], None, 0, 0)
    assert len(hits[0][0]) == 0
    hits, failed, _, _ = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], None, 0, 100)
    assert len(hits[0][0]) == 5


def test_golden_fixture(ctx):
    """The device path reproduces the committed golden vectors."""
    import golden_io

    gold = golden_io.load()
    M, L, cl = golden_io.cluster(gold)
    f = flat_from_cluster(ctx, M, L, cl)
    enc = golden_io.encoded(gold)
    hits, failed, r, mv = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)],
                                  [bytes(gold["v_seed"])], int(gold["trials"]), int(gold["k"]), want_r=True,
                                  want_mv=True)
    assert np.array_equal(r[0], gold["r"]) and np.array_equal(mv[0], gold["mv"])
    assert np.array_equal(hits[0][0], gold["top_ids"]) and np.array_equal(hits[0][1], gold["top_scores"])
    fg, ur, zv = f.verify(gold["r"], enc.v_enc, bytes(gold["v_seed"]), int(gold["trials"]))
    assert fg == -1 and np.array_equal(ur, gold["ur"]) and np.array_equal(zv, gold["zv"])


def test_budget_refuses_oversized_payload():
    c = capi()
    small = c.Context(0, vram_budget_bytes=1 << 20)  # 1 MiB: a 1000-row corpus needs ~8 MiB
    m = 1000
    with pytest.raises(c.BnError) as e:
        c.Flat.build(small, np.zeros((m, N), np.uint64), np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    assert e.value.code == c.BN_EBUDGET
    assert small.memory()[1] == 0  # nothing leaked


def test_invalid_inputs_are_rejected(ctx):
    c = capi()
    m = 4
    bad = np.zeros((m, N), np.uint64)
    bad[1, 2] = P  # not canonical
    with pytest.raises(c.BnError) as e:
        c.Flat.build(ctx, bad, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    assert e.value.code == c.BN_EINVAL
    f = c.Flat.build(ctx, np.zeros((m, N), np.uint64), np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    with pytest.raises(c.BnError) as e:
        f.query(np.zeros((1, N), np.uint64), np.zeros((1, 128), np.uint64), [([], [])], None, 0, 5)
    assert e.value.code == c.BN_EUNSUPPORTED  # no client state attached


def test_plan_and_graph_capture_match_query(ctx):
    """bn_plan_enqueue over device buffers (and inside a CUDA graph) gives
    the same hits as bn_flat_query."""
    torch = pytest.importorskip("torch")
    M, L, cl = cluster(4096, 61)
    f = flat_from_cluster(ctx, M, L, cl)
    B, trials, k = 4, 3, 16
    encs, seeds = [], []
    for b in range(B):
        v, q_seed, enc = query(L, 900 + b)
        encs.append(enc)
        seeds.append(O.domain_separate(q_seed, b"protocol2"))
    want, wf, _, _ = f.query(np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                             [(e.t_idx, e.t_sign) for e in encs], seeds, trials, k)
    dev = torch.device("cuda:0")
    t = np.zeros((B, N), np.uint32)
    tn = np.zeros(B, np.uint32)
    for b, e in enumerate(encs):
        tn[b] = e.t_idx.size
        t[b, : e.t_idx.size] = e.t_idx | np.where(e.t_sign < 0, np.uint32(0x80000000), np.uint32(0))
    d_v = torch.from_numpy(np.stack([e.v_enc for e in encs]).view(np.int64)).to(dev)
    d_g = torch.from_numpy(np.stack([e.g for e in encs]).view(np.int64)).to(dev)
    d_t = torch.from_numpy(t.view(np.int32)).to(dev)
    d_tn = torch.from_numpy(tn.view(np.int32)).to(dev)
    d_s = torch.from_numpy(np.frombuffer(b"".join(seeds), np.uint8).copy()).to(dev)
    d_ids = torch.zeros((B, k), dtype=torch.int32, device=dev)
    d_sc = torch.zeros((B, k), dtype=torch.int64, device=dev)
    d_n = torch.zeros(B, dtype=torch.int32, device=dev)
    d_f = torch.zeros(B, dtype=torch.int32, device=dev)
    plan = f.plan(B, trials, k)
    stream = torch.cuda.Stream()
    args = [x.data_ptr() for x in (d_v, d_g, d_t, d_tn, d_s, d_ids, d_sc, d_n, d_f)]
    with torch.cuda.stream(stream):
        plan.enqueue(*args, stream.cuda_stream)
    stream.synchronize()

    def check():
        ids, sc, n, fl = (d_ids.cpu().numpy().view(np.uint32), d_sc.cpu().numpy(), d_n.cpu().numpy(), d_f.cpu().numpy())
        for b in range(B):
            assert n[b] == k and fl[b] == wf[b] == -1
            assert np.array_equal(ids[b], want[b][0]) and np.array_equal(sc[b], want[b][1])

    check()
    d_ids.zero_(); d_sc.zero_(); d_n.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        plan.enqueue(*args, stream.cuda_stream)
    g.replay()
    torch.cuda.synchronize()
    check()
