"""CPU tests of the oracle: pins it against published vectors and exact
big-integer arithmetic, and restates the reference's own unit tests
(scorer-bntm/src/crypto.rs:1061-1560, params.rs:208-285)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, bigint_matvec, cluster, query, signed, uniform_fp


# ---------------------------------------------------------------- ChaCha20 pins
def test_chacha20_rfc8439_block_vector():
    # RFC 8439 section 2.3.2: key 00..1f, nonce 00000009 0000004a 00000000, counter 1.
    key = np.frombuffer(bytes(range(32)), dtype=np.uint32)
    out = O.chacha20_block(key, 1 | (0x09000000 << 32), 0x4A000000)
    want = [0xE4E7F110, 0x15593BD1, 0x1FDD0F50, 0xC47120A3, 0xC7F4D1C7, 0x0368C033, 0x9AAA2204, 0x4E6CD4C3,
            0x466482D2, 0x09AA9F07, 0x05D7C214, 0xA2028BD9, 0xD19C12B5, 0xB94E16DE, 0xE883D0CB, 0x4E3C50A2]
    assert [int(x) for x in out] == want


def test_chacha20_rfc8439_keystream_zero_key():
    # RFC 8439 appendix A.1 test vectors #1 and #2 (all-zero key and nonce,
    # block counters 0 and 1) = ChaCha20Rng::from_seed([0; 32]) output.
    ks = O.rng_u32s(bytes(32), 32).astype("<u4").tobytes()
    want0 = bytes.fromhex("76b8e0ada0f13d90405d6ae55386bd28bdd219b8a08ded1aa836efcc8b770dc7"
                          "da41597c5157488d7724e03fb8d84a376a43b8f41518a11cc387b669b2ee6586")
    want1 = bytes.fromhex("9f07e7be5551387a98ba977c732d080dcb0f29a048e3656912c6533e32ee7aed"
                          "29b721769ce64e43d57133b074d839d531ed1f28510afb45ace10a1f4b794d6f")
    assert ks[:64] == want0
    assert ks[64:] == want1


def test_next_u64_is_two_words_low_first():
    w = O.rng_u32s(bytes([3]) * 32, 10).astype(np.uint64)
    q = O.rng_u64s(bytes([3]) * 32, 5)
    assert list(q) == [int(w[2 * i]) | (int(w[2 * i + 1]) << 32) for i in range(5)]


def test_seed_from_u64_pcg32_filler():
    # rand_core's PCG32-based seed_from_u64, restated independently here.
    def pcg(state):
        out = b""
        for _ in range(8):
            state = (state * 6364136223846793005 + 11634580027462260723) % 2**64
            xs = (((state >> 18) ^ state) >> 27) & 0xFFFFFFFF
            rot = state >> 59
            x = ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF
            out += x.to_bytes(4, "little")
        return out
    for s in (0, 1, 0xC0DEBEEF, 2**64 - 1):
        assert O.seed_from_u64(s) == pcg(s)


# ---------------------------------------------------------------- params (params.rs:208-285)
def test_params_relations():
    assert abs(O.mu() - 0.125) < 1e-9
    assert O.lib.bno_verification_trials() == 3
    assert [O.lib.bno_n1(k) for k in (1, 2, 3, 4)] == [512, 256, 128, 64]
    assert O.lib.bno_n1(5) == 0  # outside the reviewed range (the reference panics)
    # mu = 1024^(0.7-1) is a hair below 1/8 in f64, so the threshold is 2^29 - 1.
    assert O.lib.bno_sparse_threshold(O.mu()) == 536870911


# ---------------------------------------------------------------- field (crypto.rs:1078-1101)
def test_mersenne_reduce_canonical():
    assert O.mersenne_reduce(0) == 0
    assert O.mersenne_reduce(P) == 0
    assert O.mersenne_reduce(2 * P) == 0
    assert O.mersenne_reduce(P - 1) == P - 1
    a, b = P - 7, P - 3
    assert O.mersenne_reduce(a * b) == (a * b) % P
    rng = np.random.default_rng(5)
    for _ in range(200):
        x = int(rng.integers(0, 2**63)) << 64 | int(rng.integers(0, 2**63)) << 1
        assert O.mersenne_reduce(x) == x % P


def test_field_ops_match_naive():
    for a, b in [(0, 0), (1, 1), (P - 1, P - 1), (12345, 67890), (P - 1, 0), (0, P - 1)]:
        assert O.lib.bno_add_mod(a, b) == (a + b) % P
        assert O.lib.bno_sub_mod(a, b) == (a - b) % P
        assert O.lib.bno_mul_mod(a, b) == (a * b) % P


def test_fp_to_signed():
    assert O.fp_to_signed(5) == 5
    assert O.fp_to_signed(P - 5) == -5
    assert O.fp_to_signed(P // 2 - 1) == P // 2 - 1
    assert O.fp_to_signed(P // 2) == P // 2 - P


# ---------------------------------------------------------------- matvec (crypto.rs:1150-1226)
@pytest.mark.parametrize("rows,cols", [(100, 512), (100, 1024)])
def test_matvec_matches_bigint(rows, cols):
    mat = uniform_fp((rows, cols), 0xC0DEBEEF)
    vec = uniform_fp(cols, 0xC0DEBEEF + 1)
    want = bigint_matvec(mat, vec)
    assert [int(x) for x in O.matvec(mat, rows, cols, vec)] == want
    assert [int(x) for x in O.matvec(mat, rows, cols, vec, avx512=True)] == want


@pytest.mark.parametrize("rows,cols", [(100, 512), (100, 1024)])
def test_matvec_transpose_matches_bigint(rows, cols):
    mat = uniform_fp((rows, cols), 0xA5)
    vec = uniform_fp(rows, 0xA6)
    want = bigint_matvec(mat.T, vec)
    assert [int(x) for x in O.matvec_transpose(mat, rows, cols, vec)] == want


@pytest.mark.parametrize("B", [1, 8, 64])
def test_compute_products_batch_matches_per_query(B):
    m = 16
    mat = uniform_fp((m, N), 57)
    vecs = uniform_fp((B, N), 58 + B)
    got = O.matvec_batch(mat, m, N, vecs)
    for b in range(B):
        assert np.array_equal(got[b], O.matvec(mat, m, N, vecs[b]))


def test_extreme_residues():
    mat = np.full((4, N), P - 1, np.uint64)
    vec = np.full(N, P - 1, np.uint64)
    assert [int(x) for x in O.matvec(mat, 4, N, vec)] == bigint_matvec(mat, vec)


# ---------------------------------------------------------------- protocol (crypto.rs:1231-1376)
def test_protocol_roundtrip_recovers_mv_exactly():
    M, L, cl = cluster(16, 7, uniform=True)
    v = uniform_fp(N, 8)
    enc = O.encode_query(v, L, bytes([9]) * 32)
    r = O.matvec(cl.m_enc, 16, N, enc.v_enc)
    assert [int(x) for x in O.decode_scores(r, cl, L, enc)] == bigint_matvec(M, v)


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_delta_sweep_recall_exact(k):
    n1 = 1024 >> k
    M = uniform_fp((16, N), 60 + k)
    L = O.generate_subspace(bytes([70 + k]) * 32, N, n1)
    cl = O.encrypt_cluster(M.reshape(-1), 16, L, bytes([80 + k]) * 32, n1=n1)
    v = uniform_fp(N, 90 + k)
    enc = O.encode_query(v, L, bytes([90 + k]) * 32, n1=n1)
    r = O.matvec(cl.m_enc, 16, N, enc.v_enc)
    assert [int(x) for x in O.decode_scores(r, cl, L, enc)] == bigint_matvec(M, v)


def test_two_independent_queries():
    M, L, cl = cluster(16, 11, uniform=True)
    for qs in (bytes([13]) * 32, bytes([17]) * 32):
        v = uniform_fp(N, qs[0])
        enc = O.encode_query(v, L, qs)
        r = O.matvec(cl.m_enc, 16, N, enc.v_enc)
        assert [int(x) for x in O.decode_scores(r, cl, L, enc)] == bigint_matvec(M, v)


def test_h_s_regeneration_deterministic_and_cached():
    H1, S1 = O.regenerate_h_s(bytes([42]) * 32, 8)
    H2, S2 = O.regenerate_h_s(bytes([42]) * 32, 8)
    assert np.array_equal(H1, H2) and np.array_equal(S1.idx, S2.idx) and np.array_equal(S1.sign, S2.sign)
    M, L, cl = cluster(16, 51, uniform=True)
    He, Se = O.regenerate_h_s(O.derive_h_seed(7, 0), 16)
    assert np.array_equal(cl.h_mat, He) and np.array_equal(cl.s_mat.idx, Se.idx)


def test_s_density_matches_mu():
    _, S = O.regenerate_h_s(bytes([99]) * 32, 64)
    mean = S.idx.size / 64
    assert abs(mean - 128) < 64
    assert set(np.unique(S.sign)) <= {-1, 1}
    for i in range(64):  # sorted column indices per row
        row = S.idx[int(S.rowptr[i]) : int(S.rowptr[i + 1])]
        assert np.all(np.diff(row.astype(np.int64)) > 0)


def test_encrypt_cluster_definition():
    """M_enc = M + H L^T + S and AL = M L, re-derived with Python integers."""
    M, L, cl = cluster(3, 21, uniform=True)
    Lm = L.reshape(N, 128)
    H = cl.h_mat.reshape(3, 128)
    for i in range(3):
        s = {int(cl.s_mat.idx[c]): int(cl.s_mat.sign[c]) for c in range(int(cl.s_mat.rowptr[i]), int(cl.s_mat.rowptr[i + 1]))}
        for j in range(0, N, 97):
            hl = sum(int(H[i, k]) * int(Lm[j, k]) for k in range(128))
            assert int(cl.m_enc[i * N + j]) == (int(M[i, j]) + hl + s.get(j, 0)) % P
        for k in range(0, 128, 31):
            assert int(cl.a_l[i * 128 + k]) == sum(int(M[i, j]) * int(Lm[j, k]) for j in range(N)) % P


# ---------------------------------------------------------------- Protocol 2 (crypto.rs:1414-1474)
def test_verification_passes_on_honest_server():
    M, L, cl = cluster(16, 21, uniform=True)
    for b in range(16):
        enc = O.encode_query(uniform_fp(N, 100 + b), L, bytes([b]) * 32)
        r = O.matvec(cl.m_enc, 16, N, enc.v_enc)
        f, ur, zv = O.verify_response(r, cl.m_enc, 16, N, enc.v_enc, 3, bytes([b ^ 0xAA]) * 32)
        assert f == -1 and np.array_equal(ur, zv)


def test_verification_values_match_bigint():
    M, L, cl = cluster(12, 31, uniform=True)
    enc = O.encode_query(uniform_fp(N, 32), L, bytes([34]) * 32)
    r = O.matvec(cl.m_enc, 12, N, enc.v_enc)
    seed = bytes([35]) * 32
    f, ur, zv = O.verify_response(r, cl.m_enc, 12, N, enc.v_enc, 4, seed)
    draws = O.rng_u64s(seed, 4 * 12) & np.uint64(P)
    Me = cl.m_enc.reshape(12, N)
    for t in range(4):
        u = [int(x) for x in draws[t * 12 : (t + 1) * 12]]
        assert int(ur[t]) == sum(a * int(b) for a, b in zip(u, r)) % P
        z = [sum(u[i] * int(Me[i, j]) for i in range(12)) % P for j in range(N)]
        assert int(zv[t]) == sum(a * int(b) for a, b in zip(z, enc.v_enc)) % P


@pytest.mark.parametrize("pos", [0, 8, 15])
def test_verification_detects_tampered_response(pos):
    M, L, cl = cluster(16, 31, uniform=True)
    enc = O.encode_query(uniform_fp(N, 33), L, bytes([34]) * 32)
    r = O.matvec(cl.m_enc, 16, N, enc.v_enc)
    r[pos] = (int(r[pos]) + 1) % P
    f, ur, zv = O.verify_response(r, cl.m_enc, 16, N, enc.v_enc, 3, bytes([35]) * 32)
    assert f == 0 and ur[0] != zv[0]


# ---------------------------------------------------------------- rank + whole query (lib.rs)
def test_topk_canonical_order_and_cap():
    s = np.array([5, 9, 9, -3, 7, 9], np.int64)
    ids, sc = O.topk(s, 4)
    assert list(ids) == [1, 2, 5, 4] and list(sc) == [9, 9, 9, 7]
    ids, sc = O.topk(s, 100)  # k capped at the candidate count (lib.rs:1028-1041)
    assert len(ids) == 6


def test_score_flat_int8_scores_are_exact_dot_products():
    M, L, cl = cluster(300, 3)
    v, qs, _ = query(L, 4)
    f, ids, sc, _, _ = O.score_flat(cl, L, v, qs, trials=3, k=10)
    assert f == -1
    exact = signed(M) @ signed(v)
    order = sorted(range(300), key=lambda i: (-exact[i], i))[:10]
    assert list(ids) == order and list(sc) == [int(exact[i]) for i in order]


def test_quantise_vector_semantics():
    v = np.array([0.5, -0.5, 1.5, -2.5, 0.0, 3.2], np.float32)
    q = O.quantise_vector(v, q=1)
    # f64::round rounds half away from zero; negatives wrap to p - k.
    assert [int(x) for x in q[:6]] == [1, P - 1, 2, P - 3, 0, 3]
    assert np.all(q[6:] == 0)
    q2 = O.quantise_vector(np.array([1.0, -1.0], np.float32))
    assert int(q2[0]) == 1 << 20 and int(q2[1]) == P - (1 << 20)


# ---------------------------------------------------------------- IVF routing (ivf-index)
def test_probe_route_and_kmeans_small():
    rng = np.random.default_rng(3)
    data = rng.standard_normal((400, 16)).astype(np.float32)
    cents = O.kmeans_train(data, 8, seed=42, max_iter=25)
    assert cents.shape == (8, 16) and np.isfinite(cents).all()
    asg = O.assign(data, cents)
    assert set(np.unique(asg)) <= set(range(8))
    q = data[5]
    pr = O.probe_route(cents, q, 3)
    d = [float(np.sqrt(((q - c) ** 2).sum())) for c in cents]
    assert list(pr) == sorted(range(8), key=lambda i: (d[i], i))[:3]
    assert list(O.probe_route(cents, q, 100)) == sorted(range(8), key=lambda i: (d[i], i))
