"""GPU parity of the IVF path (device CSR of inverted lists) against the
oracle; restates scorer-bntm/src/ivf.rs:1904-2423 on the device path."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, P, int8_matrix
from ivfutil import IvfCase

pytestmark = pytest.mark.gpu

SIZES = [50, 0, 3, 200, 1, 0, 97, 400, 33]


def capi():
    from bn_b200 import capi as c

    return c


@pytest.fixture(scope="module")
def case():
    return IvfCase(SIZES)


@pytest.fixture(scope="module")
def ivf(ctx, case):
    c = capi()
    m_enc, a_l, h, rp, ix, sg = case.concat()
    v = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    v.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    return v


def test_compute_products_per_list(case, ivf):
    v = int8_matrix(1, 768, 3)[0]
    enc = O.encode_query(v, case.L, bytes([4]) * 32)
    for ci in range(case.nlist):
        got = ivf.compute_products(ci, enc.v_enc)
        if case.sizes[ci] == 0:
            assert got is None  # Ok(None) for an empty list
        else:
            cl = case.clusters[ci]
            assert np.array_equal(got, O.matvec(cl.m_enc, cl.m, N, enc.v_enc))
    assert ivf.compute_products(case.nlist + 3, enc.v_enc) is None  # out of range


def test_decode_dense_terms_per_list(case, ivf):
    g = (np.arange(128, dtype=np.uint64) * np.uint64(977)) % np.uint64(P)
    x = (np.arange(128, dtype=np.uint64) * np.uint64(31337) + np.uint64(5)) % np.uint64(P)
    for ci in (0, 3, 8):
        cl = case.clusters[ci]
        want = [(int(a) + int(b)) % P for a, b in zip(O.matvec(cl.a_l, cl.m, 128, g), O.matvec(cl.h_mat, cl.m, 128, x))]
        assert [int(t) for t in ivf.decode_dense_terms(ci, g, x)] == want


@pytest.fixture(params=["tensor", "cuda_core"])
def engine(request, ctx):
    c = capi()
    ctx.set_engine(c.ENGINE_TENSOR if request.param == "tensor" else c.ENGINE_CUDA_CORE)
    yield request.param
    ctx.set_engine(c.ENGINE_TENSOR)


@pytest.mark.parametrize("trials", [0, 3, 20])
def test_query_matches_oracle(case, ivf, engine, trials):
    rng = np.random.default_rng(trials)
    B, nprobe, k = 5, 4, 25
    probes = np.stack([rng.permutation(case.nlist)[:nprobe] for _ in range(B)]).astype(np.uint32)
    probes[0] = [1, 5, 4, 2]  # mostly empty lists
    encs, seeds, want = [], [], []
    for b in range(B):
        q_seed = O.derive_h_seed(99, b)
        enc = O.encode_query(int8_matrix(1, 768, 40 + b)[0], case.L, q_seed)
        vs = O.domain_separate(q_seed, b"protocol2")
        encs.append(enc)
        seeds.append(vs)
        want.append(case.oracle_score(list(probes[b]), enc, vs, trials, k))
    hits, fc, ft = ivf.query(probes, np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                             [(e.t_idx, e.t_sign) for e in encs], seeds if trials else None, trials, k)
    for b in range(B):
        assert fc[b] == -1 and ft[b] == -1
        assert np.array_equal(hits[b][0], want[b][0]) and np.array_equal(hits[b][1], want[b][1])


def test_all_lists_probed_single_list_equals_flat(ctx):
    """ivf.rs:2045-2078: one list probed in full == the flat scorer."""
    c = capi()
    one = IvfCase([321], seed=8)
    m_enc, a_l, h, rp, ix, sg = one.concat()
    v = c.Ivf.build(ctx, one.offsets, np.arange(321, dtype=np.uint32), m_enc, a_l, h)
    v.attach_client(one.L, one.M.reshape(-1), rp, ix, sg)
    f = c.Flat.build(ctx, m_enc, a_l, h, 321)
    f.attach_client(one.L, one.M.reshape(-1), rp, ix, sg)
    q_seed = bytes([5]) * 32
    enc = O.encode_query(int8_matrix(1, 768, 6)[0], one.L, q_seed)
    vs = [O.domain_separate(q_seed, b"protocol2")]
    hi, fc, ft = v.query(np.zeros((1, 1), np.uint32), enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], vs, 3, 10)
    hf, ff, _, _ = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], vs, 3, 10)
    assert np.array_equal(hi[0][0], hf[0][0]) and np.array_equal(hi[0][1], hf[0][1])


def test_verify_tampered_list(case, ivf, engine):
    ci = 7
    cl = case.clusters[ci]
    enc = O.encode_query(int8_matrix(1, 768, 12)[0], case.L, bytes([13]) * 32)
    r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
    seed = bytes([14]) * 32
    f0, ur0, zv0 = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, 3, seed)
    fg, urg, zvg = ivf.verify(ci, r, enc.v_enc, seed, 3)
    assert f0 == fg == -1 and np.array_equal(ur0, urg) and np.array_equal(zv0, zvg)
    r[123] = (int(r[123]) + 1) % P
    assert ivf.verify(ci, r, enc.v_enc, seed, 3)[0] == 0


def test_device_encrypted_ivf_matches(ctx, case, ivf):
    c = capi()
    m_enc, a_l, h, rp, ix, sg = case.concat()
    d = c.Ivf.build_from_plain(ctx, case.offsets, case.ids, case.M.reshape(-1), case.L, h, rp, ix, sg)
    enc = O.encode_query(int8_matrix(1, 768, 77)[0], case.L, bytes([78]) * 32)
    pr = np.array([[3, 7, 0, 8, 6]], np.uint32)
    a = ivf.query(pr, enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [bytes(32)], 3, 40)
    b = d.query(pr, enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [bytes(32)], 3, 40)
    assert np.array_equal(a[0][0][0], b[0][0][0]) and np.array_equal(a[0][0][1], b[0][0][1])
