"""Key generation on the device (bn_keygen.cu) against the host keygen and
the oracle: H and S drawn from a cluster's h_seed must equal
regenerate_h_s (crypto.rs:258-270) bit for bit, and corpora built from
device-drawn keys must score exactly like corpora built from host-drawn
keys (and like the oracle)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import N, int8_matrix, query
from ivfutil import IvfCase

pytestmark = pytest.mark.gpu


def capi():
    from bn_b200 import capi as c

    return c


@pytest.mark.parametrize("m,n1", [(1, 128), (7, 64), (1000, 128), (4097, 256), (200_000, 128)])
def test_device_keys_equal_host_keys(ctx, m, n1):
    c = capi()
    seed = O.derive_h_seed(91 + m, 3)
    H, rp, ix, sg = c.keygen_h_s(ctx, seed, m, n1)
    Hh, rph, ixh, sgh = c.host_regenerate_h_s(seed, m, n1)
    assert np.array_equal(H, Hh)
    assert np.array_equal(rp, rph) and np.array_equal(ix, ixh) and np.array_equal(sg, sgh)
    if m <= 4097:  # the oracle's restatement too (the host keygen is pinned to it at every size in CPU tests)
        Ho, So = O.regenerate_h_s(seed, m, n1=n1)
        assert np.array_equal(H, Ho) and np.array_equal(rp, So.rowptr) and np.array_equal(ix, So.idx)


def test_flat_built_from_device_keys_scores_like_the_oracle(ctx):
    c = capi()
    m = 3000
    M = int8_matrix(m, 768, 9300)
    L = O.generate_subspace(bytes([5]) * 32)
    seed = O.derive_h_seed(9301, 0)
    f = c.Flat.build_keygen(ctx, M.reshape(-1), m, L, seed)
    cl = O.encrypt_cluster(M.reshape(-1), m, L, seed)
    for i in range(3):
        v, q_seed, enc = query(L, 9310 + i)
        vs = O.domain_separate(q_seed, b"protocol2")
        hits, failed, r, mv = f.query(enc.v_enc[None], enc.g[None], [(enc.t_idx, enc.t_sign)], [vs], 20, 10,
                                      want_r=True, want_mv=True)
        want_f, ids, sc, r_o, _ = O.score_flat(cl, L, v, q_seed, 20, 10, want_r=True)
        assert np.array_equal(r[0], r_o) and failed[0] == want_f == -1
        assert np.array_equal(mv[0], O.decode_scores(r_o, cl, L, enc))
        assert np.array_equal(hits[0][0], ids) and np.array_equal(hits[0][1], sc)
    f.close()


def test_ivf_built_from_device_keys_equals_host_keys(ctx):
    c = capi()
    case = IvfCase([50, 0, 3, 200, 1, 0, 97, 400, 33], upload_seed=7)
    m_enc, a_l, h, rp, ix, sg = case.concat()
    host = c.Ivf.build(ctx, case.offsets, case.ids, m_enc, a_l, h)
    host.attach_client(case.L, case.M.reshape(-1), rp, ix, sg)
    dev = c.Ivf.build_keygen(ctx, case.offsets, case.ids, case.M.reshape(-1), case.L, 7)
    rng = np.random.default_rng(3)
    B, nprobe = 4, 4
    probes = np.stack([rng.choice(case.nlist, nprobe, replace=False) for _ in range(B)]).astype(np.uint32)
    encs = [O.encode_query(case.M[10 + b], case.L, bytes([60 + b]) * 32) for b in range(B)]
    seeds = [O.domain_separate(bytes([60 + b]) * 32, b"protocol2") for b in range(B)]
    args = (probes, np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
            [(e.t_idx, e.t_sign) for e in encs], seeds, 20, 10)
    a, fa, ta = host.query(*args)
    b, fb, tb = dev.query(*args)
    for q in range(B):
        assert np.array_equal(a[q][0], b[q][0]) and np.array_equal(a[q][1], b[q][1])
        want = case.oracle_score(probes[q], encs[q], seeds[q], 20, 10)
        assert np.array_equal(b[q][0], want[0]) and np.array_equal(b[q][1], want[1])
    assert np.all(fa == -1) and np.all(fb == -1)
    for ci in range(case.nlist):  # the device-encrypted lists equal the oracle's encryption
        if case.sizes[ci]:
            v = np.arange(N, dtype=np.uint64) * np.uint64(7919)
            assert np.array_equal(dev.compute_products(ci, v), O.matvec(case.clusters[ci].m_enc, case.sizes[ci], N, v))
    host.close()
    dev.close()
