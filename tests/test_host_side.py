"""CPU parity of the product's host side (include/bn_host.h) with the oracle:
key generation, quantisation, encoding and routing consume the ChaCha
stream exactly as the reference does, so both must agree bit for bit."""
import numpy as np
import pytest

import oracle as O
from bnutil import N, int8_matrix


@pytest.fixture(scope="module")
def capi():
    from bn_b200 import capi as c

    return c


def test_seeds(capi):
    for s in (bytes(32), bytes(range(32)), bytes([7]) * 32):
        assert capi.host_domain_separate(s) == O.domain_separate(s, b"protocol2")
    for u, c in ((0, 0), (7, 3), (2**64 - 1, 4095)):
        assert capi.host_derive_h_seed(u, c) == O.derive_h_seed(u, c)
    assert capi.lib.bn_host_default_trials() == 3
    assert capi.lib.bn_host_mu() == O.mu()


@pytest.mark.parametrize("n1", [64, 128, 512])
def test_keygen_matches_oracle(capi, n1):
    assert np.array_equal(capi.host_generate_subspace(bytes([3]) * 32, n1), O.generate_subspace(bytes([3]) * 32, N, n1))
    H, rp, ix, sg = capi.host_regenerate_h_s(bytes([4]) * 32, 77, n1)
    Ho, So = O.regenerate_h_s(bytes([4]) * 32, 77, N, n1)
    assert np.array_equal(H, Ho) and np.array_equal(rp, So.rowptr)
    assert np.array_equal(ix, So.idx) and np.array_equal(sg, So.sign)


def test_keygen_lists_matches_per_list_oracle(capi):
    sizes = [5, 0, 40, 1, 17]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    H, rp, ix, sg = capi.host_regenerate_h_s_lists(9, off)
    for c, m in enumerate(sizes):
        Ho, So = O.regenerate_h_s(O.derive_h_seed(9, c), m)
        o = int(off[c])
        assert np.array_equal(H[o * 128 : (o + m) * 128], Ho[: m * 128])
        base = int(rp[o])
        assert np.array_equal(rp[o : o + m + 1] - np.uint64(base), So.rowptr)
        assert np.array_equal(ix[base : int(rp[o + m])], So.idx)


def test_quantise_and_encode_match_oracle(capi):
    rng = np.random.default_rng(1)
    v = rng.standard_normal((3, 768)).astype(np.float32)
    q = capi.host_quantise(v)
    for i in range(3):
        assert np.array_equal(q[i], O.quantise_vector(v[i]))
    assert np.array_equal(capi.host_quantise(np.array([[0.5, -0.5, 1.5, -2.5]], np.float32), q=1)[0],
                          O.quantise_vector(np.array([0.5, -0.5, 1.5, -2.5], np.float32), q=1))
    L = O.generate_subspace(bytes([1]) * 32)
    vq = int8_matrix(1, 768, 2)[0]
    ve, g, ti, ts = capi.host_encode_query(vq, L, bytes([5]) * 32)
    enc = O.encode_query(vq, L, bytes([5]) * 32)
    assert np.array_equal(ve, enc.v_enc) and np.array_equal(g, enc.g)
    assert np.array_equal(ti, enc.t_idx) and np.array_equal(ts, enc.t_sign)


def test_probe_route_matches_oracle(capi):
    rng = np.random.default_rng(4)
    cents = rng.standard_normal((64, 96)).astype(np.float32)
    qs = rng.standard_normal((10, 96)).astype(np.float32)
    got = capi.host_probe_route(cents, qs, 8)
    for i in range(10):
        assert np.array_equal(got[i], O.probe_route(cents, qs[i], 8))
