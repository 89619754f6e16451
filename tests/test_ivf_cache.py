"""Reader of the reference's on-disk BN-IVF cache (`.bntm-ivf-cache-*.bin`,
scorer-bntm/src/ivf.rs:440-560 writer, :1755-1901 loader) through the C ABI
(bn_host_ivf_cache_*), on files written in that layout by ivfcache_fmt.

CPU only: the header hash against a restatement of cache.rs fingerprint64,
round trips of every array, the per-list S regenerated from the stored
h_seed against the oracle's encryption, and the rejections the reference
also makes (magic, version, fingerprint, truncation, count mismatches)."""
from __future__ import annotations

import os
import struct

import numpy as np
import pytest

import ivfcache_fmt as F
import oracle as O
from bnutil import N, P, int8_matrix, uniform_fp

N1 = 128


def capi():
    from bn_b200 import capi as c

    return c


PARTS = [b"bntm-ivf2", struct.pack("<Q", 4), struct.pack("<Q", 42), struct.pack("<Q", 25),
         struct.pack("<Q", 13), struct.pack("<Q", 7), bytes([1]) * 32, struct.pack("<Q", N1), struct.pack("<Q", 1)]


def random_lists(sizes, dim, seed):
    rng = np.random.default_rng(seed)
    lists, next_id = [], 0
    for c, m in enumerate(sizes):
        lists.append({
            "ids": np.arange(next_id, next_id + m, dtype=np.uint32)[::-1].copy(),
            "vecs": rng.standard_normal((m, dim)).astype(np.float32),
            "h_seed": bytes(rng.integers(0, 256, 32, dtype=np.uint8)),
            "m_enc": uniform_fp((m, N), seed * 10 + c),
            "a_l": uniform_fp((m, N1), seed * 10 + c + 100),
            "m_plain": uniform_fp((m, N), seed * 10 + c + 200),
            "h": uniform_fp((m, N1), seed * 10 + c + 300),
        })
        next_id += m
    return lists


@pytest.fixture
def small_cache(tmp_path):
    sizes, dim = [3, 0, 5, 1], 6
    cen = np.random.default_rng(5).standard_normal((len(sizes), dim)).astype(np.float32)
    lists = random_lists(sizes, dim, 9)
    L = uniform_fp((N, N1), 77)
    path = tmp_path / "c.bin"
    F.write_cache(path, PARTS, cen, lists, L)
    return path, cen, lists, L


def test_fingerprint_matches_cache_rs_restatement():
    c = capi()
    assert c.cache_fingerprint([]) == 0xCBF29CE484222325 == F.fnv1a64([])
    for parts in ([b""], [b"a"], PARTS, [b"x" * 1000, b"", b"yz"]):
        assert c.cache_fingerprint(parts) == F.fnv1a64(parts)
    fp, name = c.bntm_ivf_cache_name(4, 42, 25, 13, 7, bytes([1]) * 32, N1, 1)
    assert fp == F.fnv1a64(PARTS) and name == f".bntm-ivf-cache-{fp:016x}.bin"


def test_fnv_core_matches_published_vectors():
    """The FNV-1a 64 core of the restatement, against the algorithm's published test vectors."""
    assert F.fnv1a64_raw(b"") == 0xCBF29CE484222325
    assert F.fnv1a64_raw(b"a") == 0xAF63DC4C8601EC8C
    assert F.fnv1a64_raw(b"foobar") == 0x85944171F73967E8


def test_fingerprint_properties_of_cache_rs_tests():
    """cache.rs:80-100: deterministic, scorer tags differ, part boundaries count."""
    c = capi()
    one = [b"plaintext-ivf", bytes([1, 0, 0, 0])]
    assert c.cache_fingerprint(one) == c.cache_fingerprint(list(one))
    assert c.cache_fingerprint(one) != c.cache_fingerprint([b"sap-ivf", bytes([1, 0, 0, 0])])
    assert c.cache_fingerprint([b"ab", b"c"]) != c.cache_fingerprint([b"a", b"bc"])


def test_round_trip(small_cache):
    c = capi()
    path, cen, lists, L = small_cache
    cache = c.IvfCache(path, F.fnv1a64(PARTS), N1)
    assert (cache.nlist, cache.dim, cache.rows) == (4, 6, 9)
    off, ids, cen2, hs = cache.lists()
    assert off.tolist() == [0, 3, 3, 8, 9]
    assert np.array_equal(ids, np.concatenate([x["ids"] for x in lists]))
    assert np.array_equal(cen2, cen)
    assert [bytes(h) for h in hs] == [x["h_seed"] for x in lists]
    a = cache.arrays()
    for key in ("m_enc", "a_l", "m_plain", "h"):
        assert np.array_equal(a[key], np.concatenate([x[key] for x in lists])), key
    assert np.array_equal(a["l_subspace"], L)
    assert c.IvfCache(path, 0, N1).rows == 9  # fingerprint 0 accepts any parameters


def test_empty_index(tmp_path):
    c = capi()
    path = tmp_path / "e.bin"
    F.write_cache(path, PARTS, np.zeros((0, 0), np.float32), [], uniform_fp((N, N1), 3))
    cache = c.IvfCache(path, 0, N1)
    assert (cache.nlist, cache.rows) == (0, 0)
    assert cache.lists()[0].tolist() == [0]


def test_s_regenerated_from_stored_h_seed_matches_encryption(tmp_path):
    """ivf.rs:1855-1862: S is not stored; the per-list S regenerated from the
    cached h_seed is the one the encryption used (oracle encrypt_cluster)."""
    c = capi()
    L = O.generate_subspace(bytes([1]) * 32)
    sizes, lists, want_s = [4, 0, 7], [], []
    for ci, m in enumerate(sizes):
        M = int8_matrix(m, 768, 40 + ci)
        hs = O.derive_h_seed(7, ci)
        cl = O.encrypt_cluster(M.reshape(-1), m, L, hs)
        lists.append({"ids": np.arange(m, dtype=np.uint32), "vecs": np.zeros((m, 2), np.float32), "h_seed": hs,
                      "m_enc": cl.m_enc, "a_l": cl.a_l, "m_plain": M, "h": cl.h_mat})
        want_s.append(cl.s_mat)
    path = tmp_path / "s.bin"
    F.write_cache(path, PARTS, np.zeros((3, 2), np.float32), lists, L)
    rp, ix, sg = c.IvfCache(path, 0, N1).s_lists()
    base = 0
    for ci, m in enumerate(sizes):
        s = want_s[ci]
        assert np.array_equal(rp[base : base + m + 1] - rp[base], np.asarray(s.rowptr, np.uint64))
        lo, hi = int(rp[base]), int(rp[base + m])
        assert np.array_equal(ix[lo:hi], np.asarray(s.idx, np.uint32))
        assert np.array_equal(sg[lo:hi], np.asarray(s.sign, np.int8))
        base += m


def expect_einval(path, fingerprint=0):
    c = capi()
    with pytest.raises(c.BnError) as e:
        c.IvfCache(path, fingerprint, N1)
    assert e.value.code == c.BN_EINVAL
    return str(e.value)


def patched(path, tmp_path, name, edit):
    data = bytearray(open(path, "rb").read())
    edit(data)
    out = tmp_path / name
    open(out, "wb").write(bytes(data))
    return out


def test_rejects_wrong_magic_version_fingerprint(small_cache, tmp_path):
    path = small_cache[0]
    assert "magic" in expect_einval(patched(path, tmp_path, "m.bin", lambda d: d.__setitem__(1, ord("X"))))
    assert "version" in expect_einval(patched(path, tmp_path, "v.bin", lambda d: d.__setitem__(8, 2)))
    assert "fingerprint" in expect_einval(path, F.fnv1a64(PARTS[:-1] + [struct.pack("<Q", 2)]))
    assert "cannot open" in expect_einval(tmp_path / "missing.bin")


def test_rejects_truncation_anywhere(small_cache, tmp_path):
    path = small_cache[0]
    size = os.path.getsize(path)
    # header, IVF payload, the padding and BN count, list arrays, l_subspace
    for cut in (10, 25, 60, 300, size - 8 * N * N1 - 8, size - 8 * N * N1 + 5, size - 1):
        p = patched(path, tmp_path, f"t{cut}.bin", lambda d, cut=cut: d.__delitem__(slice(cut, None)))
        expect_einval(p)


def test_rejects_inconsistent_counts(tmp_path):
    sizes, dim = [2, 3], 4
    lists = random_lists(sizes, dim, 3)
    cen = np.zeros((2, dim), np.float32)
    L = uniform_fp((N, N1), 4)
    path = tmp_path / "ok.bin"
    F.write_cache(path, PARTS, cen, lists, L)
    payload_end = 20 + 16 + 4 * dim * 2 + 8 + sum(8 + m * (4 + 4 * dim) for m in sizes)
    bn0 = payload_end + (8 - payload_end % 8) % 8
    # the BN part names three clusters
    msg = expect_einval(patched(path, tmp_path, "n.bin", lambda d: d.__setitem__(slice(bn0, bn0 + 8),
                                                                                   struct.pack("<Q", 3))))
    assert "cluster count" in msg
    # list 0 claims 1 row where the index has 2
    msg = expect_einval(patched(path, tmp_path, "r.bin", lambda d: d.__setitem__(slice(bn0 + 8, bn0 + 16),
                                                                                   struct.pack("<Q", 1))))
    assert "row count" in msg
