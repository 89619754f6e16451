"""A device IVF handle loaded from a reference-layout cache file
(ivf_from_cache: bn_host_ivf_cache_* -> bn_ivf_build -> bn_ivf_attach_client
with S regenerated from the stored h_seeds) scores exactly like the oracle's
BnTmIvfScorer::score (ivf.rs:778-823) on the same lists."""
from __future__ import annotations

import numpy as np
import pytest

import ivfcache_fmt as F
import oracle as O
from bnutil import int8_matrix
from ivfutil import IvfCase

pytestmark = pytest.mark.gpu

SIZES = [40, 0, 3, 200, 1, 97]


def test_ivf_from_cache_matches_oracle(ctx, tmp_path):
    from bn_b200 import capi as c

    case = IvfCase(SIZES, seed=17, upload_seed=7)
    dim = 8
    cen = np.random.default_rng(3).standard_normal((len(SIZES), dim)).astype(np.float32)
    lists = []
    for ci, m in enumerate(SIZES):
        o = int(case.offsets[ci])
        cl = case.clusters[ci]
        zero = np.zeros((0,), np.uint64)
        lists.append({"ids": case.ids[o : o + m], "vecs": np.zeros((m, dim), np.float32),
                      "h_seed": O.derive_h_seed(7, ci),
                      "m_enc": cl.m_enc if m else zero, "a_l": cl.a_l if m else zero,
                      "m_plain": case.M[o : o + m] if m else zero, "h": cl.h_mat if m else zero})
    path = tmp_path / "ivf.bin"
    F.write_cache(path, [b"bntm-ivf2"], cen, lists, case.L)
    ivf, cen2 = c.ivf_from_cache(ctx, str(path), F.fnv1a64([b"bntm-ivf2"]))
    assert np.array_equal(cen2, cen)
    B, nprobe, trials, k = 4, 3, 5, 10
    rng = np.random.default_rng(8)
    probes = np.stack([rng.choice(len(SIZES), nprobe, replace=False) for _ in range(B)]).astype(np.uint32)
    encs = [O.encode_query(int8_matrix(1, 768, 90 + b)[0], case.L, O.derive_h_seed(91, b)) for b in range(B)]
    seeds = [O.domain_separate(O.derive_h_seed(92, b), b"protocol2") for b in range(B)]
    hits, fc, ft = ivf.query(probes, np.stack([e.v_enc for e in encs]), np.stack([e.g for e in encs]),
                             [(e.t_idx, e.t_sign) for e in encs], seeds, trials, k)
    for b in range(B):
        ids, sc = case.oracle_score(list(probes[b]), encs[b], seeds[b], trials, k)
        assert np.array_equal(hits[b][0], ids) and np.array_equal(hits[b][1], sc), b
        assert fc[b] == -1 and ft[b] == -1
