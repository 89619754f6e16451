"""IVF routing on the device (bn_ivf_route) against the host restatement of
probe_route (ivf-index/src/ivf.rs:150-164 with the scalar l2_f32 of
distance.rs:30-36), bit for bit, and against the oracle's probe_route."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from bnutil import uniform_fp

pytestmark = pytest.mark.gpu


def empty_ivf(ctx, nlist, rows_per_list=1):
    from bn_b200 import capi as c

    off = np.arange(nlist + 1, dtype=np.uint64) * rows_per_list
    rows = nlist * rows_per_list
    return c.Ivf.build(ctx, off, np.arange(rows, dtype=np.uint32), uniform_fp((rows, 1024), 1),
                       uniform_fp((rows, 128), 2), uniform_fp((rows, 128), 3))


@pytest.mark.parametrize("nlist,d,B,nprobe", [(300, 768, 37, 8), (4096, 768, 16, 128), (5, 16, 3, 9), (1, 4, 2, 1)])
def test_route_matches_host_probe_route(ctx, nlist, d, B, nprobe):
    from bn_b200 import capi as c

    rng = np.random.default_rng(nlist + d)
    cen = rng.standard_normal((nlist, d)).astype(np.float32)
    cen /= np.linalg.norm(cen, axis=1, keepdims=True)
    q = (cen[rng.integers(0, nlist, B)] + 0.3 * rng.standard_normal((B, d)).astype(np.float32) / np.sqrt(d))
    q = q.astype(np.float32)
    v = empty_ivf(ctx, nlist)
    v.set_centroids(cen)
    got = v.route(q, nprobe)
    want = c.host_probe_route(cen, q, nprobe)
    assert got.shape == (B, min(nprobe, nlist))
    assert np.array_equal(got, want)


def test_route_ties_go_to_the_lower_list(ctx):
    """Duplicate centroids give equal distances; the lower list index ranks first."""
    from bn_b200 import capi as c

    rng = np.random.default_rng(4)
    base = rng.standard_normal((6, 32)).astype(np.float32)
    cen = np.concatenate([base, base[::-1]])  # list 6 + i duplicates list 5 - i
    q = rng.standard_normal((5, 32)).astype(np.float32)
    v = empty_ivf(ctx, 12)
    v.set_centroids(cen)
    got = v.route(q, 12)
    assert np.array_equal(got, c.host_probe_route(cen, q, 12))
    for row in got:
        pos = {int(x): i for i, x in enumerate(row)}
        for i in range(6):
            assert pos[i] < pos[11 - i]


def test_route_matches_oracle(ctx):
    rng = np.random.default_rng(6)
    cen = rng.standard_normal((64, 24)).astype(np.float32)
    q = rng.standard_normal((7, 24)).astype(np.float32)
    v = empty_ivf(ctx, 64)
    v.set_centroids(cen)
    got = v.route(q, 10)
    for b in range(7):
        assert list(got[b]) == list(O.probe_route(cen, q[b], 10))


def test_route_rejects_bad_input(ctx):
    from bn_b200 import capi as c

    v = empty_ivf(ctx, 4)
    with pytest.raises(c.BnError) as e:
        v.route(np.zeros((1, 8), np.float32), 2)  # no centroids yet
    assert e.value.code == c.BN_EINVAL
    v.set_centroids(np.zeros((4, 8), np.float32))
    with pytest.raises(c.BnError) as e:
        v.route(np.zeros((1, 8), np.float32), 0)
    assert e.value.code == c.BN_EINVAL
