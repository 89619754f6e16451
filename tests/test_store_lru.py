"""The streaming store's LRU bookkeeping (bn_lru, csrc/bn_stream.cu) with no
GPU: the behaviours the reference's CUDA-free store tests check on LruInner
(scorer-gpu-common/src/store.rs:437-540), through the C ABI."""
from __future__ import annotations

import pytest


def capi():
    from bn_b200 import capi as c

    return c


def insert_one(lru, cid, nbytes):
    evicted = lru.pre_evict(nbytes)
    assert lru.insert(cid, nbytes)
    return evicted


def test_budget_too_small_surfaces_when_first_payload_overflows():
    c = capi()
    lru = c.Lru(100)
    with pytest.raises(c.BnError) as e:
        lru.pre_evict(200)
    assert e.value.code == c.BN_EBUDGET
    assert "200" in str(e.value) and "100" in str(e.value)
    assert lru.stats()["resident_bytes"] == 0


def test_lru_evicts_oldest_then_inserts_new():
    lru = capi().Lru(250)
    dropped = []
    for cid in range(3):
        dropped += insert_one(lru, cid, 100)
    assert dropped == [0]  # cluster 0 evicts first when 2's insert hits the budget
    st = lru.stats()
    assert st["resident_bytes"] == 200 and st["evictions"] == 1 and st["uploads"] == 3


def test_touch_returns_existing_payload_and_bumps_recency():
    lru = capi().Lru(1000)
    insert_one(lru, 7, 100)
    assert lru.touch(7)
    assert not lru.touch(8)
    assert lru.stats()["gets"] == 2


def test_recency_bump_protects_recently_used_cluster():
    lru = capi().Lru(250)
    insert_one(lru, 0, 100)
    insert_one(lru, 1, 100)
    assert lru.touch(0)  # 0 is the most recently used now
    assert insert_one(lru, 2, 100) == [1]


def test_insert_returns_existing_on_race():
    lru = capi().Lru(500)
    insert_one(lru, 3, 100)
    before = lru.stats()["resident_bytes"]
    assert not lru.insert(3, 100)  # already resident: the existing entry stays, nothing is counted
    assert lru.stats()["resident_bytes"] == before


def test_pre_evict_only_evicts_enough_for_request():
    lru = capi().Lru(250)
    insert_one(lru, 0, 100)
    insert_one(lru, 1, 100)
    assert lru.pre_evict(100) == [0]
    assert lru.stats()["resident_bytes"] == 100
    assert lru.touch(1) and not lru.touch(0)


def test_cyclic_scan_keeps_the_last_entries():
    """A corpus larger than the budget scanned in full, in LRU order (the
    visiting order of bn_stream_query): each pass misses exactly the chunks
    that do not fit."""
    lru = capi().Lru(3 * 10)
    chunks, slots = 8, 3
    order = list(range(chunks))
    misses_per_pass = []
    resident = []
    for _ in range(4):
        misses = 0
        visit = resident + [c for c in order if c not in resident]
        for cid in visit:
            if not lru.touch(cid):
                misses += 1
                for e in lru.pre_evict(10):
                    resident.remove(e)
                assert lru.insert(cid, 10)
                resident.append(cid)
            else:
                resident.remove(cid)
                resident.append(cid)
        misses_per_pass.append(misses)
    assert misses_per_pass == [chunks] + [chunks - slots] * 3
