"""CPU: the oracle reproduces the committed golden fixture bit for bit."""
import numpy as np

import golden_io
import oracle as O


def test_oracle_reproduces_golden_fixture():
    gold = golden_io.load()
    M, L, cl = golden_io.cluster(gold)  # asserts the keygen hashes
    v = np.zeros(golden_io.N, np.int64)
    v[: int(gold["d"])] = gold["v"].astype(np.int64)
    vu = (v % golden_io.P).astype(np.uint64)
    enc = O.encode_query(vu, L, gold["q_seed"].tobytes())
    assert np.array_equal(enc.v_enc, gold["v_enc"]) and np.array_equal(enc.g, gold["g"])
    assert np.array_equal(enc.t_idx, gold["t_idx"]) and np.array_equal(enc.t_sign, gold["t_sign"])
    f, ids, sc, r, _ = O.score_flat(cl, L, vu, gold["q_seed"].tobytes(), int(gold["trials"]), int(gold["k"]),
                                    want_r=True)
    assert f == -1 and np.array_equal(r, gold["r"])
    assert np.array_equal(ids, gold["top_ids"]) and np.array_equal(sc, gold["top_scores"])
    assert np.array_equal(O.decode_scores(r, cl, L, enc), gold["mv"])
    fv, ur, zv = O.verify_response(r, cl.m_enc, cl.m, 1024, enc.v_enc, int(gold["trials"]), gold["v_seed"].tobytes())
    assert fv == -1 and np.array_equal(ur, gold["ur"]) and np.array_equal(zv, gold["zv"])
    assert gold["v_seed"].tobytes() == O.domain_separate(gold["q_seed"].tobytes(), b"protocol2")
