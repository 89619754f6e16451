"""Generates tests/golden/bn_small.npz: a small seeded BN instance.

The reference ships no golden vectors and its Rust toolchain is absent, so
the fixture is produced by the CPU oracle and every F_p value in it is
re-derived here with Python integers, independently of the oracle:
  r  = M_enc v_enc,  Mv = M v (plaintext, the decode target),
  ur / zv from the Freivalds draws, top-k from exact integer dot products.
Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

P, N = O.P, 1024
M_ROWS, D, TRIALS, K = 48, 96, 3, 10
KEY_SEED, UPLOAD_SEED, Q_SEED = bytes([1]) * 32, 7, bytes([9]) * 32


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    rng = np.random.default_rng(20260101)
    Mi = rng.integers(-127, 128, size=(M_ROWS, D), dtype=np.int64)
    vi = rng.integers(-127, 128, size=D, dtype=np.int64)
    M = np.zeros((M_ROWS, N), np.int64)
    M[:, :D] = Mi
    v = np.zeros(N, np.int64)
    v[:D] = vi
    Mu, vu = (M % P).astype(np.uint64), (v % P).astype(np.uint64)

    L = O.generate_subspace(KEY_SEED)
    h_seed = O.derive_h_seed(UPLOAD_SEED, 0)
    cl = O.encrypt_cluster(Mu.reshape(-1), M_ROWS, L, h_seed)
    enc = O.encode_query(vu, L, Q_SEED)
    v_seed = O.domain_separate(Q_SEED, b"protocol2")
    f, ids, sc, r, _ = O.score_flat(cl, L, vu, Q_SEED, TRIALS, K, want_r=True)
    mv = O.decode_scores(r, cl, L, enc)
    fv, ur, zv = O.verify_response(r, cl.m_enc, M_ROWS, N, enc.v_enc, TRIALS, v_seed)

    # independent big-integer checks
    me = cl.m_enc.reshape(M_ROWS, N)
    ve = [int(x) for x in enc.v_enc]
    r_big = [sum(int(a) * b for a, b in zip(row, ve)) % P for row in me]
    assert [int(x) for x in r] == r_big
    exact = [int(x) for x in (Mi @ vi)]
    assert [int(x) for x in mv] == [e % P for e in exact]
    order = sorted(range(M_ROWS), key=lambda i: (-exact[i], i))[:K]
    assert f == -1 and fv == -1 and list(ids) == order and list(sc) == [exact[i] for i in order]
    draws = [int(x) & P for x in O.rng_u64s(v_seed, TRIALS * M_ROWS)]
    for t in range(TRIALS):
        u = draws[t * M_ROWS : (t + 1) * M_ROWS]
        assert int(ur[t]) == sum(a * b for a, b in zip(u, r_big)) % P
        z = [sum(u[i] * int(me[i, j]) for i in range(M_ROWS)) % P for j in range(N)]
        assert int(zv[t]) == sum(a * b for a, b in zip(z, ve)) % P

    np.savez_compressed(
        os.path.join(HERE, "bn_small.npz"),
        M=Mi.astype(np.int8), v=vi.astype(np.int8), d=D, key_seed=np.frombuffer(KEY_SEED, np.uint8),
        upload_seed=UPLOAD_SEED, q_seed=np.frombuffer(Q_SEED, np.uint8), v_seed=np.frombuffer(v_seed, np.uint8),
        trials=TRIALS, k=K, r=r, mv=mv, top_ids=ids, top_scores=sc, ur=ur, zv=zv, v_enc=enc.v_enc, g=enc.g,
        t_idx=enc.t_idx, t_sign=enc.t_sign, sha_L=sha(L), sha_m_enc=sha(cl.m_enc), sha_a_l=sha(cl.a_l),
        sha_h=sha(cl.h_mat), sha_s=sha(np.concatenate([cl.s_mat.rowptr.view(np.uint8), cl.s_mat.idx.view(np.uint8),
                                                        cl.s_mat.sign.view(np.uint8)])))
    print("wrote bn_small.npz")


if __name__ == "__main__":
    main()
