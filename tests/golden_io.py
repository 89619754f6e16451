"""Loader of the committed golden fixture (tests/golden/bn_small.npz)."""
from __future__ import annotations

import hashlib
import os

import numpy as np

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
P, N = O.P, 1024


def load():
    return dict(np.load(os.path.join(HERE, "golden", "bn_small.npz")))


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cluster(gold):
    """Rebuilds (M, L, cluster) with the oracle and checks the keygen hashes."""
    m = gold["M"].shape[0]
    M = np.zeros((m, N), np.int64)
    M[:, : int(gold["d"])] = gold["M"].astype(np.int64)
    Mu = (M % P).astype(np.uint64)
    L = O.generate_subspace(gold["key_seed"].tobytes())
    cl = O.encrypt_cluster(Mu.reshape(-1), m, L, O.derive_h_seed(int(gold["upload_seed"]), 0))
    assert sha(L) == str(gold["sha_L"]) and sha(cl.m_enc) == str(gold["sha_m_enc"])
    assert sha(cl.a_l) == str(gold["sha_a_l"]) and sha(cl.h_mat) == str(gold["sha_h"])
    return Mu, L, cl


def encoded(gold):
    return O.Encoded(gold["v_enc"], gold["g"], gold["t_idx"], gold["t_sign"])
