"""Seeded synthetic inputs shared by the tests (oracle-built clusters)."""
from __future__ import annotations

import numpy as np

import oracle as O

N = 1024
P = O.P


def int8_matrix(m: int, d: int, seed: int) -> np.ndarray:
    """Gaussian -> L2-normalise -> int8 rows, zero-padded to n, as F_p residues."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((m, d)).astype(np.float32)
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    q = np.clip(np.rint(127.0 * x / np.maximum(np.abs(x).max(axis=1, keepdims=True), 1e-12)), -127, 127)
    out = np.zeros((m, N), np.int64)
    out[:, :d] = q
    return (out % P).astype(np.uint64)


def uniform_fp(shape, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 2**62, size=shape, dtype=np.uint64) % np.uint64(P)).astype(np.uint64)


def cluster(m: int, seed: int, d: int = 768, key_seed=bytes([1]) * 32, upload_seed: int = 7, ci: int = 0,
            uniform: bool = False):
    M = uniform_fp((m, N), seed) if uniform else int8_matrix(m, d, seed)
    L = O.generate_subspace(key_seed)
    cl = O.encrypt_cluster(M.reshape(-1), m, L, O.derive_h_seed(upload_seed, ci))
    return M, L, cl


def query(L, seed: int, d: int = 768, q_seed=None):
    v = int8_matrix(1, d, seed)[0]
    qs = q_seed if q_seed is not None else O.derive_h_seed(seed ^ 0x5155455259, 0)
    enc = O.encode_query(v, L, qs)
    return v, qs, enc


def bigint_matvec(M: np.ndarray, v: np.ndarray) -> list[int]:
    """Independent exact F_p matvec with Python integers."""
    vv = [int(x) for x in v]
    return [sum(int(a) * b for a, b in zip(row, vv)) % P for row in M]


def signed(a: np.ndarray) -> np.ndarray:
    """Residues -> signed integers (fp_to_signed), exactly."""
    s = np.asarray(a, np.uint64).astype(np.int64)
    s[s >= P // 2] -= P
    return s
