"""ctypes front-end of the CPU oracle (oracle/bn_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker.  tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg are the only callers; the product never imports
this module.  See bn_oracle.h for what is pinned and what is "parity
unpinned" (everything derived from ChaCha draws, against the reference).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbn_oracle.so")
P = (1 << 61) - 1
N = 1024

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    u64, u32, i32, i64, f64, vp = C.c_uint64, C.c_uint32, C.c_int32, C.c_int64, C.c_double, C.c_void_p
    sig = {
        "bno_mersenne_reduce128": (u64, [u64, u64]),
        "bno_add_mod": (u64, [u64, u64]),
        "bno_sub_mod": (u64, [u64, u64]),
        "bno_mul_mod": (u64, [u64, u64]),
        "bno_fp_to_signed": (i64, [u64]),
        "bno_chacha20_block": (None, [_u32p, u64, u64, _u32p]),
        "bno_seed_from_u64": (None, [u64, _u8p]),
        "bno_rng_u32s": (None, [_u8p, C.c_size_t, _u32p]),
        "bno_rng_u64s": (None, [_u8p, C.c_size_t, _u64p]),
        "bno_domain_separate": (None, [_u8p, C.c_char_p, C.c_size_t, _u8p]),
        "bno_derive_h_seed": (None, [u64, u64, _u8p]),
        "bno_mu": (f64, []),
        "bno_sparse_threshold": (u32, [f64]),
        "bno_n1": (u32, [u32]),
        "bno_verification_trials": (u32, []),
        "bno_generate_subspace": (None, [_u8p, u32, u32, _u64p]),
        "bno_regenerate_h_s": (i64, [_u8p, u64, u32, u32, f64, _u64p, _u64p, _u32p, _i8p, u64]),
        "bno_encrypt_cluster": (i64, [_u64p, u64, u32, u32, _u64p, _u8p, f64, _u64p, _u64p, _u64p,
                                      _u64p, _u32p, _i8p, u64, C.c_int]),
        "bno_quantise_vector": (None, [_f32p, u32, u32, u64, _u64p]),
        "bno_encode_query": (u32, [_u64p, _u64p, u32, u32, f64, _u8p, _u64p, _u64p, _u32p, _i8p]),
        "bno_matvec_scalar": (None, [_u64p, u64, u32, _u64p, _u64p, C.c_int]),
        "bno_have_avx512": (C.c_int, []),
        "bno_matvec_avx512": (None, [_u64p, u64, u32, _u64p, _u64p, C.c_int]),
        "bno_matvec_transpose": (None, [_u64p, u64, u32, _u64p, _u64p, C.c_int]),
        "bno_matvec_batch": (None, [_u64p, u64, u32, _u64p, u32, _u64p, C.c_int]),
        "bno_dot_product": (u64, [_u64p, _u64p, u64]),
        "bno_verify_response": (i32, [_u64p, _u64p, u64, u32, _u64p, u32, _u8p, vp, vp, C.c_int]),
        "bno_verify_shard_partials": (None, [_u64p, _u64p, u64, u32, _u64p, u32, _u8p, u64, u64, _u64p, _u64p,
                                              C.c_int]),
        "bno_l_transpose_times_vec": (None, [_u64p, u32, u32, _u64p, _u64p]),
        "bno_decode_scores": (None, [_u64p, _u64p, _u64p, _u64p, _u64p, _u32p, _i8p, _u64p, _u64p,
                                     _u64p, _u32p, _i8p, u32, u64, u32, u32, _u64p, C.c_int]),
        "bno_topk": (u32, [_i64p, vp, u64, u32, _u32p, _i64p]),
        "bno_l2_f32": (C.c_float, [_f32p, _f32p, u32]),
        "bno_probe_route": (u32, [_f32p, u32, u32, _f32p, u32, _u32p]),
        "bno_assign": (None, [_f32p, u64, u32, _f32p, u32, _u32p, C.c_int]),
        "bno_kmeans_train": (None, [_f32p, u64, u32, u32, u64, u32, _f32p, C.c_int]),
        "bno_score_flat": (i32, [_u64p, _u64p, _u64p, _u64p, _u64p, _u32p, _i8p, _u64p, u64, u32, u32,
                                 _u64p, _u8p, u32, u32, _u32p, _i64p, vp, vp, C.c_int, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()
NTHREADS = int(os.environ.get("BN_ORACLE_THREADS", str(os.cpu_count() or 1)))


def _seed(s) -> np.ndarray:
    a = np.frombuffer(bytes(s), dtype=np.uint8).copy() if not isinstance(s, np.ndarray) else s.astype(np.uint8)
    assert a.size == 32
    return np.ascontiguousarray(a)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- field
def mersenne_reduce(x: int) -> int:
    return int(lib.bno_mersenne_reduce128(x & (2**64 - 1), x >> 64))


def fp_to_signed(s: int) -> int:
    return int(lib.bno_fp_to_signed(s))


# ---------------------------------------------------------------- rng
def chacha20_block(key_words, counter: int, stream: int) -> np.ndarray:
    out = np.zeros(16, np.uint32)
    lib.bno_chacha20_block(np.ascontiguousarray(key_words, np.uint32), counter, stream, out)
    return out


def seed_from_u64(x: int) -> bytes:
    out = np.zeros(32, np.uint8)
    lib.bno_seed_from_u64(x, out)
    return out.tobytes()


def rng_u32s(seed, count: int) -> np.ndarray:
    out = np.zeros(count, np.uint32)
    lib.bno_rng_u32s(_seed(seed), count, out)
    return out


def rng_u64s(seed, count: int) -> np.ndarray:
    out = np.zeros(count, np.uint64)
    lib.bno_rng_u64s(_seed(seed), count, out)
    return out


def domain_separate(seed, tag: bytes) -> bytes:
    out = np.zeros(32, np.uint8)
    lib.bno_domain_separate(_seed(seed), tag, len(tag), out)
    return out.tobytes()


def derive_h_seed(upload_seed: int, ci: int) -> bytes:
    out = np.zeros(32, np.uint8)
    lib.bno_derive_h_seed(upload_seed, ci, out)
    return out.tobytes()


def mu() -> float:
    return float(lib.bno_mu())


# ---------------------------------------------------------------- keygen
def generate_subspace(key_seed, n=N, n1=128) -> np.ndarray:
    L = np.zeros(n * n1, np.uint64)
    lib.bno_generate_subspace(_seed(key_seed), n, n1, L)
    return L


class Sparse:
    def __init__(self, rowptr, idx, sign):
        self.rowptr, self.idx, self.sign = rowptr, idx, sign


def regenerate_h_s(h_seed, m, n=N, n1=128):
    H = np.zeros(max(m * n1, 1), np.uint64)
    rowptr = np.zeros(m + 1, np.uint64)
    cap = max(m * 256, 1024)
    while True:
        idx = np.zeros(cap, np.uint32)
        sign = np.zeros(cap, np.int8)
        nnz = lib.bno_regenerate_h_s(_seed(h_seed), m, n, n1, mu(), H, rowptr, idx, sign, cap)
        if nnz >= 0:
            return H[: m * n1], Sparse(rowptr, idx[:nnz].copy(), sign[:nnz].copy())
        cap = -nnz


class Cluster:
    """Restates crypto.rs:353-392 EncryptedCluster (owned storage)."""

    def __init__(self, m, n, n1, m_enc, a_l, m_plain, h_mat, s_mat):
        self.m, self.n, self.n1 = m, n, n1
        self.m_enc, self.a_l, self.m_plain, self.h_mat, self.s_mat = m_enc, a_l, m_plain, h_mat, s_mat


def encrypt_cluster(M: np.ndarray, m: int, L: np.ndarray, h_seed, n=N, n1=128, threads=None) -> Cluster:
    M = np.ascontiguousarray(M, np.uint64).reshape(-1)
    assert M.size == m * n
    m_enc = np.zeros(max(m * n, 1), np.uint64)
    al = np.zeros(max(m * n1, 1), np.uint64)
    H = np.zeros(max(m * n1, 1), np.uint64)
    rowptr = np.zeros(m + 1, np.uint64)
    cap = max(m * 256, 1024)
    while True:
        idx = np.zeros(cap, np.uint32)
        sign = np.zeros(cap, np.int8)
        nnz = lib.bno_encrypt_cluster(M if M.size else np.zeros(1, np.uint64), m, n, n1, L, _seed(h_seed),
                                      mu(), m_enc, al, H, rowptr, idx, sign, cap, threads or NTHREADS)
        if nnz >= 0:
            break
        cap = -nnz
    return Cluster(m, n, n1, m_enc[: m * n], al[: m * n1], M.copy(), H[: m * n1],
                   Sparse(rowptr, idx[:nnz].copy(), sign[:nnz].copy()))


# ---------------------------------------------------------------- client
def quantise_vector(v, n=N, q=1 << 20) -> np.ndarray:
    v = np.ascontiguousarray(v, np.float32)
    out = np.zeros(n, np.uint64)
    lib.bno_quantise_vector(v, v.size, n, q, out)
    return out


class Encoded:
    def __init__(self, v_enc, g, t_idx, t_sign):
        self.v_enc, self.g, self.t_idx, self.t_sign = v_enc, g, t_idx, t_sign


def encode_query(v_q: np.ndarray, L: np.ndarray, q_seed, n=N, n1=128) -> Encoded:
    v_enc = np.zeros(n, np.uint64)
    g = np.zeros(n1, np.uint64)
    ti = np.zeros(n, np.uint32)
    ts = np.zeros(n, np.int8)
    c = lib.bno_encode_query(np.ascontiguousarray(v_q, np.uint64), L, n, n1, mu(), _seed(q_seed), v_enc, g, ti, ts)
    return Encoded(v_enc, g, ti[:c].copy(), ts[:c].copy())


# ---------------------------------------------------------------- server
def matvec(mat, rows, cols, vec, avx512=False, threads=None) -> np.ndarray:
    out = np.zeros(max(rows, 1), np.uint64)
    f = lib.bno_matvec_avx512 if avx512 else lib.bno_matvec_scalar
    f(np.ascontiguousarray(mat, np.uint64).reshape(-1) if rows else np.zeros(1, np.uint64), rows, cols,
      np.ascontiguousarray(vec, np.uint64), out, threads or NTHREADS)
    return out[:rows]


compute_products = matvec


def matvec_transpose(mat, rows, cols, vec, threads=None) -> np.ndarray:
    out = np.zeros(cols, np.uint64)
    lib.bno_matvec_transpose(np.ascontiguousarray(mat, np.uint64).reshape(-1), rows, cols,
                             np.ascontiguousarray(vec, np.uint64), out, threads or NTHREADS)
    return out


def matvec_batch(mat, rows, cols, vecs: np.ndarray, threads=None) -> np.ndarray:
    vecs = np.ascontiguousarray(vecs, np.uint64).reshape(-1, cols)
    B = vecs.shape[0]
    out = np.zeros((B, rows), np.uint64)
    lib.bno_matvec_batch(np.ascontiguousarray(mat, np.uint64).reshape(-1), rows, cols, vecs.reshape(-1), B,
                         out.reshape(-1), threads or NTHREADS)
    return out


def dot_product(a, b) -> int:
    return int(lib.bno_dot_product(np.ascontiguousarray(a, np.uint64), np.ascontiguousarray(b, np.uint64), len(a)))


def verify_response(r, m_enc, m, n, v_enc, trials, v_seed, threads=None):
    """Returns (first_failed_trial or -1, ur[:ran], zv[:ran])."""
    ur = np.zeros(max(trials, 1), np.uint64)
    zv = np.zeros(max(trials, 1), np.uint64)
    f = lib.bno_verify_response(np.ascontiguousarray(r, np.uint64) if m else np.zeros(1, np.uint64),
                                np.ascontiguousarray(m_enc, np.uint64).reshape(-1) if m else np.zeros(1, np.uint64),
                                m, n, np.ascontiguousarray(v_enc, np.uint64), trials, _seed(v_seed),
                                _ptr(ur), _ptr(zv), threads or NTHREADS)
    ran = trials if f < 0 else f + 1
    return int(f), ur[:ran], zv[:ran]


def verify_shard_partials(r_shard, m_shard, rows, n, v_enc, trials, v_seed, row0, total, threads=None):
    """(ur, zv) partial sums of every trial for rows [row0, row0 + rows) of a
    corpus of `total` rows (verify_response's draws restricted to the shard)."""
    ur = np.zeros(max(trials, 1), np.uint64)
    zv = np.zeros(max(trials, 1), np.uint64)
    lib.bno_verify_shard_partials(np.ascontiguousarray(r_shard, np.uint64) if rows else np.zeros(1, np.uint64),
                                  np.ascontiguousarray(m_shard, np.uint64).reshape(-1) if rows else np.zeros(1, np.uint64),
                                  rows, n, np.ascontiguousarray(v_enc, np.uint64), trials, _seed(v_seed), row0, total,
                                  ur, zv, threads or NTHREADS)
    return ur[:trials], zv[:trials]


# ---------------------------------------------------------------- decode
def l_transpose_times_vec(L, v, n=N, n1=128):
    out = np.zeros(n1, np.uint64)
    lib.bno_l_transpose_times_vec(L, n, n1, np.ascontiguousarray(v, np.uint64), out)
    return out


def decode_scores(r, cluster: Cluster, L, enc: Encoded, threads=None) -> np.ndarray:
    m, n, n1 = cluster.m, cluster.n, cluster.n1
    out = np.zeros(max(m, 1), np.uint64)
    s = cluster.s_mat
    z = lambda a, dt: a if a.size else np.zeros(1, dt)  # noqa: E731
    lib.bno_decode_scores(z(np.ascontiguousarray(r, np.uint64), np.uint64), z(cluster.a_l, np.uint64),
                          z(cluster.m_plain, np.uint64), z(cluster.h_mat, np.uint64), s.rowptr,
                          z(s.idx, np.uint32), z(s.sign, np.int8), L, enc.v_enc, enc.g, z(enc.t_idx, np.uint32),
                          z(enc.t_sign, np.int8), enc.t_idx.size, m, n, n1, out, threads or NTHREADS)
    return out[:m]


def to_signed(mv: np.ndarray) -> np.ndarray:
    mv = mv.astype(np.uint64)
    s = mv.astype(np.int64)
    neg = mv >= np.uint64(P // 2)
    s[neg] = (mv[neg].astype(np.int64) - np.int64(P))
    return s


def topk(scores: np.ndarray, k: int, ids=None):
    scores = np.ascontiguousarray(scores, np.int64)
    kk = min(k, scores.size)
    oi = np.zeros(max(kk, 1), np.uint32)
    os_ = np.zeros(max(kk, 1), np.int64)
    idsa = None if ids is None else np.ascontiguousarray(ids, np.uint32)
    c = lib.bno_topk(scores if scores.size else np.zeros(1, np.int64), _ptr(idsa), scores.size, k, oi, os_)
    return oi[:c], os_[:c]


# ---------------------------------------------------------------- IVF
def probe_route(centroids: np.ndarray, q: np.ndarray, nprobe: int) -> np.ndarray:
    centroids = np.ascontiguousarray(centroids, np.float32)
    nlist, d = centroids.shape
    out = np.zeros(nlist, np.uint32)
    c = lib.bno_probe_route(centroids.reshape(-1), nlist, d, np.ascontiguousarray(q, np.float32), nprobe, out)
    return out[:c]


def assign(data: np.ndarray, centroids: np.ndarray, threads=None) -> np.ndarray:
    data = np.ascontiguousarray(data, np.float32)
    centroids = np.ascontiguousarray(centroids, np.float32)
    out = np.zeros(data.shape[0], np.uint32)
    lib.bno_assign(data.reshape(-1), data.shape[0], data.shape[1], centroids.reshape(-1), centroids.shape[0], out,
                   threads or NTHREADS)
    return out


def kmeans_train(data: np.ndarray, k: int, seed: int, max_iter: int, threads=None) -> np.ndarray:
    data = np.ascontiguousarray(data, np.float32)
    out = np.zeros((k, data.shape[1]), np.float32)
    lib.bno_kmeans_train(data.reshape(-1), data.shape[0], data.shape[1], k, seed, max_iter, out.reshape(-1),
                         threads or NTHREADS)
    return out


# ---------------------------------------------------------------- whole query
def score_flat(cluster: Cluster, L, v_q, q_seed, trials, k, threads=None, avx512=True, want_r=False):
    """lib.rs:326-475 with an explicit q_seed.  Returns (fail, ids, scores, r, timings_us)."""
    m, n, n1 = cluster.m, cluster.n, cluster.n1
    kk = min(k, m)
    ids = np.zeros(max(kk, 1), np.uint32)
    sc = np.zeros(max(kk, 1), np.int64)
    r = np.zeros(max(m, 1), np.uint64) if want_r else None
    tm = np.zeros(4, np.float64)
    s = cluster.s_mat
    f = lib.bno_score_flat(cluster.m_enc, cluster.a_l, cluster.m_plain, cluster.h_mat, s.rowptr,
                           s.idx if s.idx.size else np.zeros(1, np.uint32),
                           s.sign if s.sign.size else np.zeros(1, np.int8), L, m, n, n1,
                           np.ascontiguousarray(v_q, np.uint64), _seed(q_seed), trials, k, ids, sc, _ptr(r),
                           _ptr(tm), threads or NTHREADS, 1 if avx512 else 0)
    return int(f), ids[:kk], sc[:kk], (r[:m] if want_r else None), tm
