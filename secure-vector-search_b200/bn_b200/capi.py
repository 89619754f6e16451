"""ctypes bindings of the C ABI in include/bn_b200.h (libbn_b200.so).

The product path: every call lands in the sm_100a library; there is no
Python or CPU fallback.  Loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbn_b200.so")
N = 1024
P = (1 << 61) - 1
TOPK_MAX = 1024

BN_OK, BN_EINVAL, BN_ECUDA, BN_EBUDGET, BN_ENODEV, BN_EUNSUPPORTED, BN_EAGAIN, BN_EDRAW = 0, -1, -2, -3, -4, -5, -6, -7
STATUS_DRAW_HIT_P = 0x1000
ENGINE_TENSOR, ENGINE_CUDA_CORE = 0, 1
BLOCK_AUTOTUNE = 1
_NAMES = {BN_EINVAL: "EINVAL", BN_ECUDA: "ECUDA", BN_EBUDGET: "EBUDGET", BN_ENODEV: "ENODEV",
          BN_EUNSUPPORTED: "EUNSUPPORTED", BN_EAGAIN: "EAGAIN", BN_EDRAW: "EDRAW"}


class BnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built; run `python secure-vector-search_b200/build.py`")
lib = C.CDLL(LIB_PATH)

vp = C.c_void_p
u32, u64, i32 = C.c_uint32, C.c_uint64, C.c_int32


class SparseCsr(C.Structure):
    _fields_ = [("rowptr", vp), ("idx", vp), ("sign", vp)]


class ServerConfig(C.Structure):
    _fields_ = [("max_batch", u32), ("slots", u32), ("mem_budget", u64), ("max_wait_us", u32), ("trials", u32),
                ("k", u32), ("block_min", u32), ("max_queue", u32), ("queue_wait_us", u32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", u64), ("completed", u64), ("batches", u64), ("mean_batch", C.c_double),
                ("p50_us", C.c_double), ("p99_us", C.c_double), ("max_us", C.c_double),
                ("throughput_qps", C.c_double), ("peak_workspace_bytes", u64), ("block_batches", u64),
                ("rejected", u64)]


class StoreStats(C.Structure):
    _fields_ = [("gets", u64), ("uploads", u64), ("evictions", u64), ("bytes_uploaded", u64),
                ("resident_bytes", u64), ("budget_bytes", u64)]


_SIGS = {
    "bn_last_error": (C.c_char_p, []),
    "bn_build_info": (C.c_char_p, []),
    "bn_device_count": (C.c_int, [vp]),
    "bn_ctx_create": (C.c_int, [C.c_int, u64, vp]),
    "bn_ctx_destroy": (C.c_int, [vp]),
    "bn_ctx_memory": (C.c_int, [vp, vp, vp, vp]),
    "bn_ctx_set_engine": (C.c_int, [vp, C.c_int]),
    "bn_debug_plant_draw_hit": (C.c_int, [vp, C.c_int]),
    "bn_debug_set_wait_limit": (C.c_int, [vp, u64]),
    "bn_flat_build": (C.c_int, [vp, vp, vp, vp, u64, u32, u32, vp]),
    "bn_flat_attach_client": (C.c_int, [vp, vp, vp, SparseCsr]),
    "bn_flat_build_from_plain": (C.c_int, [vp, vp, u64, u32, u32, vp, vp, SparseCsr, vp]),
    "bn_flat_destroy": (C.c_int, [vp]),
    "bn_flat_info": (C.c_int, [vp, vp, vp]),
    "bn_flat_device_m_enc": (C.c_int, [vp, vp]),
    "bn_flat_compute_products": (C.c_int, [vp, vp, vp]),
    "bn_flat_compute_products_batch": (C.c_int, [vp, vp, u32, vp]),
    "bn_flat_decode_dense_terms": (C.c_int, [vp, vp, vp, vp]),
    "bn_flat_verify": (C.c_int, [vp, vp, vp, vp, u32, vp, vp, vp]),
    "bn_flat_verify_noalloc": (C.c_int, [vp, vp, vp, vp, u32, vp, vp, vp, vp]),
    "bn_flat_query": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp, vp]),
    "bn_flat_query_shard": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, vp, u32, u32, u64, u64, vp, vp, vp, vp, vp]),
    "bn_flat_plan": (C.c_int, [vp, u32, u32, u32, vp]),
    "bn_plan_enqueue": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "bn_plan_enqueue_scan": (C.c_int, [vp, vp, vp, vp]),
    "bn_plan_status": (C.c_int, [vp, vp]),
    "bn_plan_destroy": (C.c_int, [vp]),
    "bn_plan_profile": (C.c_int, [vp, u32]),
    "bn_plan_profile_read": (C.c_int, [vp, vp, u32, vp]),
    "bn_flat_block_prepare": (C.c_int, [vp]),
    "bn_flat_block_plan": (C.c_int, [vp, u32, u32, u32, u32, vp]),
    "bn_plan_block_config": (C.c_int, [vp, vp, vp]),
    "bn_plan_enqueue_block": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "bn_flat_query_block": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp]),
    "bn_flat_verify_block": (C.c_int, [vp, u32, vp, vp, vp, u32, vp, vp, vp]),
    "bn_ivf_build": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, u32, u32, vp]),
    "bn_ivf_attach_client": (C.c_int, [vp, vp, vp, SparseCsr]),
    "bn_ivf_build_from_plain": (C.c_int, [vp, u32, vp, vp, vp, u32, u32, vp, vp, SparseCsr, vp]),
    "bn_ivf_destroy": (C.c_int, [vp]),
    "bn_ivf_info": (C.c_int, [vp, vp, vp]),
    "bn_ivf_set_centroids": (C.c_int, [vp, vp, u32]),
    "bn_ivf_route": (C.c_int, [vp, u32, vp, u32, vp]),
    "bn_ivf_compute_products": (C.c_int, [vp, u32, vp, vp, vp]),
    "bn_ivf_decode_dense_terms": (C.c_int, [vp, u32, vp, vp, vp, vp]),
    "bn_ivf_verify": (C.c_int, [vp, u32, vp, vp, vp, u32, vp, vp, vp]),
    "bn_ivf_query": (C.c_int, [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp]),
    "bn_ivf_block_prepare": (C.c_int, [vp]),
    "bn_ivf_query_block": (C.c_int, [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp]),
    "bn_ivf_block_tune": (C.c_int, [vp, u32, u32]),
    "bn_ivf_block_profile": (C.c_int, [vp, C.c_int]),
    "bn_ivf_block_profile_read": (C.c_int, [vp, vp, u32, vp]),
    "bn_ivf_verify_block": (C.c_int, [vp, u32, u32, vp, vp, u64, vp, vp, u32, vp, vp, vp, vp]),
    "bn_encrypt_cluster": (C.c_int, [vp, vp, u64, u32, u32, vp, vp, SparseCsr, vp, vp]),
    "bn_keygen_h_s": (C.c_int, [vp, vp, u64, u32, vp, vp, vp, vp, u64, vp]),
    "bn_flat_build_keygen": (C.c_int, [vp, vp, u64, u32, u32, vp, vp, vp]),
    "bn_ivf_build_keygen": (C.c_int, [vp, u32, vp, vp, vp, u32, u32, vp, u64, vp]),
    "bn_server_create": (C.c_int, [vp, vp, C.POINTER(ServerConfig), vp]),
    "bn_server_submit_flat": (C.c_int, [vp, vp, vp, vp, vp, u32, vp, vp]),
    "bn_server_submit_ivf": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, u32, vp, vp]),
    "bn_server_wait": (C.c_int, [vp, u64, u32, vp, vp, vp, vp, vp, vp]),
    "bn_server_stats": (C.c_int, [vp, C.c_int, C.POINTER(ServerStats)]),
    "bn_server_destroy": (C.c_int, [vp]),
    "bn_stream_build": (C.c_int, [vp, vp, vp, vp, u64, u32, u32, vp, vp, SparseCsr, u64, u64, vp]),
    "bn_stream_build_from_plain": (C.c_int, [vp, vp, u64, u32, u32, vp, vp, SparseCsr, u64, u64, vp]),
    "bn_stream_info": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "bn_stream_query": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, vp, u32, u32, vp, vp, vp, vp]),
    "bn_stream_stats": (C.c_int, [vp, C.c_int, C.POINTER(StoreStats)]),
    "bn_stream_destroy": (C.c_int, [vp]),
    "bn_ivf_stream_build": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, u32, u32, vp, vp, SparseCsr, u64, u64, vp]),
    "bn_ivf_stream_build_keygen": (C.c_int, [vp, u32, vp, vp, vp, u32, u32, vp, u64, u64, u64, vp]),
    "bn_ivf_stream_info": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "bn_ivf_stream_query": (C.c_int, [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp]),
    "bn_ivf_stream_stats": (C.c_int, [vp, C.c_int, C.POINTER(StoreStats)]),
    "bn_ivf_stream_destroy": (C.c_int, [vp]),
    "bn_lru_create": (C.c_int, [u64, vp]),
    "bn_lru_touch": (C.c_int, [vp, u64, vp]),
    "bn_lru_pre_evict": (C.c_int, [vp, u64, vp, u32, vp]),
    "bn_lru_insert": (C.c_int, [vp, u64, u64, vp]),
    "bn_lru_stats": (C.c_int, [vp, C.POINTER(StoreStats)]),
    "bn_lru_destroy": (C.c_int, [vp]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def last_error() -> str:
    return lib.bn_last_error().decode()


def check(rc: int):
    if rc != BN_OK:
        raise BnError(rc, last_error())


def ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    return a.ctypes.data_as(vp)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _csr(rowptr, idx, sign):
    rowptr, idx, sign = _u64(rowptr), np.ascontiguousarray(idx, np.uint32), np.ascontiguousarray(sign, np.int8)
    keep = (rowptr, idx, sign)
    return SparseCsr(ptr(rowptr), ptr(idx) if idx.size else None, ptr(sign) if sign.size else None), keep


def device_count() -> int:
    n = C.c_int(0)
    check(lib.bn_device_count(C.byref(n)))
    return n.value


def build_info() -> str:
    return lib.bn_build_info().decode()


class Context:
    """bn_ctx: a device and its memory budget (gpu/mod.rs:169-200, budget.rs:132-150)."""

    def __init__(self, device: int = 0, vram_budget_bytes: int = 0):
        self.h = None
        h = vp()
        check(lib.bn_ctx_create(device, vram_budget_bytes, C.byref(h)))
        self.h = h

    def set_engine(self, engine: int):
        check(lib.bn_ctx_set_engine(self.h, engine))

    def plant_draw_hit(self, on: bool):
        """Testing hook: Protocol 2 runs behave as if a draw had equalled p."""
        check(lib.bn_debug_plant_draw_hit(self.h, 1 if on else 0))

    def set_wait_limit(self, cycles: int):
        """Testing hook: pipeline waits of later launches give up after `cycles` (0 = default)."""
        check(lib.bn_debug_set_wait_limit(self.h, cycles))

    def memory(self):
        b, u, p = u64(), u64(), u64()
        check(lib.bn_ctx_memory(self.h, C.byref(b), C.byref(u), C.byref(p)))
        return b.value, u.value, p.value

    def close(self):
        if getattr(self, "h", None):
            lib.bn_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


def _t_concat(enc_list):
    """Concatenate per-query sparse T (idx, sign) lists."""
    nnz = np.array([len(t[0]) for t in enc_list], np.uint32)
    idx = np.concatenate([np.asarray(t[0], np.uint32) for t in enc_list]) if len(enc_list) else np.zeros(0, np.uint32)
    sign = np.concatenate([np.asarray(t[1], np.int8) for t in enc_list]) if len(enc_list) else np.zeros(0, np.int8)
    return idx, sign, nnz


class Flat:
    """bn_flat: a resident flat corpus (FlatGpuState, gpu/mod.rs:279-409)."""

    def __init__(self, ctx: Context, handle, m: int, n1: int):
        self.ctx, self.h, self.m, self.n1 = ctx, handle, m, n1

    @classmethod
    def build(cls, ctx, m_enc, a_l, h, m, n1=128):
        m_enc, a_l, h = _u64(m_enc), _u64(a_l), _u64(h)
        out = vp()
        check(lib.bn_flat_build(ctx.h, ptr(m_enc), ptr(a_l), ptr(h), m, N, n1, C.byref(out)))
        return cls(ctx, out, m, n1)

    @classmethod
    def build_keygen(cls, ctx, m_q, m, L, h_seed: bytes, n1=128):
        """bn_flat_build_keygen: keys drawn on the device from h_seed."""
        m_q, L = _u64(m_q), _u64(L)
        seed = np.frombuffer(bytes(h_seed), np.uint8).copy()
        out = vp()
        check(lib.bn_flat_build_keygen(ctx.h, ptr(m_q), m, N, n1, ptr(L), ptr(seed), C.byref(out)))
        return cls(ctx, out, m, n1)

    @classmethod
    def build_from_plain(cls, ctx, m_q, m, L, H, s_rowptr, s_idx, s_sign, n1=128):
        m_q, L, H = _u64(m_q), _u64(L), _u64(H)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        out = vp()
        check(lib.bn_flat_build_from_plain(ctx.h, ptr(m_q), m, N, n1, ptr(L), ptr(H), csr, C.byref(out)))
        return cls(ctx, out, m, n1)

    def attach_client(self, L, m_plain, s_rowptr, s_idx, s_sign):
        L, m_plain = _u64(L), _u64(m_plain)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        check(lib.bn_flat_attach_client(self.h, ptr(L), ptr(m_plain), csr))

    def info(self):
        rows, b = u64(), u64()
        check(lib.bn_flat_info(self.h, C.byref(rows), C.byref(b)))
        return rows.value, b.value

    def device_m_enc(self) -> int:
        p = vp()
        check(lib.bn_flat_device_m_enc(self.h, C.byref(p)))
        return p.value

    def compute_products(self, v_enc) -> np.ndarray:
        v = _u64(v_enc)
        r = np.zeros(max(self.m, 1), np.uint64)
        check(lib.bn_flat_compute_products(self.h, ptr(v), ptr(r)))
        return r[: self.m]

    def compute_products_batch(self, v_encs) -> np.ndarray:
        v = _u64(v_encs).reshape(-1, N)
        r = np.zeros((v.shape[0], max(self.m, 1)), np.uint64)
        check(lib.bn_flat_compute_products_batch(self.h, ptr(v), v.shape[0], ptr(r)))
        return r[:, : self.m]

    def decode_dense_terms(self, g, lt_venc) -> np.ndarray:
        g, lt = _u64(g), _u64(lt_venc)
        out = np.zeros(max(self.m, 1), np.uint64)
        check(lib.bn_flat_decode_dense_terms(self.h, ptr(g), ptr(lt), ptr(out)))
        return out[: self.m]

    def verify(self, r, v_enc, v_seed: bytes, trials: int):
        r, v = _u64(r), _u64(v_enc)
        seed = np.frombuffer(bytes(v_seed), np.uint8).copy()
        f = i32(0)
        ur = np.zeros(max(trials, 1), np.uint64)
        zv = np.zeros(max(trials, 1), np.uint64)
        check(lib.bn_flat_verify(self.h, ptr(r) if r.size else None, ptr(v), ptr(seed), trials, C.byref(f), ptr(ur),
                                 ptr(zv)))
        ran = trials if f.value < 0 else f.value + 1
        return f.value, ur[:ran], zv[:ran]

    def query(self, v_enc, g, t_list, v_seeds, trials, k, want_r=False, want_mv=False):
        """t_list: per query (idx array, sign array).  v_seeds: list of 32-byte seeds or None."""
        v = _u64(v_enc).reshape(-1, N)
        B = v.shape[0]
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seeds = None if v_seeds is None else np.frombuffer(b"".join(bytes(s) for s in v_seeds), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        fl = np.zeros(B, np.int32)
        r = np.zeros((B, max(self.m, 1)), np.uint64) if want_r else None
        mv = np.zeros((B, max(self.m, 1)), np.uint64) if want_mv else None
        check(lib.bn_flat_query(self.h, B, ptr(v), ptr(gg), ptr(ti) if ti.size else None, ptr(ts) if ts.size else None,
                                ptr(tn), ptr(seeds), trials, k, ptr(ids), ptr(sc), ptr(nh), ptr(fl), ptr(r), ptr(mv)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, fl, (r[:, : self.m] if want_r else None), (mv[:, : self.m] if want_mv else None)

    def query_shard(self, v_enc, g, t_list, v_seeds, trials, k, shard_row0: int, total_rows: int):
        """bn_flat_query_shard: this handle is rows [shard_row0, shard_row0 + m) of a corpus of total_rows.
        Returns (hits with global ids, ur, zv) with ur / zv of shape (B, trials)."""
        v = _u64(v_enc).reshape(-1, N)
        B = v.shape[0]
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seeds = None if v_seeds is None else np.frombuffer(b"".join(bytes(s) for s in v_seeds), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        ur = np.zeros((B, max(trials, 1)), np.uint64)
        zv = np.zeros((B, max(trials, 1)), np.uint64)
        check(lib.bn_flat_query_shard(self.h, B, ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                                      ptr(ts) if ts.size else None, ptr(tn), ptr(seeds), trials, k, shard_row0,
                                      total_rows, ptr(ids), ptr(sc), ptr(nh), ptr(ur), ptr(zv)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, ur[:, :trials], zv[:, :trials]

    def plan(self, B: int, trials: int, k: int) -> "Plan":
        out = vp()
        check(lib.bn_flat_plan(self.h, B, trials, k, C.byref(out)))
        return Plan(self, out, B, trials, k)

    # ---- block scoring: B queries per launch, Protocol 2 with one seed per block
    def block_prepare(self):
        check(lib.bn_flat_block_prepare(self.h))

    def block_plan(self, B: int, trials: int, k: int, autotune: bool = False) -> "Plan":
        out = vp()
        check(lib.bn_flat_block_plan(self.h, B, trials, k, BLOCK_AUTOTUNE if autotune else 0, C.byref(out)))
        return Plan(self, out, B, trials, k, block=True)

    def query_block(self, v_enc, g, t_list, block_seed, trials, k, want_mv=False):
        v = _u64(v_enc).reshape(-1, N)
        B = v.shape[0]
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seed = None if block_seed is None else np.frombuffer(bytes(block_seed), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        fl = np.zeros(B, np.int32)
        mv = np.zeros((B, max(self.m, 1)), np.uint64) if want_mv else None
        check(lib.bn_flat_query_block(self.h, B, ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                                      ptr(ts) if ts.size else None, ptr(tn), ptr(seed), trials, k, ptr(ids), ptr(sc),
                                      ptr(nh), ptr(fl), ptr(mv)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, fl, (mv[:, : self.m] if want_mv else None)

    def verify_block(self, r, v_enc, block_seed, trials):
        r = _u64(r).reshape(-1, self.m)
        v = _u64(v_enc).reshape(-1, N)
        B = r.shape[0]
        seed = np.frombuffer(bytes(block_seed), np.uint8).copy()
        fl = np.zeros(B, np.int32)
        ur = np.zeros((max(trials, 1), B), np.uint64)
        zv = np.zeros((max(trials, 1), B), np.uint64)
        check(lib.bn_flat_verify_block(self.h, B, ptr(r), ptr(v), ptr(seed), trials, ptr(fl), ptr(ur), ptr(zv)))
        return fl, ur[:trials], zv[:trials]

    def close(self):
        if self.h:
            lib.bn_flat_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


class Plan:
    """bn_plan: enqueue-only form of Flat.query over device buffers (graph-capturable)."""

    def __init__(self, flat, handle, B, trials, k, block=False):
        self.flat, self.h, self.B, self.trials, self.k, self.block = flat, handle, B, trials, k, block

    def enqueue(self, d_v, d_g, d_t, d_t_nnz, d_seeds, d_ids, d_scores, d_n, d_failed, stream: int):
        """Per-query plans: d_seeds holds B seeds.  Block plans: d_seeds is the one block seed."""
        fn = lib.bn_plan_enqueue_block if self.block else lib.bn_plan_enqueue
        check(fn(self.h, d_v, d_g, d_t, d_t_nnz, d_seeds, d_ids, d_scores, d_n, d_failed, stream))

    def block_config(self):
        cfg = np.zeros(6, np.uint32)
        ms = np.zeros(2, np.float32)
        check(lib.bn_plan_block_config(self.h, ptr(cfg), ptr(ms)))
        return {"w_tile": int(cfg[0]), "stages": int(cfg[1]), "order": int(cfg[2]), "a_resident": int(cfg[3]),
                "k_panel": int(cfg[4]), "two_ksteps_per_stage": int(cfg[5]),
                "tuned_scan_ms": float(ms[0]), "tuned_ur_ms": float(ms[1])}

    def enqueue_scan(self, d_v, d_r, stream: int):
        check(lib.bn_plan_enqueue_scan(self.h, d_v, d_r, stream))

    def status(self) -> int:
        f = u32(0)
        check(lib.bn_plan_status(self.h, C.byref(f)))
        return f.value

    def profile(self, max_launches: int):
        """Time the dominant kernel of the next max_launches enqueues (CUDA events on the launch stream)."""
        check(lib.bn_plan_profile(self.h, max_launches))

    def profile_read(self, cap: int = 65536) -> np.ndarray:
        ms = np.zeros(max(cap, 1), np.float32)
        n = u32(0)
        check(lib.bn_plan_profile_read(self.h, ptr(ms), cap, C.byref(n)))
        return ms[: n.value].copy()

    def close(self):
        if self.h:
            lib.bn_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


class Ivf:
    """bn_ivf: resident inverted lists in CSR form (IvfGpuState, gpu/mod.rs:423-578)."""

    def __init__(self, ctx, handle, offsets, n1):
        self.ctx, self.h, self.offsets, self.n1 = ctx, handle, np.asarray(offsets, np.uint64), n1
        self.nlist = len(offsets) - 1

    @classmethod
    def build(cls, ctx, offsets, ids, m_enc, a_l, h, n1=128):
        off = _u64(offsets)
        ids = np.ascontiguousarray(ids, np.uint32)
        m_enc, a_l, h = _u64(m_enc), _u64(a_l), _u64(h)
        out = vp()
        check(lib.bn_ivf_build(ctx.h, len(off) - 1, ptr(off), ptr(ids), ptr(m_enc), ptr(a_l), ptr(h), N, n1,
                               C.byref(out)))
        return cls(ctx, out, off, n1)

    @classmethod
    def build_keygen(cls, ctx, offsets, ids, m_q, L, upload_seed: int, n1=128):
        """bn_ivf_build_keygen: every list's keys drawn on the device from derive_h_seed(upload_seed, list)."""
        off = _u64(offsets)
        ids = np.ascontiguousarray(ids, np.uint32)
        m_q, L = _u64(m_q), _u64(L)
        out = vp()
        check(lib.bn_ivf_build_keygen(ctx.h, len(off) - 1, ptr(off), ptr(ids), ptr(m_q), N, n1, ptr(L), upload_seed,
                                      C.byref(out)))
        return cls(ctx, out, off, n1)

    @classmethod
    def build_from_plain(cls, ctx, offsets, ids, m_q, L, H, s_rowptr, s_idx, s_sign, n1=128):
        off = _u64(offsets)
        ids = np.ascontiguousarray(ids, np.uint32)
        m_q, L, H = _u64(m_q), _u64(L), _u64(H)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        out = vp()
        check(lib.bn_ivf_build_from_plain(ctx.h, len(off) - 1, ptr(off), ptr(ids), ptr(m_q), N, n1, ptr(L), ptr(H),
                                          csr, C.byref(out)))
        return cls(ctx, out, off, n1)

    def set_centroids(self, centroids):
        """bn_ivf_set_centroids: nlist x d f32 centroids for bn_ivf_route."""
        c = np.ascontiguousarray(centroids, np.float32)
        check(lib.bn_ivf_set_centroids(self.h, ptr(c), c.shape[1]))
        self.cent_d = c.shape[1]

    def route(self, queries, nprobe: int) -> np.ndarray:
        """bn_ivf_route: the min(nprobe, nlist) nearest lists of every query, nearest first."""
        q = np.ascontiguousarray(queries, np.float32)
        if q.ndim == 1:
            q = q[None]
        out = np.zeros((q.shape[0], max(min(nprobe, self.nlist), 1)), np.uint32)
        check(lib.bn_ivf_route(self.h, q.shape[0], ptr(q), nprobe, ptr(out)))
        return out[:, : min(nprobe, self.nlist)]

    def attach_client(self, L, m_plain, s_rowptr, s_idx, s_sign):
        L, m_plain = _u64(L), _u64(m_plain)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        check(lib.bn_ivf_attach_client(self.h, ptr(L), ptr(m_plain), csr))

    def compute_products(self, ci, v_enc):
        v = _u64(v_enc)
        m = int(self.offsets[ci + 1] - self.offsets[ci]) if ci < self.nlist else 0
        r = np.zeros(max(m, 1), np.uint64)
        mo = u64()
        check(lib.bn_ivf_compute_products(self.h, ci, ptr(v), ptr(r), C.byref(mo)))
        return None if mo.value == 0 else r[: mo.value]

    def decode_dense_terms(self, ci, g, lt):
        g, lt = _u64(g), _u64(lt)
        m = int(self.offsets[ci + 1] - self.offsets[ci]) if ci < self.nlist else 0
        out = np.zeros(max(m, 1), np.uint64)
        mo = u64()
        check(lib.bn_ivf_decode_dense_terms(self.h, ci, ptr(g), ptr(lt), ptr(out), C.byref(mo)))
        return None if mo.value == 0 else out[: mo.value]

    def verify(self, ci, r, v_enc, v_seed, trials):
        r, v = _u64(r), _u64(v_enc)
        seed = np.frombuffer(bytes(v_seed), np.uint8).copy()
        f = i32(0)
        ur = np.zeros(max(trials, 1), np.uint64)
        zv = np.zeros(max(trials, 1), np.uint64)
        check(lib.bn_ivf_verify(self.h, ci, ptr(r) if r.size else None, ptr(v), ptr(seed), trials, C.byref(f),
                                ptr(ur), ptr(zv)))
        ran = trials if f.value < 0 else f.value + 1
        return f.value, ur[:ran], zv[:ran]

    def query(self, probes, v_enc, g, t_list, v_seeds, trials, k):
        pr = np.ascontiguousarray(probes, np.uint32)
        B, nprobe = pr.shape
        v = _u64(v_enc).reshape(B, N)
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seeds = None if v_seeds is None else np.frombuffer(b"".join(bytes(s) for s in v_seeds), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        fc = np.zeros(B, np.int32)
        ft = np.zeros(B, np.int32)
        check(lib.bn_ivf_query(self.h, B, nprobe, ptr(pr), ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                               ptr(ts) if ts.size else None, ptr(tn), ptr(seeds), trials, k, ptr(ids), ptr(sc),
                               ptr(nh), ptr(fc), ptr(ft)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, fc, ft

    # ---- block scoring: the batch's (query, list) pairs grouped by list, Protocol 2 per block and list
    def block_prepare(self):
        check(lib.bn_ivf_block_prepare(self.h))

    def query_block(self, probes, v_enc, g, t_list, block_seed, trials, k):
        pr = np.ascontiguousarray(probes, np.uint32)
        B, nprobe = pr.shape
        v = _u64(v_enc).reshape(B, N)
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seed = None if block_seed is None else np.frombuffer(bytes(block_seed), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        fc = np.zeros(B, np.int32)
        ft = np.zeros(B, np.int32)
        check(lib.bn_ivf_query_block(self.h, B, nprobe, ptr(pr), ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                                     ptr(ts) if ts.size else None, ptr(tn), ptr(seed), trials, k, ptr(ids), ptr(sc),
                                     ptr(nh), ptr(fc), ptr(ft)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, fc, ft

    IVF_BLOCK_STAGES = ("host_plan_pack", "h2d_operand_images", "g1_r", "g2_al_h", "g3_m_t_s_v", "topk",
                        "protocol2_u_draws", "protocol2_z_passes", "protocol2_u_dot_r", "zv_decide", "d2h")

    def block_tune(self, w_tile=0, stages=0):
        """GEMM tiling of later block calls: W rows per tile, pipeline stages (0 = automatic)."""
        check(lib.bn_ivf_block_tune(self.h, w_tile, stages))

    def block_profile(self, enable=True):
        check(lib.bn_ivf_block_profile(self.h, 1 if enable else 0))

    def block_profile_read(self):
        """Stage times (ms) of the last profiled query_block, by stage name."""
        ms = np.zeros(len(self.IVF_BLOCK_STAGES), np.float32)
        n = u32(0)
        check(lib.bn_ivf_block_profile_read(self.h, ptr(ms), len(ms), C.byref(n)))
        return {k: float(v) for k, v in zip(self.IVF_BLOCK_STAGES, ms[: n.value])}

    def pairs(self, probes):
        """(query, list, rows) of every (query, list) pair of a batch in probe order, empty lists skipped:
        the layout of the r argument of verify_block."""
        out = []
        for q, row in enumerate(np.asarray(probes)):
            for c in row:
                m = int(self.offsets[c + 1] - self.offsets[c])
                if m:
                    out.append((q, int(c), m))
        return out

    def verify_block(self, probes, r, v_enc, block_seed, trials):
        """Protocol 2 over claimed responses r (every pair's r in probe order, concatenated):
        per query (failed_cluster, failed_trial), and per pair and trial u_t . r and z_t . v."""
        pr = np.ascontiguousarray(probes, np.uint32)
        B, nprobe = pr.shape
        r = _u64(r).reshape(-1)
        v = _u64(v_enc).reshape(B, N)
        seed = np.frombuffer(bytes(block_seed), np.uint8).copy()
        npairs = len(self.pairs(pr))
        fc = np.zeros(B, np.int32)
        ft = np.zeros(B, np.int32)
        ur = np.zeros((max(npairs, 1), trials), np.uint64)
        zv = np.zeros((max(npairs, 1), trials), np.uint64)
        check(lib.bn_ivf_verify_block(self.h, B, nprobe, ptr(pr), ptr(r) if r.size else None, r.size, ptr(v),
                                      ptr(seed), trials, ptr(fc), ptr(ft), ptr(ur), ptr(zv)))
        return fc, ft, ur[:npairs], zv[:npairs]

    def close(self):
        if self.h:
            lib.bn_ivf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


class Server:
    """bn_server: continuous batching of flat and IVF queries over resident corpora."""

    def __init__(self, flat=None, ivf=None, max_batch=64, slots=4, mem_budget=0, max_wait_us=200, trials=20, k=10,
                 block_min=0, max_queue=0, queue_wait_us=0):
        self.flat, self.ivf, self.k = flat, ivf, k
        cfg = ServerConfig(max_batch, slots, mem_budget, max_wait_us, trials, k, block_min, max_queue, queue_wait_us)
        out = vp()
        check(lib.bn_server_create(flat.h if flat else None, ivf.h if ivf else None, C.byref(cfg), C.byref(out)))
        self.h = out

    def submit_flat(self, v_enc, g, t_idx, t_sign, v_seed) -> int:
        v, gg = _u64(v_enc), _u64(g)
        ti, ts = np.ascontiguousarray(t_idx, np.uint32), np.ascontiguousarray(t_sign, np.int8)
        seed = None if v_seed is None else np.frombuffer(bytes(v_seed), np.uint8).copy()
        t = u64(0)
        check(lib.bn_server_submit_flat(self.h, ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                                        ptr(ts) if ts.size else None, ti.size, ptr(seed), C.byref(t)))
        return t.value

    def submit_ivf(self, probes, v_enc, g, t_idx, t_sign, v_seed) -> int:
        pr = np.ascontiguousarray(probes, np.uint32)
        v, gg = _u64(v_enc), _u64(g)
        ti, ts = np.ascontiguousarray(t_idx, np.uint32), np.ascontiguousarray(t_sign, np.int8)
        seed = None if v_seed is None else np.frombuffer(bytes(v_seed), np.uint8).copy()
        t = u64(0)
        check(lib.bn_server_submit_ivf(self.h, pr.size, ptr(pr) if pr.size else None, ptr(v), ptr(gg),
                                       ptr(ti) if ti.size else None, ptr(ts) if ts.size else None, ti.size,
                                       ptr(seed), C.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60000):
        """(ids, scores, failed_trial, failed_cluster, latency_us); raises BnError(EAGAIN) on timeout."""
        kk = max(self.k, 1)
        ids = np.zeros(kk, np.uint32)
        sc = np.zeros(kk, np.int64)
        nh, ft, fc, lat = u32(0), i32(0), i32(0), C.c_double(0)
        check(lib.bn_server_wait(self.h, ticket, timeout_ms, ptr(ids), ptr(sc), C.byref(nh), C.byref(ft),
                                 C.byref(fc), C.byref(lat)))
        return ids[: nh.value].copy(), sc[: nh.value].copy(), ft.value, fc.value, lat.value

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        check(lib.bn_server_stats(self.h, 1 if reset else 0, C.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib.bn_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


def keygen_h_s(ctx, h_seed: bytes, m: int, n1: int = 128):
    """bn_keygen_h_s: (H, rowptr, idx, sign) drawn on the device."""
    seed = np.frombuffer(bytes(h_seed), np.uint8).copy()
    H = np.zeros(max(m * n1, 1), np.uint64)
    rowptr = np.zeros(m + 1, np.uint64)
    cap = max(m * 160, 1024)
    nnz = u64(0)
    while True:
        idx = np.zeros(cap, np.uint32)
        sign = np.zeros(cap, np.int8)
        rc = lib.bn_keygen_h_s(ctx.h, ptr(seed), m, n1, ptr(H), ptr(rowptr), ptr(idx), ptr(sign), cap, C.byref(nnz))
        if rc == BN_EINVAL and nnz.value > cap:
            cap = nnz.value
            continue
        check(rc)
        return H[: m * n1], rowptr, idx[: nnz.value], sign[: nnz.value]


def encrypt_cluster(ctx, m_q, m, L, H, s_rowptr, s_idx, s_sign, n1=128):
    m_q, L, H = _u64(m_q), _u64(L), _u64(H)
    csr, keep = _csr(s_rowptr, s_idx, s_sign)
    m_enc = np.zeros(max(m * N, 1), np.uint64)
    al = np.zeros(max(m * n1, 1), np.uint64)
    check(lib.bn_encrypt_cluster(ctx.h, ptr(m_q), m, N, n1, ptr(L), ptr(H), csr, ptr(m_enc), ptr(al)))
    return m_enc[: m * N], al[: m * n1]


# ---------------------------------------------------------------- host side (include/bn_host.h)
_HOST_SIGS = {
    "bn_host_mu": (C.c_double, []),
    "bn_host_default_trials": (u32, []),
    "bn_host_domain_separate": (None, [vp, C.c_char_p, vp]),
    "bn_host_derive_h_seed": (None, [u64, u64, vp]),
    "bn_host_generate_subspace": (None, [vp, u32, u32, vp]),
    "bn_host_regenerate_h_s": (C.c_int64, [vp, u64, u32, u32, vp, vp, vp, vp, u64]),
    "bn_host_regenerate_h_s_lists": (C.c_int64, [u64, u32, vp, u32, u32, vp, vp, vp, vp, u64]),
    "bn_host_quantise": (None, [vp, u64, u32, u32, u64, vp]),
    "bn_host_encode_query": (u32, [vp, vp, u32, u32, vp, vp, vp, vp, vp]),
    "bn_host_probe_route": (None, [vp, u32, u32, vp, u64, u32, vp]),
    "bn_host_cache_fingerprint": (u64, [vp, vp, u32]),
    "bn_host_ivf_cache_open": (C.c_int, [C.c_char_p, u64, u32, u32, C.POINTER(vp)]),
    "bn_host_ivf_cache_close": (None, [vp]),
    "bn_host_ivf_cache_info": (None, [vp, vp, vp, vp]),
    "bn_host_ivf_cache_lists": (None, [vp, vp, vp, vp, vp]),
    "bn_host_ivf_cache_arrays": (None, [vp, vp, vp, vp, vp, vp]),
}
for _name, (_res, _args) in _HOST_SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def _seed_arr(s) -> np.ndarray:
    a = np.frombuffer(bytes(s), np.uint8).copy()
    assert a.size == 32
    return a


def host_domain_separate(seed: bytes, tag: str = "protocol2") -> bytes:
    out = np.zeros(32, np.uint8)
    lib.bn_host_domain_separate(ptr(_seed_arr(seed)), tag.encode(), ptr(out))
    return out.tobytes()


def host_derive_h_seed(upload_seed: int, ci: int) -> bytes:
    out = np.zeros(32, np.uint8)
    lib.bn_host_derive_h_seed(upload_seed, ci, ptr(out))
    return out.tobytes()


def host_generate_subspace(key_seed: bytes, n1: int = 128) -> np.ndarray:
    L = np.zeros(N * n1, np.uint64)
    lib.bn_host_generate_subspace(ptr(_seed_arr(key_seed)), N, n1, ptr(L))
    return L


def host_regenerate_h_s(h_seed: bytes, m: int, n1: int = 128):
    H = np.zeros(max(m * n1, 1), np.uint64)
    rowptr = np.zeros(m + 1, np.uint64)
    cap = max(m * 160, 1024)
    while True:
        idx = np.zeros(cap, np.uint32)
        sign = np.zeros(cap, np.int8)
        nnz = lib.bn_host_regenerate_h_s(ptr(_seed_arr(h_seed)), m, N, n1, ptr(H), ptr(rowptr), ptr(idx), ptr(sign), cap)
        if nnz >= 0:
            return H[: m * n1], rowptr, idx[:nnz], sign[:nnz]
        cap = -nnz


def host_regenerate_h_s_lists(upload_seed: int, offsets, n1: int = 128):
    off = _u64(offsets)
    rows = int(off[-1])
    H = np.zeros(max(rows * n1, 1), np.uint64)
    rowptr = np.zeros(rows + 1, np.uint64)
    cap = max(rows * 160, 1024)
    while True:
        idx = np.zeros(cap, np.uint32)
        sign = np.zeros(cap, np.int8)
        nnz = lib.bn_host_regenerate_h_s_lists(upload_seed, len(off) - 1, ptr(off), N, n1, ptr(H), ptr(rowptr),
                                               ptr(idx), ptr(sign), cap)
        if nnz >= 0:
            return H[: rows * n1], rowptr, idx[:nnz], sign[:nnz]
        cap = -nnz


def host_quantise(v, q: int = 1 << 20) -> np.ndarray:
    v = np.ascontiguousarray(v, np.float32)
    if v.ndim == 1:
        v = v[None]
    out = np.zeros((v.shape[0], N), np.uint64)
    lib.bn_host_quantise(ptr(v), v.shape[0], v.shape[1], N, q, ptr(out))
    return out


def host_encode_query(v_q, L, q_seed: bytes, n1: int = 128):
    v_q, L = _u64(v_q), _u64(L)
    v_enc = np.zeros(N, np.uint64)
    g = np.zeros(n1, np.uint64)
    ti = np.zeros(N, np.uint32)
    ts = np.zeros(N, np.int8)
    c = lib.bn_host_encode_query(ptr(v_q), ptr(L), N, n1, ptr(_seed_arr(q_seed)), ptr(v_enc), ptr(g), ptr(ti), ptr(ts))
    return v_enc, g, ti[:c].copy(), ts[:c].copy()


def host_probe_route(centroids, queries, nprobe: int) -> np.ndarray:
    c = np.ascontiguousarray(centroids, np.float32)
    q = np.ascontiguousarray(queries, np.float32)
    if q.ndim == 1:
        q = q[None]
    np_ = min(nprobe, c.shape[0])
    out = np.zeros((q.shape[0], np_), np.uint32)
    lib.bn_host_probe_route(ptr(c), c.shape[0], c.shape[1], ptr(q), q.shape[0], nprobe, ptr(out))
    return out


# ---------------------------------------------------------------- reference IVF cache files
def cache_fingerprint(parts) -> int:
    """scorer-core/src/cache.rs fingerprint64 of byte strings `parts`."""
    bufs = [np.frombuffer(bytes(pt), np.uint8).copy() if len(pt) else np.zeros(1, np.uint8) for pt in parts]
    ptrs = (vp * max(len(bufs), 1))(*[b.ctypes.data for b in bufs])
    lens = np.array([len(pt) for pt in parts] or [0], np.uint64)
    return int(lib.bn_host_cache_fingerprint(ptrs, ptr(lens), len(parts)))


def bntm_ivf_cache_parts(n_centroids: int, train_seed: int, max_iter: int, n_vectors: int, upload_seed: int,
                         key_seed: bytes, n1: int, quantisation_q: int) -> list:
    """The reference's fingerprint parts of a BN-IVF cache (scorer-bntm/src/ivf.rs:321-331)."""
    le = lambda x: int(x).to_bytes(8, "little")
    return [b"bntm-ivf2", le(n_centroids), le(train_seed), le(max_iter), le(n_vectors), le(upload_seed),
            bytes(key_seed), le(n1), le(quantisation_q)]


def bntm_ivf_cache_name(*args, **kw) -> tuple:
    """(fingerprint, file name) of the reference's cache for these parameters (ivf.rs:332-337)."""
    fp = cache_fingerprint(bntm_ivf_cache_parts(*args, **kw))
    return fp, f".bntm-ivf-cache-{fp:016x}.bin"


class IvfCache:
    """A `.bntm-ivf-cache-*.bin` file of the reference, mapped and indexed
    (bn_host_ivf_cache_open); fingerprint 0 accepts any parameters."""

    def __init__(self, path: str, fingerprint: int = 0, n1: int = 128):
        self.h = None
        h = vp()
        check(lib.bn_host_ivf_cache_open(str(path).encode(), fingerprint, N, n1, C.byref(h)))
        self.h, self.n1 = h, n1
        nl, dim, rows = u32(0), u32(0), u64(0)
        lib.bn_host_ivf_cache_info(self.h, C.byref(nl), C.byref(dim), C.byref(rows))
        self.nlist, self.dim, self.rows = nl.value, dim.value, rows.value

    def lists(self):
        """(list_offsets, ids, centroids [nlist, dim] f32, h_seeds [nlist, 32] u8)."""
        off = np.zeros(self.nlist + 1, np.uint64)
        ids = np.zeros(max(self.rows, 1), np.uint32)
        cen = np.zeros((max(self.nlist, 1), max(self.dim, 1)), np.float32)
        hs = np.zeros((max(self.nlist, 1), 32), np.uint8)
        lib.bn_host_ivf_cache_lists(self.h, ptr(off), ptr(ids), ptr(cen), ptr(hs))
        return off, ids[: self.rows], cen[: self.nlist, : self.dim], hs[: self.nlist]

    def arrays(self):
        """Concatenated list-order arrays: m_enc [rows, n], a_l [rows, n1],
        m_plain [rows, n], h [rows, n1], l_subspace [n, n1]."""
        r, n1 = self.rows, self.n1
        me, mp = np.zeros((max(r, 1), N), np.uint64), np.zeros((max(r, 1), N), np.uint64)
        al, hh = np.zeros((max(r, 1), n1), np.uint64), np.zeros((max(r, 1), n1), np.uint64)
        L = np.zeros((N, n1), np.uint64)
        lib.bn_host_ivf_cache_arrays(self.h, ptr(me), ptr(al), ptr(mp), ptr(hh), ptr(L))
        return {"m_enc": me[:r], "a_l": al[:r], "m_plain": mp[:r], "h": hh[:r], "l_subspace": L}

    def s_lists(self):
        """S of every list, regenerated from its h_seed (crypto.rs:258-270),
        concatenated in list order as one CSR (rowptr, idx, sign)."""
        off, _, _, hs = self.lists()
        rowptr, idx, sign = [np.zeros(1, np.uint64)], [], []
        base = 0
        for c in range(self.nlist):
            m = int(off[c + 1] - off[c])
            _, rp, ix, sg = host_regenerate_h_s(hs[c].tobytes(), m, self.n1)
            rowptr.append(rp[1:] + np.uint64(base))
            idx.append(ix)
            sign.append(sg)
            base += len(ix)
        cat = lambda xs, t: np.concatenate(xs).astype(t) if xs else np.zeros(0, t)
        return np.concatenate(rowptr).astype(np.uint64), cat(idx, np.uint32), cat(sign, np.int8)

    def close(self):
        if self.h:
            lib.bn_host_ivf_cache_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


def ivf_from_cache(ctx, path: str, fingerprint: int = 0, n1: int = 128):
    """Device IVF handle (server and client state) from a reference cache
    file: bn_ivf_build on its m_enc / a_l / h and ids, then
    bn_ivf_attach_client with its L, m_plain and the regenerated S.
    Returns (Ivf, centroids) -- the centroids route queries
    (host_probe_route)."""
    cache = IvfCache(path, fingerprint, n1)
    off, ids, cen, _ = cache.lists()
    a = cache.arrays()
    rp, ix, sg = cache.s_lists()
    cache.close()
    v = Ivf.build(ctx, off, ids, a["m_enc"].reshape(-1), a["a_l"].reshape(-1), a["h"].reshape(-1), n1=n1)
    v.attach_client(a["l_subspace"].reshape(-1), a["m_plain"].reshape(-1), rp, ix, sg)
    return v, cen


def _store_stats(st: StoreStats) -> dict:
    return {f: getattr(st, f) for f, _ in StoreStats._fields_}


class Stream:
    """bn_stream: a flat corpus streamed through device memory in chunks
    (the reference's ClusterStore, scorer-gpu-common/src/store.rs:247-395)."""

    def __init__(self, ctx: Context, handle, m: int, n1: int):
        self.ctx, self.h, self.m, self.n1 = ctx, handle, m, n1

    @classmethod
    def build(cls, ctx, m_enc, a_l, h, m, L, m_plain, s_rowptr, s_idx, s_sign, chunk_rows, budget_bytes, n1=128):
        m_enc, a_l, h, L, m_plain = _u64(m_enc), _u64(a_l), _u64(h), _u64(L), _u64(m_plain)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        out = vp()
        check(lib.bn_stream_build(ctx.h, ptr(m_enc), ptr(a_l), ptr(h), m, N, n1, ptr(L), ptr(m_plain), csr,
                                  chunk_rows, budget_bytes, C.byref(out)))
        return cls(ctx, out, m, n1)

    @classmethod
    def build_from_plain(cls, ctx, m_q, m, L, H, s_rowptr, s_idx, s_sign, chunk_rows, budget_bytes, n1=128):
        m_q, L, H = _u64(m_q), _u64(L), _u64(H)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        out = vp()
        check(lib.bn_stream_build_from_plain(ctx.h, ptr(m_q), m, N, n1, ptr(L), ptr(H), csr, chunk_rows,
                                             budget_bytes, C.byref(out)))
        return cls(ctx, out, m, n1)

    def info(self) -> dict:
        rows, chunks, slots, sb, hb = u64(), u32(), u32(), u64(), u64()
        check(lib.bn_stream_info(self.h, C.byref(rows), C.byref(chunks), C.byref(slots), C.byref(sb), C.byref(hb)))
        return {"rows": rows.value, "chunks": chunks.value, "slots": slots.value, "slot_bytes": sb.value,
                "host_bytes": hb.value}

    def query(self, v_enc, g, t_list, v_seeds, trials, k):
        """Same arguments as Flat.query; returns (hits, failed_trial)."""
        v = _u64(v_enc).reshape(-1, N)
        B = v.shape[0]
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seeds = None if v_seeds is None else np.frombuffer(b"".join(bytes(s) for s in v_seeds), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        fl = np.zeros(B, np.int32)
        check(lib.bn_stream_query(self.h, B, ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                                  ptr(ts) if ts.size else None, ptr(tn), ptr(seeds), trials, k, ptr(ids), ptr(sc),
                                  ptr(nh), ptr(fl)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, fl

    def stats(self, reset=False) -> dict:
        st = StoreStats()
        check(lib.bn_stream_stats(self.h, 1 if reset else 0, C.byref(st)))
        return _store_stats(st)

    def close(self):
        if getattr(self, "h", None):
            lib.bn_stream_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


class IvfStream:
    """bn_ivf_stream: an IVF corpus streamed through device memory in chunks of
    whole lists (the reference's per-cluster ClusterStore uploads)."""

    def __init__(self, ctx: Context, handle, nlist: int, n1: int):
        self.ctx, self.h, self.nlist, self.n1 = ctx, handle, nlist, n1

    @classmethod
    def build(cls, ctx, offsets, ids, m_enc, a_l, h, L, m_plain, s_rowptr, s_idx, s_sign, chunk_rows, budget_bytes,
              n1=128):
        off = np.ascontiguousarray(offsets, np.uint64)
        ids = np.ascontiguousarray(ids, np.uint32)
        m_enc, a_l, h, L, m_plain = _u64(m_enc), _u64(a_l), _u64(h), _u64(L), _u64(m_plain)
        csr, keep = _csr(s_rowptr, s_idx, s_sign)
        out = vp()
        check(lib.bn_ivf_stream_build(ctx.h, off.size - 1, ptr(off), ptr(ids), ptr(m_enc), ptr(a_l), ptr(h), N, n1,
                                      ptr(L), ptr(m_plain), csr, chunk_rows, budget_bytes, C.byref(out)))
        return cls(ctx, out, off.size - 1, n1)

    @classmethod
    def build_keygen(cls, ctx, offsets, ids, m_q, L, upload_seed: int, chunk_rows, budget_bytes, n1=128):
        off = np.ascontiguousarray(offsets, np.uint64)
        ids = np.ascontiguousarray(ids, np.uint32)
        m_q, L = _u64(m_q), _u64(L)
        out = vp()
        check(lib.bn_ivf_stream_build_keygen(ctx.h, off.size - 1, ptr(off), ptr(ids), ptr(m_q), N, n1, ptr(L),
                                             upload_seed, chunk_rows, budget_bytes, C.byref(out)))
        return cls(ctx, out, off.size - 1, n1)

    def info(self) -> dict:
        rows, chunks, slots, sb, hb = u64(), u32(), u32(), u64(), u64()
        check(lib.bn_ivf_stream_info(self.h, C.byref(rows), C.byref(chunks), C.byref(slots), C.byref(sb),
                                     C.byref(hb)))
        return {"rows": rows.value, "chunks": chunks.value, "slots": slots.value, "slot_bytes": sb.value,
                "host_bytes": hb.value}

    def query(self, probes, v_enc, g, t_list, v_seeds, trials, k):
        """Same arguments as Ivf.query; returns (hits, failed_cluster, failed_trial)."""
        pr = np.ascontiguousarray(probes, np.uint32)
        B, nprobe = pr.shape
        v = _u64(v_enc).reshape(B, N)
        gg = _u64(g).reshape(B, self.n1)
        ti, ts, tn = _t_concat(t_list)
        seeds = None if v_seeds is None else np.frombuffer(b"".join(bytes(s) for s in v_seeds), np.uint8).copy()
        kk = max(k, 1)
        ids = np.zeros((B, kk), np.uint32)
        sc = np.zeros((B, kk), np.int64)
        nh = np.zeros(B, np.uint32)
        fc = np.zeros(B, np.int32)
        ft = np.zeros(B, np.int32)
        check(lib.bn_ivf_stream_query(self.h, B, nprobe, ptr(pr), ptr(v), ptr(gg), ptr(ti) if ti.size else None,
                                      ptr(ts) if ts.size else None, ptr(tn), ptr(seeds), trials, k, ptr(ids), ptr(sc),
                                      ptr(nh), ptr(fc), ptr(ft)))
        hits = [(ids[b, : nh[b]].copy(), sc[b, : nh[b]].copy()) for b in range(B)]
        return hits, fc, ft

    def stats(self, reset=False) -> dict:
        st = StoreStats()
        check(lib.bn_ivf_stream_stats(self.h, 1 if reset else 0, C.byref(st)))
        return _store_stats(st)

    def close(self):
        if getattr(self, "h", None):
            lib.bn_ivf_stream_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


class Lru:
    """bn_lru: the store's CUDA-free LRU bookkeeping (LruInner, store.rs:133-245)."""

    def __init__(self, budget_bytes: int):
        out = vp()
        check(lib.bn_lru_create(budget_bytes, C.byref(out)))
        self.h = out

    def touch(self, cid: int) -> bool:
        hit = C.c_int(0)
        check(lib.bn_lru_touch(self.h, cid, C.byref(hit)))
        return bool(hit.value)

    def pre_evict(self, nbytes: int) -> list:
        """Evicted ids, least recently used first; BnError(BN_EBUDGET) when nbytes cannot fit."""
        cap = 4096
        ev = np.zeros(cap, np.uint64)
        n = u32(0)
        check(lib.bn_lru_pre_evict(self.h, nbytes, ptr(ev), cap, C.byref(n)))
        return [int(x) for x in ev[: n.value]]

    def insert(self, cid: int, nbytes: int) -> bool:
        ins = C.c_int(0)
        check(lib.bn_lru_insert(self.h, cid, nbytes, C.byref(ins)))
        return bool(ins.value)

    def stats(self) -> dict:
        st = StoreStats()
        check(lib.bn_lru_stats(self.h, C.byref(st)))
        return _store_stats(st)

    def close(self):
        if getattr(self, "h", None):
            lib.bn_lru_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):
            pass
