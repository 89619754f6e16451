"""Writer of the reference's BN-IVF cache file layout, for the reader's
tests (test infrastructure; the product only reads these files).

Restates the byte layout of scorer-bntm/src/ivf.rs:440-560 (the streaming
writer inside BnTmIvfScorer's index build, whose loader is ivf.rs:1755-1901),
scorer-core/src/cache.rs:46-52 (header) and ivf-index/src/ivf.rs:68-89 (IVF
payload): integers little-endian, f32 vectors, u64 residues."""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"\x89SVScach"
VERSION = 1


def fnv1a64_raw(data: bytes) -> int:
    """FNV-1a 64 of a byte string (offset basis 0xcbf29ce484222325, prime 0x100000001b3)."""
    h = 0xCBF29CE484222325
    for b in data:
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def fnv1a64(parts) -> int:
    """cache.rs:23-38 fingerprint64: FNV-1a 64 over the u64-LE-length-prefixed parts."""
    return fnv1a64_raw(b"".join(struct.pack("<Q", len(p)) + bytes(p) for p in parts))


def write_cache(path, parts, centroids, lists, l_subspace, n1=128, fingerprint=None):
    """lists: one dict per cluster with ids (m,), vecs (m, dim) f32, h_seed
    (32 bytes), m_enc (m, 1024), a_l (m, n1), m_plain (m, 1024), h (m, n1)."""
    centroids = np.asarray(centroids, np.float32)
    dim = centroids.shape[1] if centroids.size else 0
    out = bytearray()
    out += MAGIC + struct.pack("<I", VERSION)
    out += struct.pack("<Q", fnv1a64(parts) if fingerprint is None else fingerprint)
    out += struct.pack("<QQ", dim, len(centroids)) + centroids.astype("<f4").tobytes()
    out += struct.pack("<Q", len(lists))
    for c in lists:
        out += struct.pack("<Q", len(c["ids"]))
        for i, v in zip(c["ids"], np.asarray(c["vecs"], np.float32).reshape(len(c["ids"]), dim)):
            out += struct.pack("<I", int(i)) + v.astype("<f4").tobytes()
    out += b"\x00" * ((8 - len(out) % 8) % 8)
    out += struct.pack("<Q", len(lists))
    for c in lists:
        m = len(c["ids"])
        out += struct.pack("<Q", m) + bytes(c["h_seed"])
        for key, w in (("m_enc", 1024), ("a_l", n1), ("m_plain", 1024), ("h", n1)):
            out += np.asarray(c[key], np.uint64).reshape(m, w).astype("<u8").tobytes()
    out += np.asarray(l_subspace, np.uint64).astype("<u8").tobytes()
    with open(path, "wb") as f:
        f.write(bytes(out))
    return len(out)
