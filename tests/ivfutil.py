"""Small IVF instances built list by list with the oracle (ivf.rs:627-653)."""
from __future__ import annotations

import numpy as np

import oracle as O
from bnutil import N, P, int8_matrix


class IvfCase:
    def __init__(self, sizes, seed=5, d=768, key_seed=bytes([2]) * 32, upload_seed=7, n1=128):
        self.sizes = list(sizes)
        self.n1 = n1
        self.nlist = len(sizes)
        total = sum(sizes)
        self.M = int8_matrix(total, d, seed)
        self.ids = np.random.default_rng(seed).permutation(total).astype(np.uint32)
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
        self.L = O.generate_subspace(key_seed, n1=n1)
        self.clusters = []
        for ci, m in enumerate(sizes):
            o = int(self.offsets[ci])
            self.clusters.append(O.encrypt_cluster(self.M[o : o + m].reshape(-1), m, self.L,
                                                   O.derive_h_seed(upload_seed, ci), n1=n1) if m else None)

    def concat(self):
        cs = [c for c in self.clusters if c is not None]
        m_enc = np.concatenate([c.m_enc for c in cs])
        a_l = np.concatenate([c.a_l for c in cs])
        h = np.concatenate([c.h_mat for c in cs])
        rowptr = [np.zeros(1, np.uint64)]
        idx, sign, base = [], [], 0
        for c in cs:
            rowptr.append(c.s_mat.rowptr[1:] + np.uint64(base))
            idx.append(c.s_mat.idx)
            sign.append(c.s_mat.sign)
            base += int(c.s_mat.rowptr[-1])
        return m_enc, a_l, h, np.concatenate(rowptr), np.concatenate(idx), np.concatenate(sign)

    def oracle_score(self, probes, enc, v_seed, trials, k):
        """BnTmIvfScorer::score CPU path (ivf.rs:778-823) for given probes."""
        allid, allsc = [], []
        for ci in probes:
            cl = self.clusters[ci]
            if cl is None:
                continue
            r = O.matvec(cl.m_enc, cl.m, N, enc.v_enc)
            if trials:
                f, _, _ = O.verify_response(r, cl.m_enc, cl.m, N, enc.v_enc, trials, v_seed)
                if f >= 0:
                    return ("fail", ci, f)
            mv = O.decode_scores(r, cl, self.L, enc)
            o = int(self.offsets[ci])
            allid.append(self.ids[o : o + cl.m])
            allsc.append(O.to_signed(mv))
        if not allid:
            return np.zeros(0, np.uint32), np.zeros(0, np.int64)
        return O.topk(np.concatenate(allsc), k, ids=np.concatenate(allid))
