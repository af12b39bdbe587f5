"""Test adapter: a shard's phase-1 and phase-2 computations by the oracle (the reference's
Index::route / candidates / rerank restated), with the methods of sieve_gpu.Index that the
two-phase protocol of sieve_gpu.shard calls. It is the checker the GPU shards are compared to,
and it lets the protocol's exchange run on CPU ranks."""
import numpy as np

import oracle as O


class OracleShard:
    def __init__(self, arrays: dict):
        self.oi = O.OracleIndex(arrays)
        self.k = int(arrays["k"])

    def route(self, q256, params):
        return [self.oi.route(q, params.to_c()) for q in np.asarray(q256, np.float32)]

    def candidates_probes(self, q256, probes, params, allow=None):
        out = []
        for q, (sc, cl) in zip(np.asarray(q256, np.float32), probes):
            out.append(self.oi.candidates(q, np.asarray(sc, np.float32), np.asarray(cl, np.uint32), params.to_c(),
                                          allow))
        return out

    def rerank(self, q768, q256, cands, params):
        k = max(params.k, 1)
        nq = len(cands)
        sc = np.zeros((nq, k), np.float32)
        ids = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        for i, (e, r, w) in enumerate(cands):
            w = np.zeros(len(r), np.float32) if w is None else w
            s, o = self.oi.rerank(q768[i], q256[i], e, r, w, params.to_c())
            cnt[i] = len(o)
            sc[i, : len(o)], ids[i, : len(o)] = s, o
        return sc[:, : params.k], ids[:, : params.k], cnt
