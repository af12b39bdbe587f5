"""Test model of the reference's live layer (src/live.rs) on the oracle: inserts encoded by the
oracle's restatement of Live::apply_insert, per-cluster delta lists scanned right after each base
list, tombstones hiding rows, external ids. Searching it builds the index a View with those delta
lists and tombstones amounts to: every cluster's base blocks followed by its delta list's blocks
(the scan admits them in that order; padding slots inside are skipped as PAD), the delta rows
appended to the corpus rows, and every live row allowed. It is the checker the GPU's live index is
compared with."""
import numpy as np

import oracle as O


class OracleLive:
    def __init__(self, arrays: dict, soar_lambda: float | None = 1.0):
        self.base = arrays
        self.n, self.k = int(arrays["n"]), int(arrays["k"])
        cents = np.asarray(arrays["centroids"], np.float32).reshape(self.k, 256)
        self.cents_rot = np.stack([O.rotation_apply(arrays["rotation"], c) for c in cents]).astype(np.float32)
        self.soar, self.lam = soar_lambda is not None, float(soar_lambda or 0.0)
        self.oi = O.OracleIndex(arrays)
        self.lists = [[] for _ in range(self.k)]  # (code [32], mul, err, row)
        self.rows, self.norm, self.t2, self.t2n, self.ext = [], [], [], [], []
        self.deleted, self.by_ext = set(), {}

    def current(self, e: int):
        if e in self.by_ext:
            return self.by_ext[e]
        return e if e < self.n and e not in self.deleted else None

    def insert(self, ext_ids, vecs):
        for e, v in zip(ext_ids, np.asarray(vecs, np.float32)):
            row, nrm, pair, codes, fac, t2, t2n = self.oi.live_encode(self.cents_rot, self.soar, self.lam, v)
            old = self.current(int(e))
            if old is not None:
                self.deleted.add(old)
            rid = self.n + len(self.ext)
            self.ext.append(int(e))
            self.by_ext[int(e)] = rid
            self.rows.append(row)
            self.norm.append(nrm)
            self.t2.append(t2)
            self.t2n.append(t2n)
            for h in range(2):
                if pair[h] != 0xFFFFFFFF:
                    self.lists[int(pair[h])].append((codes[h].copy(), fac[h, 0], fac[h, 1], rid))

    def delete(self, ext_ids):
        for e in ext_ids:
            rid = self.current(int(e))
            if rid is not None:
                self.deleted.add(rid)
                self.by_ext.pop(int(e), None)

    def merged(self) -> dict:
        a = self.base
        boff = np.asarray(a["block_off"], np.int64)
        blocks = np.asarray(a["blocks"]).reshape(-1, 1024)
        ids = np.asarray(a["ids"]).reshape(-1, 32)
        fac = np.asarray(a["factors"]).reshape(-1, 64)
        ob, oi, of, off = [], [], [], [0]
        for c in range(self.k):
            ob.append(blocks[boff[c]:boff[c + 1]])
            oi.append(ids[boff[c]:boff[c + 1]])
            of.append(fac[boff[c]:boff[c + 1]])
            nb = boff[c + 1] - boff[c]
            lst = self.lists[c]
            for i in range(0, len(lst), 32):
                part = lst[i:i + 32]
                ob.append(O.pack_block(np.stack([x[0] for x in part]))[None])
                bid = np.full(32, 0xFFFFFFFF, np.uint32)
                bf = np.zeros(64, np.float32)
                for j, x in enumerate(part):
                    bid[j], bf[2 * j], bf[2 * j + 1] = x[3], x[1], x[2]
                oi.append(bid[None])
                of.append(bf[None])
                nb += 1
            off.append(off[-1] + nb)
        out = dict(a)
        out["block_off"] = np.asarray(off, np.uint64)
        out["blocks"] = np.concatenate(ob).reshape(-1)
        out["ids"] = np.concatenate(oi).reshape(-1)
        out["factors"] = np.concatenate(of).reshape(-1)
        d = len(self.rows)
        out["n"] = self.n + d
        if d:
            out["rerank"] = np.concatenate([a["rerank"], np.stack(self.rows)])
            out["norm256"] = np.concatenate([a["norm256"], np.asarray(self.norm, np.float32)])
            if a.get("tier2_codes") is not None:
                out["tier2_codes"] = np.concatenate([a["tier2_codes"], np.stack(self.t2)])
                out["tier2_norm"] = np.concatenate([a["tier2_norm"], np.asarray(self.t2n, np.float32)])
        return out

    def search_batch(self, q768, q256, params):
        m = self.merged()
        oi = O.OracleIndex(m)
        nrows = int(m["n"])
        alive = np.ones(nrows, bool)
        alive[list(self.deleted)] = False
        pad = (-nrows) % 64
        bits = np.packbits(np.concatenate([alive, np.zeros(pad, bool)]), bitorder="little").view(np.uint64)
        k = max(params.k, 1)
        sc = np.zeros((len(q768), k), np.float32)
        ids = np.zeros((len(q768), k), np.uint32)
        cnt = np.zeros(len(q768), np.uint32)
        for i in range(len(q768)):
            s, o, _ = oi.search(q768[i], q256[i], params.to_c(), bits)
            cnt[i] = len(o)
            sc[i, : len(o)] = s
            ids[i, : len(o)] = [r if r < self.n else self.ext[r - self.n] for r in o]
        return sc[:, : params.k], ids[:, : params.k], cnt
