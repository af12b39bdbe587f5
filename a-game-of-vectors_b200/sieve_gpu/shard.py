"""Cluster sharding across GPUs with the reference's two-phase merge (src/shard.rs).

Clusters are partitioned across ranks (one process per GPU) by the reference's longest-processing-
time balance on stored slots (`assign`, src/shard.rs:31-46), and each rank's index holds only the
slots of the clusters it owns (`shard_arrays`; centroids and corpus rows are whole on every rank,
so routing is global and every rank can rerank any row it returns). A batch runs as the
reference's two-phase protocol (Client::two_phase, src/shard.rs:249-299), with the TCP rounds
replaced by collectives over the ranks:

  1. every rank routes the batch against the global centroids (the same probe lists on every
     rank) and scans the probes it owns: Index::candidates over given probes, (estimate, row,
     error) triples (`phase1`, sg_candidates_probes);
  2. one all-gather of the triples; every rank makes the same global cut (`global_cut`): the best
     `cand` estimates of the union, deduplicated by row, bound-pruned, and the rows split back to
     the rank that returned each (estimates are calibrated inner products, so they compare across
     ranks);
  3. every rank reranks its share (`phase2`, sg_rerank), and a second all-gather brings the
     (score, row) lists to every rank, which keep each row's best score and the top k (`merge`).

With Rerank::None the estimates are the answer and the second round is skipped; Rerank::Ssd(r)
cuts to r globally before it; Rerank::Tiered(r) gives each rank its share ceil(r * rows / n) of r,
as the reference's coordinator does. The union is cut by (estimate desc, row asc) where the
reference's unstable sort leaves ties unspecified.

The exchange is `torch.distributed.all_gather_object` (NCCL between GPUs, gloo on the host).
Phase 1 and phase 2 take any object with the `Index` methods route / candidates_probes / rerank,
so the protocol runs unchanged over other implementations of them.
"""
from __future__ import annotations

import math

import numpy as np

from .index import Params, Rerank
from . import _abi


# ---- ownership (src/shard.rs:31-46) ----------------------------------------------------------
def cluster_slots(block_off) -> np.ndarray:
    """Index::slots of every cluster: stored slots, padding included."""
    b = np.asarray(block_off, np.int64)
    return (b[1:] - b[:-1]) * _abi.BLOCK


def assign(sizes, shards: int) -> np.ndarray:
    """Owner shard of every cluster: clusters by (size desc, cluster asc), each to the shard of
    least load (ties to the lower shard)."""
    sizes = np.asarray(sizes, np.int64)
    order = sorted(range(sizes.size), key=lambda c: (-int(sizes[c]), c))
    load = [0] * shards
    owner = np.zeros(sizes.size, np.uint16)
    for c in order:
        s = min(range(shards), key=lambda x: (load[x], x))
        load[s] += int(sizes[c])
        owner[c] = s
    return owner


def shard_arrays(arrays: dict, owner: np.ndarray, me: int) -> dict:
    """The index arrays of shard `me`: every cluster keeps its number, the clusters other shards
    own hold no blocks; centroids, rotation, corpus rows and tier-2 files are shared."""
    boff = np.asarray(arrays["block_off"], np.int64)
    k = boff.size - 1
    keep = np.asarray(owner)[:k] == me
    nb = np.where(keep, boff[1:] - boff[:-1], 0)
    out = dict(arrays)
    new_off = np.zeros(k + 1, np.int64)
    new_off[1:] = np.cumsum(nb)
    blocks = np.asarray(arrays["blocks"]).reshape(-1, _abi.BLOCK_BYTES)
    ids = np.asarray(arrays["ids"]).reshape(-1, _abi.BLOCK)
    sel = np.concatenate([np.arange(boff[c], boff[c + 1]) for c in range(k) if keep[c]] or
                         [np.zeros(0, np.int64)]).astype(np.int64)
    out["block_off"] = new_off.astype(np.uint64)
    out["blocks"] = np.ascontiguousarray(blocks[sel]).reshape(-1)
    out["ids"] = np.ascontiguousarray(ids[sel]).reshape(-1)
    if arrays.get("factors") is not None:
        f = np.asarray(arrays["factors"]).reshape(-1, _abi.BLOCK * 2)
        out["factors"] = np.ascontiguousarray(f[sel]).reshape(-1)
    out.pop("sizes", None)
    return out


# ---- the protocol ------------------------------------------------------------------------------
def budget_cut(probe, slots: np.ndarray, budget: int | None):
    """Index::route's scan budget (src/ivf.rs:601-611) with the global cluster sizes: clusters in
    score order while the slots taken stay within the budget, at least one."""
    sc, cl = probe
    if budget is None or len(cl) == 0:
        return sc, cl
    used = np.cumsum(slots[np.asarray(cl, np.int64)])
    keep = max(int(np.searchsorted(used, budget, side="right")), 1)
    return sc[:keep], cl[:keep]


def phase1(index, owner: np.ndarray, me: int, slots: np.ndarray, q256, params: Params, allow=None):
    """Route every query against the global centroids and scan the probes this shard owns:
    per query (estimates, rows, error widths)."""
    rp = Params(params.nprobe, params.cand, params.rerank, params.k, params.prune, params.margin, None)
    routes = [budget_cut(r, slots, params.budget) for r in index.route(q256, rp)]
    mine = []
    for sc, cl in routes:
        m = np.asarray(owner)[np.asarray(cl, np.int64)] == me
        mine.append((np.asarray(sc)[m], np.asarray(cl)[m]))
    return index.candidates_probes(q256, mine, params, allow)


def prune_threshold(est, err, m: int, w: float) -> float:
    """ivf::prune_threshold (src/ivf.rs:540-550): the m-th largest est - w*err (total order)."""
    if m == 0 or len(est) < m:
        return -math.inf
    lo = np.sort((np.asarray(est, np.float32) - np.float32(w) * np.asarray(err, np.float32)).astype(np.float32))
    return float(lo[::-1][m - 1])


def global_cut(triples: list, params: Params, shards: int):
    """The coordinator's cut of one query (src/shard.rs:252-299). triples[s] = shard s's
    (estimates, rows, error widths). Returns ('answer', [(est, row)]) when the estimates are the
    answer (Rerank::None), else ('rerank', rows[s], params[s]): each shard's (estimate, row) share
    and the params of its rerank round."""
    all_ = []
    for s, (est, rows, err) in enumerate(triples):
        all_.extend((float(e), int(r), float(w), s) for e, r, w in zip(est, rows, err))
    # the best `cand` of the union (each shard sent its best `cand`), ties by row
    all_.sort(key=lambda x: (-x[0], x[1], x[3]))
    all_ = all_[: params.cand]
    # one entry per row: its best estimate
    all_.sort(key=lambda x: (x[1], -x[0], x[3]))
    dedup, last = [], None
    for x in all_:
        if x[1] != last:
            dedup.append(x)
            last = x[1]
    all_ = dedup
    if params.prune is not None:
        m, w = params.prune
        tau = prune_threshold([x[0] for x in all_], [x[2] for x in all_], m, w)
        wf = np.float32(w)
        all_ = [x for x in all_ if float(np.float32(x[0]) + wf * np.float32(x[2])) >= tau]
    n = len(all_)
    kind = params.rerank.kind
    if kind == _abi.RERANK_NONE:
        return ("answer", [(x[0], x[1]) for x in all_])
    rerank = params.rerank
    if kind == _abi.RERANK_SSD:
        all_.sort(key=lambda x: (-x[0], x[1]))
        all_ = all_[: params.rerank.r]
    rows = [[] for _ in range(shards)]
    for x in all_:
        rows[x[3]].append((x[0], x[1]))
    ps = []
    for s in range(shards):
        if kind == _abi.RERANK_SSD:
            rr = Rerank.ssd(len(rows[s]))
        elif kind == _abi.RERANK_TIERED:
            rr = Rerank.tiered(-(-rerank.r * len(rows[s]) // max(n, 1)))
        else:
            rr = rerank
        ps.append(Params(params.nprobe, params.cand, rr, params.k, None, params.margin, params.budget))
    return ("rerank", rows, ps)


def phase2(index, q768, q256, cuts: list, me: int):
    """Rerank this shard's share of every query (queries grouped by their rerank params)."""
    nq = len(cuts)
    out = [[] for _ in range(nq)]
    groups: dict = {}
    for i, c in enumerate(cuts):
        if c[0] == "rerank" and c[1][me]:
            p = c[2][me]
            key = (p.rerank.kind, p.rerank.r)
            groups.setdefault(key, (p, []))[1].append(i)
    for p, qs in groups.values():
        cands = [(np.array([e for e, _ in cuts[i][1][me]], np.float32),
                  np.array([r for _, r in cuts[i][1][me]], np.uint32), None) for i in qs]
        sc, ids, cnt = index.rerank(np.asarray(q768)[qs], None if q256 is None else np.asarray(q256)[qs], cands, p)
        for j, i in enumerate(qs):
            out[i] = [(float(sc[j, t]), int(ids[j, t])) for t in range(int(cnt[j]))]
    return out


def merge(cut, results: list, k: int):
    """The coordinator's final merge (src/shard.rs:238-246): each row's best score over the
    shards, then the top k by (score desc, row asc)."""
    pairs = cut[1] if cut[0] == "answer" else [x for r in results for x in r]
    best: dict = {}
    for v, r in pairs:
        if r not in best or v > best[r]:
            best[r] = v
    top = sorted(best.items(), key=lambda x: (-x[1], x[0]))[:k]
    return [(v, r) for r, v in top]


class ShardedIndex:
    """This rank's shard of an index searched with the two-phase merge over a process group."""

    def __init__(self, index, owner: np.ndarray, slots: np.ndarray, me: int, shards: int, group=None):
        self.index, self.owner, self.slots = index, np.asarray(owner), np.asarray(slots)
        self.me, self.shards, self.group = me, shards, group

    def _all_gather(self, obj) -> list:
        import torch.distributed as dist

        out = [None] * self.shards
        dist.all_gather_object(out, obj, group=self.group)
        return out

    def search_batch(self, q768, q256, params: Params, allow=None):
        """Every rank returns the same (scores [nq, k], ids [nq, k], counts [nq])."""
        q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
        if q256 is None:
            p = q768[:, : _abi.PDIM]
            q256 = (p / np.sqrt((p * p).sum(1, keepdims=True, dtype=np.float32))).astype(np.float32)
        cands = phase1(self.index, self.owner, self.me, self.slots, q256, params, allow)
        every = self._all_gather([(np.asarray(e), np.asarray(r), np.asarray(w)) for e, r, w in cands])
        cuts = [global_cut([every[s][i] for s in range(self.shards)], params, self.shards)
                for i in range(q768.shape[0])]
        mine = phase2(self.index, q768, q256, cuts, self.me)
        results = self._all_gather(mine)
        return pack([merge(cuts[i], [results[s][i] for s in range(self.shards)], params.k)
                     for i in range(q768.shape[0])], params.k)


def pack(lists: list, k: int):
    """Per-query (score, row) lists as (scores [nq, k], ids [nq, k], counts [nq])."""
    nq = len(lists)
    sc = np.zeros((nq, max(k, 1)), np.float32)
    ids = np.zeros((nq, max(k, 1)), np.uint32)
    cnt = np.zeros(nq, np.uint32)
    for i, lst in enumerate(lists):
        cnt[i] = len(lst)
        for t, (v, r) in enumerate(lst):
            sc[i, t], ids[i, t] = v, r
    return sc[:, :k], ids[:, :k], cnt
