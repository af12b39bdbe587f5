"""The reference's query API over the GPU library: `Index`, `Params`, `Rerank`, `Timing`.

Mirrors ivf::Index / ivf::Params / ivf::Rerank / ivf::Timing (src/ivf.rs:410-633) and the config
strings of the search binary (src/bin/search.rs:180-218). Every call goes through the C ABI in
include/sieve_gpu.h; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_int, c_uint32, c_uint64, c_void_p
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import SgParams, SgStats, SgTiming, check, lib, make_arrays, ptr


# ---- ivf::Rerank (src/ivf.rs:425-439) -----------------------------------------------------------
@dataclass(frozen=True)
class Rerank:
    kind: int
    r: int = 0

    @staticmethod
    def none() -> "Rerank":
        return Rerank(_abi.RERANK_NONE)

    @staticmethod
    def prefix() -> "Rerank":
        return Rerank(_abi.RERANK_PREFIX)

    @staticmethod
    def full() -> "Rerank":
        return Rerank(_abi.RERANK_FULL)

    @staticmethod
    def tiered(r: int) -> "Rerank":
        return Rerank(_abi.RERANK_TIERED, r)

    @staticmethod
    def ssd(r: int) -> "Rerank":
        return Rerank(_abi.RERANK_SSD, r)

    def __str__(self) -> str:
        return {0: "none", 1: "prefix", 2: "full", 3: f"tiered{self.r}", 4: f"ssd{self.r}"}[self.kind]


# ---- ivf::Params (src/ivf.rs:441-460) ------------------------------------------------------------
@dataclass
class Params:
    nprobe: int
    cand: int
    rerank: Rerank = field(default_factory=Rerank.full)
    k: int = 10
    prune: tuple[int, float] | None = None
    margin: float | None = None
    budget: int | None = None

    def to_c(self) -> SgParams:
        p = SgParams()
        p.nprobe, p.cand, p.k = self.nprobe, self.cand, self.k
        p.rerank_kind, p.rerank_r = self.rerank.kind, self.rerank.r
        if self.prune is not None:
            p.has_prune, p.prune_m, p.prune_w = 1, int(self.prune[0]), float(self.prune[1])
        if self.margin is not None:
            p.has_margin, p.margin = 1, float(self.margin)
        if self.budget is not None:
            p.has_budget, p.budget = 1, int(self.budget)
        return p


def parse_config(s: str, nclusters: int) -> tuple[str, Params]:
    """`nprobe:cand:rerank[:bM[xW]][:pD][:sN[k]]` as src/bin/search.rs:180-218 (k is 100)."""
    f = s.split(":")
    if len(f) < 3:
        raise ValueError(f"config {s}: expected nprobe:cand:rerank[:bM[xW]][:pD][:sN[k]]")
    np_, cand, rr, opts = f[0], f[1], f[2], f[3:]
    prune = margin = budget = None
    for o in opts:
        key, v = o[:1], o[1:]
        if key == "b":
            m, _, w = v.partition("x")
            prune = (int(m), float(w) if w else 1.0)
        elif key == "p":
            margin = float(v)
        elif key == "s":
            mul = 1000 if v.endswith("k") else 1
            budget = int(v.rstrip("k")) * mul
        else:
            raise ValueError(f"config option {o}: expected bM[xW], pD or sN[k]")
    nprobe = nclusters if np_ == "all" else int(np_)
    if rr == "none":
        rerank = Rerank.none()
    elif rr == "prefix":
        rerank = Rerank.prefix()
    elif rr == "full":
        rerank = Rerank.full()
    elif rr.startswith("tiered"):
        rerank = Rerank.tiered(int(rr[len("tiered"):]))
    elif rr.startswith("ssd"):
        rerank = Rerank.ssd(int(rr[len("ssd"):]))
    else:
        raise ValueError("rerank must be none, prefix, full, tieredN or ssdN")
    label = f"ivf {np_} probes, {cand} cand, rerank {rr}"
    if prune is not None:
        label += f", bound-pruned at rank {prune[0]}, width {prune[1]:g}"
    if margin is not None:
        label += f", probe margin {margin:g}"
    if budget is not None:
        label += f", scan budget {budget}"
    return label, Params(nprobe, int(cand), rerank, 100, prune, margin, budget)


# ---- ivf::Timing (src/ivf.rs:521-538) ----------------------------------------------------------
@dataclass
class Timing:
    route: int = 0
    scan: int = 0
    rerank: int = 0
    tier2: int = 0
    scanned: int = 0
    reranked: int = 0
    probed: int = 0
    fetch: int = 0
    wait: int = 0

    def add(self, t: SgTiming) -> None:
        for name, _ in SgTiming._fields_:
            setattr(self, name, getattr(self, name) + getattr(t, name))


def _f32(a, rows: int, dim: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.reshape(rows, dim)


def allow_bitset(rows, n: int) -> np.ndarray:
    """View::allow as u64 words (bit r of word r/64 set for every allowed row)."""
    bits = np.zeros((n + 63) // 64, np.uint64)
    rows = np.asarray(rows, dtype=np.int64)
    np.bitwise_or.at(bits, rows >> 6, np.left_shift(np.uint64(1), (rows & 63).astype(np.uint64)))
    return bits


class Index:
    """A RaBitQ IVF index with its corpus resident in one GPU's HBM (ivf::Index + ivf::Corpus)."""

    def __init__(self, handle: c_void_p, device: int):
        self._h = handle
        self.device = device
        k, n, nb, t2 = c_uint32(), c_uint64(), c_uint64(), c_uint32()
        check(lib().sg_index_info(self._h, byref(k), byref(n), byref(nb), byref(t2)))
        self.k, self.n, self.nblocks, self.has_tier2 = k.value, n.value, nb.value, bool(t2.value)

    # ivf::Corpus::open + ivf::Index::open (src/ivf.rs:75-90, :553-578)
    @classmethod
    def open(cls, ingest_dir: str, index_dir: str, device: int = 0) -> "Index":
        h = c_void_p()
        check(lib().sg_open_ivf(ingest_dir.encode(), index_dir.encode(), c_int(device), byref(h)))
        return cls(h, device)

    @classmethod
    def from_arrays(cls, arrays: dict, device: int = 0, codes: bool = False) -> "Index":
        """Uploads the arrays; codes=True also uploads the rows' sign codes (codes.bin) for
        flat_hamming."""
        st, keep = make_arrays(arrays, codes=codes)
        h = c_void_p()
        check(lib().sg_open_ivf_arrays(byref(st), c_int(device), byref(h)))
        del keep
        return cls(h, device)

    def close(self) -> None:
        if self._h:
            check(lib().sg_close(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_timing(self, on: bool) -> None:
        """Per-stage device timing of every search (read back with last_stats)."""
        check(lib().sg_set_timing(self._h, c_int(1 if on else 0)))

    def last_stats(self) -> dict:
        st = SgStats()
        check(lib().sg_last_stats(self._h, byref(st)))
        return {name: getattr(st, name) for name, _ in SgStats._fields_ if not name.startswith("reserved")}

    def tuning(self) -> dict:
        t = _abi.SgTuning()
        check(lib().sg_get_tuning(self._h, byref(t)))
        return {name: getattr(t, name) for name, _ in _abi.SgTuning._fields_}

    def set_tuning(self, **fields) -> None:
        t = _abi.SgTuning(**{**self.tuning(), **fields})
        check(lib().sg_set_tuning(self._h, byref(t)))

    def autotune(self, nq: int, d_q768: int, params: Params, d_q256: int | None = None, reps: int = 2) -> dict:
        """sg_autotune on nq device-resident queries: the chosen shapes and the batch's device
        time before and after (ms)."""
        p = params.to_c()
        t = _abi.SgTuning()
        ms = (ctypes.c_float * 2)()
        check(lib().sg_autotune(self._h, c_uint32(nq), c_void_p(d_q768), c_void_p(d_q256) if d_q256 else None,
                                byref(p), c_uint32(reps), byref(t), ms))
        out = {name: getattr(t, name) for name, _ in _abi.SgTuning._fields_}
        out.update(ms_before=round(ms[0], 4), ms_after=round(ms[1], 4))
        return out

    def set_route_precision(self, bf16: bool) -> None:
        check(lib().sg_set_route_precision(self._h, c_int(_abi.ROUTE_BF16 if bf16 else _abi.ROUTE_FP32)))

    # Index::search / search_view (src/ivf.rs:621-633), batched
    def search_batch(self, q768, q256=None, params: Params | None = None, allow=None,
                     timing: Timing | None = None):
        """Returns (scores [nq, k], ids [nq, k], counts [nq]) best first per query."""
        q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
        nq = q768.shape[0]
        q2 = None if q256 is None else _f32(q256, nq, _abi.PDIM)
        p = params.to_c()
        k = max(p.k, 1)
        sc = np.zeros((nq, k), np.float32)
        ids = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        t = SgTiming()
        check(lib().sg_search(self._h, c_uint32(nq), ptr(q768), ptr(q2), byref(p), ptr(al),
                              c_uint64(0 if al is None else al.size), ptr(sc), ptr(ids), ptr(cnt),
                              byref(t)))
        if timing is not None:
            timing.add(t)
        return sc[:, : p.k], ids[:, : p.k], cnt

    def search_into(self, q768: np.ndarray, params: Params, out_scores: np.ndarray,
                    out_ids: np.ndarray, out_counts: np.ndarray, q256: np.ndarray | None = None) -> None:
        """sg_search into caller-owned host buffers (pinned buffers make the copies direct)."""
        nq = q768.shape[0]
        p = params.to_c()
        check(lib().sg_search(self._h, c_uint32(nq), ptr(q768), ptr(q256), byref(p), None, c_uint64(0),
                              ptr(out_scores), ptr(out_ids), ptr(out_counts), None))

    def search(self, q768, q256, params: Params, allow=None, timing: Timing | None = None):
        """One query: list of (score, row) best first, like Index::search."""
        sc, ids, cnt = self.search_batch(np.asarray(q768)[None], None if q256 is None else np.asarray(q256)[None],
                                         params, allow, timing)
        return [(float(sc[0, i]), int(ids[0, i])) for i in range(int(cnt[0]))]

    def search_device(self, nq: int, d_q768: int, d_q256: int | None, params: Params,
                      d_out_scores: int, d_out_ids: int, d_out_counts: int, stream: int = 0) -> None:
        """sg_search_device over raw device pointers (e.g. torch tensors' data_ptr())."""
        p = params.to_c()
        check(lib().sg_search_device(self._h, c_uint32(nq), c_void_p(d_q768),
                                     c_void_p(d_q256) if d_q256 else None, byref(p), None, c_uint64(0),
                                     c_void_p(d_out_scores), c_void_p(d_out_ids), c_void_p(d_out_counts),
                                     c_void_p(stream)))

    # flat_hamming_rerank of the search binary (src/bin/search.rs:251-269)
    def flat_hamming(self, q768, q256=None, cand: int = 1000, k: int = 100):
        """The flat Hamming baseline: (scores [nq, k], ids [nq, k], counts [nq]), best first."""
        q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
        nq = q768.shape[0]
        q2 = None if q256 is None else _f32(q256, nq, _abi.PDIM)
        sc = np.zeros((nq, max(k, 1)), np.float32)
        ids = np.zeros((nq, max(k, 1)), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        check(lib().sg_flat_hamming(self._h, c_uint32(nq), ptr(q768), ptr(q2), c_uint32(cand), c_uint32(k),
                                    ptr(sc), ptr(ids), ptr(cnt)))
        return sc[:, :k], ids[:, :k], cnt

    # Index::route (src/ivf.rs:589-613)
    def route(self, q256, params: Params):
        q = np.ascontiguousarray(q256, np.float32).reshape(-1, _abi.PDIM)
        nq = q.shape[0]
        P = max(min(params.nprobe, self.k), 1)
        sc = np.zeros((nq, P), np.float32)
        cl = np.zeros((nq, P), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        p = params.to_c()
        check(lib().sg_route(self._h, c_uint32(nq), ptr(q), byref(p), ptr(sc), ptr(cl), ptr(cnt)))
        return [(sc[i, : cnt[i]], cl[i, : cnt[i]]) for i in range(nq)]

    # the centroid scores of Index::route (src/ivf.rs:592, blas::gemm_abt) at the routing precision
    def route_scores(self, q256) -> np.ndarray:
        q = np.ascontiguousarray(q256, np.float32).reshape(-1, _abi.PDIM)
        nq = q.shape[0]
        out = np.zeros((nq, self.k), np.float32)
        if nq:
            check(lib().sg_route_scores(self._h, c_uint32(nq), ptr(q), ptr(out)))
        return out

    # Index::candidates (src/ivf.rs:647-729) after the index's own routing
    def candidates(self, q256, params: Params, allow=None):
        q = np.ascontiguousarray(q256, np.float32).reshape(-1, _abi.PDIM)
        nq = q.shape[0]
        c = max(params.cand, 1)
        est = np.zeros((nq, c), np.float32)
        ids = np.zeros((nq, c), np.uint32)
        err = np.zeros((nq, c), np.float32)
        cnt = np.zeros(nq, np.uint32)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        p = params.to_c()
        check(lib().sg_candidates(self._h, c_uint32(nq), ptr(q), byref(p), ptr(al),
                                  c_uint64(0 if al is None else al.size), ptr(est), ptr(ids), ptr(err),
                                  ptr(cnt)))
        return [(est[i, : cnt[i]], ids[i, : cnt[i]], err[i, : cnt[i]]) for i in range(nq)]

    # Index::candidates over given probe lists (src/ivf.rs:647-729), a shard's phase 1
    def candidates_probes(self, q256, probes, params: Params, allow=None):
        """probes: per query (centroid scores, clusters) in scan order. Returns per query
        (estimates, rows, error widths) in row order."""
        q = np.ascontiguousarray(q256, np.float32).reshape(-1, _abi.PDIM)
        nq = q.shape[0]
        P = max(min(params.nprobe, self.k), 1)
        ps = np.zeros((nq, P), np.float32)
        pc = np.zeros((nq, P), np.uint32)
        pn = np.zeros(nq, np.uint32)
        for i, (sc, cl) in enumerate(probes):
            pn[i] = len(cl)
            ps[i, : len(cl)] = sc
            pc[i, : len(cl)] = cl
        c = max(params.cand, 1)
        est = np.zeros((nq, c), np.float32)
        ids = np.zeros((nq, c), np.uint32)
        err = np.zeros((nq, c), np.float32)
        cnt = np.zeros(nq, np.uint32)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        p = params.to_c()
        check(lib().sg_candidates_probes(self._h, c_uint32(nq), ptr(q), ptr(ps), ptr(pc), ptr(pn), byref(p),
                                         ptr(al), c_uint64(0 if al is None else al.size), ptr(est), ptr(ids),
                                         ptr(err), ptr(cnt)))
        return [(est[i, : cnt[i]], ids[i, : cnt[i]], err[i, : cnt[i]]) for i in range(nq)]

    # Index::rerank of given candidates (src/ivf.rs:734-815), a shard's phase 2
    def rerank(self, q768, q256, cands, params: Params):
        """cands: per query (estimates, rows, error widths or None). Returns (scores [nq, k],
        ids [nq, k], counts [nq]) best first."""
        q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
        nq = q768.shape[0]
        q2 = None if q256 is None else _f32(q256, nq, _abi.PDIM)
        stride = max([len(c[1]) for c in cands] + [1])
        est = np.zeros((nq, stride), np.float32)
        ids = np.zeros((nq, stride), np.uint32)
        err = np.zeros((nq, stride), np.float32)
        cn = np.zeros(nq, np.uint32)
        for i, (e, r, w) in enumerate(cands):
            cn[i] = len(r)
            est[i, : len(r)] = e
            ids[i, : len(r)] = r
            if w is not None:
                err[i, : len(r)] = w
        p = params.to_c()
        k = max(p.k, 1)
        sc = np.zeros((nq, k), np.float32)
        oid = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        check(lib().sg_rerank(self._h, c_uint32(nq), ptr(q768), ptr(q2), ptr(est), ptr(ids), ptr(err), ptr(cn),
                              c_uint32(stride), byref(p), ptr(sc), ptr(oid), ptr(cnt)))
        return sc[:, : p.k], oid[:, : p.k], cnt

    # rabitq::Query::new (src/rabitq.rs:119-125)
    def query_prep(self, q256):
        q = np.ascontiguousarray(q256, np.float32).reshape(-1, _abi.PDIM)
        nq = q.shape[0]
        tables = np.zeros((nq, 64, 16), np.uint8)
        sc, bi, a, b = (np.zeros(nq, np.float32) for _ in range(4))
        check(lib().sg_query_prep(self._h, c_uint32(nq), ptr(q), ptr(tables), ptr(sc), ptr(bi), ptr(a), ptr(b)))
        return tables, sc, bi, a, b


class Context:
    """ivf::Scratch (src/ivf.rs:497-513) on the GPU: one thread's stream, device scratch and captured
    graphs over a shared Index. Threads that each search through their own Context run at once
    (sg_search on the Index itself serialises its callers); a Context serves one call at a time."""

    def __init__(self, index: Index):
        self.index = index
        self._c = c_void_p()
        check(lib().sg_context_open(index._h, byref(self._c)))

    def close(self) -> None:
        if self._c:
            check(lib().sg_context_close(self._c))
            self._c = None

    def __enter__(self) -> "Context":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # Index::search(&self, &Corpus, q768, q256, &Params, &mut Scratch, &mut Timing), batched
    def search_batch(self, q768, q256=None, params: Params | None = None, allow=None,
                     timing: Timing | None = None):
        """Returns (scores [nq, k], ids [nq, k], counts [nq]) best first per query."""
        q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
        nq = q768.shape[0]
        q2 = None if q256 is None else _f32(q256, nq, _abi.PDIM)
        p = params.to_c()
        k = max(p.k, 1)
        sc = np.zeros((nq, k), np.float32)
        ids = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        t = SgTiming()
        check(lib().sg_search_ctx(self._c, c_uint32(nq), ptr(q768), ptr(q2), byref(p), ptr(al),
                                  c_uint64(0 if al is None else al.size), ptr(sc), ptr(ids), ptr(cnt),
                                  byref(t)))
        if timing is not None:
            timing.add(t)
        return sc[:, : p.k], ids[:, : p.k], cnt

    def search_device(self, nq: int, d_q768: int, d_q256: int | None, params: Params,
                      d_out_scores: int, d_out_ids: int, d_out_counts: int, stream: int = 0) -> None:
        """sg_search_device_ctx over raw device pointers."""
        p = params.to_c()
        check(lib().sg_search_device_ctx(self._c, c_uint32(nq), c_void_p(d_q768),
                                         c_void_p(d_q256) if d_q256 else None, byref(p), None, c_uint64(0),
                                         c_void_p(d_out_scores), c_void_p(d_out_ids), c_void_p(d_out_counts),
                                         c_void_p(stream)))

    def last_stats(self) -> dict:
        st = SgStats()
        check(lib().sg_context_last_stats(self._c, byref(st)))
        return {name: getattr(st, name) for name, _ in SgStats._fields_ if not name.startswith("reserved")}


def lut_scan(tables: np.ndarray, blocks: np.ndarray) -> np.ndarray:
    """lut::scan (src/lut.rs:96-102) on the GPU: u16 scores, 32 per block."""
    tables = np.ascontiguousarray(tables, np.uint8)
    groups = tables.size // 16
    blocks = np.ascontiguousarray(blocks, np.uint8)
    nb = blocks.size // (groups * 16)
    out = np.zeros(nb * 32, np.uint16)
    check(lib().sg_lut_scan(c_uint32(groups), ptr(tables), ptr(blocks), c_uint64(nb), ptr(out)))
    return out


def lut_scan_batch(tables: np.ndarray, blocks: np.ndarray) -> np.ndarray:
    """lut::scan (src/lut.rs:96-102, 64 groups) of many queries at once on the tcgen05 tensor
    cores: tables [nq, 1024] u8, blocks [nblocks * 1024] u8 -> u16 scores [nq, nblocks * 32]."""
    tables = np.ascontiguousarray(tables, np.uint8).reshape(-1, 64 * 16)
    blocks = np.ascontiguousarray(blocks, np.uint8)
    nb = blocks.size // (64 * 16)
    out = np.zeros((tables.shape[0], nb * 32), np.uint16)
    check(lib().sg_lut_scan_batch(c_uint32(tables.shape[0]), ptr(tables), ptr(blocks), c_uint64(nb), ptr(out)))
    return out


def dot_i8i8(query: np.ndarray, rows: np.ndarray) -> np.ndarray:
    """quant::dot_i8i8 (src/quant.rs:113-125) of one query against many rows, on the GPU."""
    query = np.ascontiguousarray(query, np.int8)
    rows = np.ascontiguousarray(rows, np.int8).reshape(-1, query.size)
    out = np.zeros(rows.shape[0], np.int32)
    check(lib().sg_dot_i8i8(ptr(query), ptr(rows), c_uint64(rows.shape[0]), c_uint32(query.size), ptr(out)))
    return out
