"""bigann::Index / Params / Timing (src/bigann.rs:604-747) over the GPU library: billion-scale L2
search over int8 rows of 100 dims, every record and base row resident in HBM.

`BigannIndex.search_batch` is Index::search for a batch of queries; `route` and `candidates`
expose the first two stages for parity tests. `parse_config` reads the spacev binary's config
grammar nprobe:cand[:refine[:mMARGIN]] (src/bin/spacev.rs:213-218).
"""
from __future__ import annotations

from ctypes import byref, c_int, c_uint32, c_uint64, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import SgBigannParams, SgBigannTiming, check, lib, make_bigann_arrays, ptr


@dataclass
class BigannParams:
    """bigann::Params (src/bigann.rs:610-623)."""

    nprobe: int
    cand: int = 500
    k: int = 10
    refine: int = 0
    margin: float = 0.0
    route_fp32: bool = False  # exact FP32 dots of every leaf instead of the tensor-core routing

    def to_c(self) -> SgBigannParams:
        return SgBigannParams(int(self.nprobe), int(self.cand), int(self.k), int(self.refine),
                              float(self.margin), int(bool(self.route_fp32)))


def parse_config(cfg: str, k: int = 10) -> BigannParams:
    f = cfg.split(":")
    nprobe = int(f[0])
    cand = int(f[1]) if len(f) > 1 else 500
    refine = int(f[2]) if len(f) > 2 else 0
    margin = float(f[3].lstrip("m")) if len(f) > 3 else 0.0
    return BigannParams(nprobe, cand, k, refine, margin)


@dataclass
class BigannTiming:
    """bigann::Timing (src/bigann.rs:624-632), device nanoseconds."""

    route: int = 0
    scan: int = 0
    io_wait: int = 0
    rerank: int = 0
    scanned: int = 0
    probes: int = 0

    def add(self, t: SgBigannTiming) -> None:
        for name, _ in SgBigannTiming._fields_:
            setattr(self, name, getattr(self, name) + getattr(t, name))


def _i8(q, nq=None) -> np.ndarray:
    q = np.ascontiguousarray(q, np.int8).reshape(-1, _abi.BG_DIM)
    return q


class BigannIndex:
    """bigann::Index with its records and base rows resident in one GPU's HBM."""

    def __init__(self, handle: c_void_p, device: int):
        self._h = handle
        self.device = device
        k, n, nb, bits = c_uint32(), c_uint64(), c_uint64(), c_uint32()
        check(lib().sg_bigann_info(self._h, byref(k), byref(n), byref(nb), byref(bits)))
        self.k, self.n, self.nblocks, self.bits = k.value, n.value, nb.value, bits.value

    @classmethod
    def open(cls, index_dir: str, base_dir: str, device: int = 0) -> "BigannIndex":
        h = c_void_p()
        check(lib().sg_open_bigann(index_dir.encode(), base_dir.encode(), c_int(device), byref(h)))
        return cls(h, device)

    @classmethod
    def from_arrays(cls, arrays: dict, device: int = 0) -> "BigannIndex":
        st, keep = make_bigann_arrays(arrays)
        h = c_void_p()
        check(lib().sg_open_bigann_arrays(byref(st), c_int(device), byref(h)))
        del keep
        return cls(h, device)

    def route_fallbacks(self) -> int:
        """Passes since open in which a query's tensor-core routing fell back to exact FP32 dots
        of every leaf (same results, slower)."""
        n = c_uint64()
        check(lib().sg_bigann_route_fallbacks(self._h, byref(n)))
        return n.value

    def close(self) -> None:
        if self._h:
            check(lib().sg_close_bigann(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search_batch(self, q, params: BigannParams, timing: BigannTiming | None = None):
        """Index::search for every row of q: (scores [nq, k], ids [nq, k], counts [nq])."""
        q = _i8(q)
        nq = q.shape[0]
        p = params.to_c()
        k = max(p.k, 1)
        sc = np.zeros((nq, k), np.float32)
        ids = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        t = SgBigannTiming()
        check(lib().sg_search_bigann(self._h, c_uint32(nq), ptr(q), byref(p), ptr(sc), ptr(ids), ptr(cnt),
                                     byref(t) if timing is not None else None))
        if timing is not None:
            timing.add(t)
        return sc[:, : p.k], ids[:, : p.k], cnt

    def search_into(self, q: np.ndarray, params: BigannParams, out_scores: np.ndarray,
                    out_ids: np.ndarray, out_counts: np.ndarray) -> None:
        """sg_search_bigann into caller-owned host buffers (pinned buffers make the copies direct)."""
        p = params.to_c()
        check(lib().sg_search_bigann(self._h, c_uint32(q.shape[0]), ptr(q), byref(p), ptr(out_scores),
                                     ptr(out_ids), ptr(out_counts), None))

    def search(self, q, params: BigannParams, timing: BigannTiming | None = None):
        """One query: list of (score, row) best first, like bigann::Index::search."""
        sc, ids, cnt = self.search_batch(np.asarray(q)[None], params, timing)
        return [(float(sc[0, i]), int(ids[0, i])) for i in range(int(cnt[0]))]

    def search_device(self, nq: int, d_q: int, params: BigannParams, d_out_scores: int,
                      d_out_ids: int, d_out_counts: int, stream: int = 0) -> None:
        p = params.to_c()
        check(lib().sg_search_bigann_device(self._h, c_uint32(nq), c_void_p(d_q), byref(p),
                                            c_void_p(d_out_scores), c_void_p(d_out_ids),
                                            c_void_p(d_out_counts), c_void_p(stream)))

    def route(self, q, params: BigannParams):
        q = _i8(q)
        nq = q.shape[0]
        P = max(min(params.nprobe, self.k), 1)
        probe = np.zeros((nq, P), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        p = params.to_c()
        check(lib().sg_bigann_route(self._h, c_uint32(nq), ptr(q), byref(p), ptr(probe), ptr(cnt)))
        return [probe[i, : cnt[i]] for i in range(nq)]

    def candidates(self, q, params: BigannParams):
        q = _i8(q)
        nq = q.shape[0]
        c = max(params.cand, 1)
        ids = np.zeros((nq, c), np.uint32)
        est = np.zeros((nq, c), np.float32)
        nx = np.zeros((nq, c), np.float32)
        cnt = np.zeros(nq, np.uint32)
        p = params.to_c()
        check(lib().sg_bigann_candidates(self._h, c_uint32(nq), ptr(q), byref(p), ptr(ids), ptr(est),
                                         ptr(nx), ptr(cnt)))
        return [(ids[i, : cnt[i]], est[i, : cnt[i]], nx[i, : cnt[i]]) for i in range(nq)]
