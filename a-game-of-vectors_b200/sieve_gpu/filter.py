"""filter::Filter / filter::Plan / filter::search (src/filter.rs) over the GPU library.

A `Filter` is an allow bitset resident on the index's GPU with its allowed rows (ascending) and
allowed slots per cluster, built on the device as Filter::new builds them (src/filter.rs:27-38).
`search` runs one of the reference's plans for a batch of queries: Post (the unfiltered probes,
disallowed rows skipped at admission), Expand(target) (clusters in route order until `target`
allowed slots are covered), Brute (exact int8 scores of every allowed row), or Auto.
"""
from __future__ import annotations

from ctypes import byref, c_int, c_uint32, c_uint64, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import SgTiming, check, lib, ptr
from .index import Index, Params, Timing, _f32

BRUTE_MAX = 250_000        # filter::BRUTE_MAX (src/filter.rs:55)
POST_MIN = 0.3             # filter::POST_MIN (src/filter.rs:57)
EXPAND_TARGET = 200_000    # filter::EXPAND_TARGET (src/filter.rs:59)

POST, EXPAND, BRUTE, AUTO = 0, 1, 2, 3


@dataclass(frozen=True)
class Plan:
    """filter::Plan (src/filter.rs:42-53): kind POST / EXPAND / BRUTE / AUTO; target for EXPAND."""

    kind: int
    target: int = 0

    @staticmethod
    def post() -> "Plan":
        return Plan(POST)

    @staticmethod
    def expand(target: int) -> "Plan":
        return Plan(EXPAND, int(target))

    @staticmethod
    def brute() -> "Plan":
        return Plan(BRUTE)

    @staticmethod
    def auto() -> "Plan":
        return Plan(AUTO)

    def resolve(self, f: "Filter", n: int) -> "Plan":
        """Plan::resolve (src/filter.rs:62-71)."""
        kind = lib().sg_plan_resolve(c_int(self.kind), c_uint64(f.nrows), c_uint64(n))
        if self.kind == AUTO and kind == EXPAND:
            return Plan(EXPAND, EXPAND_TARGET)
        return self if kind == self.kind else Plan(kind)


class Filter:
    """filter::Filter (src/filter.rs:18-38) on the index's GPU. Free it (close) before the index."""

    def __init__(self, allow, index: Index):
        self.allow = np.ascontiguousarray(allow, np.uint64)
        self.index = index
        self._h = c_void_p()
        check(lib().sg_filter_new(index._h, ptr(self.allow), c_uint64(self.allow.size), byref(self._h)))
        n = c_uint64()
        check(lib().sg_filter_info(self._h, byref(n), None, None))
        self.nrows = n.value

    @property
    def rows(self) -> np.ndarray:
        out = np.zeros(max(self.nrows, 1), np.uint32)
        check(lib().sg_filter_info(self._h, None, None, ptr(out)))
        return out[: self.nrows]

    @property
    def per_cluster(self) -> np.ndarray:
        out = np.zeros(self.index.k, np.uint32)
        check(lib().sg_filter_info(self._h, None, ptr(out), None))
        return out

    def close(self) -> None:
        if self._h:
            check(lib().sg_filter_free(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def search_batch(index: Index, f: Filter, plan: Plan, q768, q256, params: Params,
                 timing: Timing | None = None):
    """filter::search (src/filter.rs:74-110) for a batch: (scores [nq, k], ids [nq, k], counts)."""
    q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
    nq = q768.shape[0]
    q2 = None if q256 is None else _f32(q256, nq, _abi.PDIM)
    p = params.to_c()
    k = max(p.k, 1)
    sc = np.zeros((nq, k), np.float32)
    ids = np.zeros((nq, k), np.uint32)
    cnt = np.zeros(nq, np.uint32)
    t = SgTiming()
    check(lib().sg_filter_search(index._h, f._h, c_int(plan.kind), c_uint64(plan.target), c_uint32(nq),
                                 ptr(q768), ptr(q2), byref(p), ptr(sc), ptr(ids), ptr(cnt), byref(t)))
    if timing is not None:
        timing.add(t)
    return sc[:, : p.k], ids[:, : p.k], cnt


def search(index: Index, f: Filter, plan: Plan, q768, q256, params: Params,
           timing: Timing | None = None):
    """One query: list of (score, row) best first, like filter::search."""
    sc, ids, cnt = search_batch(index, f, plan, np.asarray(q768)[None],
                                None if q256 is None else np.asarray(q256)[None], params, timing)
    return [(float(sc[0, i]), int(ids[0, i])) for i in range(int(cnt[0]))]
