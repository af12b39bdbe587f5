"""The serving loop (continuous batching) over an Index, behind sg_server_* of the C ABI.

Requests are single queries; a dispatcher thread in the library batches whatever is pending
each time one of its execution contexts frees up, so requests that arrive while others run on
the GPU join the next batch and batches overlap. Each result equals the query's result alone.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_int, c_uint32, c_uint64, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import check, lib, ptr
from .index import Index, Params


class SgServerConfig(ctypes.Structure):
    _fields_ = [("max_batch", c_uint32), ("contexts", c_uint32), ("scratch_bytes", c_uint64),
                ("max_pending", c_uint32), ("reserved", c_uint32)]


class SgRequestInfo(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_float), ("service_ms", ctypes.c_float), ("batch", c_uint32),
                ("retried", c_uint32)]


class SgServerStats(ctypes.Structure):
    _fields_ = [(n, c_uint64) for n in ("submitted", "completed", "rejected", "batches",
                                        "queries_batched", "retried")] + \
               [("pending", c_uint32), ("in_flight", c_uint32)]


@dataclass
class RequestInfo:
    queue_ms: float
    service_ms: float
    batch: int
    retried: bool


class Server:
    """sg_server over an open Index. Filters (sieve_gpu.filter.Filter) must outlive the requests
    that use them."""

    def __init__(self, index: Index, max_batch: int = 1024, contexts: int = 2,
                 scratch_bytes: int = 0, max_pending: int = 0):
        self.index = index
        cfg = SgServerConfig(max_batch, contexts, scratch_bytes, max_pending, 0)
        self._h = c_void_p()
        check(lib().sg_server_start(index._h, byref(cfg), byref(self._h)))
        self._k = {}

    def submit(self, q768, q256=None, params: Params | None = None, filter=None) -> int:
        q = np.ascontiguousarray(q768, np.float32).reshape(_abi.DIM)
        q2 = None if q256 is None else np.ascontiguousarray(q256, np.float32).reshape(_abi.PDIM)
        p = params.to_c()
        t = c_uint64()
        check(lib().sg_server_submit(self._h, ptr(q), ptr(q2), byref(p),
                                     filter._h if filter is not None else None, byref(t)))
        self._k[t.value] = p.k
        return t.value

    def poll(self, ticket: int, wait_ms: int = -1):
        """(scores, ids, RequestInfo) when the request is done; None on timeout."""
        k = max(self._k.get(ticket, 1), 1)
        sc = np.zeros(k, np.float32)
        ids = np.zeros(k, np.uint32)
        n = c_uint32()
        info = SgRequestInfo()
        rc = lib().sg_server_poll(self._h, c_uint64(ticket), c_int(wait_ms), ptr(sc), ptr(ids), byref(n),
                                  byref(info))
        if rc == -5:  # SG_ERR_TIMEOUT: still running
            return None
        check(rc)
        self._k.pop(ticket, None)
        m = n.value
        return sc[:m], ids[:m], RequestInfo(info.queue_ms, info.service_ms, info.batch, bool(info.retried))

    def replay(self, arrival_s, q768_pool, which, params: Params, filters=(), filter_of=None):
        """Open-loop load from a library thread (sg_server_replay): request i goes at arrival_s[i]
        seconds after the start with query q768_pool[which[i]] and filters[filter_of[i]] (no
        filter where filter_of[i] < 0). Returns (latency ms per request, batch size per request,
        wall seconds from the first arrival to the last result)."""
        n = len(which)
        arr = np.ascontiguousarray(np.round(np.asarray(arrival_s) * 1e9), np.uint64)
        pool = np.ascontiguousarray(q768_pool, np.float32).reshape(-1, _abi.DIM)
        wh = np.ascontiguousarray(which, np.uint32)
        fs = (c_void_p * max(len(filters), 1))(*[f._h for f in filters])
        fo = None if filter_of is None else np.ascontiguousarray(filter_of, np.int32)
        lat = np.zeros(n, np.float32)
        bat = np.zeros(n, np.uint32)
        wall = ctypes.c_double()
        p = params.to_c()
        check(lib().sg_server_replay(self._h, c_uint32(n), ptr(arr), ptr(pool), ptr(wh), byref(p),
                                     fs if filters else None, ptr(fo), ptr(lat), ptr(bat), byref(wall)))
        return lat, bat, wall.value

    def stats(self) -> dict:
        st = SgServerStats()
        check(lib().sg_server_get_stats(self._h, byref(st)))
        return {name: getattr(st, name) for name, _ in SgServerStats._fields_}

    def stop(self) -> None:
        if self._h:
            check(lib().sg_server_stop(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()
