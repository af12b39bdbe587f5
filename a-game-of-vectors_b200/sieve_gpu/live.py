"""Live updates over an Index on the GPU: ivf's live layer (src/live.rs), behind sg_live_* of the
C ABI. Inserts are encoded on the device as Live::apply_insert encodes them and join
per-centroid delta lists scanned after each base list; deletes tombstone rows; results carry
external ids (corpus rows keep their row number, inserted rows the id they were inserted under)."""
from __future__ import annotations

from ctypes import byref, c_float, c_uint32, c_uint64, c_void_p

import numpy as np

from . import _abi
from ._abi import check, lib, ptr
from .index import Index, Params


class Live:
    """Live::open over an open Index (which must then be searched through this object)."""

    def __init__(self, index: Index, max_rows: int, soar_lambda: float | None = 1.0):
        self.index = index
        self._h = c_void_p()
        lam = -1.0 if soar_lambda is None else float(soar_lambda)
        check(lib().sg_live_open(index._h, c_uint64(max_rows), c_float(lam), byref(self._h)))

    def close(self) -> None:
        if self._h:
            check(lib().sg_live_close(self._h))
            self._h = None

    def __enter__(self) -> "Live":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def insert(self, ext_ids, vecs) -> None:
        """Live::insert: unit 768-d vectors under external ids (an id already live is replaced)."""
        e = np.ascontiguousarray(ext_ids, np.uint32).reshape(-1)
        v = np.ascontiguousarray(vecs, np.float32).reshape(e.size, _abi.DIM)
        check(lib().sg_live_insert(self._h, c_uint32(e.size), ptr(e), ptr(v)))

    def delete(self, ext_ids) -> None:
        """Live::delete: unknown ids are ignored."""
        e = np.ascontiguousarray(ext_ids, np.uint32).reshape(-1)
        check(lib().sg_live_delete(self._h, c_uint32(e.size), ptr(e)))

    def search_batch(self, q768, q256=None, params: Params | None = None):
        """Live::search for many queries: (scores [nq, k], external ids [nq, k], counts [nq])."""
        q768 = np.ascontiguousarray(q768, np.float32).reshape(-1, _abi.DIM)
        nq = q768.shape[0]
        q2 = None if q256 is None else np.ascontiguousarray(q256, np.float32).reshape(nq, _abi.PDIM)
        p = params.to_c()
        k = max(p.k, 1)
        sc = np.zeros((nq, k), np.float32)
        ids = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        check(lib().sg_live_search(self._h, c_uint32(nq), ptr(q768), ptr(q2), byref(p), ptr(sc), ptr(ids), ptr(cnt)))
        return sc[:, : p.k], ids[:, : p.k], cnt

    def info(self) -> dict:
        r, s, d = c_uint64(), c_uint64(), c_uint64()
        check(lib().sg_live_info(self._h, byref(r), byref(s), byref(d)))
        return {"delta_rows": r.value, "delta_slots": s.value, "deleted": d.value}
