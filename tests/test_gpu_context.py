"""Search contexts (ivf::Scratch on the GPU): threads that each search one shared index through
their own context get exactly the results of serial calls, and overlap on the device.

The reference shares one Index across rayon workers, each with its own Scratch
(src/bin/search.rs:312-323); sg_context is that Scratch, so concurrent callers no longer serialise
on the index's default context.
"""
import threading
import time

import numpy as np
import pytest

import oracle as O
from fixtures import index_a
from sieve_gpu import Context, Index, Params, Rerank

pytestmark = pytest.mark.gpu

PARAMS = [Params(16, 500, Rerank.full(), 10), Params(8, 300, Rerank.tiered(100), 10)]


def test_context_equals_index_search_and_oracle():
    arrays, q768, q256, _ = index_a()
    ix = Index.from_arrays(arrays)
    oi = O.OracleIndex(arrays)
    try:
        with Context(ix) as ctx:
            for p in PARAMS:
                sc, ids, cnt = ctx.search_batch(q768, None, p)
                sc0, ids0, cnt0 = ix.search_batch(q768, None, p)
                assert np.array_equal(cnt, cnt0)
                assert np.array_equal(ids, ids0) and np.array_equal(sc, sc0)
                for i in range(0, q768.shape[0], 7):
                    s, o, _ = oi.search(q768[i], q256[i], p.to_c())
                    assert np.array_equal(ids[i, : cnt[i]], o) and np.array_equal(sc[i, : cnt[i]], s)
    finally:
        ix.close()


def test_four_threads_four_contexts_match_serial_and_overlap():
    arrays, q768, _, _ = index_a()
    ix = Index.from_arrays(arrays)
    p = PARAMS[0]
    nthreads, calls = 4, 12
    # every thread runs every query set: a batch of 64 queries, rotated per call
    batches = [np.roll(q768, 3 * j, axis=0)[:64].copy() for j in range(calls)]
    try:
        want = [ix.search_batch(b, None, p) for b in batches]
        ctxs = [Context(ix) for _ in range(nthreads)]
        for c in ctxs:  # warm each context (workspace, graphs) outside the timed runs
            for b in batches[:2]:
                c.search_batch(b, None, p)
        got = [[None] * calls for _ in range(nthreads)]
        errors = []

        def run(t):
            try:
                for j in range(calls):
                    got[t][j] = ctxs[t].search_batch(batches[j], None, p)
            except Exception as e:  # reported on the main thread
                errors.append(e)

        t0 = time.perf_counter()
        for t in range(nthreads):
            run(t)
        serial = time.perf_counter() - t0
        serial_got = [row[:] for row in got]
        ths = [threading.Thread(target=run, args=(t,)) for t in range(nthreads)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        parallel = time.perf_counter() - t0
        assert not errors, errors
        for t in range(nthreads):
            for j in range(calls):
                for a, b, c in ((got[t][j], want[j], serial_got[t][j]),):
                    assert all(np.array_equal(x, y) for x, y in zip(a, b))
                    assert all(np.array_equal(x, y) for x, y in zip(c, b))
        assert parallel < serial, (parallel, serial)
        for c in ctxs:
            c.close()
    finally:
        ix.close()
