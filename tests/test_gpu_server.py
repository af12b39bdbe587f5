"""The serving loop (sg_server_*): requests submitted from several threads with mixed params and
per-request filters are batched and overlapped on the GPU, and every result equals the query
run alone (sg_search of that one query) and the oracle."""
import os
import threading

import numpy as np
import pytest

import oracle as O
from fixtures import index_a
from sieve_gpu import Index, Params, Rerank, Server, SieveError, allow_bitset
from sieve_gpu import filter as F

pytestmark = pytest.mark.gpu

CONFIGS = [Params(16, 500, Rerank.full(), 10), Params(8, 300, Rerank.tiered(100), 20),
           Params(32, 1000, Rerank.full(), 10, prune=(10, 0.5))]


@pytest.fixture(scope="module")
def env():
    arrays, q768, q256, _ = index_a()
    ix = Index.from_arrays(arrays)
    n = arrays["n"]
    r = np.random.default_rng(3)
    allows = [allow_bitset(np.nonzero(r.random(n) < f)[0], n) for f in (0.3, 0.02)]
    filters = [F.Filter(a, ix) for a in allows]
    yield ix, arrays, q768, q256, allows, filters
    for f in filters:
        f.close()
    ix.close()


def requests(q768, q256, nreq, seed):
    r = np.random.default_rng(seed)
    out = []
    for i in range(nreq):
        qi = int(r.integers(0, q768.shape[0]))
        out.append((qi, int(r.integers(0, len(CONFIGS))), int(r.integers(-1, 2)), bool(r.integers(0, 2))))
    return out  # (query, config, filter index or -1, with q256)


def alone(ix, q768, q256, allows, req):
    qi, ci, fi, hq = req
    sc, ids, cnt = ix.search_batch(q768[qi:qi + 1], q256[qi:qi + 1] if hq else None, CONFIGS[ci],
                                   allow=None if fi < 0 else allows[fi])
    return sc[0, : cnt[0]], ids[0, : cnt[0]]


def run_mix(srv, ix, q768, q256, filters, reqs, threads=4):
    out = [None] * len(reqs)

    def worker(t):
        mine = list(range(t, len(reqs), threads))
        tickets = []
        for j in mine:
            qi, ci, fi, hq = reqs[j]
            tickets.append(srv.submit(q768[qi], q256[qi] if hq else None, CONFIGS[ci],
                                      None if fi < 0 else filters[fi]))
        for j, tk in zip(mine, tickets):
            out[j] = srv.poll(tk, wait_ms=-1)

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return out


def test_results_in_the_mix_equal_results_alone(env):
    ix, arrays, q768, q256, allows, filters = env
    reqs = requests(q768, q256, 400, 1)
    with Server(ix, max_batch=256, contexts=3) as srv:
        got = run_mix(srv, ix, q768, q256, filters, reqs)
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["batches"] < len(reqs)  # batching happened
    for req, (sc, ids, info) in zip(reqs, got):
        s1, i1 = alone(ix, q768, q256, allows, req)
        assert np.array_equal(ids, i1) and np.array_equal(sc, s1), req
        assert info.batch >= 1 and info.service_ms >= 0


def test_mix_matches_oracle(env):
    ix, arrays, q768, q256, allows, filters = env
    oi = O.OracleIndex(arrays)
    reqs = requests(q768, q256, 60, 2)
    with Server(ix, max_batch=64, contexts=2) as srv:
        got = run_mix(srv, ix, q768, q256, filters, reqs, threads=2)
    for (qi, ci, fi, hq), (sc, ids, _) in zip(reqs, got):
        p = CONFIGS[ci].to_c()
        al = None if fi < 0 else allows[fi]
        s, o, _ = oi.search(q768[qi], q256[qi], p, al)
        assert np.array_equal(ids, o) and np.array_equal(sc, s)


def test_overflowing_queries_are_rerun_alone(env):
    ix0, arrays, q768, q256, allows, _ = env
    os.environ["SIEVE_GPU_SOFT_CAP"] = "64"
    try:
        ix = Index.from_arrays(arrays)
    finally:
        del os.environ["SIEVE_GPU_SOFT_CAP"]
    try:
        p = Params(16, 500, Rerank.full(), 10)
        with Server(ix, max_batch=128, contexts=2) as srv:
            tickets = [srv.submit(q768[i], q256[i], p) for i in range(q768.shape[0])]
            got = [srv.poll(t) for t in tickets]
            assert srv.stats()["retried"] > 0
        sc, ids, cnt = ix0.search_batch(q768, q256, p)
        for i, (s1, i1, info) in enumerate(got):
            assert np.array_equal(i1, ids[i, : cnt[i]]) and np.array_equal(s1, sc[i, : cnt[i]])
    finally:
        ix.close()


def test_admission_refuses_requests_that_cannot_fit(env):
    ix, arrays, q768, q256, allows, filters = env
    with Server(ix, max_batch=16, contexts=1, scratch_bytes=1024) as srv:
        with pytest.raises(SieveError):
            srv.submit(q768[0], q256[0], CONFIGS[0])
        assert srv.stats()["rejected"] == 1


def test_poll_timeout_and_stop_drains(env):
    ix, arrays, q768, q256, allows, filters = env
    srv = Server(ix, max_batch=32, contexts=1)
    tickets = [srv.submit(q768[i % q768.shape[0]], None, CONFIGS[0]) for i in range(100)]
    first = srv.poll(tickets[0], wait_ms=0)  # may still be running
    assert first is None or first[1].size == 10
    done = [srv.poll(t, wait_ms=-1) for t in tickets[1:]]
    srv.stop()
    assert all(d is not None for d in done)
