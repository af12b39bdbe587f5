"""CUDA-graph replay of the search pipeline: a call shape seen twice is captured and replayed from
then on. Replayed batches must equal direct launches and the oracle bit for bit, including when
the inputs, the allow bitset or the routing precision change between replays."""
import os

import numpy as np
import pytest

import oracle as O
from fixtures import index_a
from sieve_gpu import Index, Params, Rerank, allow_bitset

pytestmark = pytest.mark.gpu


def open_env(arrays, **env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return Index.from_arrays(arrays)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.fixture(scope="module")
def pair():
    arrays, q768, q256, _ = index_a()
    g = open_env(arrays, SIEVE_GPU_GRAPHS=1)
    d = open_env(arrays, SIEVE_GPU_GRAPHS=0)
    yield g, d, O.OracleIndex(arrays), arrays, q768, q256
    g.close()
    d.close()


def same(a, b):
    sa, ia, na = a
    sb, ib, nb = b
    assert np.array_equal(na, nb)
    for i in range(na.size):
        n = int(na[i])
        assert np.array_equal(ia[i, :n], ib[i, :n])
        assert np.array_equal(sa[i, :n], sb[i, :n])


@pytest.mark.parametrize("nq", [1, 96, 148])
def test_replay_equals_direct_and_oracle(pair, nq):
    g, d, oi, arrays, q768, q256 = pair
    p = Params(16, 600, Rerank.full(), 10)
    want = d.search_batch(q768[:nq], q256[:nq], p)
    for rep in range(4):  # direct, capture, replay, replay
        got = g.search_batch(q768[:nq], q256[:nq], p)
        same(got, want)
    s, o, cnt, _ = oi.search_batch(q768[:nq], q256[:nq], p.to_c(), threads=4)
    same(want, (s, o, cnt))


def test_replay_reads_new_inputs(pair):
    g, d, oi, arrays, q768, q256 = pair
    p = Params(8, 300, Rerank.tiered(100), 10)
    nq = 100
    for off in (0, 48, 24, 0):  # same shape, different queries every call
        got = g.search_batch(q768[off:off + nq], q256[off:off + nq], p)
        same(got, d.search_batch(q768[off:off + nq], q256[off:off + nq], p))


def test_replay_reads_new_allow_bitset(pair):
    g, d, oi, arrays, q768, q256 = pair
    p = Params(16, 400, Rerank.full(), 10)
    n = arrays["n"]
    r = np.random.default_rng(5)
    for rep in range(4):
        allow = allow_bitset(np.nonzero(r.random(n) < 0.3 + 0.2 * rep)[0], n)
        got = g.search_batch(q768[:64], q256[:64], p, allow=allow)
        same(got, d.search_batch(q768[:64], q256[:64], p, allow=allow))


def test_replay_follows_route_precision(pair):
    g, d, oi, arrays, q768, q256 = pair
    p = Params(12, 500, Rerank.full(), 10)
    for prec in (True, False, True, False):
        g.set_route_precision(prec)
        d.set_route_precision(prec)
        for rep in range(3):
            same(g.search_batch(q768, q256, p), d.search_batch(q768, q256, p))


def test_replay_with_derived_prefix_and_params_mix(pair):
    g, d, oi, arrays, q768, q256 = pair
    configs = [Params(4, 100, Rerank.none(), 10), Params(16, 800, Rerank.prefix(), 20),
               Params(32, 1500, Rerank.full(), 10, prune=(10, 0.5))]
    for rep in range(3):
        for p in configs:
            same(g.search_batch(q768[:77], None, p), d.search_batch(q768[:77], None, p))
            same(g.search_batch(q768[:77], q256[:77], p), d.search_batch(q768[:77], q256[:77], p))
