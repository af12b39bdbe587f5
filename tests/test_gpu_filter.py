"""GPU parity of filter::Filter::new and filter::search (src/filter.rs) against the oracle: the
allowed rows and per-cluster counts, and every plan (Post, Expand(target), Brute, Auto), bit-exact
(scores and rows)."""
import numpy as np
import pytest

import oracle as O
from fixtures import index_a, index_b
from sieve_gpu import Index, Params, Rerank, allow_bitset
from sieve_gpu import filter as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env_a():
    arrays, q768, q256, _ = index_a()
    ix = Index.from_arrays(arrays)
    yield ix, O.OracleIndex(arrays), arrays, q768, q256
    ix.close()


def make_allow(n, frac, seed, extra_words=0):
    rows = np.random.default_rng(seed).permutation(n)[: int(round(frac * n))]
    allow = allow_bitset(rows, n)
    if extra_words:
        allow = np.concatenate([allow, np.full(extra_words, np.uint64(0xFFFFFFFFFFFFFFFF))])
    return allow, np.sort(rows).astype(np.uint32)


def check_plan(ix, oi, f, allow, rows, plan: F.Plan, q768, q256, p: Params, use_q256=True):
    sc, ids, cnt = F.search_batch(ix, f, plan, q768, q256 if use_q256 else None, p)
    pcl = oi.filter_per_cluster(allow)
    for i in range(q768.shape[0]):
        s, o = oi.filter_search(allow, rows, pcl, plan.kind, plan.target, q768[i], q256[i], p.to_c())
        assert cnt[i] == s.size, i
        assert np.array_equal(ids[i, : cnt[i]], o), i
        assert np.array_equal(sc[i, : cnt[i]], s), i
        allowed = (allow[(o >> 6).astype(np.int64)] >> (o & 63).astype(np.uint64)) & np.uint64(1)
        assert np.all(allowed == 1)


@pytest.mark.parametrize("frac,extra", [(0.0, 0), (0.001, 0), (0.05, 0), (0.5, 3), (1.0, 0)])
def test_filter_new_matches_oracle(env_a, frac, extra):
    ix, oi, arrays, q768, q256 = env_a
    n = arrays["n"]
    allow, rows = make_allow(n, frac, 11, extra)
    with F.Filter(allow, ix) as f:
        assert f.nrows == rows.size  # bits past row n-1 name no row
        assert np.array_equal(f.rows, rows)
        assert np.array_equal(f.per_cluster, oi.filter_per_cluster(allow))


@pytest.mark.parametrize("frac", [0.3, 0.02])
def test_plan_post(env_a, frac):
    ix, oi, arrays, q768, q256 = env_a
    allow, rows = make_allow(arrays["n"], frac, 3)
    with F.Filter(allow, ix) as f:
        check_plan(ix, oi, f, allow, rows, F.Plan.post(), q768, q256, Params(16, 500, Rerank.full(), 10))


@pytest.mark.parametrize("target", [0, 1, 3000, 20000, 10**9])
@pytest.mark.parametrize("frac", [0.2, 0.01])
def test_plan_expand(env_a, frac, target):
    ix, oi, arrays, q768, q256 = env_a
    allow, rows = make_allow(arrays["n"], frac, 5)
    with F.Filter(allow, ix) as f:
        check_plan(ix, oi, f, allow, rows, F.Plan.expand(target), q768, q256,
                   Params(16, 500, Rerank.tiered(100), 10))


def test_plan_expand_params_mix(env_a):
    ix, oi, arrays, q768, q256 = env_a
    allow, rows = make_allow(arrays["n"], 0.05, 8)
    with F.Filter(allow, ix) as f:
        for p in (Params(8, 200, Rerank.none(), 20), Params(4, 1000, Rerank.prefix(), 10, prune=(10, 0.5)),
                  Params(64, 300, Rerank.full(), 10, margin=0.05, budget=2000)):
            check_plan(ix, oi, f, allow, rows, F.Plan.expand(4000), q768, q256, p, use_q256=False)


@pytest.mark.parametrize("frac,k", [(0.02, 10), (0.2, 100), (0.0002, 10), (0.0, 10)])
def test_plan_brute(env_a, frac, k):
    ix, oi, arrays, q768, q256 = env_a
    allow, rows = make_allow(arrays["n"], frac, 9)
    with F.Filter(allow, ix) as f:
        check_plan(ix, oi, f, allow, rows, F.Plan.brute(), q768, q256, Params(16, 500, Rerank.full(), k))


def test_plan_auto(env_a):
    ix, oi, arrays, q768, q256 = env_a
    allow, rows = make_allow(arrays["n"], 0.1, 2)
    with F.Filter(allow, ix) as f:
        assert F.Plan.auto().resolve(f, ix.n) == F.Plan.brute()  # 2,000 rows <= BRUTE_MAX
        check_plan(ix, oi, f, allow, rows, F.Plan.auto(), q768, q256, Params(16, 500, Rerank.full(), 10))


def test_expand_batch_equals_single(env_a):
    ix, oi, arrays, q768, q256 = env_a
    allow, rows = make_allow(arrays["n"], 0.05, 4)
    p = Params(16, 500, Rerank.full(), 10)
    with F.Filter(allow, ix) as f:
        sc, ids, cnt = F.search_batch(ix, f, F.Plan.expand(5000), q768, q256, p)
        for i in range(0, q768.shape[0], 11):
            one = F.search(ix, f, F.Plan.expand(5000), q768[i], q256[i], p)
            assert [r for _, r in one] == list(ids[i, : cnt[i]])
            assert [s for s, _ in one] == list(sc[i, : cnt[i]])


def test_expand_on_index_with_duplicates():
    arrays, q768, q256, _ = index_b()
    ix = Index.from_arrays(arrays)
    try:
        oi = O.OracleIndex(arrays)
        allow, rows = make_allow(arrays["n"], 0.1, 6)
        with F.Filter(allow, ix) as f:
            check_plan(ix, oi, f, allow, rows, F.Plan.expand(3000), q768, q256,
                       Params(4, 400, Rerank.full(), 10))
    finally:
        ix.close()


def test_filter_of_another_index_is_rejected(env_a):
    ix, oi, arrays, q768, q256 = env_a
    other = Index.from_arrays(arrays)
    try:
        allow, _ = make_allow(arrays["n"], 0.1, 1)
        with F.Filter(allow, other) as f:
            with pytest.raises(Exception):
                F.search_batch(ix, f, F.Plan.post(), q768[:2], q256[:2], Params(8, 100))
    finally:
        other.close()
