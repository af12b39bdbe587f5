"""GPU parity of the bigann query path (src/bigann.rs:653-747) against the oracle, through the C
ABI: probe lists, candidates (row, estimate, |x|^2) and final (score, row) lists, bit-exact, for
1-, 2- and 3-bit indexes, with and without the refined shortlist, with the margin rule, and with
shortlists small enough to compact many times inside one scan step."""
import numpy as np
import pytest

import oracle as O
from fixtures import bigann_a, bigann_b, bigann_c
from sieve_gpu.bigann import BigannIndex, BigannParams, BigannTiming

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[1, 2, 3], ids=["bits1", "bits2", "bits3"])
def env(request):
    ix, q = bigann_a(request.param)
    g = BigannIndex.from_arrays(ix)
    yield g, O.OracleBigann(ix), ix, q
    g.close()


@pytest.fixture(scope="module")
def env_b():
    ix, q = bigann_b()
    g = BigannIndex.from_arrays(ix)
    yield g, O.OracleBigann(ix), ix, q
    g.close()


def cp(p: BigannParams):
    return p.to_c()


@pytest.mark.parametrize("route_fp32", [False, True], ids=["tc", "fp32"])
@pytest.mark.parametrize("nprobe,margin", [(1, 0.0), (12, 0.0), (40, 0.0), (40, 0.05), (40, 0.3), (10**6, 0.0)])
def test_route_matches_oracle(env, nprobe, margin, route_fp32):
    g, ob, ix, q = env
    p = BigannParams(nprobe, 100, 10, 0, margin, route_fp32)
    got = g.route(q, p)
    for i in range(q.shape[0]):
        want, _, _ = ob.route(q[i], cp(p))
        assert np.array_equal(got[i], want), i


@pytest.fixture(scope="module")
def env_c():
    ix, q = bigann_c()
    g = BigannIndex.from_arrays(ix)
    yield g, O.OracleBigann(ix), ix, q
    g.close()


# 10,240 leaves: nprobe 1..300 take the subset threshold (cap 8,192 or 32 nprobe entries per
# query); 320 emits every leaf (640 subset leaves < 2 nprobe); 4096 the largest nprobe.
@pytest.mark.parametrize("route_fp32", [False, True], ids=["tc", "fp32"])
@pytest.mark.parametrize("nprobe,margin", [(1, 0.0), (64, 0.0), (64, 0.2), (300, 0.0), (320, 0.05), (4096, 0.0)])
def test_route_many_leaves_matches_oracle(env_c, nprobe, margin, route_fp32):
    g, ob, ix, q = env_c
    p = BigannParams(nprobe, 100, 10, 0, margin, route_fp32)
    before = g.route_fallbacks()
    got = g.route(q, p)
    for i in range(q.shape[0]):
        want, _, _ = ob.route(q[i], cp(p))
        assert np.array_equal(got[i], want), i
    if not route_fp32 and nprobe <= 320:
        # the rescoring windows fit: no query needed the exact fallback
        assert g.route_fallbacks() == before


def test_search_many_leaves_matches_oracle(env_c):
    g, ob, ix, q = env_c
    p = BigannParams(64, 200, 10, 0, 0.1)
    sc, ids, cnt = g.search_batch(q, p)
    for i in range(q.shape[0]):
        ws, wo, _ = ob.search(q[i], cp(p))
        assert np.array_equal(ids[i, : cnt[i]], wo), i
        assert np.array_equal(sc[i, : cnt[i]], ws), i


CASES = [(8, 100, 10, 0), (8, 100, 10, 500), (16, 40, 10, 60), (16, 10, 5, 30), (4, 3, 3, 0),
         (40, 300, 100, 2000), (6, 1, 1, 1)]


@pytest.mark.parametrize("nprobe,cand,k,refine", CASES)
def test_candidates_match_oracle(env, nprobe, cand, k, refine):
    g, ob, ix, q = env
    p = BigannParams(nprobe, cand, k, refine)
    got = g.candidates(q, p)
    for i in range(q.shape[0]):
        ids, est, nx, _ = ob.candidates(q[i], cp(p))
        gi, ge, gn = got[i]
        assert np.array_equal(gi, ids), i
        assert np.array_equal(ge, est), i
        assert np.array_equal(gn, nx), i


@pytest.mark.parametrize("nprobe,cand,k,refine", CASES)
def test_search_matches_oracle(env, nprobe, cand, k, refine):
    g, ob, ix, q = env
    p = BigannParams(nprobe, cand, k, refine)
    sc, ids, cnt = g.search_batch(q, p)
    s, o, c, _ = ob.search_batch(q, cp(p), threads=4)
    assert np.array_equal(cnt, c)
    for i in range(q.shape[0]):
        assert np.array_equal(ids[i, : cnt[i]], o[i, : c[i]]), i
        assert np.array_equal(sc[i, : cnt[i]], s[i, : c[i]]), i


@pytest.mark.parametrize("refine", [0, 100, 400])
@pytest.mark.parametrize("cand", [5, 50])
def test_large_leaves_many_compactions(env_b, cand, refine):
    g, ob, ix, q = env_b
    p = BigannParams(8, cand, 10, refine)
    got = g.candidates(q, p)
    for i in range(q.shape[0]):
        ids, est, nx, _ = ob.candidates(q[i], cp(p))
        assert np.array_equal(got[i][0], ids), i
        assert np.array_equal(got[i][1], est), i
    sc, gid, cnt = g.search_batch(q, p)
    s, o, c, _ = ob.search_batch(q, cp(p), threads=4)
    assert np.array_equal(cnt, c)
    for i in range(q.shape[0]):
        assert np.array_equal(gid[i, : cnt[i]], o[i, : c[i]]) and np.array_equal(sc[i, : cnt[i]], s[i, : c[i]])


def test_margin_search(env):
    g, ob, ix, q = env
    p = BigannParams(64, 200, 10, 500, 0.1)
    sc, ids, cnt = g.search_batch(q, p)
    s, o, c, _ = ob.search_batch(q, cp(p), threads=4)
    assert np.array_equal(cnt, c)
    for i in range(q.shape[0]):
        assert np.array_equal(ids[i, : cnt[i]], o[i, : c[i]]) and np.array_equal(sc[i, : cnt[i]], s[i, : c[i]])


def test_zero_cand_and_zero_k(env):
    g, ob, ix, q = env
    sc, ids, cnt = g.search_batch(q[:4], BigannParams(8, 0, 10))
    assert np.all(cnt == 0)
    sc, ids, cnt = g.search_batch(q[:4], BigannParams(8, 50, 0))
    assert np.all(cnt == 0)


def test_timing_counts(env):
    g, ob, ix, q = env
    t = BigannTiming()
    p = BigannParams(8, 100, 10, 200)
    g.search_batch(q, p, t)
    want = sum(int(ob.candidates(q[i], cp(p))[3]) for i in range(q.shape[0]))
    assert t.scanned == want and t.probes == 8 * q.shape[0]
    assert t.route > 0 and t.scan > 0 and t.rerank > 0


def test_open_from_files(env, tmp_path):
    from sieve_gpu import bigann_builder as BB

    g, ob, ix, q = env
    BB.write_files(ix, str(tmp_path / "idx"), str(tmp_path / "base"))
    g2 = BigannIndex.open(str(tmp_path / "idx"), str(tmp_path / "base"))
    try:
        p = BigannParams(8, 100, 10, 300)
        a = g.search_batch(q, p)
        b = g2.search_batch(q, p)
        assert np.array_equal(a[2], b[2])
        for i in range(q.shape[0]):
            n = int(a[2][i])
            assert np.array_equal(a[0][i, :n], b[0][i, :n]) and np.array_equal(a[1][i, :n], b[1][i, :n])
    finally:
        g2.close()


def test_invalid_params_are_rejected(env):
    from sieve_gpu import SieveError

    g, ob, ix, q = env
    with pytest.raises(SieveError):
        g.search_batch(q[:1], BigannParams(8, 5000, 10))
    with pytest.raises(SieveError):
        g.search_batch(q[:1], BigannParams(8, 100, 10, 0, float("nan")))
