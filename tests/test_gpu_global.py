"""GPU parity of the global sign-code ablation (src/ivf.rs:700-717) and the flat Hamming baseline
(src/bin/search.rs:251-269) against the oracle, through the C ABI.

A global-code index has no rotation.f32 / factors.f32: the LUT is built on the unrotated prefix,
candidates are the best u16 LUT scores with ties by row (scores tie often: they are integers
below 16,320), their estimates lut.to_float(score), and their error widths infinite. The bar is
bit-exact (score, row) lists and candidate triples under every scan the batch may take.
"""
import numpy as np
import pytest

import oracle as O
from fixtures import index_g
from sieve_gpu import Index, Params, Rerank

pytestmark = pytest.mark.gpu

PARAMS = [Params(4, 300, Rerank.full(), 10), Params(8, 500, Rerank.tiered(60), 10),
          Params(6, 200, Rerank.none(), 10), Params(6, 200, Rerank.prefix(), 10),
          Params(16, 100, Rerank.full(), 10, prune=(10, 1.0)), Params(3, 40, Rerank.ssd(20), 5)]


@pytest.fixture(scope="module", params=["1", "2", "0"], ids=["auto", "tc", "alu"])
def gpu_g(request):
    import os

    old = os.environ.get("SIEVE_GPU_MMA")
    os.environ["SIEVE_GPU_MMA"] = request.param
    try:
        arrays, q768, q256 = index_g()
        ix = Index.from_arrays(arrays, codes=True)
    finally:
        if old is None:
            del os.environ["SIEVE_GPU_MMA"]
        else:
            os.environ["SIEVE_GPU_MMA"] = old
    yield ix, O.OracleIndex(arrays), arrays, q768, q256
    ix.close()


@pytest.mark.parametrize("pi", range(len(PARAMS)))
def test_global_search_matches_oracle(gpu_g, pi):
    ix, oi, _, q768, q256 = gpu_g
    p = PARAMS[pi]
    sc, ids, cnt = ix.search_batch(q768, None, p)
    for i in range(q768.shape[0]):
        s, o, _ = oi.search(q768[i], q256[i], p.to_c())
        assert np.array_equal(ids[i, : cnt[i]], o), i
        assert np.array_equal(sc[i, : cnt[i]], s), i


def test_global_candidates_match_oracle(gpu_g):
    ix, oi, _, q768, q256 = gpu_g
    p = Params(6, 250, Rerank.full(), 10)
    got = ix.candidates(q256[:24], p)
    for i in range(24):
        ps, pc = oi.route(q256[i], p.to_c())
        e, r, w = oi.candidates(q256[i], ps, pc, p.to_c())
        assert np.array_equal(got[i][1], r) and np.array_equal(got[i][0], e)
        assert np.all(np.isinf(got[i][2]))


@pytest.mark.parametrize("cand,k", [(300, 10), (1000, 100), (7, 3)])
def test_flat_hamming_matches_oracle(gpu_g, cand, k):
    ix, oi, arrays, q768, q256 = gpu_g
    sc, ids, cnt = ix.flat_hamming(q768, None, cand=cand, k=k)
    for i in range(q768.shape[0]):
        s, o = oi.flat_hamming(arrays["codes"], q768[i], q256[i], cand, k)
        assert np.array_equal(ids[i, : cnt[i]], o), i
        assert np.array_equal(sc[i, : cnt[i]], s), i


def test_flat_hamming_needs_codes():
    arrays, q768, _ = index_g()
    ix = Index.from_arrays(arrays)
    try:
        from sieve_gpu import SieveError

        with pytest.raises(SieveError) as e:
            ix.flat_hamming(q768[:2])
        assert e.value.status == -7
    finally:
        ix.close()
