"""The autotuner and the tuning controls (sg_autotune, sg_get_tuning, sg_set_tuning).

Every tuning of the batched path — the per-cluster split between the ALU and tcgen05 scans, the
ALU chunk size and CTAs per SM, the seed budget — must return exactly the same results: the
tests compare full result lists bit for bit across tunings, and against the oracle.
"""
import numpy as np
import pytest
import torch

import oracle as O
from fixtures import index_a
from sieve_gpu import Index, Params, Rerank, SieveError

pytestmark = pytest.mark.gpu


def batch(q768, reps):
    return np.ascontiguousarray(np.tile(q768, (reps, 1)), np.float32)


@pytest.fixture(scope="module")
def tuned():
    arrays, q768, q256, _ = index_a()
    ix = Index.from_arrays(arrays)
    yield ix, arrays, batch(q768, 2)  # 128 queries: the batched path
    ix.close()


def run(ix, q, p):
    return ix.search_batch(q, None, p)


@pytest.mark.parametrize("tmin", [1, 2, 6, 1000000])
def test_split_threshold_exact(tuned, tmin):
    ix, arrays, q = tuned
    p = Params(16, 500, Rerank.full(), 10)
    base = run(ix, q, p)
    old = ix.tuning()
    try:
        ix.set_tuning(tc_min_queries=tmin)
        got = run(ix, q, p)
    finally:
        ix.set_tuning(**old)
    for a, b in zip(base, got):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("field,value", [("chunk_blocks", 512), ("seed_blocks", 128), ("scan_ctas_per_sm", 1)])
def test_shapes_exact(tuned, field, value):
    ix, arrays, q = tuned
    p = Params(24, 400, Rerank.tiered(80), 10)
    base = run(ix, q, p)
    old = ix.tuning()
    try:
        ix.set_tuning(**{field: value})
        got = run(ix, q, p)
    finally:
        ix.set_tuning(**old)
    for a, b in zip(base, got):
        assert np.array_equal(a, b)


def test_autotune_keeps_results(tuned):
    ix, arrays, q = tuned
    p = Params(16, 500, Rerank.full(), 10)
    base = run(ix, q, p)
    dq = torch.as_tensor(q, device="cuda:0")
    old = ix.tuning()
    try:
        res = ix.autotune(q.shape[0], dq.data_ptr(), p, reps=1)
        assert res["ms_after"] <= res["ms_before"] * 1.0001
        assert ix.tuning() == {k: res[k] for k in old}
        got = run(ix, q, p)
        for a, b in zip(base, got):
            assert np.array_equal(a, b)
        # and the oracle agrees with the tuned index
        oi = O.OracleIndex(arrays)
        for i in range(0, q.shape[0], 17):
            s, o, _ = oi.search(q[i], O.prefix(q[i])[0], p.to_c())
            assert np.array_equal(got[1][i, : got[2][i]], o) and np.array_equal(got[0][i, : got[2][i]], s)
    finally:
        ix.set_tuning(**old)


def test_set_tuning_rejects_bad_values(tuned):
    ix, _, _ = tuned
    for bad in ({"chunk_blocks": 1024}, {"seed_blocks": 0}, {"scan_ctas_per_sm": 3}, {"tc_min_queries": 0}):
        with pytest.raises(SieveError):
            ix.set_tuning(**bad)


def test_autotune_rejects_small_batches(tuned):
    ix, _, q = tuned
    dq = torch.as_tensor(q[:8], device="cuda:0")
    with pytest.raises(SieveError):
        ix.autotune(8, dq.data_ptr(), Params(16, 500, Rerank.full(), 10))
