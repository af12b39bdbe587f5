"""Live updates on the GPU (src/live.rs) against the oracle's live model (tests/live_oracle.py):
the device's insert encoding, delta lists scanned after each base list, tombstones and upserts
give bit-exact (score, external id) lists under every scan the batch may take."""
import numpy as np
import pytest

from fixtures import index_a
from live_oracle import OracleLive
from sieve_gpu import Index, Params, Rerank
from sieve_gpu.live import Live

pytestmark = pytest.mark.gpu

PARAMS = [Params(16, 500, Rerank.full(), 10), Params(12, 300, Rerank.tiered(80), 10),
          Params(8, 200, Rerank.none(), 10), Params(12, 300, Rerank.prefix(), 10),
          Params(24, 400, Rerank.full(), 10, prune=(10, 1.0))]


def scenario(live, model, mix):
    """Three insert batches (new vectors, copies of corpus rows, an upsert of a corpus row and of
    an inserted row), deletes of corpus and inserted rows."""
    rng = np.random.default_rng(3)
    a = mix.queries(300, sigma=0.3, seed=11).numpy().astype(np.float32)
    b = mix.rows(1000, 40).numpy().astype(np.float32)
    for obj in (live, model):
        obj.insert(np.arange(2_000_000, 2_000_300), a)
        obj.insert(np.arange(3_000_000, 3_000_040), b)
        obj.delete([1000, 1001, 2_000_005, 77, 99_999_999])
        obj.insert([1002, 2_000_010], a[:2][::-1].copy())
    return rng


@pytest.fixture(scope="module", params=["1", "0"], ids=["auto", "alu"])
def live_pair(request):
    import os

    old = os.environ.get("SIEVE_GPU_MMA")
    os.environ["SIEVE_GPU_MMA"] = request.param
    try:
        arrays, q768, q256, mix = index_a()
        ix = Index.from_arrays(arrays)
    finally:
        if old is None:
            del os.environ["SIEVE_GPU_MMA"]
        else:
            os.environ["SIEVE_GPU_MMA"] = old
    live = Live(ix, max_rows=1000, soar_lambda=1.0)
    model = OracleLive(arrays, 1.0)
    scenario(live, model, mix)
    # queries: the fixture's, plus copies of inserted and deleted rows
    extra = np.concatenate([mix.queries(300, sigma=0.3, seed=11).numpy()[:12], mix.rows(1000, 4).numpy()])
    q = np.concatenate([q768, extra]).astype(np.float32)
    qp = q[:, :256] / np.linalg.norm(q[:, :256], axis=1, keepdims=True)
    yield live, model, q, qp.astype(np.float32)
    live.close()
    ix.close()


def test_live_info(live_pair):
    live, model, _, _ = live_pair
    info = live.info()
    assert info["delta_rows"] == len(model.ext) == 342
    assert info["delta_slots"] == sum(len(x) for x in model.lists)
    assert info["deleted"] == len(model.deleted)


@pytest.mark.parametrize("pi", range(len(PARAMS)))
def test_live_search_matches_oracle(live_pair, pi):
    live, model, q, qp = live_pair
    p = PARAMS[pi]
    sc, ids, cnt = live.search_batch(q, qp, p)
    wsc, wids, wcnt = model.search_batch(q, qp, p)
    for i in range(q.shape[0]):
        assert cnt[i] == wcnt[i], i
        assert np.array_equal(ids[i, : cnt[i]], wids[i, : cnt[i]]), i
        assert np.array_equal(sc[i, : cnt[i]], wsc[i, : cnt[i]]), i


def test_deleted_rows_never_return(live_pair):
    live, model, q, qp = live_pair
    _, ids, cnt = live.search_batch(q, qp, PARAMS[0])
    gone = {1000, 1001, 2_000_005, 77}
    for i in range(q.shape[0]):
        assert not gone & set(ids[i, : cnt[i]].tolist())
