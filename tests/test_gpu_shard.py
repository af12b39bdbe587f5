"""Cluster sharding on the GPU: each shard's phase 1 (Index::candidates over the probes it owns,
sg_candidates_probes) and phase 2 (Index::rerank of its share, sg_rerank) against the oracle
shards of tests/shard_oracle.py, bit for bit, and the whole two-phase protocol of two GPU shards
against the same protocol run on the oracle shards. The shards share one GPU here (each an index
of its own clusters); the exchange between ranks is covered on gloo ranks in tests/test_shard.py.
"""
import numpy as np
import pytest

from fixtures import index_a, index_b
from shard_oracle import OracleShard
from sieve_gpu import Index, Params, Rerank
from sieve_gpu import shard as S
from test_shard import PARAMS, run_protocol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["a", "b"])
def shards(request):
    arrays, q768, q256, _ = (index_a if request.param == "a" else index_b)()
    slots = S.cluster_slots(arrays["block_off"])
    owner = S.assign(slots, 2)
    parts = [S.shard_arrays(arrays, owner, s) for s in range(2)]
    gpu = [Index.from_arrays(p) for p in parts]
    yield gpu, [OracleShard(p) for p in parts], owner, slots, q768, q256
    for g in gpu:
        g.close()


@pytest.mark.parametrize("pi", range(len(PARAMS)))
def test_phase1_matches_oracle(shards, pi):
    gpu, orc, owner, slots, q768, q256 = shards
    p = PARAMS[pi]
    for s in range(2):
        got = S.phase1(gpu[s], owner, s, slots, q256, p)
        want = S.phase1(orc[s], owner, s, slots, q256, p)
        for (ge, gr, gw), (we, wr, ww) in zip(got, want):
            assert np.array_equal(gr, wr) and np.array_equal(ge, we) and np.array_equal(gw, ww)


@pytest.mark.parametrize("pi", range(len(PARAMS)))
def test_protocol_matches_oracle(shards, pi):
    gpu, orc, owner, slots, q768, q256 = shards
    p = PARAMS[pi]
    got = run_protocol(gpu, owner, slots, q768, q256, p)
    want = run_protocol(orc, owner, slots, q768, q256, p)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_rerank_of_given_candidates_matches_oracle(shards):
    """sg_rerank on an arbitrary candidate list (every row of a probe list's first 50 slots)."""
    gpu, orc, owner, slots, q768, q256 = shards
    ids_all = np.arange(0, 3000, 7, dtype=np.uint32)
    est = np.linspace(1.0, 0.0, ids_all.size).astype(np.float32)
    err = np.full(ids_all.size, 0.01, np.float32)
    cands = [(est, ids_all, err)] * 8
    for p in (Params(1, 0, Rerank.full(), 10), Params(1, 0, Rerank.tiered(40), 10),
              Params(1, 0, Rerank.none(), 5, prune=(10, 0.5)), Params(1, 0, Rerank.prefix(), 10)):
        got = gpu[0].rerank(q768[:8], q256[:8], cands, p)
        want = orc[0].rerank(q768[:8], q256[:8], cands, p)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
