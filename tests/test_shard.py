"""Cluster sharding with the two-phase merge (src/shard.rs), host side: the LPT ownership, the
per-shard index arrays, the coordinator's cut and merge, and the protocol's two all-gathers on
two gloo ranks on the CPU, each shard's computations done by the oracle (tests/shard_oracle.py).
The GPU shards are compared with the same oracle shards in tests/test_gpu_shard.py."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fixtures import index_a
from shard_oracle import OracleShard
from sieve_gpu import Params, Rerank
from sieve_gpu import shard as S

PARAMS = [Params(12, 300, Rerank.full(), 10), Params(16, 400, Rerank.tiered(80), 10),
          Params(8, 200, Rerank.none(), 10), Params(12, 300, Rerank.ssd(60), 10),
          Params(24, 300, Rerank.full(), 10, prune=(10, 1.0), margin=0.3, budget=8000)]


def test_balance_evens_out_load():
    """src/shard.rs:336-340."""
    sizes = [9, 7, 5, 4, 3, 2]
    owner = S.assign(sizes, 2)
    load = [sum(s for s, o in zip(sizes, owner) if o == x) for x in (0, 1)]
    assert load == [15, 15]


def test_shard_arrays_partition_the_slots():
    arrays = index_a()[0]
    sizes = S.cluster_slots(arrays["block_off"])
    owner = S.assign(sizes, 3)
    parts = [S.shard_arrays(arrays, owner, s) for s in range(3)]
    ids = np.asarray(arrays["ids"]).reshape(-1, 32)
    boff = np.asarray(arrays["block_off"], np.int64)
    for c in range(int(arrays["k"])):
        p = parts[owner[c]]
        pb = np.asarray(p["block_off"], np.int64)
        assert np.array_equal(np.asarray(p["ids"]).reshape(-1, 32)[pb[c]:pb[c + 1]], ids[boff[c]:boff[c + 1]])
        for s in range(3):
            if s != owner[c]:
                pbs = np.asarray(parts[s]["block_off"], np.int64)
                assert pbs[c] == pbs[c + 1]
    assert sum(int(np.asarray(p["block_off"])[-1]) for p in parts) == int(boff[-1])


def run_protocol(shards, owner, slots, q768, q256, params):
    """The protocol in one process: every shard's phase 1, the cut, every shard's phase 2, the
    merge (what the ranks do between their all-gathers)."""
    n = len(shards)
    cands = [S.phase1(sh, owner, s, slots, q256, params) for s, sh in enumerate(shards)]
    cuts = [S.global_cut([cands[s][i] for s in range(n)], params, n) for i in range(q768.shape[0])]
    res = [S.phase2(sh, q768, q256, cuts, s) for s, sh in enumerate(shards)]
    return S.pack([S.merge(cuts[i], [res[s][i] for s in range(n)], params.k) for i in range(q768.shape[0])],
                  params.k)


def test_two_shards_recall_matches_one_node():
    """The merged lists rank about as a single node would (src/shard.rs:1-16; the reference
    shows two-phase recall equal to single-node recall). They are not identical: a shard
    deduplicates its own candidates, so a row whose two SOAR copies it holds takes one place of its
    cut instead of two and the union can hold a row the single node's cut missed. Every query keeps
    at least 8 of the single node's top 10, and the scores at each rank are never lower."""
    arrays, q768, q256, _ = index_a()
    slots = S.cluster_slots(arrays["block_off"])
    owner = S.assign(slots, 2)
    shards = [OracleShard(S.shard_arrays(arrays, owner, s)) for s in range(2)]
    one = OracleShard(arrays)
    p = PARAMS[0]
    sc, ids, cnt = run_protocol(shards, owner, slots, q768, q256, p)
    for i in range(q768.shape[0]):
        s, o, _ = one.oi.search(q768[i], q256[i], p.to_c())
        assert len(set(ids[i, : cnt[i]].tolist()) & set(o.tolist())) >= 8
        assert cnt[i] == len(o) and np.all(sc[i, : cnt[i]] >= s)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, pi: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        arrays, q768, q256, _ = index_a()
        slots = S.cluster_slots(arrays["block_off"])
        owner = S.assign(slots, world)
        sh = S.ShardedIndex(OracleShard(S.shard_arrays(arrays, owner, rank)), owner, slots, rank, world)
        out = sh.search_batch(q768, q256, PARAMS[pi])
        q.put((rank, [x.tolist() for x in out]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("pi", [0, 1, 2])
def test_two_gloo_ranks_run_the_protocol(pi):
    """Two ranks, each holding its shard, exchange candidates and reranked lists by all-gather and
    both return exactly the lists of the protocol run in one process."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, pi, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    arrays, q768, q256, _ = index_a()
    slots = S.cluster_slots(arrays["block_off"])
    owner = S.assign(slots, 2)
    want = run_protocol([OracleShard(S.shard_arrays(arrays, owner, s)) for s in range(2)], owner, slots, q768,
                        q256, PARAMS[pi])
    for r in range(2):
        for a, b in zip(got[r], want):
            assert np.array_equal(np.asarray(a, dtype=b.dtype), b)
