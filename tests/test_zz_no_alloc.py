"""sg_search_noalloc: the search entry point for callers that must not allocate device memory
while they serve queries (a latency-critical serving thread, where cudaFree synchronises the
device and cudaMalloc can wait behind running kernels; a host whose device-memory budget is fixed
up front). It takes all scratch from one fixed device array instead of cudaMalloc.

Checked through the C ABI against sg_search, bit for bit (the tolerance the parity tests use),
with two calls in a row per query: the array keeps the previous call's contents, so the second
call shows that everything that must start from zero is cleared. Covered: the derived and the
given 256-d prefix, an allow bitset, the result count never reading SG_COUNT_FAILED on a call
that ran, and the rejection of params whose scratch exceeds the array. This file sorts last so
that a run stopping at the first failure has already run every other test.
"""
from ctypes import byref, c_uint64, c_void_p

import numpy as np
import pytest

from fixtures import index_a
from sieve_gpu import Index, Params, Rerank, SieveError, allow_bitset
from sieve_gpu._abi import check, lib

pytestmark = pytest.mark.gpu

COUNT_FAILED = 0xFFFFFFFF


def _noalloc(ix, dq768, dq256, cp, dallow, words, out_s, out_i, out_n, stream):
    check(lib().sg_search_noalloc(
        ix._h, c_void_p(dq768), c_void_p(dq256) if dq256 else None, byref(cp),
        c_void_p(dallow) if dallow else None, c_uint64(words), c_void_p(out_s.data_ptr()),
        c_void_p(out_i.data_ptr()), c_void_p(out_n.data_ptr()), c_void_p(stream.cuda_stream)))


@pytest.mark.parametrize("params", [Params(8, 500, Rerank.full(), 10),
                                    Params(16, 300, Rerank.tiered(100), 10),
                                    Params(12, 200, Rerank.prefix(), 5, prune=(10, 1.0))])
@pytest.mark.parametrize("given_q256", [False, True], ids=["derived_q256", "given_q256"])
@pytest.mark.parametrize("filtered", [False, True], ids=["all_rows", "allow_bitset"])
def test_noalloc_search_equals_search(params, given_q256, filtered):
    import torch

    arrays, q768, q256, _ = index_a()
    ix = Index.from_arrays(arrays)
    try:
        nq = 6
        allow = None
        if filtered:  # every third row, and the self-match rows the queries copy
            allow = allow_bitset(np.arange(0, int(arrays["n"]), 3), int(arrays["n"]))
        sc, ids, cnt = ix.search_batch(q768[:nq], q256[:nq] if given_q256 else None, params, allow)
        dev = torch.device("cuda", ix.device)
        dq = torch.as_tensor(q768[:nq]).to(dev).contiguous()
        dq2 = torch.as_tensor(q256[:nq]).to(dev).contiguous()
        dal = torch.as_tensor(allow.view(np.int64)).to(dev) if filtered else None
        k = params.k
        out_s = torch.empty(k, dtype=torch.float32, device=dev)
        out_i = torch.empty(k, dtype=torch.int32, device=dev)
        out_n = torch.empty(1, dtype=torch.int32, device=dev)
        cp = params.to_c()
        stream = torch.cuda.current_stream(dev)
        for i in range(nq):
            for _ in range(2):  # two calls in a row on the same scratch
                out_s.fill_(-7.0)
                out_i.fill_(-1)
                out_n.fill_(-2)
                _noalloc(ix, dq[i].data_ptr(), dq2[i].data_ptr() if given_q256 else None, cp,
                         dal.data_ptr() if filtered else None, 0 if allow is None else allow.size,
                         out_s, out_i, out_n, stream)
                stream.synchronize()
                n = int(out_n.cpu().numpy().view(np.uint32)[0])
                assert n != COUNT_FAILED, "the device reported a failure"
                assert n == int(cnt[i])
                got_ids = out_i.cpu().numpy().view(np.uint32)[:n]
                got_sc = out_s.cpu().numpy()[:n]
                assert np.array_equal(got_ids, ids[i, :n])
                assert np.array_equal(got_sc, sc[i, :n])
    finally:
        ix.close()


def _one_big_cluster(slots: int = 3_000_000, rows: int = 1000) -> dict:
    """An index of one cluster holding `slots` slots over `rows` corpus rows (ids cycle through
    the rows): large enough that one query's exact candidate bound exceeds the fixed array."""
    nb = slots // 32
    r = np.random.default_rng(7)
    return {
        "n": rows, "k": 1,
        "centroids": np.ones((1, 256), np.float32) / 16.0,
        "block_off": np.array([0, nb], np.uint64),
        "ids": (np.arange(nb * 32, dtype=np.uint64) % rows).astype(np.uint32),
        "blocks": np.zeros(nb * 1024, np.uint8),
        "factors": np.tile(np.array([1.0, 0.0], np.float32), nb * 32),
        "rotation": np.where(r.random(768) < 0.5, -1.0, 1.0).astype(np.float32),
        "rerank": r.integers(-127, 128, (rows, 768), dtype=np.int8),
        "quant_scale": np.full(768, 127.0, np.float32),
    }


def test_noalloc_rejects_params_beyond_the_array():
    """Params whose buffers need more than the fixed 32 MiB array are refused before any device
    work, with SG_ERR_INVALID; the output buffers are left untouched."""
    import torch

    ix = Index.from_arrays(_one_big_cluster())
    try:
        dev = torch.device("cuda", ix.device)
        q = np.zeros((1, 768), np.float32)
        q[0, 0] = 1.0
        dq = torch.as_tensor(q).to(dev).contiguous()
        out_s = torch.full((10,), -7.0, dtype=torch.float32, device=dev)
        out_i = torch.full((10,), -1, dtype=torch.int32, device=dev)
        out_n = torch.full((1,), -2, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev)
        # 4096 candidates over 1,465 scan chunks: the candidate buffer is bounded by the cluster's
        # 3M slots, 36 MB at 12 B each, beyond the 32 MiB array
        big = Params(1, 4096, Rerank.full(), 10).to_c()
        with pytest.raises(SieveError) as e:
            _noalloc(ix, dq[0].data_ptr(), None, big, None, 0, out_s, out_i, out_n, stream)
        assert e.value.status == -1 and "scratch" in str(e.value)
        stream.synchronize()
        assert int(out_n.item()) == -2 and float(out_s[0].item()) == -7.0
    finally:
        ix.close()
