"""sg_search_noalloc: the search entry point for callers that must not allocate device memory
while they serve queries (a latency-critical serving thread, where cudaFree synchronises the
device and cudaMalloc can wait behind running kernels; a host whose device-memory budget is fixed
up front). It takes all scratch from one fixed device array instead of cudaMalloc.

Checked through the C ABI against sg_search, bit for bit (the tolerance the parity tests use),
with two calls in a row per query: the array keeps the previous call's contents, so the second
call shows that everything that must start from zero is cleared. This file sorts last so that a
run stopping at the first failure has already run every other test.
"""
from ctypes import byref, c_uint64, c_void_p

import numpy as np
import pytest

from fixtures import index_a
from sieve_gpu import Index, Params, Rerank
from sieve_gpu._abi import check, lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("params", [Params(8, 500, Rerank.full(), 10),
                                    Params(16, 300, Rerank.tiered(100), 10),
                                    Params(12, 200, Rerank.prefix(), 5, prune=(10, 1.0))])
def test_noalloc_search_equals_search(params):
    import torch

    arrays, q768, q256, _ = index_a()
    ix = Index.from_arrays(arrays)
    try:
        nq = 6
        sc, ids, cnt = ix.search_batch(q768[:nq], None, params)
        dev = torch.device("cuda", ix.device)
        dq = torch.as_tensor(q768[:nq]).to(dev).contiguous()
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
                out_n.fill_(-1)
                check(lib().sg_search_noalloc(
                    ix._h, c_void_p(dq[i].data_ptr()), None, byref(cp), None, c_uint64(0),
                    c_void_p(out_s.data_ptr()), c_void_p(out_i.data_ptr()), c_void_p(out_n.data_ptr()),
                    c_void_p(stream.cuda_stream)))
                stream.synchronize()
                n = int(out_n.item())
                assert n == int(cnt[i])
                got_ids = out_i.cpu().numpy().view(np.uint32)[:n]
                got_sc = out_s.cpu().numpy()[:n]
                assert np.array_equal(got_ids, ids[i, :n])
                assert np.array_equal(got_sc, sc[i, :n])
    finally:
        ix.close()
