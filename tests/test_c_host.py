"""The C ABI from a C host: tests/host_search.c (gcc, C99, pthreads) opens an index from the
reference's files and searches through sg_search and through two threads' search contexts.
The CPU test compiles it against include/sieve_gpu.h with every warning an error; the GPU test
runs it and compares its results with the Python API's, bit for bit."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "a-game-of-vectors_b200", "sieve_gpu", "_lib")


def build(tmp_path) -> str:
    exe = str(tmp_path / "host_search")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-O2",
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "host_search.c"), "-o", exe,
           "-L", LIBDIR, "-lsieve_gpu", f"-Wl,-rpath,{LIBDIR}", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_host_compiles(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libsieve_gpu.so")):
        pytest.skip("the CUDA library is not built")
    build(tmp_path)


@pytest.mark.gpu
def test_c_host_matches_python(tmp_path):
    from fixtures import index_a
    from sieve_gpu import Index, Params, Rerank, builder

    arrays, q768, _, _ = index_a()
    ing, idx = str(tmp_path / "ingest"), str(tmp_path / "index")
    builder.write_files(arrays, arrays, ing, idx)
    qf = tmp_path / "q.f32"
    q768.astype(np.float32).tofile(qf)
    out = tmp_path / "out.bin"
    exe = build(tmp_path)
    r = subprocess.run([exe, ing, idx, str(qf), str(q768.shape[0]), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nq, k = q768.shape[0], 10
    raw = np.fromfile(out, np.uint8)
    ix = Index.open(ing, idx)
    try:
        sc, ids, cnt = ix.search_batch(q768, None, Params(16, 500, Rerank.full(), k))
    finally:
        ix.close()
    off = 0
    for _ in range(3):
        c = raw[off:off + nq * 4].view(np.uint32)
        off += nq * 4
        s = raw[off:off + nq * k * 4].view(np.float32).reshape(nq, k)
        off += nq * k * 4
        i = raw[off:off + nq * k * 4].view(np.uint32).reshape(nq, k)
        off += nq * k * 4
        assert np.array_equal(c, cnt)
        for q in range(nq):
            assert np.array_equal(i[q, : c[q]], ids[q, : cnt[q]]) and np.array_equal(s[q, : c[q]], sc[q, : cnt[q]])
