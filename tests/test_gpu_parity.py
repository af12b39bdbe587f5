"""GPU parity: every kernel and the whole query path against the CPU oracle, through the C ABI.

Bar: integer LUT scores, int8 dots, probe lists, candidate (estimate, row, error) triples and
final (score, row) lists are bit-exact. Float estimates equal the oracle's because both run the
reference's f32 operations in the reference's order; the tolerance is therefore zero (the
north-star allowance of 1e-5 relative is not needed).
"""
import numpy as np
import pytest

import oracle as O
from fixtures import index_a, index_b, index_c, index_d
from sieve_gpu import Index, Params, Rerank, allow_bitset, dot_i8i8, lut_scan
from sieve_gpu._abi import SgParams

pytestmark = pytest.mark.gpu


def cparams(p: Params) -> SgParams:
    return p.to_c()


def open_with(arrays, scan_mode: str):
    """Opens an index with the scan chosen by SIEVE_GPU_MMA (0 ALU, 1 automatic, 2 tensor-core);
    a suffix "h" selects the exact one-hot tcgen05 contraction instead of the bound pass
    (SIEVE_GPU_TC=2)."""
    import os

    tc = "2" if scan_mode.endswith("h") else "1"
    env = {"SIEVE_GPU_MMA": scan_mode.rstrip("h"), "SIEVE_GPU_TC": tc}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return Index.from_arrays(arrays)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.fixture(scope="module", params=["1", "2", "2h", "0"], ids=["auto", "tc", "onehot", "alu"])
def gpu_a(request):
    arrays, q768, q256, _ = index_a()
    ix = open_with(arrays, request.param)
    yield ix, O.OracleIndex(arrays), arrays, q768, q256
    ix.close()


@pytest.fixture(scope="module", params=["1", "2", "2h"], ids=["auto", "tc", "onehot"])
def gpu_b(request):
    arrays, q768, q256, _ = index_b()
    ix = open_with(arrays, request.param)
    yield ix, O.OracleIndex(arrays), arrays, q768, q256
    ix.close()


# ---- kernels ---------------------------------------------------------------------------------
@pytest.mark.parametrize("groups", [64, 32])
@pytest.mark.parametrize("seed", range(4))
def test_lut_scan_matches_oracle(groups, seed):
    r = np.random.default_rng(seed)
    q = r.uniform(-1, 1, groups * 4).astype(np.float32)
    tables, _, _ = O.lut_new(q)
    blocks = r.integers(0, 256, (777, groups * 16), dtype=np.uint8)
    assert np.array_equal(lut_scan(tables, blocks), O.scan(tables, blocks))


def test_lut_scan_extremes():
    tables = np.full((64, 16), 255, np.uint8)
    blocks = np.random.default_rng(1).integers(0, 256, (64, 1024), dtype=np.uint8)
    got = lut_scan(tables, blocks)
    assert np.all(got == 64 * 255)
    tables[:, 0] = 0
    zero = np.zeros((3, 1024), np.uint8)
    assert np.all(lut_scan(tables, zero) == 0)
    assert np.array_equal(lut_scan(tables, blocks), O.scan(tables, blocks))


@pytest.mark.parametrize("dim", [768, 256, 100, 4])
def test_dot_i8i8_matches_oracle(dim):
    r = np.random.default_rng(dim)
    q = r.integers(-128, 128, dim, dtype=np.int8)
    rows = r.integers(-128, 128, (513, dim), dtype=np.int8)
    rows[0] = -128
    q2 = q.copy()
    got = dot_i8i8(q, rows)
    want = np.array([O.dot_i8i8(q2, x) for x in rows], np.int32)
    assert np.array_equal(got, want)


def test_query_prep_matches_oracle(gpu_a):
    ix, oi, arrays, q768, q256 = gpu_a
    tables, sc, bi, a, b = ix.query_prep(q256)
    for i in range(q256.shape[0]):
        t, s, bb, aa, b2 = O.query_new(arrays["rotation"], q256[i])
        assert np.array_equal(tables[i], t)
        assert (sc[i], bi[i], a[i], b[i]) == (np.float32(s), np.float32(bb), np.float32(aa), np.float32(b2))


# ---- routing ---------------------------------------------------------------------------------
ROUTE_CASES = [
    Params(8, 100),
    Params(16, 100, margin=0.05),
    Params(64, 100),
    Params(200, 100),
    Params(12, 100, budget=3000),
    Params(12, 100, budget=1),
    Params(12, 100, margin=0.0),
]


@pytest.mark.parametrize("bf16", [False, True])
@pytest.mark.parametrize("case", range(len(ROUTE_CASES)))
def test_route_matches_oracle(gpu_a, bf16, case):
    ix, oi, arrays, q768, q256 = gpu_a
    p = ROUTE_CASES[case]
    ix.set_route_precision(bf16)
    got = ix.route(q256, p)
    ix.set_route_precision(True)
    for i in range(q256.shape[0]):
        s, c = oi.route(q256[i], cparams(p))
        assert np.array_equal(got[i][1], c), f"query {i}"
        assert np.array_equal(got[i][0], s), f"query {i}"


def _bf16(x: np.ndarray) -> np.ndarray:
    """f32 -> bf16 (round to nearest even), returned as f32; finite inputs."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


@pytest.fixture(scope="module", params=["a", "c"])
def gpu_route(request):
    arrays, q768, q256, _ = (index_a if request.param == "a" else index_c)()
    ix = Index.from_arrays(arrays)
    yield ix, O.OracleIndex(arrays), arrays, q768, q256
    ix.close()


@pytest.fixture(scope="module", params=["a", "c", "d"])
def gpu_route_scores(request):
    arrays, q768, q256, _ = {"a": index_a, "c": index_c, "d": index_d}[request.param]()
    ix = Index.from_arrays(arrays)
    yield ix, None, arrays, q768, q256
    ix.close()


def test_route_scores_fp32_bit_exact(gpu_route_scores):
    """FP32 routing scores are blas::gemm_abt's sequential sums (src/blas.rs:46-52) bit for bit."""
    ix, _, arrays, q768, q256 = gpu_route_scores
    ix.set_route_precision(False)
    try:
        got = ix.route_scores(q256)
    finally:
        ix.set_route_precision(True)
    want = O.gemm_abt(q256, arrays["centroids"])
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_route_scores_bf16_gemm(gpu_route_scores):
    """The tcgen05 BF16 GEMM: every (query, centroid) score equals the exact product of the
    bf16-rounded operands up to FP32 accumulation error (512 * 2^-23 * sum|q_i c_i|), and lies
    within the rescoring window's delta = 0.0085 |q| max|c| of the FP32 score."""
    ix, _, arrays, q768, q256 = gpu_route_scores
    got = ix.route_scores(q256)
    cent = np.asarray(arrays["centroids"], np.float32)
    qb, cb = _bf16(q256).astype(np.float64), _bf16(cent).astype(np.float64)
    exact = qb @ cb.T
    acc_tol = 512 * 2.0**-23 * (np.abs(qb) @ np.abs(cb).T) + 1e-30
    err = np.abs(got.astype(np.float64) - exact)
    assert np.all(err <= acc_tol), f"max excess {np.max(err - acc_tol)}"
    fp32 = O.gemm_abt(q256, cent).astype(np.float64)
    delta = 0.0085 * np.linalg.norm(q256, axis=1)[:, None] * np.max(np.linalg.norm(cent, axis=1))
    assert np.all(np.abs(got - fp32) <= delta)
    # the scores differ from FP32's (the GEMM ran in bf16), so the check above is not vacuous
    assert np.any(got != fp32.astype(np.float32))


@pytest.mark.parametrize("bf16", [False, True])
@pytest.mark.parametrize("p", [Params(20, 100), Params(300, 100), Params(40, 100, margin=0.1)])
def test_route_many_tiles_matches_oracle(gpu_route, bf16, p):
    ix, oi, arrays, q768, q256 = gpu_route
    ix.set_route_precision(bf16)
    try:
        got = ix.route(q256, p)
    finally:
        ix.set_route_precision(True)
    for i in range(q256.shape[0]):
        s, c = oi.route(q256[i], cparams(p))
        assert np.array_equal(got[i][1], c), f"query {i}"
        assert np.array_equal(got[i][0], s), f"query {i}"


# ---- candidates ------------------------------------------------------------------------------
CAND_CASES = [Params(8, 500), Params(16, 200), Params(4, 3000), Params(64, 1), Params(32, 4096)]


@pytest.mark.parametrize("case", range(len(CAND_CASES)))
@pytest.mark.parametrize("which", ["a", "b"])
def test_candidates_match_oracle(gpu_a, gpu_b, case, which):
    ix, oi, arrays, q768, q256 = gpu_a if which == "a" else gpu_b
    p = CAND_CASES[case]
    if which == "b":
        p = Params(min(p.nprobe, 8), p.cand)
    got = ix.candidates(q256, p)
    for i in range(q256.shape[0]):
        s, c = oi.route(q256[i], cparams(p))
        e, ids, err = oi.candidates(q256[i], s, c, cparams(p))
        assert np.array_equal(got[i][1], ids), f"query {i}"
        assert np.array_equal(got[i][0], e), f"query {i}"
        assert np.array_equal(got[i][2], err), f"query {i}"


# ---- the whole path ---------------------------------------------------------------------------
SEARCH_CASES = [
    Params(8, 500, Rerank.full(), 10),
    Params(16, 1000, Rerank.full(), 100),
    Params(8, 500, Rerank.tiered(200), 10),
    Params(8, 500, Rerank.prefix(), 10),
    Params(8, 500, Rerank.none(), 10),
    Params(8, 500, Rerank.ssd(100), 10),
    Params(8, 500, Rerank.full(), 10, prune=(10, 1.0)),
    Params(8, 500, Rerank.tiered(50), 10, prune=(10, 0.5)),
    Params(32, 500, Rerank.full(), 10, margin=0.1),
    Params(32, 500, Rerank.full(), 10, budget=4000),
    Params(4, 20, Rerank.full(), 50),
    Params(8, 300, Rerank.full(), 0),
]


def check_search(ix, oi, q768, q256, p, allow=None):
    sc, ids, cnt = ix.search_batch(q768, q256, p, allow=allow)
    for i in range(q768.shape[0]):
        s, o, _ = oi.search(q768[i], q256[i], cparams(p), allow=allow)
        assert cnt[i] == s.size, f"query {i}"
        assert np.array_equal(ids[i, : cnt[i]], o), f"query {i}"
        assert np.array_equal(sc[i, : cnt[i]], s), f"query {i}"


@pytest.mark.parametrize("case", range(len(SEARCH_CASES)))
def test_search_matches_oracle_a(gpu_a, case):
    ix, oi, arrays, q768, q256 = gpu_a
    check_search(ix, oi, q768, q256, SEARCH_CASES[case])


@pytest.mark.parametrize("case", [0, 2, 3, 5, 6])
def test_search_matches_oracle_b_ties(gpu_b, case):
    ix, oi, arrays, q768, q256 = gpu_b
    p = SEARCH_CASES[case]
    check_search(ix, oi, q768, q256, Params(min(p.nprobe, 8), p.cand, p.rerank, p.k, p.prune))


def test_search_without_q256_derives_the_prefix(gpu_a):
    ix, oi, arrays, q768, q256 = gpu_a
    p = Params(8, 500, Rerank.full(), 10)
    a = ix.search_batch(q768, None, p)
    b = ix.search_batch(q768, q256, p)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("frac", [0.5, 0.05, 0.0])
def test_search_with_allow_filter(gpu_a, frac):
    ix, oi, arrays, q768, q256 = gpu_a
    n = arrays["n"]
    rows = np.random.default_rng(7).permutation(n)[: int(frac * n)]
    allow = allow_bitset(rows, n)
    check_search(ix, oi, q768, q256, Params(16, 500, Rerank.full(), 10), allow=allow)


def test_short_allow_bitset_hides_the_tail(gpu_a):
    ix, oi, arrays, q768, q256 = gpu_a
    allow = allow_bitset(np.arange(5000), 5000)  # words cover rows < 5056 only
    check_search(ix, oi, q768, q256, Params(16, 500, Rerank.full(), 10), allow=allow)


def test_batch_equals_single(gpu_a):
    ix, oi, arrays, q768, q256 = gpu_a
    p = Params(16, 500, Rerank.tiered(100), 10)
    sc, ids, cnt = ix.search_batch(q768, q256, p)
    for i in range(0, q768.shape[0], 7):
        s1, i1, c1 = ix.search_batch(q768[i : i + 1], q256[i : i + 1], p)
        assert c1[0] == cnt[i]
        assert np.array_equal(i1[0, : c1[0]], ids[i, : cnt[i]])
        assert np.array_equal(s1[0, : c1[0]], sc[i, : cnt[i]])


def test_empty_batch(gpu_a):
    ix = gpu_a[0]
    sc, ids, cnt = ix.search_batch(np.zeros((0, 768), np.float32), None, Params(8, 100))
    assert cnt.size == 0


def test_open_from_files_matches_arrays(gpu_a, tmp_path):
    ix, oi, arrays, q768, q256 = gpu_a
    from sieve_gpu import builder

    corpus = {k: arrays[k] for k in ("n", "rerank", "norm256", "codes", "quant_scale")}
    builder.write_files(corpus, arrays, str(tmp_path / "ingest"), str(tmp_path / "index"))
    ix2 = Index.open(str(tmp_path / "ingest"), str(tmp_path / "index"))
    p = Params(8, 500, Rerank.tiered(100), 10)
    a = ix.search_batch(q768, q256, p)
    b = ix2.search_batch(q768, q256, p)
    ix2.close()
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_invalid_params_are_rejected(gpu_a):
    from sieve_gpu import SieveError

    ix, oi, arrays, q768, q256 = gpu_a
    with pytest.raises(SieveError):
        ix.search_batch(q768[:1], q256[:1], Params(8, 5000))
    with pytest.raises(SieveError):
        ix.search_batch(q768[:1], q256[:1], Params(8, 100, Rerank(9)))


def test_buffer_overflow_retry_gives_exact_results(monkeypatch):
    """A candidate buffer too small for the batch makes queries overflow; they are re-run with
    the exact bound and must still equal the oracle."""
    arrays, q768, q256, _ = index_a()
    monkeypatch.setenv("SIEVE_GPU_SOFT_CAP", "600")
    ix = Index.from_arrays(arrays)
    monkeypatch.delenv("SIEVE_GPU_SOFT_CAP")
    try:
        check_search(ix, O.OracleIndex(arrays), q768, q256, Params(16, 500, Rerank.full(), 10))
    finally:
        ix.close()
