"""Pins of the CPU oracle: ports of the reference's own unit and property tests.

The reference (a Rust crate) cannot be built here and ships no golden vectors, so these ports,
with their known answers and properties, are what ties the oracle to the reference. Each test
names the Rust test it ports. Property tests (proptest in the reference) run over seeded cases.
"""
import numpy as np
import pytest

import oracle as O

CASES = 64


def rust_unit(rng: O.Rng, d: int = 256) -> np.ndarray:
    """`unit` of src/rabitq.rs:138-145: sum of 4 uniforms minus 0.5 per dim, normalised."""
    v = np.empty(d, np.float32)
    two53 = np.float32(1 << 53)
    for i in range(d):
        s = np.float32(-0.0)
        for _ in range(4):
            s = np.float32(s + (np.float32(rng.next() >> 11) / two53 - np.float32(0.5)))
        v[i] = s
    return O.normalize(v)[0]


# ---- src/lut.rs:203-221 kernel_matches_reference --------------------------------------------
@pytest.mark.parametrize("seed", range(CASES))
def test_kernel_matches_reference(seed):
    r = np.random.default_rng(seed)
    q = r.uniform(-1.0, 1.0, 256).astype(np.float32)
    codes = r.integers(0, 256, (32, 32), dtype=np.uint8)
    tables, _, _ = O.lut_new(q)
    block = O.pack_block(codes)
    got = O.scan(tables, block)
    for k in range(32):
        assert got[k] == O.score_code(tables, codes[k])


# ---- src/lut.rs:223-234 quantized_score_tracks_float ----------------------------------------
@pytest.mark.parametrize("seed", range(CASES))
def test_quantized_score_tracks_float(seed):
    r = np.random.default_rng(1000 + seed)
    q = r.uniform(-0.2, 0.2, 256).astype(np.float32)
    code = r.integers(0, 256, 32, dtype=np.uint8)
    tables, scale, bias = O.lut_new(q)
    exact = O.float_score(q, code)
    approx = O.lut_to_float(scale, bias, O.score_code(tables, code))
    bound = 64.0 * 0.5 / scale + 1e-4
    assert abs(exact - approx) <= bound


# ---- src/lut.rs:237-253 narrow_codes_use_the_same_kernel ------------------------------------
def test_narrow_codes_use_the_same_kernel():
    q = np.cos(np.arange(128, dtype=np.float32) * np.float32(0.91)).astype(np.float32)
    tables, _, _ = O.lut_new(q)
    assert tables.shape == (32, 16)
    codes = np.array([[(k * 37 + i * 11) % 256 for i in range(16)] for k in range(32)], np.uint8)
    block = O.pack_block(codes, groups=32)
    got = O.scan(tables, block)
    for k in range(32):
        assert got[k] == O.score_code(tables, codes[k])
        assert np.array_equal(O.unpack_slot(block, 32, k), codes[k])


# ---- src/lut.rs:255-266 partial_block_pads_with_zero_codes -----------------------------------
def test_partial_block_pads_with_zero_codes():
    q = np.sin(np.arange(256, dtype=np.float32) * np.float32(0.37)).astype(np.float32)
    tables, _, _ = O.lut_new(q)
    c = np.full(32, 0xA5, np.uint8)
    block = O.pack_block(c[None, :])
    got = O.scan(tables, block)
    assert got[0] == O.score_code(tables, c)
    assert got[1] == O.score_code(tables, np.zeros(32, np.uint8))


# ---- src/lut.rs:268-273 hamming_counts_bits --------------------------------------------------
def test_hamming_counts_bits():
    assert O.hamming(np.full(32, 0xFF, np.uint8), np.full(32, 0x0F, np.uint8)) == 4 * 32


# ---- src/rabitq.rs:147-157 rotation_is_orthogonal ---------------------------------------------
def test_rotation_is_orthogonal():
    rng = O.Rng(1)
    signs = O.rotation_signs(3)
    a, b = rust_unit(rng), rust_unit(rng)
    ra, rb = O.rotation_apply(signs, a), O.rotation_apply(signs, b)
    assert abs(O.dot_f32(ra, ra) - 1.0) < 1e-4
    assert abs(O.dot_f32(ra, rb) - O.dot_f32(a, b)) < 1e-4


def test_rotation_norm_is_exact_at_256():
    assert O.lib().or_rotation_norm(256) == np.float32(1.0 / 4096.0)


# ---- src/rabitq.rs:159-187 estimate_is_within_bound -------------------------------------------
def test_estimate_is_within_bound():
    rng = O.Rng(2)
    signs = O.rotation_signs(5)
    inside, trials, sq = 0, 2000, 0.0
    for _ in range(trials):
        x = rust_unit(rng)
        u = rust_unit(rng)
        c = O.normalize((x + np.float32(0.8) * u).astype(np.float32))[0]
        q = rust_unit(rng)
        xr, cr = O.rotation_apply(signs, x), O.rotation_apply(signs, c)
        code, mul, err = O.rabitq_encode(xr, cr)
        tables, scale, bias, a, b = O.query_new(signs, q)
        est = O.estimate(a, b, O.dot_f32(c, q), mul, O.score_code(tables, code))
        truth = O.dot_f32(x, q)
        sq += (est - truth) ** 2
        if abs(est - truth) <= err * 1.1:
            inside += 1
    assert inside / trials > 0.95, f"{inside}/{trials} inside the bound"
    assert (sq / trials) ** 0.5 < 0.05


# ---- src/quant.rs:147-159 sign_code_bits ---------------------------------------------------------
def test_sign_code_bits():
    p = np.full(256, -1.0, np.float32)
    p[0], p[9], p[255] = 0.5, 0.1, 2.0
    c = O.sign_code(p)
    assert c[0] == 1 and c[1] == 1 << 1 and c[31] == 1 << 7
    assert sum(bin(int(x)).count("1") for x in c) == 3


# ---- src/quant.rs:161-171 int8_roundtrip_and_dot --------------------------------------------------
def test_int8_roundtrip_and_dot():
    v = ((np.arange(768) * 37 % 101).astype(np.float32) - np.float32(50.0)) / np.float32(50.0)
    v = O.normalize(v)[0]
    scale = O.int8_fit(v[None, :])
    c = O.int8_encode(scale, v)
    w = O.int8_query_weights(scale, v)
    approx = O.dot_i8(w, c)
    assert abs(approx - 1.0) < 0.01


# ---- src/quant.rs:173-179 sdot_matches_scalar (the CPU side: scalar == numpy int dot) ------------
@pytest.mark.parametrize("seed", range(16))
def test_dot_i8i8_matches_integer_dot(seed):
    r = np.random.default_rng(seed)
    a = r.integers(-128, 128, 768, dtype=np.int8)
    b = r.integers(-128, 128, 768, dtype=np.int8)
    assert O.dot_i8i8(a, b) == int(np.dot(a.astype(np.int64), b.astype(np.int64)))
    assert O.dot_i8i8(a[:256], b[:256]) == int(np.dot(a[:256].astype(np.int64), b[:256].astype(np.int64)))


# ---- src/tier2.rs:81-96 table_score_matches_reconstruction ---------------------------------------
def test_tier2_table_score_matches_reconstruction():
    x = [0x2545F4914F6CDD1D]
    M = (1 << 64) - 1

    def rnd():
        v = x[0]
        v ^= (v << 13) & M
        v ^= v >> 7
        v ^= (v << 17) & M
        x[0] = v
        return np.float32(np.float32(v >> 11) / np.float32(1 << 53) - np.float32(0.5))

    rows = np.array([rnd() for _ in range(256 * 64)], np.float32).reshape(64, 256)
    sigma = O.tier2_fit(rows)
    q = np.array([rnd() for _ in range(256)], np.float32)
    tables = O.tier2_tables(sigma, q)
    levels = np.array([-1.510, -0.4528, 0.4528, 1.510], np.float32)
    for r in rows[:8]:
        code, norm = O.tier2_encode(sigma, r)
        lv = np.array([(code[i >> 2] >> ((i & 3) * 2)) & 3 for i in range(256)])
        recon = (levels[lv] * sigma).astype(np.float32)
        want = np.float32(-0.0)
        for a, b in zip(q, recon):
            want = np.float32(want + np.float32(a * b))
        want = np.float32(want / np.float32(norm))
        assert abs(O.tier2_score(tables, code, norm) - want) < 1e-4


# ---- src/topk.rs:69-82 matches_full_sort -----------------------------------------------------------
@pytest.mark.parametrize("seed", range(CASES))
def test_topk_matches_full_sort(seed):
    r = np.random.default_rng(seed)
    n = int(r.integers(0, 2000))
    k = int(r.integers(1, 64))
    scores = r.integers(0, 500, n).astype(np.float32)
    got, ids = O.topk(scores, np.arange(n, dtype=np.uint32), k)
    want = np.sort(scores)[::-1][:k]
    assert np.array_equal(got, want)
    # canonical tie order: equal scores come out by ascending id
    for i in range(1, got.size):
        assert got[i - 1] > got[i] or (got[i - 1] == got[i] and ids[i - 1] < ids[i])


def test_topk_keeps_lowest_ids_among_ties():
    scores = np.array([3, 1, 3, 3, 2, 3], np.float32)
    got, ids = O.topk(scores, np.array([10, 11, 12, 13, 14, 15], np.uint32), 2)
    assert list(ids) == [10, 12]


# ---- src/ivf.rs:856-868 prune_threshold_is_mth_lower_bound -------------------------------------
def test_prune_threshold_is_mth_lower_bound():
    est = np.array([0.9, 0.7, 0.7, 0.3], np.float32)
    err = np.array([0.1, 0.2, 0.05, 0.2], np.float32)
    tau = O.prune_threshold(est, err, 2, 1.0)
    assert tau == np.float32(0.65)
    assert O.prune_threshold(est, err, 5, 1.0) == -np.inf
    kept = [i for i in range(4) if np.float32(est[i] + err[i]) >= tau]
    assert kept == [0, 1, 2]
    assert O.prune_threshold(est, err, 2, 0.5) > tau


# ---- src/filter.rs:157-165 auto_plan -------------------------------------------------------------
def test_auto_plan():
    n = 10_000_000
    assert O.plan_resolve(3, 250_000, n) == 2
    assert O.plan_resolve(3, 1_000_000, n) == 1
    assert O.plan_resolve(3, 3_000_000, n) == 0
    assert O.plan_resolve(1, 1, n) == 1


# ---- src/eval.rs:61-64 recall_counts_overlap --------------------------------------------------
def test_recall_counts_overlap():
    assert O.recall_at(2, [1, 2, 3], [2, 9, 1]) == 0.5


# ---- src/blas.rs:58-65 small_product -------------------------------------------------------------
def test_gemm_small_product():
    a = np.array([[1, 2, 3], [4, 5, 6]], np.float32)
    b = np.array([[1, 0, 1], [0, 1, 0]], np.float32)
    assert O.gemm_abt(a, b).ravel().tolist() == [4.0, 2.0, 10.0, 5.0]


# ---- rng known answers: splitmix64 reference values ----------------------------------------------
def test_splitmix64_known_values():
    r = O.Rng(0)
    # splitmix64 from seed 0: published first outputs of the generator
    assert r.next() == 0xE220A8397B1DCDAF
    assert r.next() == 0x6E789E6AA1B965F4
