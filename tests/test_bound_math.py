"""CPU checks of the arithmetic the tensor-core bound pass relies on (csrc/scan_tcf.cu), restated
in numpy and run against the oracle's tables and exact scores:

- the integer bound gamma*D + R_lo <= s <= gamma*D + R_hi of the LUT score s from per-query s8
  weights and residual ranges (k_filter_prep), on tables built by Query::new
  (src/rabitq.rs:119-125) and scores from lut::scan (src/lut.rs:116-126);
- the K order of the A columns (bits s, s+8, s+16, s+24 of code word i in column 8i + s) and the
  weights stored in that order;
- the exact float form of the score bound (gamma*D written into the bits of 1.5 * 2^23, plus
  R - 1.5 * 2^23);
- the monotone estimate bound: the estimate's own f32 operations at the bound of the score
  (src/rabitq.rs:127-130) bound the exact estimate from above.
"""
import numpy as np
import pytest

import oracle as O

MAGIC_BITS = 0x4B400000
MAGIC = np.float32(12582912.0)  # 1.5 * 2^23


def filter_prep(t: np.ndarray):
    """The weights, gamma and summed residual range of one query's [64, 16] u8 tables."""
    t = t.astype(np.int64)
    w = np.stack([t[:, 1 << j] - t[:, 0] for j in range(4)], 1)  # [G, 4]
    gam = 2 if np.any((w > 127) | (w < -127)) else 1
    w = np.sign(w) * (np.abs(w) // gam)  # C division truncates toward zero
    bits = (np.arange(16)[:, None] >> np.arange(4)) & 1  # [16, 4]: nibble c's bits
    v = t - gam * (w @ bits.T)  # [G, 16]: T_g[c] - gamma * L_g[c]
    return w.reshape(-1), gam, int(v.max(1).sum()), int(v.min(1).sum())


def code_bits(code: np.ndarray) -> np.ndarray:
    """Bit d of a 32-byte code (prefix dimension d): nibble d/4, bit d%4."""
    return np.unpackbits(code, bitorder="little").astype(np.int64)


def a_row(code: np.ndarray) -> np.ndarray:
    """The producers' A row: 64 columns of 4 bytes, column 8i + s = bits s, s+8, s+16, s+24 of
    little-endian code word i."""
    words = code.view("<u4")
    row = np.zeros(256, np.int64)
    for i in range(8):
        for s in range(8):
            for j in range(4):
                row[4 * (8 * i + s) + j] = (int(words[i]) >> (8 * j + s)) & 1
    return row


def k_order_weights(w: np.ndarray) -> np.ndarray:
    """k_filter_prep's store: thread g's weight m (dimension 4g + m, bit b = 4(g%8) + m of word
    g/8) goes to K byte 32(g/8) + 4(b%8) + b/8."""
    out = np.zeros(256, np.int64)
    for g in range(64):
        for m in range(4):
            b = 4 * (g & 7) + m
            out[32 * (g >> 3) + 4 * (b & 7) + (b >> 3)] = w[4 * g + m]
    return out


def queries(n: int, seed: int):
    rng = np.random.default_rng(seed)
    signs = O.rotation_signs(7)
    for _ in range(n):
        q = rng.standard_normal(256).astype(np.float32)
        yield O.query_new(signs, q / np.linalg.norm(q))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_score_lies_within_the_integer_bound(seed):
    rng = np.random.default_rng(seed)
    for t, _sc, _bi, _a, _b in queries(8, seed):
        w, gam, rhi, rlo = filter_prep(t)
        assert np.all(np.abs(w) <= 127)
        for _ in range(64):
            code = rng.integers(0, 256, 32, dtype=np.uint8)
            s = O.score_code(t, code)
            D = int(code_bits(code) @ w)
            assert gam * D + rlo <= s <= gam * D + rhi


def test_extreme_codes_lie_within_the_bound():
    for t, *_ in queries(4, 9):
        w, gam, rhi, rlo = filter_prep(t)
        for code in (np.zeros(32, np.uint8), np.full(32, 255, np.uint8), np.full(32, 0x5A, np.uint8)):
            s = O.score_code(t, code)
            D = int(code_bits(code) @ w)
            assert gam * D + rlo <= s <= gam * D + rhi


def test_k_order_of_a_and_b_gives_the_same_product():
    rng = np.random.default_rng(5)
    w = rng.integers(-127, 128, 256)
    wk = k_order_weights(w)
    assert sorted(wk.tolist()) == sorted(w.tolist())  # a permutation
    for _ in range(200):
        code = rng.integers(0, 256, 32, dtype=np.uint8)
        assert int(a_row(code) @ wk) == int(code_bits(code) @ w)


def test_float_form_of_the_score_bound_is_exact():
    # |D| <= 256 * 127 and |R| <= 64 * (255 + 2 * 4 * 127): the bound's whole range
    rng = np.random.default_rng(11)
    dmax, rmax = 256 * 127, 64 * (255 + 8 * 127)
    for gam in (1, 2):
        D = np.concatenate([np.array([-dmax, -1, 0, 1, dmax]), rng.integers(-dmax, dmax + 1, 20000)])
        R = np.concatenate([np.array([-rmax, 0, rmax, -rmax, rmax]), rng.integers(-rmax, rmax + 1, 20000)])
        bits = (D * gam + MAGIC_BITS).astype(np.uint32)
        F = bits.view(np.float32)
        Rp = R.astype(np.float32) - MAGIC  # exact: an integer below 2^24 in magnitude
        assert np.all(Rp.astype(np.float64) == R - 12582912.0)
        sb = F + Rp
        assert np.all(sb.astype(np.float64) == gam * D + R)


def est32(a, b, cent, mul, s):
    """cent + mul * (a * s + b), rounded to f32 after each operation (src/rabitq.rs:127-130) for
    any integer s, including bounds outside the u16 range of a score."""
    f = np.float32
    return f(f(cent) + f(f(mul) * f(f(f(a) * f(s)) + f(b))))


@pytest.mark.parametrize("seed", [4, 6])
def test_estimate_at_the_score_bound_bounds_the_estimate(seed):
    rng = np.random.default_rng(seed)
    for t, _sc, _bi, a, b in queries(4, seed):
        w, gam, rhi, rlo = filter_prep(t)
        for _ in range(64):
            code = rng.integers(0, 256, 32, dtype=np.uint8)
            s = O.score_code(t, code)
            D = int(code_bits(code) @ w)
            cent = float(np.float32(rng.uniform(-1, 1)))
            for mul in (float(np.float32(rng.uniform(0, 3))), float(np.float32(-rng.uniform(0, 3))), 0.0):
                sb = gam * D + (rhi if mul >= 0 else rlo)
                exact = est32(a, b, cent, mul, s)
                assert exact == np.float32(O.estimate(a, b, cent, mul, s))
                assert est32(a, b, cent, mul, sb) >= exact


def test_admission_key_finds_its_probe():
    """k_tc_recheck's lookup: probe r's slots hold admission keys probe_off[r] ..
    probe_off[r] + slots(r) - 1 (offsets in probe order, src/ivf.rs:663-675), so the last probe
    whose offset is at most a key owns it, with empty clusters (equal offsets) in between."""
    rng = np.random.default_rng(21)
    for _ in range(50):
        sizes = rng.integers(0, 5, rng.integers(1, 40)) * 32  # padded slots; zero = empty cluster
        off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        for r, n in enumerate(sizes):
            for key in range(off[r], off[r] + n):
                lo, hi = 0, len(off)  # the kernel's search: the first offset above the key
                while lo < hi:
                    mid = (lo + hi) >> 1
                    if off[mid] <= key:
                        lo = mid + 1
                    else:
                        hi = mid
                assert lo - 1 == r
