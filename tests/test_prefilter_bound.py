"""The integer prefilter of the transposed bound pass (tct_prefilter, csrc/scan_tcf.cu), restated
and checked on the CPU: for every pair whose weight product D is at or below the prefilter's
floor, the float bound the kernel evaluates (the estimate's operations of src/rabitq.rs:127-130 at
the score bound gamma * D + R_hi, each rounded to f32) stays below the admission threshold, for
every mul in the cluster's range. So skipping those pairs never changes an admission."""
import math

import numpy as np

F = np.float32
DMAX = 256 * 127


def prefilter(cent, a, b, gam, rhi, T, m0, m1):
    """The restatement: Df such that D <= Df cannot reach T (None: no prefilter)."""
    if not (m0 >= 0 and m1 >= m0 and math.isfinite(m1) and a > 0 and gam > 0):
        return None
    mag = abs(cent) + m1 * (abs(a) * (gam * DMAX + abs(rhi)) + abs(b)) + abs(T)
    tl = T - 16.0 * 2.0 ** -24 * mag
    m = m1 if tl > cent else m0
    if not m > 0:
        return None
    ds = (((tl - cent) / m - b) / a - rhi) / gam
    if not math.isfinite(ds):
        return None
    df = math.floor(ds) - 1.0
    if df < -DMAX - 1:
        return None
    return int(min(df, DMAX))


def bound(cent, a, b, gam, rhi, mul, d):
    """The kernel's float bound, operation by operation in f32 (no fused multiply-add)."""
    sb = F(F(F(gam) * F(d)) + F(rhi))
    return F(F(cent) + F(F(mul) * F(F(F(a) * sb) + F(b))))


def test_prefilter_never_rejects_an_admissible_pair():
    rng = np.random.default_rng(5)
    checked = 0
    for _ in range(4000):
        # magnitudes of a query's LUT constants and a cluster's factors: a = 2/scale ~ 1e-3..1e-1,
        # b ~ -10..10, R_hi ~ 0..2000, cent ~ -1..1, mul ~ 0..0.5, thresholds near cent
        a = float(F(10 ** rng.uniform(-3.5, -0.5)))
        b = float(F(rng.uniform(-20, 20)))
        gam = float(rng.choice([1.0, 2.0]))
        rhi = float(F(rng.uniform(-100, 3000)))
        cent = float(F(rng.uniform(-1, 1)))
        m0 = float(F(rng.uniform(0, 0.3))) * float(rng.random() < 0.8)
        m1 = float(F(m0 + rng.uniform(0, 0.4)))
        T = float(F(cent + rng.normal(0, 0.3)))
        df = prefilter(cent, a, b, gam, rhi, T, m0, m1)
        if df is None:
            continue
        muls = [m0, m1] + [float(F(x)) for x in rng.uniform(m0, m1, 4)]
        ds = [df, df - 1, df - 7] + [int(x) for x in rng.integers(-DMAX, df + 1, 3)] if df >= -DMAX else [df]
        for d in ds:
            if d < -DMAX:
                continue
            for mul in muls:
                assert bound(cent, a, b, gam, rhi, mul, d) < F(T), (cent, a, b, gam, rhi, T, m0, m1, d, mul)
                checked += 1
    assert checked > 10000


def test_prefilter_is_tight_enough_to_matter():
    """Just above the floor a pair can pass: the prefilter only drops pairs the bound drops."""
    cent, a, b, gam, rhi, m0, m1 = 0.2, 0.01, -3.0, 1.0, 500.0, 0.05, 0.3
    T = 0.3
    df = prefilter(cent, a, b, gam, rhi, T, m0, m1)
    assert df is not None
    # some D a few units above the floor reaches T at mul = m1
    assert any(bound(cent, a, b, gam, rhi, m1, d) >= F(T) for d in range(df + 1, df + 40))
