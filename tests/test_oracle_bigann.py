"""CPU pins of the bigann oracle (src/bigann.rs): the reference's own refinement test, the
TopK equivalences the GPU path relies on, and the builder's record layout and files."""
import numpy as np
import pytest

import oracle as O
from fixtures import bigann_a, bigann_b


def gauss(rng: O.Rng) -> np.ndarray:
    v = np.empty(128, np.float32)
    for i in range(128):
        s = np.float32(0.0)
        for _ in range(12):
            s = np.float32(s + np.float32(rng.below(1000)) / np.float32(1000.0))
        v[i] = np.float32(s - np.float32(6.0))
    return v


def sign_code(r: np.ndarray) -> np.ndarray:
    c = np.zeros(16, np.uint8)
    for i in range(128):
        if r[i] > 0:
            c[i >> 3] |= 1 << (i & 7)
    return c


def test_refined_estimate_is_exact_on_its_own_residual_and_sharpens_with_bits():
    """src/bigann.rs:799-819."""
    rng = O.Rng(9)
    err = np.zeros(4)
    for _ in range(200):
        r, q = gauss(rng), gauss(rng)
        truth = float(np.dot(r.astype(np.float64), q.astype(np.float64)))
        for bits in (2, 3):
            planes, f = O.bg_refine_encode(r, bits)
            npl = (bits - 1) * 16
            tab, off = O.bg_refiner(r, bits)
            self_est = O.bg_refiner_estimate(tab, off, bits, sign_code(r), planes[:npl], f)
            rr = float(np.sum(r.astype(np.float64) ** 2))
            assert abs(self_est - rr) < 1e-3 * rr
            tq, oq = O.bg_refiner(q, bits)
            err[bits] += (O.bg_refiner_estimate(tq, oq, bits, sign_code(r), planes[:npl], f) - truth) ** 2
    assert err[3] < 0.5 * err[2]


def all_estimates(ix, q, probe, dots):
    """Every probed slot's 1-bit estimate in scan order (numpy f32, the reference's operations)."""
    qp = np.zeros(128, np.float32)
    qp[:100] = q
    qr = O.rotation_apply(ix["rotation"], qp)
    tables, scale, bias = O.lut_new(qr)
    a = np.float32(2.0) / np.float32(scale)
    s = np.float32(-0.0)
    for v in qr:
        s = np.float32(s + v)
    b = np.float32(np.float32(2.0) * np.float32(bias) - s)
    bo = ix["block_off"].astype(np.int64)
    est, ids, slots = [], [], []
    for c in probe:
        b0, b1 = bo[c], bo[c + 1]
        if b1 == b0:
            continue
        sc = O.scan(tables, ix["blocks"].reshape(-1, 512)[b0:b1]).astype(np.float32)
        sl = np.arange(b0 * 32, b1 * 32)
        f = ix["factors"].reshape(-1, 2)[sl]
        e = (np.float32(2.0) * (np.float32(dots[c]) + f[:, 0] * (a * sc + b))) - f[:, 1]
        keep = ix["ids"][sl] != 0xFFFFFFFF
        est.append(e[keep].astype(np.float32))
        ids.append(ix["ids"][sl][keep])
        slots.append(sl[keep])
    return np.concatenate(est), np.concatenate(ids), np.concatenate(slots)


@pytest.mark.parametrize("cand", [1, 10, 100, 700])
def test_candidates_without_refine_are_the_canonical_top(cand):
    ix, qs = bigann_a(1)
    ob = O.OracleBigann(ix)
    for q in qs[:20]:
        p = ob.params(12, cand, 10)
        probe, _, dots = ob.route(q, p)
        ids, est, nx, _ = ob.candidates(q, p)
        e, i, _ = all_estimates(ix, q, probe, dots)
        order = np.lexsort((np.arange(e.size), -e.astype(np.float64)))[:cand]
        assert np.array_equal(ids, i[order])
        assert np.array_equal(est, e[order])


def test_route_is_top_nprobe_by_l2_score_with_margin_prefix():
    ix, qs = bigann_a(2)
    ob = O.OracleBigann(ix)
    leaves = ix["leaves"].reshape(-1, 100).astype(np.float64)
    for q in qs[:16]:
        probe, sc, dots = ob.route(q, ob.params(20, 100, 10))
        ref = 2.0 * leaves @ q.astype(np.float64) - (leaves ** 2).sum(1)
        assert set(probe) == set(np.argsort(-ref, kind="stable")[:20]) or np.allclose(
            np.sort(ref[probe]), np.sort(np.sort(ref)[-20:]), rtol=1e-5)
        assert np.all(np.diff(sc) <= 0)
        pm, scm, _ = ob.route(q, ob.params(20, 100, 10, margin=0.05))
        assert np.array_equal(pm, probe[: pm.size]) and pm.size >= 1
        qq = float(np.sum(q.astype(np.float64) ** 2))
        assert np.all(qq - scm <= (qq - scm[0]) * 1.05 * (1 + 1e-6))


def test_refined_candidates_carry_refined_estimates():
    ix, qs = bigann_b()
    ob = O.OracleBigann(ix)
    for q in qs[:6]:
        p = ob.params(4, 50, 10, refine=300)
        ids, est, nx, _ = ob.candidates(q, p)
        p0 = ob.params(4, 50, 10)
        ids0, est0, _, _ = ob.candidates(q, p0)
        assert ids.size == 50 and np.all(np.diff(est) <= 0)
        assert not np.array_equal(est, est0)  # the refined estimates differ from the 1-bit ones


def test_builder_record_layout():
    ix, _ = bigann_a(2)
    n, k = ix["n"], ix["k"]
    bo = ix["block_off"].astype(np.int64)
    ids = ix["ids"]
    seen = np.zeros(n, np.int64)
    for c in range(k):
        s = ids[bo[c] * 32:bo[c + 1] * 32]
        real = s[s != 0xFFFFFFFF]
        assert np.all(s[:real.size] != 0xFFFFFFFF) and np.all(np.diff(real.astype(np.int64)) > 0)
        seen[real] += 1
    assert np.all(seen == 1)  # every row stored once
    f = ix["factors"].reshape(-1, 2)
    live = ids != 0xFFFFFFFF
    base = ix["base"].astype(np.float64)
    assert np.allclose(f[live, 1], (base[ids[live]] ** 2).sum(1), rtol=1e-6)


def test_bigann_files_round_trip(tmp_path):
    from sieve_gpu import bigann_builder as BB

    ix, _ = bigann_a(3)
    BB.write_files(ix, str(tmp_path / "idx"), str(tmp_path / "base"))
    back = BB.read_files(str(tmp_path / "idx"), str(tmp_path / "base"))
    for key in ("block_off", "ids", "blocks", "factors", "ext", "rotation", "leaves", "base", "coarse"):
        assert np.array_equal(np.asarray(back[key]).ravel(), np.asarray(ix[key]).ravel()), key
    assert back["bits"] == 3 and back["k"] == ix["k"] and back["n"] == ix["n"]


def test_oracle_search_recall():
    from sieve_gpu import bigann_builder as BB
    import torch

    ix, qs = bigann_a(2)
    ob = O.OracleBigann(ix)
    gt, _ = BB.ground_truth(torch.as_tensor(ix["base"]), torch.as_tensor(qs[:64]), 10)
    s, o, cnt, _ = ob.search_batch(qs[:64], ob.params(16, 200, 10, refine=1000), threads=4)
    rec = np.mean([len(set(o[i, :cnt[i]]) & set(gt[i])) / 10 for i in range(64)])
    assert rec > 0.95
    assert np.all(np.diff(s, axis=1) <= 0)
