"""CPU tests of bench.py's reporting helpers: the parity count against the CPU leg, recall@10,
the serving knee, the domain allowlists of the filtered serving load, and the distinct-slot count
of a batch."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _lists():
    ids = np.array([[5, 3, 9], [1, 2, 0]], np.uint32)
    sc = np.array([[0.9, 0.8, 0.7], [0.5, 0.4, 0.0]], np.float32)
    cnt = np.array([3, 2], np.uint32)
    return ids, sc, cnt


def test_parity_counts_identical_lists_as_matching():
    ids, sc, cnt = _lists()
    cpu = {"ids": ids.copy(), "sc": sc.copy(), "cnt": cnt.copy(), "tied": np.array([False, False])}
    p = bench.parity_check(ids, sc, cnt, cpu)
    assert (p["queries"], p["mismatched"], p["tied_boundary"], p["tied_and_differing"]) == (2, 0, 0, 0)


def test_parity_separates_tied_boundaries_from_mismatches():
    ids, sc, cnt = _lists()
    cpu = {"ids": ids.copy(), "sc": sc.copy(), "cnt": cnt.copy(), "tied": np.array([False, True])}
    gpu_ids = ids.copy()
    gpu_ids[1, 1] = 7  # the tied query differs
    p = bench.parity_check(gpu_ids, sc, cnt, cpu)
    assert (p["mismatched"], p["tied_boundary"], p["tied_and_differing"]) == (0, 1, 1)
    gpu_sc = sc.copy()
    gpu_sc[0, 2] = np.nextafter(np.float32(0.7), np.float32(1))  # one ulp on an untied query
    p = bench.parity_check(ids, gpu_sc, cnt, cpu)
    assert p["mismatched"] == 1
    p = bench.parity_check(ids, sc, np.array([2, 2], np.uint32), cpu)  # a shorter list
    assert p["mismatched"] == 1


def test_recall10_counts_overlap_in_the_first_ten():
    gt = np.arange(20).reshape(2, 10)
    ids = np.stack([np.arange(10), np.array([10, 11, 12, 99, 98, 97, 96, 95, 94, 93])])
    assert bench.recall10(ids, np.array([10, 10]), gt) == (1.0 + 0.3) / 2
    assert bench.recall10(ids, np.array([5, 10]), gt) == (0.5 + 0.3) / 2


def test_serving_knee_takes_the_fastest_rate_within_the_limit():
    rows = [
        {"offered_qps": 10000.0, "achieved_qps": 9990.0, "p99_ms": 2.0},
        {"offered_qps": 20000.0, "achieved_qps": 19950.0, "p99_ms": 4.9},
        {"offered_qps": 30000.0, "achieved_qps": 29900.0, "p99_ms": 5.2},  # over the p99 limit
        {"offered_qps": 40000.0, "achieved_qps": 30000.0, "p99_ms": 4.0},  # does not keep up
    ]
    k = bench.serving_knee(rows, [0.5, 0.5])  # plain path: 2000 queries/s
    assert k["offered_qps"] == 20000.0 and abs(k["vs_plain"] - 19950.0 / 2000.0) < 1e-9
    assert bench.serving_knee([{"offered_qps": 1.0, "achieved_qps": 1.0, "p99_ms": 9.0}], [1.0])["offered_qps"] is None
    assert bench.serving_knee([], [1.0]) is None


def test_domain_allowlist_allows_whole_domains_up_to_the_selectivity():
    rng = np.random.default_rng(3)
    dom = rng.integers(0, bench.N_DOMAINS, 200_000).astype(np.uint16)
    for sel in (0.001, 0.01, 0.1, 0.5):
        bits = bench.domain_allowlist(dom, sel)
        mask = np.unpackbits(bits.view(np.uint8), bitorder="little")[: dom.size].astype(bool)
        assert mask.sum() >= sel * dom.size
        allowed = np.unique(dom[mask])
        # whole domains: every row of an allowed domain is allowed, and no other row is
        assert np.array_equal(mask, np.isin(dom, allowed))
        # domains are taken in the order of (h * golden).rotate_left(17) (src/bin/search.rs:
        # 598-620): the allowed ones are a prefix of that order, and the last one crossed the target
        h = np.arange(bench.N_DOMAINS, dtype=np.uint64)
        with np.errstate(over="ignore"):
            x = h * np.uint64(bench.GOLDEN)
        order = np.argsort((x << np.uint64(17)) | (x >> np.uint64(47)), kind="stable")
        pos = np.empty(bench.N_DOMAINS, np.int64)
        pos[order] = np.arange(bench.N_DOMAINS)
        counts = np.bincount(dom, minlength=bench.N_DOMAINS)
        taken = order[: pos[allowed].max() + 1]
        assert set(taken[counts[taken] > 0].tolist()) == set(allowed.tolist())
        last = taken[-1]
        assert mask.sum() - counts[last] < sel * dom.size


def test_distinct_slots_counts_each_probed_cluster_once():
    routes = [np.array([0, 2]), np.array([2, 3]), np.array([1])]
    slots = np.array([10, 20, 30, 40])
    assert bench.distinct_slots(routes, 0, 2, slots) == 10 + 30 + 40
    assert bench.distinct_slots(routes, 1, 2, slots) == 20 + 30 + 40
