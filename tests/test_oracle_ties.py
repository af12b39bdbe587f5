"""The oracle's two TopK tie rules (src/topk.rs:4-62) and its record of tied cuts.

The reference's TopK rejects pushes with score <= threshold and cuts a full buffer with
select_nth_unstable_by, so which of several equal scores survives at the k-th place is
unspecified there. The oracle keeps a canonical rule (score desc, id asc) and a restatement of
the reference's own mechanics; every TopK records whether its k-th place was tied, and the two
rules may only disagree on queries so recorded.
"""
import numpy as np
import pytest

import oracle as O
from fixtures import index_b


@pytest.fixture
def reference_rule():
    O.set_tie_rule(O.TIE_REFERENCE)
    yield
    O.set_tie_rule(O.TIE_CANONICAL)


def test_distinct_scores_are_never_tied():
    r = np.random.default_rng(3)
    scores = r.permutation(5000).astype(np.float32)
    for k in (1, 10, 100, 4999):
        s, i, tied = O.topk(scores, np.arange(5000, dtype=np.uint32), k, tied=True)
        assert not tied
        assert np.array_equal(s, np.sort(scores)[::-1][:k])


def test_tied_cut_is_recorded_under_both_rules(reference_rule):
    scores = np.array([5, 5, 5, 4, 3, 5, 2], np.float32)
    ids = np.arange(7, dtype=np.uint32)
    s, i, tied = O.topk(scores, ids, 2, tied=True)
    assert tied and np.array_equal(s, [5, 5])
    # the reference rule keeps two of the four 5s (which two is the selection's choice), sorted
    assert set(i.tolist()) <= {0, 1, 2, 5} and i[0] < i[1]
    O.set_tie_rule(O.TIE_CANONICAL)
    s, i, tied = O.topk(scores, ids, 2, tied=True)
    assert tied and np.array_equal(i, [0, 1])
    # a tie strictly inside the kept set is no boundary tie
    s, i, tied = O.topk(scores, ids, 5, tied=True)
    assert not tied and np.array_equal(i, [0, 1, 2, 5, 3])


def test_reference_rule_rejects_equal_to_threshold(reference_rule):
    # k = 2: after [9, 8, 7, 6] the buffer (2k) is cut to {9, 8}, threshold 8; a later 8 is
    # rejected by `score <= threshold`, so the tie is recorded
    s, i, tied = O.topk(np.array([9, 8, 7, 6, 8], np.float32), np.arange(5, dtype=np.uint32), 2, tied=True)
    assert np.array_equal(i, [0, 1]) and tied


def test_rules_differ_only_on_tied_queries():
    """Index B holds 400 exact duplicates and queries near them: estimates and int8 scores tie.
    Per query, the canonical and the reference rule give the same list unless a cut was tied."""
    arrays, q768, q256, _ = index_b()
    oi = O.OracleIndex(arrays)
    from sieve_gpu import Params, Rerank

    # k = 3 cuts through the five copies of a duplicated row that a query near it ranks first
    for params in (Params(4, 300, Rerank.full(), 3), Params(8, 200, Rerank.tiered(50), 3)):
        p = params.to_c()
        s0, o0, c0, _, t0 = oi.search_batch(q768, q256, p, tied=True)
        O.set_tie_rule(O.TIE_REFERENCE)
        try:
            s1, o1, c1, _, t1 = oi.search_batch(q768, q256, p, tied=True)
        finally:
            O.set_tie_rule(O.TIE_CANONICAL)
        assert np.array_equal(c0, c1)
        differ = np.array([not (np.array_equal(o0[i, :c0[i]], o1[i, :c1[i]]) and
                                np.array_equal(s0[i, :c0[i]], s1[i, :c1[i]])) for i in range(len(c0))])
        assert not np.any(differ & ~(t0 | t1))
        assert t0.any(), "index B's duplicate rows make some cut tied"
