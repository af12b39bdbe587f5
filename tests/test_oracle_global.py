"""The global sign-code ablation (src/ivf.rs:700-717) and the flat Hamming baseline
(src/bin/search.rs:251-269, hamming src/lut.rs:156-165) in the oracle, against a direct numpy
restatement of the same steps on a small index built without RaBitQ (ivf::build with
rabitq: false: every slot holds its row's sign code, no rotation.f32 / factors.f32)."""
import numpy as np

import oracle as O
from fixtures import index_g
from sieve_gpu import Params, Rerank


def test_global_index_has_no_rabitq_files():
    arrays, _, _ = index_g()
    assert arrays["rotation"] is None and arrays["factors"] is None
    # every slot holds its row's sign code
    boff, ids = arrays["block_off"].astype(np.int64), arrays["ids"]
    blocks = arrays["blocks"].reshape(-1, 1024)
    for s in range(0, int(boff[-1]) * 32, 997):
        if ids[s] != 0xFFFFFFFF:
            assert np.array_equal(O.unpack_slot(blocks[s // 32], 64, s % 32), arrays["codes"][ids[s]])


def test_global_candidates_match_numpy_restatement():
    arrays, q768, q256 = index_g()
    oi = O.OracleIndex(arrays)
    boff, ids = arrays["block_off"].astype(np.int64), arrays["ids"]
    blocks = arrays["blocks"].reshape(-1, 1024)
    p = Params(6, 200, Rerank.full(), 10).to_c()
    for i in range(q768.shape[0]):
        ps, pc = oi.route(q256[i], p)
        est, got_ids, err = oi.candidates(q256[i], ps, pc, p)
        tables, scale, bias = O.lut_new(q256[i])
        items = []
        for c in pc:
            sc = O.scan(tables, blocks[boff[c]:boff[c + 1]])
            for j, row in enumerate(ids[boff[c] * 32:boff[c + 1] * 32]):
                if row != 0xFFFFFFFF:
                    items.append((-int(sc[j]), int(row)))
        items.sort()
        kept = items[:200]  # TopK(cand) by (score desc, row asc), then dedup by row
        want = sorted({row: s for s, row in reversed(kept)}.items())
        assert np.array_equal(got_ids, [r for r, _ in want])
        assert np.array_equal(est, np.array([O.lut_to_float(scale, bias, -s) for _, s in want], np.float32))
        assert np.all(np.isinf(err))


def test_global_search_prunes_nothing():
    """Infinite error widths: bound pruning keeps every candidate (src/ivf.rs:736-739)."""
    arrays, q768, q256 = index_g()
    oi = O.OracleIndex(arrays)
    base = Params(6, 200, Rerank.full(), 10)
    pruned = Params(6, 200, Rerank.full(), 10, prune=(10, 1.0))
    for i in range(4):
        s0, o0, _ = oi.search(q768[i], q256[i], base.to_c())
        s1, o1, _ = oi.search(q768[i], q256[i], pruned.to_c())
        assert np.array_equal(o0, o1) and np.array_equal(s0, s1)


def test_hamming_counts_bits():
    """src/lut.rs:243-247: a code against its complement differs in every bit."""
    a = np.random.default_rng(0).integers(0, 256, 32, dtype=np.uint8)
    assert O.hamming(a, ~a) == 256 and O.hamming(a, a) == 0


def test_flat_hamming_matches_numpy_restatement():
    arrays, q768, q256 = index_g()
    oi = O.OracleIndex(arrays)
    codes = arrays["codes"]
    bits = np.unpackbits(codes, axis=1, bitorder="little")
    for i in range(4):
        s, o = oi.flat_hamming(codes, q768[i], q256[i], cand=300, k=10)
        qb = np.unpackbits(O.sign_code(q256[i]), bitorder="little")
        sim = 256 - (bits != qb).sum(1)
        order = np.lexsort((np.arange(len(sim)), -sim))[:300]
        w = O.int8_query_weights(arrays["quant_scale"], q768[i])
        d = [(O.dot_i8(w, arrays["rerank"][r]), int(r)) for r in order]
        d.sort(key=lambda x: (-x[0], x[1]))
        assert np.array_equal(o, [r for _, r in d[:10]])
        assert np.array_equal(s, np.array([x for x, _ in d[:10]], np.float32))
