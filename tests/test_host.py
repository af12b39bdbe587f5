"""CPU tests of the host side: the C ABI's exports, the builder's layouts against the oracle,
the reference file formats, config parsing, and the oracle's search over a built index."""
import os
import re

import numpy as np
import pytest
import torch

import oracle as O
from fixtures import index_a
from sieve_gpu import Params, Rerank, builder, parse_config
from sieve_gpu import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "sieve_gpu.h")).read()
    declared = set(re.findall(r"^\s*(?:const char\*|int)\s+(sg_\w+)\(", header, re.M))
    assert declared == set(_abi.EXPORTS)
    L = _abi.lib()
    for name in declared:
        assert hasattr(L, name), name


def test_library_reports_errors_without_aborting():
    import ctypes

    L = _abi.lib()
    h = ctypes.c_void_p()
    rc = L.sg_open_ivf(b"/nonexistent-dir", b"/nonexistent-dir", 0, ctypes.byref(h))
    assert rc == -2 and b"cannot open" in L.sg_last_error()
    assert L.sg_lut_scan(7, None, None, 0, None) == -1
    assert L.sg_dot_i8i8(None, None, 0, 3, None) == -1
    # argument checks come before any device call
    assert L.sg_route_scores(None, 1, None, None) == -1 and b"null" in L.sg_last_error()
    assert L.sg_route(None, 1, None, None, None, None, None) == -1


def test_abi_struct_layouts():
    assert ctypes_size(_abi.SgParams) == 56
    assert ctypes_size(_abi.SgTiming) == 72
    assert ctypes_size(_abi.SgStats) == 8 * 4 + 8 + 4 * 8 + 8
    assert ctypes_size(_abi.SgIvfArrays) == 8 + 8 + 13 * 8


def ctypes_size(t):
    import ctypes

    return ctypes.sizeof(t)


def test_parse_config():
    label, p = parse_config("64:500:tiered200:b10x0.5:p0.12:s100k", 4096)
    assert (p.nprobe, p.cand, p.rerank, p.k) == (64, 500, Rerank.tiered(200), 100)
    assert p.prune == (10, 0.5) and p.margin == 0.12 and p.budget == 100000
    _, p = parse_config("all:100:full:b10", 77)
    assert p.nprobe == 77 and p.prune == (10, 1.0)
    with pytest.raises(ValueError):
        parse_config("8:100:bogus", 8)


def test_splitmix_stream_matches_oracle_rng():
    r = O.Rng(42)
    want = [r.next() for _ in range(10)]
    assert [int(x) for x in builder.splitmix_stream(42, 10)] == want
    assert np.array_equal(builder.rotation_signs(11), O.rotation_signs(11))


def test_builder_rotation_is_the_reference_rotation():
    signs = O.rotation_signs(11)
    v = np.random.default_rng(0).standard_normal((5, 256)).astype(np.float32)
    got = builder.rotate(torch.as_tensor(signs), torch.as_tensor(v)).numpy()
    for i in range(5):
        assert np.array_equal(got[i], O.rotation_apply(signs, v[i]))


def test_builder_pack_is_the_reference_pack_block():
    r = np.random.default_rng(3)
    codes = r.integers(0, 256, (4, 32, 32), dtype=np.uint8)
    got = builder.pack_blocks(torch.as_tensor(codes)).numpy()
    for b in range(4):
        assert np.array_equal(got[b], O.pack_block(codes[b]))


def test_built_index_layout():
    arrays, q768, q256, _ = index_a()
    k, bo, ids = arrays["k"], arrays["block_off"].astype(np.int64), arrays["ids"]
    assert bo[0] == 0 and np.all(np.diff(bo) >= 0) and ids.size == bo[-1] * 32
    seen = np.zeros(arrays["n"], np.int64)
    for c in range(k):
        s = ids[bo[c] * 32 : bo[c + 1] * 32]
        real = s[s != 0xFFFFFFFF]
        assert np.all(s[: real.size] != 0xFFFFFFFF) and np.all(s[real.size :] == 0xFFFFFFFF)
        assert np.all(np.diff(real.astype(np.int64)) > 0)  # row order inside a cluster
        seen[real] += 1
    assert np.all(seen == 2)  # SOAR: every row in exactly two clusters
    # each slot's code is the sign code of the rotated residual to its cluster
    signs = arrays["rotation"]
    cr = np.stack([O.rotation_apply(signs, c) for c in arrays["centroids"].reshape(k, 256)])
    scale = arrays["quant_scale"][:256]
    for c in (0, 5):
        s0 = bo[c] * 32
        blk = arrays["blocks"][bo[c] * 1024 : (bo[c] + 1) * 1024]
        for j in range(3):
            row = ids[s0 + j]
            x = O.normalize(arrays["rerank"][row, :256].astype(np.float32) / scale)[0]
            code, mul, err = O.rabitq_encode(O.rotation_apply(signs, x), cr[c])
            assert np.array_equal(O.unpack_slot(blk, 64, j), code)
            f = arrays["factors"][2 * (s0 + j) : 2 * (s0 + j) + 2]
            assert abs(f[0] - mul) <= 1e-4 * abs(mul) and abs(f[1] - err) <= 1e-3 * abs(err) + 1e-6


def test_reference_files_round_trip(tmp_path):
    arrays, *_ = index_a()
    corpus = {k: arrays[k] for k in ("n", "rerank", "norm256", "codes", "quant_scale")}
    builder.write_files(corpus, arrays, str(tmp_path / "i"), str(tmp_path / "x"))
    back = builder.read_files(str(tmp_path / "i"), str(tmp_path / "x"))
    for key in list(builder.CORPUS_FILES) + list(builder.INDEX_FILES):
        assert np.array_equal(np.asarray(back[key]).ravel(), np.asarray(arrays[key]).ravel()), key


def test_oracle_search_is_sane():
    arrays, q768, q256, mix = index_a()
    oi = O.OracleIndex(arrays)
    gt = builder.ground_truth(mix, torch.as_tensor(q768), k=10)
    p = Params(16, 1000, Rerank.full(), 10).to_c()
    s, o, cnt, scanned = oi.search_batch(q768, q256, p, threads=4)
    rec = np.mean([O.recall_at(10, o[i, : cnt[i]], gt[i]) for i in range(len(q768))])
    assert rec > 0.8
    assert np.all(np.diff(s, axis=1) <= 0)
    for i in range(0, len(q768), 9):
        s1, o1, _ = oi.search(q768[i], q256[i], p)
        assert np.array_equal(o1, o[i, : cnt[i]])


def test_plan_resolve_is_the_reference_auto_plan():
    """src/filter.rs:157-165 auto_plan, through the library's host-side sg_plan_resolve."""
    from sieve_gpu import filter as F

    class Fake:
        def __init__(self, rows):
            self.nrows = rows

    n = 10_000_000
    assert F.Plan.auto().resolve(Fake(F.BRUTE_MAX), n) == F.Plan.brute()
    assert F.Plan.auto().resolve(Fake(1_000_000), n) == F.Plan.expand(F.EXPAND_TARGET)
    assert F.Plan.auto().resolve(Fake(3_000_000), n) == F.Plan.post()
    assert F.Plan.expand(7).resolve(Fake(1), n) == F.Plan.expand(7)
    for rows in (0, 1, 250_000, 250_001, 2_999_999, 3_000_000, 10_000_000):
        for plan in range(4):
            got = _abi.lib().sg_plan_resolve(plan, _abi.c_uint64(rows), _abi.c_uint64(n))
            assert got == O.plan_resolve(plan, rows, n)
