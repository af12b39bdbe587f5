"""Committed golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the oracle):
the CPU test checks the oracle still reproduces them; the GPU test checks the CUDA path does."""
import os

import numpy as np
import pytest

import oracle as O
from sieve_gpu import Params, Rerank

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_ivf():
    z = np.load(os.path.join(HERE, "ivf_small.npz"))
    arrays = {k: z[k] for k in ("rerank", "norm256", "codes", "quant_scale", "centroids", "block_off",
                                "ids", "blocks", "factors", "rotation", "tier2_sigma", "tier2_codes",
                                "tier2_norm")}
    arrays["n"], arrays["k"] = int(z["n"]), int(z["k"])
    return z, arrays


def case_params(v) -> Params:
    nprobe, cand, kind, r, k, pm, pw, margin = v
    return Params(int(nprobe), int(cand), Rerank(int(kind), int(r)), int(k),
                  None if pm < 0 else (int(pm), float(pw)), None if margin < 0 else float(margin))


CASES = ["full", "tiered", "prefix", "none", "pruned", "margin"]


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_golden(case):
    z, arrays = load_ivf()
    oi = O.OracleIndex(arrays)
    p = case_params(z[f"{case}_params"]).to_c()
    for i in range(z["q768"].shape[0]):
        s, o, _ = oi.search(z["q768"][i], z["q256"][i], p)
        n = int(z[f"{case}_counts"][i])
        assert s.size == n
        assert np.array_equal(o, z[f"{case}_ids"][i, :n])
        assert np.array_equal(s, z[f"{case}_scores"][i, :n])


def test_oracle_lut_golden():
    z = np.load(os.path.join(HERE, "lut_small.npz"))
    t, s, b = O.lut_new(z["q32"])
    assert np.array_equal(t, z["tables32"]) and s == z["scale32"] and b == z["bias32"]
    assert np.array_equal(O.scan(t, z["block32"]), z["scores32"])
    for k in range(32):
        assert z["scores32"][k] == O.score_code(t, z["codes32"][k])
    t64, s64, b64 = O.lut_new(z["q64"])
    assert np.array_equal(t64, z["tables64"])
    assert np.array_equal(O.scan(t64, z["blocks64"]), z["scores64"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_golden(case):
    from sieve_gpu import Index

    z, arrays = load_ivf()
    ix = Index.from_arrays(arrays)
    try:
        p = case_params(z[f"{case}_params"])
        sc, ids, cnt = ix.search_batch(z["q768"], z["q256"], p)
        assert np.array_equal(cnt, z[f"{case}_counts"])
        for i in range(cnt.size):
            n = int(cnt[i])
            assert np.array_equal(ids[i, :n], z[f"{case}_ids"][i, :n])
            assert np.array_equal(sc[i, :n], z[f"{case}_scores"][i, :n])
    finally:
        ix.close()


@pytest.mark.gpu
def test_gpu_lut_golden():
    from sieve_gpu import lut_scan

    z = np.load(os.path.join(HERE, "lut_small.npz"))
    assert np.array_equal(lut_scan(z["tables32"], z["block32"]), z["scores32"])
    assert np.array_equal(lut_scan(z["tables64"], z["blocks64"]), z["scores64"])
