"""Regenerates tests/golden/*.npz: small seeded inputs and the oracle's outputs on them.

    python tests/golden/make_golden.py

ivf_small.npz  a 512-row corpus + 8-cluster RaBitQ index (built by sieve_gpu.builder on the CPU),
               12 queries, and the oracle's probe lists, candidates and final lists for several
               parameter sets (keys `<case>_<field>`).
lut_small.npz  the reference's deterministic LUT test inputs (src/lut.rs:237-266: q[i] = cos(0.91 i),
               code[k][i] = (37k + 11i) mod 256, G = 32; q[i] = sin(0.37 i), G = 64) with tables and
               scan outputs.
The outputs come from the oracle (oracle/sieve_oracle.c); the tests check that the oracle still
reproduces them and that the GPU path matches them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "a-game-of-vectors_b200"), os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from sieve_gpu import Params, Rerank, builder, synth  # noqa: E402

CASES = {
    "full": Params(4, 200, Rerank.full(), 10),
    "tiered": Params(4, 200, Rerank.tiered(40), 10),
    "prefix": Params(3, 150, Rerank.prefix(), 8),
    "none": Params(8, 100, Rerank.none(), 10),
    "pruned": Params(5, 200, Rerank.full(), 10, prune=(10, 0.5)),
    "margin": Params(8, 300, Rerank.ssd(60), 10, margin=0.05),
}
ARRAY_KEYS = ["rerank", "norm256", "codes", "quant_scale", "centroids", "block_off", "ids", "blocks",
              "factors", "rotation", "tier2_sigma", "tier2_codes", "tier2_norm"]


def make_ivf():
    mix = synth.Mixture(n=512, n_centers=8, seed=21)
    corpus = builder.ingest(mix)
    ix = builder.build_ivf(corpus, k=8, sample_n=512, iters=6)
    arrays = {**corpus, **ix}
    q768 = mix.queries(12, sigma=0.35).numpy().astype(np.float32)
    q256 = np.stack([O.prefix(v)[0] for v in q768]).astype(np.float32)
    oi = O.OracleIndex(arrays)
    out = {k: np.asarray(arrays[k]) for k in ARRAY_KEYS}
    out.update(n=np.uint64(arrays["n"]), k=np.uint32(arrays["k"]), q768=q768, q256=q256)
    for name, p in CASES.items():
        cp = p.to_c()
        k = max(p.k, 1)
        sc = np.zeros((12, k), np.float32)
        ids = np.zeros((12, k), np.uint32)
        cnt = np.zeros(12, np.uint32)
        for i in range(12):
            s, o, _ = oi.search(q768[i], q256[i], cp)
            sc[i, : s.size], ids[i, : s.size], cnt[i] = s, o, s.size
        out[f"{name}_scores"], out[f"{name}_ids"], out[f"{name}_counts"] = sc, ids, cnt
        out[f"{name}_params"] = np.array([p.nprobe, p.cand, p.rerank.kind, p.rerank.r, p.k,
                                          -1 if p.prune is None else p.prune[0],
                                          -1.0 if p.prune is None else p.prune[1],
                                          -1.0 if p.margin is None else p.margin], np.float64)
    np.savez_compressed(os.path.join(HERE, "ivf_small.npz"), **out)


def make_lut():
    q32 = np.cos(np.arange(128, dtype=np.float32) * np.float32(0.91)).astype(np.float32)
    codes = np.array([[(k * 37 + i * 11) % 256 for i in range(16)] for k in range(32)], np.uint8)
    t32, s32, b32 = O.lut_new(q32)
    blk32 = O.pack_block(codes, groups=32)
    q64 = np.sin(np.arange(256, dtype=np.float32) * np.float32(0.37)).astype(np.float32)
    t64, s64, b64 = O.lut_new(q64)
    rng = np.random.default_rng(123)
    blocks64 = rng.integers(0, 256, (16, 1024), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "lut_small.npz"), q32=q32, codes32=codes, tables32=t32,
                        scale32=np.float32(s32), bias32=np.float32(b32), block32=blk32,
                        scores32=O.scan(t32, blk32), q64=q64, tables64=t64, scale64=np.float32(s64),
                        bias64=np.float32(b64), blocks64=blocks64, scores64=O.scan(t64, blocks64))


if __name__ == "__main__":
    make_ivf()
    make_lut()
    for f in ("ivf_small.npz", "lut_small.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
