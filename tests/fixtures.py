"""Seeded small corpora and indexes shared by the tests (built on the CPU with the builder).

INDEX_A: 20,000 rows, 64 clusters, SOAR, 2-bit tier — clusters of about one scan chunk.
INDEX_B: 30,000 rows with 400 exact duplicates, 8 clusters — clusters span several scan chunks,
         and the duplicates make exactly tied estimates and tied int8 scores.
INDEX_C: 12,000 rows, 300 clusters, 150 queries — several routing GEMM tiles on both axes.
INDEX_D: 16,384 rows, 4096 clusters, 4096 queries — the routing GEMM at full size.
INDEX_G: 6,000 rows, 16 clusters, built without RaBitQ: global sign codes, no rotation/factors;
         96 queries (16 copies of rows) so the batched path runs.
Queries come from the same mixtures (sigma 0.35) plus copies of corpus rows (self-matches).
"""
from __future__ import annotations

import functools

import numpy as np
import torch

from sieve_gpu import builder, synth

import oracle as O


def prefixes(q768: np.ndarray) -> np.ndarray:
    return np.stack([O.prefix(v)[0] for v in q768]).astype(np.float32)


@functools.lru_cache(maxsize=None)
def index_a():
    torch.manual_seed(0)
    mix = synth.Mixture(n=20000, n_centers=64, seed=3)
    corpus = builder.ingest(mix)
    ix = builder.build_ivf(corpus, k=64, sample_n=20000, iters=8)
    arrays = {**corpus, **ix}
    q = mix.queries(48, sigma=0.35).numpy()
    rows = mix.rows(100, 16).numpy()  # self-match queries
    q768 = np.concatenate([q, rows]).astype(np.float32)
    return arrays, q768, prefixes(q768), mix


@functools.lru_cache(maxsize=None)
def index_b():
    mix = synth.Mixture(n=30000, n_centers=24, seed=5)
    corpus = builder.ingest(mix)
    # 400 exact duplicates: rows 0..99 repeated 4 more times at the end
    dup = np.concatenate([corpus["rerank"][:100]] * 4)
    corpus["rerank"] = np.concatenate([corpus["rerank"], dup])
    corpus["norm256"] = np.concatenate([corpus["norm256"], np.tile(corpus["norm256"][:100], 4)])
    corpus["codes"] = np.concatenate([corpus["codes"], np.tile(corpus["codes"][:100], (4, 1))])
    corpus["n"] = corpus["rerank"].shape[0]
    ix = builder.build_ivf(corpus, k=8, sample_n=30400, iters=6)
    arrays = {**corpus, **ix}
    q = mix.queries(24, sigma=0.35).numpy()
    # queries near the duplicated rows: ties among their copies
    rows = (corpus["rerank"][:8].astype(np.float32) / corpus["quant_scale"])
    rows /= np.linalg.norm(rows, axis=1, keepdims=True)
    q768 = np.concatenate([q, rows]).astype(np.float32)
    return arrays, q768, prefixes(q768), mix


@functools.lru_cache(maxsize=None)
def index_c():
    """300 clusters over 12,000 rows and 150 queries: routing tiles of 128 centroids x 64 queries
    with a partial last tile on both axes."""
    torch.manual_seed(1)
    mix = synth.Mixture(n=12000, n_centers=96, seed=11)
    corpus = builder.ingest(mix)
    ix = builder.build_ivf(corpus, k=300, sample_n=12000, iters=3)
    arrays = {**corpus, **ix}
    q768 = mix.queries(150, sigma=0.35).numpy().astype(np.float32)
    return arrays, q768, prefixes(q768), mix


@functools.lru_cache(maxsize=None)
def index_d():
    """4096 clusters over 16,384 rows and a batch of 4096 queries: the routing GEMM at full size
    (K = 4096 centroids x 4096 queries, 32 x 64 tiles)."""
    torch.manual_seed(2)
    mix = synth.Mixture(n=16384, n_centers=256, seed=13)
    corpus = builder.ingest(mix)
    ix = builder.build_ivf(corpus, k=4096, sample_n=16384, iters=1)
    arrays = {**corpus, **ix}
    q768 = mix.queries(4096, sigma=0.35).numpy().astype(np.float32)
    return arrays, q768, prefixes(q768), mix


@functools.lru_cache(maxsize=None)
def index_g():
    """ivf::build with rabitq: false (src/ivf.rs:366-372): every slot holds its row's global sign
    code; the index has no rotation.f32 / factors.f32 (the ablation of src/ivf.rs:700-717)."""
    torch.manual_seed(4)
    mix = synth.Mixture(n=6000, n_centers=24, seed=17)
    corpus = builder.ingest(mix)
    ix = builder.build_ivf(corpus, k=16, sample_n=6000, iters=4, rabitq=False)
    arrays = {**corpus, **ix}
    q = mix.queries(80, sigma=0.35).numpy()
    rows = mix.rows(50, 16).numpy()  # self-match queries: every slot of their row ties
    q768 = np.concatenate([q, rows]).astype(np.float32)
    return arrays, q768, prefixes(q768)


@functools.lru_cache(maxsize=None)
def bigann_a(bits: int):
    """bigann: 20,000 int8 rows (64 mixture centres) plus 200 exact duplicates, 8 x 16 leaves;
    64 queries from the mixture and 16 copies of base rows."""
    from sieve_gpu import bigann_builder as BB

    sp = BB.Spacev(20000, 64, seed=5, device="cpu")
    base = sp.rows(0, 20000)
    base = torch.cat([base, base[:200]])
    ix = BB.build_bigann(base, 8, 16, bits=bits, sample_n=20200, iters=6)
    q = torch.cat([sp.queries(64), base[1000:1016]]).numpy()
    return ix, q


@functools.lru_cache(maxsize=None)
def bigann_c():
    """bigann with many small leaves: 30,000 int8 rows, 64 x 160 = 10,240 leaves (more than the
    8,192 past which the tensor-core routing takes its threshold from a 1/16 subset of the leaves),
    duplicate leaves where a top cluster holds fewer rows than 160 (tied route scores); 40 queries
    from the mixture and 8 copies of leaf centres' nearest base rows."""
    from sieve_gpu import bigann_builder as BB

    sp = BB.Spacev(30000, 256, seed=13, device="cpu")
    base = sp.rows(0, 30000)
    ix = BB.build_bigann(base, 64, 160, bits=1, sample_n=30000, iters=4)
    q = torch.cat([sp.queries(40), base[5000:5008]]).numpy()
    return ix, q


@functools.lru_cache(maxsize=None)
def bigann_b():
    """bigann with few, large leaves (2 x 4 of about 5,000 slots): scan steps span whole chunks
    and the shortlist compacts many times inside one leaf."""
    from sieve_gpu import bigann_builder as BB

    sp = BB.Spacev(40000, 16, seed=9, device="cpu")
    base = sp.rows(0, 40000)
    ix = BB.build_bigann(base, 2, 4, bits=3, sample_n=40000, iters=5)
    return ix, sp.queries(24).numpy()
