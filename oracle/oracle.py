"""Python view of the CPU oracle (oracle/sieve_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm, as the checker. The product (a-game-of-vectors_b200/) never imports it.

Each wrapper names the reference function it restates; sieve_oracle.h lists the file:line map,
the float rules and the tie convention. Parity pin: the reference's own unit and property tests,
ported in tests/test_oracle_*.py (the reference ships no golden vectors and cannot be built here).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from ctypes import POINTER, c_double, c_float, c_int, c_uint16, c_uint32, c_uint64, c_void_p

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "a-game-of-vectors_b200"))
from sieve_gpu._abi import (SgBigannParams, SgBigannTiming, SgIvfArrays, SgParams, SgTiming,  # noqa: E402
                            make_arrays, make_bigann_arrays)

HERE = os.path.dirname(os.path.abspath(__file__))


def build(native: bool = False) -> str:
    """Compiles the oracle; native=True builds a -march=native copy for timing on this host."""
    out = "_build/native" if native else "_build"
    cmd = ["make", "-s", "-C", HERE, f"OUT={out}"]
    if native:
        cmd.append("ARCH=-march=native")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, out, "liboracle.so")


_libs: dict = {}


def lib(native: bool = False) -> ctypes.CDLL:
    key = "native" if native else "portable"
    if key in _libs:
        return _libs[key]
    path = os.path.join(HERE, "_build/native" if native else "_build", "liboracle.so")
    if native or not os.path.exists(path):
        path = build(native)
    L = ctypes.CDLL(path)
    L.or_rng_next.restype = c_uint64
    L.or_rng_below.restype = c_uint64
    L.or_rotation_norm.restype = c_float
    L.or_score_code.restype = c_uint16
    L.or_float_score.restype = c_float
    L.or_lut_to_float.restype = c_float
    L.or_lut_to_float.argtypes = [c_float, c_float, c_uint16]
    L.or_hamming.restype = c_uint32
    L.or_estimate.restype = c_float
    L.or_estimate.argtypes = [c_float, c_float, c_float, c_float, c_uint16]
    for f in ("or_normalize", "or_prefix", "or_dot_i8", "or_dot_f32", "or_query_i8",
              "or_tier2_encode", "or_tier2_score"):
        getattr(L, f).restype = c_float
    L.or_tier2_score.argtypes = [c_void_p, c_void_p, c_float]
    L.or_dot_i8i8.restype = ctypes.c_int32
    L.or_topk.restype = c_uint32
    L.or_route.restype = c_uint32
    L.or_candidates.restype = c_uint32
    L.or_prune_threshold.restype = c_float
    L.or_prune_threshold.argtypes = [c_void_p, c_void_p, c_uint32, c_uint32, c_float]
    L.or_rerank.restype = c_uint32
    L.or_search.restype = c_uint32
    L.or_search_batch.restype = c_uint64
    L.or_flat_hamming.restype = c_uint32
    L.or_tie_rule.restype = c_int
    L.or_last_tied.restype = c_int
    L.or_plan_resolve.restype = c_int
    L.or_filter_search.restype = c_uint32
    L.or_recall_at.restype = c_double
    for f in ("or_bg_refine_encode", "or_bg_refiner_estimate"):
        getattr(L, f).restype = c_float
    L.or_bg_refiner_estimate.argtypes = [c_void_p, c_float, c_uint32, c_void_p, c_void_p, c_float]
    for f in ("or_bg_extra", "or_bg_route", "or_bg_candidates", "or_bg_rerank", "or_bg_search"):
        getattr(L, f).restype = c_uint32
    L.or_bg_search_batch.restype = c_uint64
    _libs[key] = L
    return L


def P(a: np.ndarray) -> c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return c_void_p(a.ctypes.data)


def f32(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.float32)


# ---- primitives ----------------------------------------------------------------------------
class Rng:
    """splitmix64 (src/ivf.rs:119-135)."""

    def __init__(self, seed: int):
        self.s = c_uint64(seed)

    def next(self) -> int:
        return lib().or_rng_next(ctypes.byref(self.s))

    def below(self, n: int) -> int:
        return lib().or_rng_below(ctypes.byref(self.s), c_uint64(n))


def rotation_signs(seed: int, d: int = 256) -> np.ndarray:
    """Rotation::with_dim (src/rabitq.rs:40-44)."""
    out = np.empty(3 * d, np.float32)
    lib().or_rotation_signs(c_uint64(seed), c_uint32(d), P(out))
    return out


def rotation_apply(signs: np.ndarray, v) -> np.ndarray:
    """Rotation::apply (src/rabitq.rs:60-69)."""
    v = f32(v).copy()
    lib().or_rotation_apply(P(f32(signs)), c_uint32(v.size), P(v))
    return v


def rabitq_encode(xr, cr):
    """rabitq::encode (src/rabitq.rs:88-108) -> (code, mul, err)."""
    xr, cr = f32(xr), f32(cr)
    code = np.zeros(xr.size // 8, np.uint8)
    me = np.zeros(2, np.float32)
    lib().or_rabitq_encode(P(xr), P(cr), c_uint32(xr.size), P(code), P(me))
    return code, float(me[0]), float(me[1])


def lut_new(q):
    """Lut::new (src/lut.rs:33-55) -> (tables [G,16] u8, scale, bias)."""
    q = f32(q)
    G = q.size // 4
    t = np.zeros((G, 16), np.uint8)
    sc, bi = c_float(), c_float()
    lib().or_lut_new(P(q), c_uint32(G), P(t), ctypes.byref(sc), ctypes.byref(bi))
    return t, sc.value, bi.value


def score_code(tables: np.ndarray, code) -> int:
    code = np.ascontiguousarray(code, np.uint8)
    return int(lib().or_score_code(P(np.ascontiguousarray(tables)), c_uint32(tables.shape[0]), P(code)))


def float_score(q, code) -> float:
    q, code = f32(q), np.ascontiguousarray(code, np.uint8)
    return lib().or_float_score(P(q), c_uint32(q.size), P(code))


def lut_to_float(scale: float, bias: float, s: int) -> float:
    return lib().or_lut_to_float(scale, bias, s)


def pack_block(codes, groups: int = 64) -> np.ndarray:
    """pack_block (src/lut.rs:72-82): up to 32 raw codes of groups/2 bytes."""
    codes = np.ascontiguousarray(codes, np.uint8).reshape(-1, groups // 2)
    out = np.zeros(groups * 16, np.uint8)
    lib().or_pack_block(P(codes), c_uint32(codes.shape[0]), c_uint32(groups), P(out))
    return out


def unpack_slot(block, groups: int, k: int) -> np.ndarray:
    block = np.ascontiguousarray(block, np.uint8)
    out = np.zeros(groups // 2, np.uint8)
    lib().or_unpack_slot(P(block), c_uint32(groups), c_uint32(k), P(out))
    return out


def scan(tables: np.ndarray, blocks) -> np.ndarray:
    """lut::scan with scan_block_scalar (src/lut.rs:96-126)."""
    tables = np.ascontiguousarray(tables, np.uint8)
    G = tables.shape[0]
    blocks = np.ascontiguousarray(blocks, np.uint8)
    nb = blocks.size // (G * 16)
    out = np.zeros(nb * 32, np.uint16)
    lib().or_scan(P(tables), c_uint32(G), P(blocks), c_uint64(nb), P(out))
    return out


def hamming(a, b) -> int:
    a, b = np.ascontiguousarray(a, np.uint8), np.ascontiguousarray(b, np.uint8)
    return int(lib().or_hamming(P(a), P(b), c_uint32(a.size)))


def query_new(signs, q):
    """rabitq::Query::new (src/rabitq.rs:119-125) -> (tables, scale, bias, a, b)."""
    q = f32(q)
    G = q.size // 4
    t = np.zeros((G, 16), np.uint8)
    sc, bi, a, b = c_float(), c_float(), c_float(), c_float()
    lib().or_query_new(P(f32(signs)), c_uint32(q.size), P(q), P(t), ctypes.byref(sc),
                       ctypes.byref(bi), ctypes.byref(a), ctypes.byref(b))
    return t, sc.value, bi.value, a.value, b.value


def estimate(a, b, cent, mul, s) -> float:
    return lib().or_estimate(a, b, cent, mul, int(s))


def normalize(v) -> tuple[np.ndarray, float]:
    v = f32(v).copy()
    n = lib().or_normalize(P(v), c_uint32(v.size))
    return v, n


def prefix(full) -> tuple[np.ndarray, float]:
    full = f32(full)
    out = np.zeros(256, np.float32)
    n = lib().or_prefix(P(full), P(out))
    return out, n


def sign_code(prefix_vec) -> np.ndarray:
    p = f32(prefix_vec)
    out = np.zeros(32, np.uint8)
    lib().or_sign_code(P(p), P(out))
    return out


def int8_fit(rows) -> np.ndarray:
    rows = f32(rows).reshape(-1, 768)
    sc = np.zeros(768, np.float32)
    lib().or_int8_fit(P(rows), c_uint64(rows.shape[0]), P(sc))
    return sc


def int8_encode(scale, v) -> np.ndarray:
    out = np.zeros(768, np.int8)
    lib().or_int8_encode(P(f32(scale)), P(f32(v)), P(out))
    return out


def int8_query_weights(scale, q) -> np.ndarray:
    q = f32(q)
    w = np.zeros(q.size, np.float32)
    lib().or_int8_query_weights(P(f32(scale)), P(q), c_uint32(q.size), P(w))
    return w


def dot_i8(w, x) -> float:
    w, x = f32(w), np.ascontiguousarray(x, np.int8)
    return lib().or_dot_i8(P(w), P(x), c_uint32(w.size))


def dot_f32(a, b) -> float:
    a, b = f32(a), f32(b)
    return lib().or_dot_f32(P(a), P(b), c_uint32(a.size))


def query_i8(w) -> tuple[np.ndarray, float]:
    w = f32(w)
    out = np.zeros(w.size, np.int8)
    s = lib().or_query_i8(P(w), c_uint32(w.size), P(out))
    return out, s


def dot_i8i8(a, b) -> int:
    a, b = np.ascontiguousarray(a, np.int8), np.ascontiguousarray(b, np.int8)
    return int(lib().or_dot_i8i8(P(a), P(b), c_uint32(a.size)))


def tier2_fit(rows) -> np.ndarray:
    rows = f32(rows).reshape(-1, 256)
    s = np.zeros(256, np.float32)
    lib().or_tier2_fit(P(rows), c_uint64(rows.shape[0]), P(s))
    return s


def tier2_encode(sigma, p) -> tuple[np.ndarray, float]:
    out = np.zeros(64, np.uint8)
    n = lib().or_tier2_encode(P(f32(sigma)), P(f32(p)), P(out))
    return out, n


def tier2_tables(sigma, q) -> np.ndarray:
    t = np.zeros((64, 256), np.float32)
    lib().or_tier2_tables(P(f32(sigma)), P(f32(q)), P(t))
    return t


def tier2_score(tables, code, norm) -> float:
    return lib().or_tier2_score(P(f32(tables)), P(np.ascontiguousarray(code, np.uint8)), float(norm))


def topk(scores, ids, k: int, tied: bool = False):
    """TopK::new(k), push in order, into_sorted (src/topk.rs) under the current tie rule; with
    tied=True also whether the cut at the k-th place was tied."""
    scores, ids = f32(scores), np.ascontiguousarray(ids, np.uint32)
    os_, oi = np.zeros(max(k, 1), np.float32), np.zeros(max(k, 1), np.uint32)
    L = lib()
    L.or_clear_tied()
    m = L.or_topk(P(scores), P(ids), c_uint64(scores.size), c_uint32(k), P(os_), P(oi))
    if tied:
        return os_[:m], oi[:m], bool(L.or_last_tied())
    return os_[:m], oi[:m]


def gemm_abt(a, b) -> np.ndarray:
    a, b = f32(a), f32(b)
    m, k = a.shape
    n = b.shape[0]
    c = np.zeros((m, n), np.float32)
    lib().or_gemm_abt(P(a), P(b), c_uint64(m), c_uint64(n), c_uint64(k), P(c))
    return c


def prune_threshold(est, err, m: int, w: float) -> float:
    est, err = f32(est), f32(err)
    return lib().or_prune_threshold(P(est), P(err), c_uint32(est.size), c_uint32(m), c_float(w))


def recall_at(k: int, got, truth) -> float:
    got, truth = np.ascontiguousarray(got, np.uint32), np.ascontiguousarray(truth, np.uint32)
    return lib().or_recall_at(c_uint32(k), P(got), c_uint32(got.size), P(truth), c_uint32(truth.size))


def plan_resolve(plan: int, allowed_rows: int, n: int) -> int:
    return lib().or_plan_resolve(c_int(plan), c_uint64(allowed_rows), c_uint64(n))


# ---- the query path over an index ------------------------------------------------------------
def build_ivf(corpus: dict, k: int, sample_n: int, iters: int, balance: float | None = None,
              soar_lambda: float | None = 1.0) -> dict:
    """ivf::build (src/ivf.rs:268-395) with RaBitQ codes, on the corpus's int8 rows: the arrays
    of the index files (centroids, tier-2 files, block_off, ids, blocks, factors, rotation)."""
    n = int(corpus["n"])
    rer = np.ascontiguousarray(corpus["rerank"], np.int8)
    scale = f32(corpus["quant_scale"])
    cents = np.zeros((k, 256), np.float32)
    sigma = np.zeros(256, np.float32)
    t2 = np.zeros((n, 64), np.uint8)
    t2n = np.zeros(n, np.float32)
    boff = np.zeros(k + 1, np.uint64)
    maxb = (2 * n + 31) // 32 + k
    ids = np.zeros(maxb * 32, np.uint32)
    blocks = np.zeros(maxb * 1024, np.uint8)
    fac = np.zeros(maxb * 64, np.float32)
    L = lib()
    L.or_build_ivf.restype = c_uint64
    nb = L.or_build_ivf(c_uint64(n), P(rer), P(scale), c_uint32(k), c_uint64(sample_n), c_uint32(iters),
                        c_int(balance is not None), c_float(balance or 0.0), c_int(soar_lambda is not None),
                        c_float(soar_lambda or 0.0), P(cents), P(sigma), P(t2), P(t2n), P(boff), P(ids),
                        P(blocks), P(fac), c_uint64(maxb))
    assert nb <= maxb
    return {"n": n, "k": k, "centroids": cents, "tier2_sigma": sigma, "tier2_codes": t2, "tier2_norm": t2n,
            "block_off": boff, "ids": ids[: nb * 32], "blocks": blocks[: nb * 1024], "factors": fac[: nb * 64],
            "rotation": rotation_signs(11)}


TIE_CANONICAL, TIE_REFERENCE = 0, 1


def set_tie_rule(rule: int, native: bool = False) -> None:
    """The tie rule of every TopK (sieve_oracle.h): TIE_CANONICAL keeps the k best by (score desc,
    id asc); TIE_REFERENCE restates src/topk.rs's `<=` rejection and select-by-score cut."""
    lib(native).or_set_tie_rule(c_int(rule))


class OracleIndex:
    """ivf::Index + ivf::Corpus over in-memory arrays (the same dict the GPU index opens)."""

    def __init__(self, arrays: dict, native: bool = False):
        self.st, self._keep = make_arrays(arrays)
        self._arrays = arrays
        self.k = int(arrays["k"])
        self.n = int(arrays["n"])
        self.L = lib(native)

    def route(self, q256, p: SgParams):
        q = f32(q256)
        cap = max(min(p.nprobe, self.k), 1)
        s, c = np.zeros(cap, np.float32), np.zeros(cap, np.uint32)
        m = self.L.or_route(ctypes.byref(self.st), P(q), ctypes.byref(p), P(s), P(c))
        return s[:m], c[:m]

    def candidates(self, q256, probe_scores, probe_clusters, p: SgParams, allow=None):
        q = f32(q256)
        ps, pc = f32(probe_scores), np.ascontiguousarray(probe_clusters, np.uint32)
        cap = max(p.cand, 1)
        e, i, r = np.zeros(cap, np.float32), np.zeros(cap, np.uint32), np.zeros(cap, np.float32)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        scanned = c_uint64(0)
        m = self.L.or_candidates(ctypes.byref(self.st), P(q), P(ps), P(pc), c_uint32(ps.size),
                                 ctypes.byref(p), None if al is None else P(al),
                                 c_uint64(0 if al is None else al.size), P(e), P(i), P(r),
                                 ctypes.byref(scanned))
        return e[:m], i[:m], r[:m]

    def rerank(self, q768, q256, est, ids, err, p: SgParams):
        est, ids, err = f32(est), np.ascontiguousarray(ids, np.uint32), f32(err)
        k = max(p.k, 1)
        s, o = np.zeros(k, np.float32), np.zeros(k, np.uint32)
        m = self.L.or_rerank(ctypes.byref(self.st), P(f32(q768)), P(f32(q256)), P(est), P(ids),
                             P(err), c_uint32(est.size), ctypes.byref(p), P(s), P(o), None)
        return s[:m], o[:m]

    def search(self, q768, q256, p: SgParams, allow=None):
        k = max(p.k, 1)
        s, o = np.zeros(k, np.float32), np.zeros(k, np.uint32)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        t = SgTiming()
        m = self.L.or_search(ctypes.byref(self.st), P(f32(q768)), P(f32(q256)), ctypes.byref(p),
                             None if al is None else P(al), c_uint64(0 if al is None else al.size),
                             P(s), P(o), ctypes.byref(t))
        return s[:m], o[:m], t

    def search_batch(self, q768, q256, p: SgParams, allow=None, threads: int = 1, tied: bool = False):
        """(scores, ids, counts, scanned) of many queries; with tied=True also a per-query flag
        that some TopK on its path cut a tie at its k-th place."""
        q768, q256 = f32(q768), f32(q256)
        nq = q768.shape[0]
        k = max(p.k, 1)
        s = np.zeros((nq, k), np.float32)
        o = np.zeros((nq, k), np.uint32)
        cnt = np.zeros(nq, np.uint32)
        tie = np.zeros(nq, np.uint8)
        al = None if allow is None else np.ascontiguousarray(allow, np.uint64)
        scanned = self.L.or_search_batch(ctypes.byref(self.st), c_uint32(nq), P(q768), P(q256),
                                         ctypes.byref(p), None if al is None else P(al),
                                         c_uint64(0 if al is None else al.size), c_int(threads),
                                         P(s), P(o), P(cnt), P(tie))
        if tied:
            return s, o, cnt, scanned, tie.astype(bool)
        return s, o, cnt, scanned

    def live_encode(self, cents_rot, soar: bool, lam: float, v):
        """Live::apply_insert's encoding of one unit 768-d row (src/live.rs:318-350): (int8 row,
        prefix norm, (primary, secondary or PAD), codes [2, 32], factors [2, 2], tier-2 code, norm)."""
        row = np.zeros(768, np.int8)
        nrm, t2n = c_float(), c_float()
        pair = np.zeros(2, np.uint32)
        codes = np.zeros((2, 32), np.uint8)
        fac = np.zeros((2, 2), np.float32)
        t2 = np.zeros(64, np.uint8)
        self.L.or_live_encode(ctypes.byref(self.st), P(f32(cents_rot)), c_int(1 if soar else 0), c_float(lam),
                              P(f32(v)), P(row), ctypes.byref(nrm), P(pair), P(codes), P(fac), P(t2),
                              ctypes.byref(t2n))
        return row, nrm.value, pair, codes, fac, t2, t2n.value

    def flat_hamming(self, codes, q768, q256, cand: int, k: int):
        """The search binary's flat Hamming baseline (src/bin/search.rs:251-269) over codes.bin."""
        codes = np.ascontiguousarray(codes, np.uint8)
        s, o = np.zeros(max(k, 1), np.float32), np.zeros(max(k, 1), np.uint32)
        a = self._arrays
        m = self.L.or_flat_hamming(P(codes), c_uint64(codes.size // 32), P(np.ascontiguousarray(a["rerank"])),
                                   P(f32(a["quant_scale"])), P(f32(q768)), P(f32(q256)), c_uint32(cand),
                                   c_uint32(k), P(s), P(o))
        return s[:m], o[:m]

    def filter_per_cluster(self, allow) -> np.ndarray:
        al = np.ascontiguousarray(allow, np.uint64)
        out = np.zeros(self.k, np.uint32)
        self.L.or_filter_per_cluster(ctypes.byref(self.st), P(al), c_uint64(al.size), P(out))
        return out

    def filter_search(self, allow, rows, per_cluster, plan: int, expand_target: int, q768, q256,
                      p: SgParams):
        al = np.ascontiguousarray(allow, np.uint64)
        rows = np.ascontiguousarray(rows, np.uint32)
        pcl = np.ascontiguousarray(per_cluster, np.uint32)
        k = max(p.k, 1)
        s, o = np.zeros(k, np.float32), np.zeros(k, np.uint32)
        m = self.L.or_filter_search(ctypes.byref(self.st), P(al), c_uint64(al.size), P(rows),
                                    c_uint64(rows.size), P(pcl), c_int(plan), c_uint64(expand_target),
                                    P(f32(q768)), P(f32(q256)), ctypes.byref(p), P(s), P(o))
        return s[:m], o[:m]


__all__ = [name for name in dir() if not name.startswith("_")]


# ---- bigann (src/bigann.rs) --------------------------------------------------------------------
def bg_refine_encode(r, bits: int):
    """refine_encode (src/bigann.rs:65-108): (planes [(MAX_BITS-1)*16] u8, f)."""
    r = f32(r)
    planes = np.zeros(2 * 16, np.uint8)
    f = lib().or_bg_refine_encode(P(r), c_uint32(bits), P(planes))
    return planes, f


def bg_refiner(qr, bits: int):
    """Refiner::new (src/bigann.rs:575-585): (tables [16, 256] f32, off)."""
    qr = f32(qr)
    tab = np.zeros((16, 256), np.float32)
    off = c_float()
    lib().or_bg_refiner_new(P(qr), c_uint32(bits), P(tab), ctypes.byref(off))
    return tab, off.value


def bg_refiner_estimate(tab, off: float, bits: int, sign, planes, f: float) -> float:
    tab = f32(tab)
    sign, planes = np.ascontiguousarray(sign, np.uint8), np.ascontiguousarray(planes, np.uint8)
    return lib().or_bg_refiner_estimate(P(tab), off, bits, P(sign), P(planes), f)


class OracleBigann:
    """bigann::Index over in-memory arrays (the dict the GPU bigann index opens)."""

    def __init__(self, arrays: dict, native: bool = False):
        self.st, self._keep = make_bigann_arrays(arrays)
        self.k = int(arrays["k"])
        self.L = lib(native)

    @staticmethod
    def params(nprobe, cand, k, refine=0, margin=0.0) -> SgBigannParams:
        return SgBigannParams(int(nprobe), int(cand), int(k), int(refine), float(margin), 0)

    def route(self, q, p: SgBigannParams):
        q = np.ascontiguousarray(q, np.int8)
        probe = np.zeros(max(self.k, 1), np.uint32)
        sc = np.zeros(max(self.k, 1), np.float32)
        dots = np.zeros(max(self.k, 1), np.float32)
        m = self.L.or_bg_route(ctypes.byref(self.st), P(q), ctypes.byref(p), P(probe), P(sc), P(dots))
        return probe[:m], sc[:m], dots

    def candidates(self, q, p: SgBigannParams):
        q = np.ascontiguousarray(q, np.int8)
        probe, _, dots = self.route(q, p)
        c = max(p.cand, 1)
        ids, est, nx = np.zeros(c, np.uint32), np.zeros(c, np.float32), np.zeros(c, np.float32)
        scanned = c_uint64()
        m = self.L.or_bg_candidates(ctypes.byref(self.st), P(q), P(probe), c_uint32(probe.size), P(dots),
                                    ctypes.byref(p), P(ids), P(est), P(nx), ctypes.byref(scanned))
        return ids[:m], est[:m], nx[:m], scanned.value

    def search(self, q, p: SgBigannParams):
        q = np.ascontiguousarray(q, np.int8)
        k = max(p.k, 1)
        s, o = np.zeros(k, np.float32), np.zeros(k, np.uint32)
        t = SgBigannTiming()
        m = self.L.or_bg_search(ctypes.byref(self.st), P(q), ctypes.byref(p), P(s), P(o), ctypes.byref(t))
        return s[:m], o[:m], t

    def search_batch(self, q, p: SgBigannParams, threads: int = 0):
        q = np.ascontiguousarray(q, np.int8).reshape(-1, 100)
        nq, k = q.shape[0], max(p.k, 1)
        s, o, cnt = np.zeros((nq, k), np.float32), np.zeros((nq, k), np.uint32), np.zeros(nq, np.uint32)
        scanned = self.L.or_bg_search_batch(ctypes.byref(self.st), c_uint32(nq), P(q), ctypes.byref(p),
                                            c_int(threads or os.cpu_count() or 1), P(s), P(o), P(cnt))
        return s[:, : p.k], o[:, : p.k], cnt, scanned
