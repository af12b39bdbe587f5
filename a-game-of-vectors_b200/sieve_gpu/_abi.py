"""ctypes view of include/sieve_gpu.h and the loader of the CUDA library.

The library is built in-tree (``build_ext.py``) into ``sieve_gpu/_lib/libsieve_gpu.so``. There is
no CPU fallback: if the library is missing, or no CUDA device is visible, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsieve_gpu.so")

SG_OK = 0
STATUS_NAMES = {
    -1: "SG_ERR_INVALID",
    -2: "SG_ERR_IO",
    -3: "SG_ERR_OOM",
    -4: "SG_ERR_DEVICE",
    -5: "SG_ERR_TIMEOUT",
    -6: "SG_ERR_ADMISSION",
    -7: "SG_ERR_UNSUPPORTED",
}

DIM, PDIM, CODE_BYTES, GROUPS, BLOCK, BLOCK_BYTES, TIER2_BYTES = 768, 256, 32, 64, 32, 1024, 64
PAD = 0xFFFFFFFF

RERANK_NONE, RERANK_PREFIX, RERANK_FULL, RERANK_TIERED, RERANK_SSD = 0, 1, 2, 3, 4
ROUTE_FP32, ROUTE_BF16 = 0, 1


class SgParams(ctypes.Structure):
    """sg_params: ivf::Params (src/ivf.rs:441-460)."""

    _fields_ = [
        ("nprobe", c_uint32),
        ("cand", c_uint32),
        ("rerank_kind", c_uint32),
        ("rerank_r", c_uint32),
        ("k", c_uint32),
        ("has_prune", c_uint32),
        ("prune_m", c_uint32),
        ("prune_w", c_float),
        ("has_margin", c_uint32),
        ("margin", c_float),
        ("has_budget", c_uint32),
        ("reserved", c_uint32),
        ("budget", c_uint64),
    ]


class SgTiming(ctypes.Structure):
    """sg_timing: ivf::Timing (src/ivf.rs:521-538)."""

    _fields_ = [
        (name, c_uint64)
        for name in ("route", "scan", "rerank", "tier2", "scanned", "reranked", "probed", "fetch", "wait")
    ]


class SgStats(ctypes.Structure):
    """sg_stats: device stage times and counters of the last search."""

    _fields_ = [(n, c_float) for n in ("ms_prep", "ms_route_gemm", "ms_route_select", "ms_scan",
                                        "ms_cut", "ms_rerank", "ms_tier2", "ms_total")] + [
        ("launches", c_uint32), ("reserved", c_uint32), ("scanned", c_uint64), ("probed", c_uint64),
        ("reranked", c_uint64), ("buffered", c_uint64), ("ms_seed", c_float), ("retried", c_uint32)]


class SgTuning(ctypes.Structure):
    """sg_tuning: the autotuned shapes of the batched path."""

    _fields_ = [("tc_min_queries", c_uint32), ("chunk_blocks", c_uint32), ("scan_ctas_per_sm", c_uint32),
                ("seed_blocks", c_uint32), ("tc_split", c_uint32)]


class SgIvfArrays(ctypes.Structure):
    """sg_ivf_arrays: the contents of the reference's corpus and index files."""

    _fields_ = [
        ("n", c_uint64),
        ("k", c_uint32),
        ("centroids", c_void_p),
        ("block_off", c_void_p),
        ("ids", c_void_p),
        ("blocks", c_void_p),
        ("factors", c_void_p),
        ("rotation", c_void_p),
        ("tier2_sigma", c_void_p),
        ("tier2_codes", c_void_p),
        ("tier2_norm", c_void_p),
        ("rerank", c_void_p),
        ("norm256", c_void_p),
        ("quant_scale", c_void_p),
        ("codes", c_void_p),
    ]


# name -> (dtype, per-row shape) of every array an IVF index holds, in sg_ivf_arrays order.
ARRAY_FIELDS = {
    "centroids": np.float32,
    "block_off": np.uint64,
    "ids": np.uint32,
    "blocks": np.uint8,
    "factors": np.float32,
    "rotation": np.float32,
    "tier2_sigma": np.float32,
    "tier2_codes": np.uint8,
    "tier2_norm": np.float32,
    "rerank": np.int8,
    "norm256": np.float32,
    "quant_scale": np.float32,
    "codes": np.uint8,
}


def ptr(a: np.ndarray | None) -> c_void_p | None:
    """Address of a C-contiguous numpy array (None for a missing optional array)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return c_void_p(a.ctypes.data)


def make_arrays(arrays: dict, codes: bool = False) -> tuple[SgIvfArrays, list]:
    """Fills an SgIvfArrays from a dict of numpy arrays; returns it with the arrays it points
    into (the caller keeps them alive while the struct is used). The rows' global sign codes
    (codes.bin) are passed only with codes=True: only the flat Hamming baseline reads them."""
    keep = []
    st = SgIvfArrays()
    st.n = int(arrays["n"])
    st.k = int(arrays["k"])
    for name, dt in ARRAY_FIELDS.items():
        a = arrays.get(name) if (name != "codes" or codes) else None
        if a is not None:
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
        setattr(st, name, ptr(a))
    return st, keep


# ---- bigann (src/bigann.rs) ----------------------------------------------------------------
BG_DIM, BG_PDIM, BG_GROUPS, BG_CODE, BG_BLOCK_BYTES, BG_MAX_BITS = 100, 128, 32, 16, 512, 3


class SgBigannParams(ctypes.Structure):
    """sg_bigann_params: bigann::Params."""

    _fields_ = [("nprobe", c_uint32), ("cand", c_uint32), ("k", c_uint32), ("refine", c_uint32),
                ("margin", c_float), ("route_fp32", c_uint32)]


class SgBigannTiming(ctypes.Structure):
    """sg_bigann_timing: bigann::Timing, in nanoseconds."""

    _fields_ = [(n, c_uint64) for n in ("route", "scan", "io_wait", "rerank", "scanned", "probes")]


class SgBigannArrays(ctypes.Structure):
    """sg_bigann_arrays: a bigann index's records (de-interleaved) and its base rows."""

    _fields_ = [
        ("n", c_uint64),
        ("k", c_uint32),
        ("bits", c_uint32),
        ("leaves", c_void_p),
        ("block_off", c_void_p),
        ("ids", c_void_p),
        ("blocks", c_void_p),
        ("factors", c_void_p),
        ("ext", c_void_p),
        ("rotation", c_void_p),
        ("base", c_void_p),
    ]


BIGANN_FIELDS = {
    "leaves": np.float32,
    "block_off": np.uint64,
    "ids": np.uint32,
    "blocks": np.uint8,
    "factors": np.float32,
    "ext": np.uint8,
    "rotation": np.float32,
    "base": np.int8,
}


def bg_extra(bits: int) -> int:
    """bigann::refine_bytes (src/bigann.rs:110-113): planes of the low bits - 1 bits, then f."""
    return (bits - 1) * BG_CODE + 4 if bits > 1 else 0


def make_bigann_arrays(arrays: dict) -> tuple[SgBigannArrays, list]:
    keep = []
    st = SgBigannArrays()
    st.n = int(arrays["n"])
    st.k = int(arrays["k"])
    st.bits = int(arrays["bits"])
    for name, dt in BIGANN_FIELDS.items():
        a = arrays.get(name)
        if a is not None and a.size:
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
        else:
            a = None
        setattr(st, name, ptr(a))
    return st, keep


class SieveError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libsieve_gpu.so (no fallback: a missing library is an error)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SieveError(-4, f"CUDA library not built: {LIB_PATH} (run build_ext.py)")
    L = ctypes.CDLL(LIB_PATH)
    for name in EXPORTS:
        getattr(L, name).restype = c_int
    L.sg_last_error.restype = c_char_p
    L.sg_version.restype = c_char_p
    _lib = L
    return L


# Every symbol include/sieve_gpu.h declares; the CPU suite checks the library exports them.
EXPORTS = [
    "sg_last_error",
    "sg_version",
    "sg_open_ivf",
    "sg_open_ivf_arrays",
    "sg_close",
    "sg_index_info",
    "sg_set_route_precision",
    "sg_set_timing",
    "sg_last_stats",
    "sg_search",
    "sg_search_device",
    "sg_context_open",
    "sg_context_close",
    "sg_search_ctx",
    "sg_search_device_ctx",
    "sg_context_last_stats",
    "sg_search_noalloc",
    "sg_flat_hamming",
    "sg_route",
    "sg_route_scores",
    "sg_candidates",
    "sg_candidates_probes",
    "sg_rerank",
    "sg_live_open",
    "sg_live_close",
    "sg_live_insert",
    "sg_live_delete",
    "sg_live_search",
    "sg_live_info",
    "sg_filter_new",
    "sg_filter_info",
    "sg_filter_free",
    "sg_plan_resolve",
    "sg_filter_search",
    "sg_server_start",
    "sg_server_submit",
    "sg_server_poll",
    "sg_server_get_stats",
    "sg_server_replay",
    "sg_server_stop",
    "sg_open_bigann",
    "sg_open_bigann_arrays",
    "sg_close_bigann",
    "sg_bigann_info",
    "sg_bigann_route_fallbacks",
    "sg_search_bigann",
    "sg_search_bigann_device",
    "sg_bigann_route",
    "sg_bigann_candidates",
    "sg_query_prep",
    "sg_get_tuning",
    "sg_set_tuning",
    "sg_autotune",
    "sg_lut_scan",
    "sg_lut_scan_batch",
    "sg_dot_i8i8",
]


def check(status: int) -> None:
    if status != SG_OK:
        msg = lib().sg_last_error()
        raise SieveError(status, msg.decode() if msg else "")


__all__ = [
    "SgParams",
    "SgTiming",
    "SgTuning",
    "SgIvfArrays",
    "make_arrays",
    "ptr",
    "lib",
    "check",
    "SieveError",
    "EXPORTS",
    "POINTER",
    "c_uint32",
    "c_uint64",
    "c_void_p",
    "c_float",
    "c_int",
]
