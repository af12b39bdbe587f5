"""sieve_gpu — the sieve IVF query path (RaBitQ 1-bit LUT scan, 2-bit tier, int8 rerank) on one
B200, behind the C ABI of include/sieve_gpu.h. `Index`, `Context` (Scratch), `Params`, `Rerank`, `Timing`
mirror the reference's ivf module; `filter` mirrors filter::Filter / Plan / search; `Server` is the serving
loop (continuous batching); `bigann` is the billion-scale L2 path; `builder` and `bigann_builder`
write the reference's index files; `synth` makes the seeded synthetic corpora the workloads run on.
"""
from .index import (Context, Index, Params, Rerank, Timing, allow_bitset, dot_i8i8, lut_scan,
                    lut_scan_batch, parse_config)
from ._abi import SieveError
from . import filter
from .server import Server

__all__ = ["Index", "Context", "Params", "Rerank", "Timing", "parse_config", "allow_bitset", "lut_scan", "lut_scan_batch",
           "dot_i8i8", "SieveError", "filter", "Server"]
