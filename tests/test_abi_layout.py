"""The ctypes mirrors of the C ABI's structs against the header itself: a small C program built
with gcc from include/sieve_gpu.h prints every struct's size and every field's offset, and the
Python side must agree field for field (a drift here would pass garbage across the boundary)."""
import os
import shutil
import subprocess

import pytest

from sieve_gpu import _abi
from sieve_gpu import server

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = {
    "sg_params": _abi.SgParams,
    "sg_timing": _abi.SgTiming,
    "sg_stats": _abi.SgStats,
    "sg_tuning": _abi.SgTuning,
    "sg_ivf_arrays": _abi.SgIvfArrays,
    "sg_bigann_params": _abi.SgBigannParams,
    "sg_bigann_timing": _abi.SgBigannTiming,
    "sg_bigann_arrays": _abi.SgBigannArrays,
    "sg_server_config": server.SgServerConfig,
    "sg_request_info": server.SgRequestInfo,
    "sg_server_stats": server.SgServerStats,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sieve_gpu.h"', "int main(void) {"]
    for cname, py in PAIRS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            c, f, v = ln.split()
            got[(c, f)] = int(v)
    for cname, py in PAIRS.items():
        assert got[(cname, "size")] == ctypes_sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def ctypes_sizeof(t):
    import ctypes

    return ctypes.sizeof(t)
