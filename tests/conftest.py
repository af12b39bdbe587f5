"""Test setup: import paths for the product package and the oracle, and the `gpu` marker.

`-m "not gpu"` runs here without a GPU (oracle pins, host logic, ABI exports);
`-m gpu` runs the parity tests through the C ABI on a B200.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "a-game-of-vectors_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
