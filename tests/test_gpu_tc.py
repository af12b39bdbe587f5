"""The tcgen05 contraction of the batched scan (sg_lut_scan_batch) against the oracle's lut::scan.

The tensor-core scan computes every (query, slot) LUT score of a work item as one u8 x u8 -> s32
matrix product over the one-hot expansion of the codes; the scores must equal the reference's
scalar scan (src/lut.rs:116-126) bit for bit, for every query and slot, including the padded
query columns (N rounded up to 16), the ragged last tile of a block range and multi-item grids.
"""
import numpy as np
import pytest

import oracle as O
from sieve_gpu import lut_scan_batch

pytestmark = pytest.mark.gpu


def tables_for(r, nq):
    return np.stack([O.lut_new(r.uniform(-1, 1, 256).astype(np.float32))[0].reshape(-1) for _ in range(nq)])


@pytest.mark.parametrize("nq,nblocks", [(1, 1), (16, 4), (17, 5), (64, 37), (130, 70), (257, 129)])
def test_lut_scan_batch_matches_oracle(nq, nblocks):
    r = np.random.default_rng(nq * 1000 + nblocks)
    tables = tables_for(r, nq)
    blocks = r.integers(0, 256, (nblocks, 1024), dtype=np.uint8)
    got = lut_scan_batch(tables, blocks)
    assert got.shape == (nq, nblocks * 32)
    for i in range(nq):
        assert np.array_equal(got[i], O.scan(tables[i].reshape(64, 16), blocks)), f"query {i}"


def test_lut_scan_batch_extremes():
    r = np.random.default_rng(5)
    full = np.full((3, 1024), 255, np.uint8)
    blocks = r.integers(0, 256, (9, 1024), dtype=np.uint8)
    assert np.all(lut_scan_batch(full, blocks) == 64 * 255)
    tables = tables_for(r, 20)
    tables[:, ::16] = 0  # entry 0 of every group zero: all-zero codes score 0
    assert np.all(lut_scan_batch(tables, np.zeros((2, 1024), np.uint8)) == 0)
    ones = np.full((2, 1024), 0xFF, np.uint8)  # nibble 15 in every group of every slot
    want = tables.reshape(20, 64, 16)[:, :, 15].astype(np.int64).sum(1)
    assert np.array_equal(lut_scan_batch(tables, ones), np.repeat(want[:, None], 64, 1))


def test_lut_scan_batch_repeatable():
    r = np.random.default_rng(9)
    tables = tables_for(r, 40)
    blocks = r.integers(0, 256, (100, 1024), dtype=np.uint8)
    a = lut_scan_batch(tables, blocks)
    b = lut_scan_batch(tables, blocks)
    assert np.array_equal(a, b)
