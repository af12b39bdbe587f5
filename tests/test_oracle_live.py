"""The oracle's restatement of the live layer (src/live.rs) on the CPU: the insert encoding of
Live::apply_insert and the search over base lists, delta lists and tombstones."""
import numpy as np

from fixtures import index_a
from live_oracle import OracleLive
from sieve_gpu import Params, Rerank

P = Params(16, 500, Rerank.full(), 10)


def test_insert_encodes_the_int8_row_as_ingest_does():
    """A corpus vector inserted again quantises to its corpus row (Int8Quantizer::encode)."""
    arrays, _, _, mix = index_a()
    L = OracleLive(arrays)
    v = mix.rows(123, 3).numpy()
    L.insert([900001, 900002, 900003], v)
    for j in range(3):
        assert np.array_equal(L.rows[j], arrays["rerank"][123 + j])
    # every row takes a primary and a SOAR secondary slot
    assert sum(len(x) for x in L.lists) == 6


def test_inserted_copy_ranks_with_its_original():
    arrays, _, _, mix = index_a()
    L = OracleLive(arrays)
    v = mix.rows(777, 1).numpy()
    L.insert([424242], v)
    q256 = v[:, :256] / np.linalg.norm(v[:, :256], axis=1, keepdims=True)
    sc, ids, cnt = L.search_batch(v, q256.astype(np.float32), P)
    top = set(ids[0, :2].tolist())
    assert top == {777, 424242} and sc[0, 0] == sc[0, 1]


def test_delete_and_upsert_hide_the_old_rows():
    arrays, _, _, mix = index_a()
    L = OracleLive(arrays)
    v = mix.rows(50, 2).numpy()
    q256 = (v[:, :256] / np.linalg.norm(v[:, :256], axis=1, keepdims=True)).astype(np.float32)
    L.delete([50])
    _, ids, cnt = L.search_batch(v, q256, P)
    assert 50 not in ids[0, : cnt[0]]
    L.insert([51], v[:1])  # upsert corpus row 51 with row 50's vector
    _, ids, cnt = L.search_batch(v, q256, P)
    assert ids[0, 0] == 51 and 51 not in ids[1, : cnt[1]]
    L.insert([51], v[1:])  # and back: the delta row replaced before is tombstoned
    _, ids, cnt = L.search_batch(v, q256, P)
    assert ids[1, 0] == 51 and list(ids[0, : cnt[0]]).count(51) == 0
