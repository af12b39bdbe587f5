"""CPU checks of the error bounds behind the tensor-core routing windows, restated in numpy: the
BF16 GEMM score of a centroid (or a bigann leaf) lies within delta of the reference's sequential
FP32 score for every accumulation order tried (sequential, reversed, pairwise, and in 16-element
K steps as the MMA chain takes them). A window of 2 delta below the nprobe-th approximate score
therefore holds every exact top-nprobe centroid, which is what the exact rescoring relies on
(csrc/route.cu k_route_select; csrc/bg_route.cu items 1-2 of its header).
"""
import numpy as np
import pytest

f32 = np.float32


def bf16(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to bfloat16, returned as float32 (finite inputs)."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def seq_sum(terms: np.ndarray) -> np.ndarray:
    """Sequential f32 sum from -0.0 over the last axis (the reference's loop order)."""
    s = np.full(terms.shape[:-1], -0.0, np.float32)
    for k in range(terms.shape[-1]):
        s = (s + terms[..., k]).astype(np.float32)
    return s


def pair_sum(terms: np.ndarray) -> np.ndarray:
    t = terms.astype(np.float32)
    while t.shape[-1] > 1:
        if t.shape[-1] % 2:
            t = np.concatenate([t, np.zeros(t.shape[:-1] + (1,), np.float32)], -1)
        t = (t[..., 0::2] + t[..., 1::2]).astype(np.float32)
    return t[..., 0]


def step_sum(terms: np.ndarray, step: int = 16) -> np.ndarray:
    """Each K step of `step` products summed, then the steps accumulated in order."""
    k = terms.shape[-1]
    pad = (-k) % step
    t = np.concatenate([terms, np.zeros(terms.shape[:-1] + (pad,), np.float32)], -1).astype(np.float32)
    parts = pair_sum(t.reshape(t.shape[:-1] + (-1, step)))
    return seq_sum(parts)


ORDERS = {
    "sequential": seq_sum,
    "reversed": lambda t: seq_sum(t[..., ::-1]),
    "pairwise": pair_sum,
    "k-steps": step_sum,
}


def ref_dot(q: np.ndarray, c: np.ndarray) -> np.ndarray:
    """The reference's f32 dot: products rounded, summed sequentially from -0.0."""
    return seq_sum((q * c).astype(np.float32))


@pytest.mark.parametrize("positive", [False, True])
def test_ivf_bf16_score_within_window_delta(positive):
    rng = np.random.default_rng(3 if positive else 4)
    n, d = 4000, 256
    q = rng.standard_normal((n, d)).astype(np.float32)
    c = rng.standard_normal((n, d)).astype(np.float32)
    if positive:  # every term of one sign: the accumulation errors cannot cancel
        q, c = np.abs(q), np.abs(c)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    c *= rng.uniform(0.5, 1.5, (n, 1)).astype(np.float32) / np.linalg.norm(c, axis=1, keepdims=True)
    cmax = float(np.linalg.norm(c, axis=1).max())
    qn = np.linalg.norm(q.astype(np.float64), axis=1)
    delta = 0.0085 * qn * cmax
    s = ref_dot(q, c).astype(np.float64)
    prod = (bf16(q) * bf16(c)).astype(np.float32)  # exact: 8-bit by 8-bit significands
    for name, acc in ORDERS.items():
        err = np.abs(acc(prod).astype(np.float64) - s)
        assert np.all(err <= delta), (name, float((err / delta).max()))


@pytest.mark.parametrize("spread", [40.0, 120.0])
def test_bigann_hi_lo_score_within_delta(spread):
    rng = np.random.default_rng(int(spread))
    n, d, kcols = 3000, 100, 208
    q = rng.integers(-127, 128, (n, d)).astype(np.float32)
    c = (rng.standard_normal((n, d)) * spread).astype(np.float32)
    cn2 = seq_sum((c * c).astype(np.float32))  # the leaf's squared norm, f32
    cmax = float(np.sqrt((c.astype(np.float64) ** 2).sum(1)).max())
    qn = np.sqrt((q.astype(np.float64) ** 2).sum(1))
    delta = 5e-4 * qn * cmax + 2.0 ** -22 * cmax * cmax
    # the reference: s = 2 <q, c> - |c|^2 in f32
    s = (f32(2) * ref_dot(q, c) - cn2).astype(np.float32).astype(np.float64)
    hi = bf16(c)
    lo = bf16((c - hi).astype(np.float32))  # c - hi is exact in f32
    terms = np.zeros((n, kcols), np.float32)  # [q, 0 x 4, q, 0 x 4] against [hi, 0 x 4, lo, 0 x 4]
    terms[:, :d] = q * hi
    terms[:, 104:104 + d] = q * lo
    for name, acc in ORDERS.items():
        st = (f32(2) * acc(terms) - cn2).astype(np.float32).astype(np.float64)
        err = np.abs(st - s)
        assert np.all(err <= delta), (name, float((err / delta).max()))
