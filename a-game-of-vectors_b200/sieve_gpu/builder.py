"""Offline ingest and IVF build, writing the reference's arrays (torch on CPU or GPU).

This is the input side of the query path, not the path itself: it produces the arrays that
`Index` uploads to HBM, in exactly the layouts of the reference's files
(`ingest`: src/bin/ingest.rs:117-140; `ivf::build`: src/ivf.rs:268-395):

  corpus  rerank.i8 [n,768] int8, norm256.f32 [n], codes.bin [n,32] (global sign codes),
          quant.f32 [768]
  index   centroids.f32 [k,256], block_off.u64 [k+1], ids.u32 [nblocks*32] (PAD-filled),
          blocks.bin [nblocks*1024] (nibble-transposed), factors.f32 [nblocks*32, 2] = [mul, err],
          rotation.f32 [3*256], tier2.sigma [256], tier2.bin [n,64], tier2.norm [n]

The steps follow the reference: sample 42 / k-means seed 7 / rotation seed 11 (splitmix64),
spherical k-means with the optional split step, SOAR secondary assignment among the 16 nearest
centroids, RaBitQ residual codes per slot, cluster-major packing in row order. Float sums here
use torch's reduction order, so centroids and factors match the reference to rounding, not
bit for bit; the query path's parity is checked on whatever arrays this produces.
"""
from __future__ import annotations

import os

import numpy as np
import torch

PDIM, DIM, BLOCK, GROUPS = 256, 768, 32, 64
PAD = 0xFFFFFFFF
SOAR_CAND = 16
GOLDEN = np.uint64(0x9E3779B97F4A7C15)


# ---- splitmix64 (src/ivf.rs:119-135), vectorised over the stream index ------------------------
def splitmix_stream(seed: int, count: int, start: int = 0) -> np.ndarray:
    """Outputs start..start+count of Rng::new(seed).next()."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


class Rng:
    """Sequential splitmix64 with a position counter (draws in the reference's order)."""

    def __init__(self, seed: int):
        self.seed, self.pos = seed, 0

    def below_many(self, n: int, count: int) -> np.ndarray:
        v = splitmix_stream(self.seed, count, self.pos) % np.uint64(n)
        self.pos += count
        return v.astype(np.int64)

    def below(self, n: int) -> int:
        return int(self.below_many(n, 1)[0])


def rotation_signs(seed: int, d: int = PDIM) -> np.ndarray:
    """Rotation::with_dim (src/rabitq.rs:40-44)."""
    bits = splitmix_stream(seed, 3 * d) & np.uint64(1)
    return np.where(bits == 1, 1.0, -1.0).astype(np.float32)


def fwht(v: torch.Tensor) -> torch.Tensor:
    """Unnormalised FWHT along the last dim, the same butterflies as src/rabitq.rs:73-84."""
    n = v.shape[-1]
    h = 1
    while h < n:
        x = v.reshape(*v.shape[:-1], n // (2 * h), 2, h)
        a, b = x[..., 0, :], x[..., 1, :]
        v = torch.stack((a + b, a - b), dim=-2).reshape(*v.shape[:-1], n)
        h *= 2
    return v


def rotate(signs: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """Rotation::apply (src/rabitq.rs:60-69) on every row of v."""
    d = v.shape[-1]
    for r in range(3):
        v = fwht(v * signs[r * d:(r + 1) * d])
    norm = np.float32(np.power(np.float32(d), np.float32(-1.5)))
    return v * float(norm)


def round_away(v: torch.Tensor) -> torch.Tensor:
    """f32::round (half away from zero); torch.round is half-to-even."""
    r = torch.round(v)
    t = torch.trunc(v)
    half = (v - t).abs() == 0.5
    return torch.where(half, t + torch.sign(v), r)


def pack_bits(b: torch.Tensor) -> torch.Tensor:
    """[.., 8m] bools -> [.., m] uint8, bit i of byte i/8 at position i%8."""
    w = (1 << torch.arange(8, device=b.device, dtype=torch.int32))
    return (b.reshape(*b.shape[:-1], -1, 8).to(torch.int32) * w).sum(-1).to(torch.uint8)


def normalise_rows(x: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    n = x.norm(dim=1)
    inv = torch.where(n > 0, 1.0 / n, torch.ones_like(n))
    return x * inv[:, None], n


# ---- ingest (src/bin/ingest.rs:117-140) ---------------------------------------------------------
def ingest(mix, batch: int = 65536, device: str | None = None) -> dict:
    """Encodes a Mixture into the corpus arrays (host numpy)."""
    dev = torch.device(device or mix.device)
    n = mix.n
    rerank = np.empty((n, DIM), np.int8)
    norm256 = np.empty(n, np.float32)
    codes = np.empty((n, PDIM // 8), np.uint8)
    scale = None
    for s in range(0, n, batch):
        x = mix.rows(s, min(batch, n - s)).to(dev)
        p, nrm = normalise_rows(x[:, :PDIM])
        if scale is None:  # Int8Quantizer::fit on the first batch (src/quant.rs:42-50)
            m = torch.clamp(x.abs().amax(0), min=1e-6)
            scale = 127.0 / m
        q = torch.clamp(round_away(x * scale), -127, 127).to(torch.int8)
        e = s + x.shape[0]
        rerank[s:e] = q.cpu().numpy()
        norm256[s:e] = nrm.cpu().numpy()
        codes[s:e] = pack_bits(p > 0).cpu().numpy()
    return {"n": n, "rerank": rerank, "norm256": norm256, "codes": codes,
            "quant_scale": scale.float().cpu().numpy()}


def prefix_f32(rerank_rows: torch.Tensor, scale256: torch.Tensor) -> torch.Tensor:
    """Corpus::prefix_f32 (src/ivf.rs:110-116): int8 prefix / scale, renormalised."""
    return normalise_rows(rerank_rows[:, :PDIM].float() / scale256)[0]


# ---- k-means (src/ivf.rs:188-254) --------------------------------------------------------------
def kmeans(sample: torch.Tensor, k: int, iters: int, seed: int, balance: float | None) -> torch.Tensor:
    n = sample.shape[0]
    rng = Rng(seed)
    cents = sample[torch.as_tensor(rng.below_many(n, k), device=sample.device)].clone()
    for it in range(iters):
        a = torch.argmax(sample @ cents.T, dim=1)
        counts = torch.bincount(a, minlength=k)
        sums = torch.zeros_like(cents).index_add_(0, a, sample)
        cnt = counts.cpu().numpy()
        for c in np.nonzero(cnt == 0)[0]:
            cents[c] = sample[rng.below(n)]
        nz = torch.as_tensor(np.nonzero(cnt)[0], device=sample.device)
        cents[nz] = normalise_rows(sums[nz])[0]
        if balance is not None and it + 2 < iters:
            split_large(sample, a, cnt, cents, balance, rng)
    return cents


def split_large(sample, a, counts: np.ndarray, cents, r: float, rng: Rng) -> int:
    """src/ivf.rs:227-254: move the smallest centroids onto members of oversized clusters."""
    k = counts.size
    mean = a.shape[0] / k
    order = np.argsort(-counts, kind="stable")
    large = [c for c in order if counts[c] > r * mean]
    large = large[: len(large)]
    small = []
    for c in order[::-1]:
        if len(small) >= len(large) or not counts[c] < 0.5 * mean:
            break
        small.append(c)
    if not small:
        return 0
    a_np = a.cpu().numpy()
    for big, tiny in zip(large, small):
        members = np.nonzero(a_np == big)[0]
        pick = members[rng.below(members.size)]
        cents[tiny] = sample[int(pick)]
    return len(small)


# ---- Tier2 (src/tier2.rs:18-40) ----------------------------------------------------------------
LEVELS = torch.tensor([-1.510, -0.4528, 0.4528, 1.510], dtype=torch.float32)
T2_T = 0.9816


def tier2_fit(sample: torch.Tensor) -> torch.Tensor:
    n = max(sample.shape[0], 1)
    ss = (sample * sample).double().sum(0)
    return torch.clamp(torch.sqrt(ss / n).float(), min=1e-6)


def tier2_encode(sigma: torch.Tensor, p: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    t = T2_T * sigma
    lv = torch.where(p < -t, 0, torch.where(p < 0, 1, torch.where(p < t, 2, 3)))
    v = LEVELS.to(p.device)[lv] * sigma
    nrm = torch.sqrt((v * v).sum(1))
    sh = (2 * torch.arange(4, device=p.device)).repeat(PDIM // 4)
    code = (lv << sh).reshape(-1, PDIM // 4, 4).sum(-1).to(torch.uint8)
    return code, nrm


# ---- RaBitQ encode (src/rabitq.rs:88-108), batched ---------------------------------------------
def rabitq_encode(xr: torch.Tensor, cr: torch.Tensor):
    r = xr - cr
    d = float(xr.shape[1])
    nr2 = (r * r).sum(1)
    l1 = r.abs().sum(1)
    code = pack_bits(r > 0)
    nr = torch.sqrt(nr2)
    od = l1 / (nr * np.sqrt(d))
    inner = (1.0 - od * od) / (od * od * (d - 1.0))
    err = nr * 1.9 * torch.sqrt(torch.clamp(inner, min=0.0))
    mul = nr2 / l1
    zero = l1 < 1e-12
    mul = torch.where(zero, torch.zeros_like(mul), mul)
    err = torch.where(zero, torch.zeros_like(err), err)
    return code, mul, err


# ---- build (src/ivf.rs:268-395) ------------------------------------------------------------------
def build_ivf(corpus: dict, k: int, sample_n: int = 262144, iters: int = 10,
              balance: float | None = None, soar_lambda: float | None = 1.0,
              device: str = "cpu", chunk: int = 131072, rabitq: bool = True) -> dict:
    """Trains and packs an IVF index over corpus arrays; returns host numpy arrays. With
    rabitq=False every slot holds its row's global sign code (codes.bin) and the index has no
    rotation.f32 / factors.f32, as ivf::build(.., rabitq: false) writes (src/ivf.rs:366-372)."""
    dev = torch.device(device)
    n = int(corpus["n"])
    rer = corpus["rerank"]
    scale256 = torch.as_tensor(corpus["quant_scale"][:PDIM], device=dev)
    rng = Rng(42)
    sample_n = min(sample_n, n)
    idx = rng.below_many(n, sample_n)
    sample = prefix_f32(torch.as_tensor(rer[idx], device=dev), scale256)
    cents = kmeans(sample, k, iters, 7, balance)
    sigma = tier2_fit(sample)
    del sample
    signs = torch.as_tensor(rotation_signs(11), device=dev)
    cents_rot = rotate(signs, cents)
    gram = cents @ cents.T if soar_lambda is not None else None

    t2_codes = np.empty((n, PDIM // 4), np.uint8)
    t2_norm = np.empty(n, np.float32)
    slot_cluster, slot_row, slot_code, slot_mul, slot_err = [], [], [], [], []
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        x = prefix_f32(torch.as_tensor(rer[s:e], device=dev), scale256)
        c2, nn = tier2_encode(sigma, x)
        t2_codes[s:e] = c2.cpu().numpy()
        t2_norm[s:e] = nn.cpu().numpy()
        scores = x @ cents.T
        rows = torch.arange(s, e, device=dev, dtype=torch.int64)
        if soar_lambda is None:
            prim = torch.argmax(scores, dim=1)
            pairs = [(prim, rows)]
        else:
            top_v, top_i = torch.topk(scores, min(SOAR_CAND, k), dim=1)
            prim = top_i[:, 0]
            if k > 1:
                x_c1 = top_v[:, 0]
                r2 = torch.clamp(2.0 - 2.0 * x_c1, min=1e-12)
                r_x = 1.0 - x_c1
                x_c = top_v[:, 1:]
                r_c = x_c - gram[prim[:, None], top_i[:, 1:]]
                along = r_x[:, None] - r_c
                loss = (2.0 - 2.0 * x_c) + soar_lambda * along * along / r2[:, None]
                sec = top_i[:, 1:].gather(1, torch.argmin(loss, dim=1, keepdim=True))[:, 0]
                pairs = [(prim, rows), (sec, rows)]
            else:
                pairs = [(prim, rows)]
        xr = rotate(signs, x) if rabitq else None
        gcode = None if rabitq else torch.as_tensor(corpus["codes"][s:e], device=dev)
        for c, r in pairs:
            if rabitq:
                code, mul, err = rabitq_encode(xr, cents_rot[c])
            else:
                code = gcode
                mul = err = torch.zeros(e - s, device=dev)
            slot_cluster.append(c)
            slot_row.append(r)
            slot_code.append(code)
            slot_mul.append(mul)
            slot_err.append(err)
        del scores
    cl = torch.cat(slot_cluster)
    rw = torch.cat(slot_row)
    key = cl * (n + 1) + rw
    order = torch.argsort(key)
    cl, rw = cl[order], rw[order]
    code = torch.cat(slot_code)[order]
    mul = torch.cat(slot_mul)[order]
    err = torch.cat(slot_err)[order]
    del slot_code, slot_mul, slot_err

    sizes = torch.bincount(cl, minlength=k)
    nb = (sizes + BLOCK - 1) // BLOCK
    block_off = torch.zeros(k + 1, dtype=torch.int64, device=dev)
    block_off[1:] = torch.cumsum(nb, 0)
    slot_start = torch.zeros(k + 1, dtype=torch.int64, device=dev)
    slot_start[1:] = torch.cumsum(sizes, 0)
    rank = torch.arange(cl.shape[0], device=dev) - slot_start[cl]
    pos = block_off[cl] * BLOCK + rank
    nblocks = int(block_off[-1])
    codes_p = torch.zeros(nblocks * BLOCK, PDIM // 8, dtype=torch.uint8, device=dev)
    codes_p[pos] = code
    ids = torch.full((nblocks * BLOCK,), PAD, dtype=torch.int64, device=dev)
    ids[pos] = rw
    factors = torch.zeros(nblocks * BLOCK, 2, dtype=torch.float32, device=dev)
    factors[pos, 0] = mul
    factors[pos, 1] = err
    blocks = pack_blocks(codes_p.reshape(nblocks, BLOCK, PDIM // 8))
    return {
        "n": n, "k": k,
        "centroids": cents.float().cpu().numpy(),
        "block_off": block_off.cpu().numpy().astype(np.uint64),
        "ids": ids.cpu().numpy().astype(np.uint32),
        "blocks": blocks.cpu().numpy().reshape(-1),
        "factors": factors.cpu().numpy().reshape(-1) if rabitq else None,
        "rotation": signs.cpu().numpy() if rabitq else None,
        "tier2_sigma": sigma.cpu().numpy(),
        "tier2_codes": t2_codes,
        "tier2_norm": t2_norm,
        "sizes": sizes.cpu().numpy(),
    }


def pack_blocks(codes: torch.Tensor) -> torch.Tensor:
    """pack_block (src/lut.rs:72-82) for [nb, 32, CB] raw codes -> [nb, G*16] bytes."""
    nb, _, cb = codes.shape
    g = cb * 2
    lo = codes & 0x0F
    hi = codes >> 4
    nib = torch.stack((lo, hi), dim=-1).reshape(nb, BLOCK, g)  # nibble g of slot k
    out = nib[:, :16, :] | (nib[:, 16:, :] << 4)  # [nb, k(16), g]
    return out.transpose(1, 2).contiguous().reshape(nb, g * 16)


# ---- exact ground truth (src/bin/ingest.rs:42-77) -----------------------------------------------
def ground_truth(mix, queries: torch.Tensor, k: int = 100, chunk: int = 262144) -> np.ndarray:
    """Exact top-k row ids by FP32 inner product over the unit-length 768-d rows."""
    q = queries.float()
    best_v = torch.full((q.shape[0], k), -float("inf"), device=q.device)
    best_i = torch.zeros((q.shape[0], k), dtype=torch.int64, device=q.device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, mix.n, chunk):
            x = mix.rows(s, min(chunk, mix.n - s)).to(q.device)
            sc = q @ x.T
            v, i = torch.topk(sc, min(k, sc.shape[1]), dim=1)
            allv = torch.cat((best_v, v), 1)
            alli = torch.cat((best_i, i + s), 1)
            tv, ti = torch.topk(allv, k, dim=1)
            best_v, best_i = tv, alli.gather(1, ti)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return best_i.cpu().numpy().astype(np.uint32)


# ---- the reference's file formats (src/store.rs:31-44: raw little-endian arrays) ---------------
CORPUS_FILES = {"rerank": "rerank.i8", "norm256": "norm256.f32", "codes": "codes.bin",
                "quant_scale": "quant.f32"}
INDEX_FILES = {"centroids": "centroids.f32", "block_off": "block_off.u64", "ids": "ids.u32",
               "blocks": "blocks.bin", "factors": "factors.f32", "rotation": "rotation.f32",
               "tier2_sigma": "tier2.sigma", "tier2_codes": "tier2.bin", "tier2_norm": "tier2.norm"}


def write_files(corpus: dict, index: dict, ingest_dir: str, index_dir: str) -> None:
    os.makedirs(ingest_dir, exist_ok=True)
    os.makedirs(index_dir, exist_ok=True)
    for key, name in CORPUS_FILES.items():
        np.ascontiguousarray(corpus[key]).tofile(os.path.join(ingest_dir, name))
    n = int(corpus["n"])
    # docids.{bin,off}: Corpus::open maps them; synthetic rows are named by their number.
    names = [f"doc{i}".encode() for i in range(n)]
    off = np.zeros(n + 1, np.uint64)
    off[1:] = np.cumsum([len(x) for x in names])
    with open(os.path.join(ingest_dir, "docids.bin"), "wb") as f:
        f.write(b"".join(names))
    off.tofile(os.path.join(ingest_dir, "docids.off"))
    for key, name in INDEX_FILES.items():
        if index.get(key) is not None:
            np.ascontiguousarray(index[key]).tofile(os.path.join(index_dir, name))


def read_files(ingest_dir: str, index_dir: str) -> dict:
    """Reads a reference corpus + index directory into the arrays dict Index takes."""
    dt = {"rerank": np.int8, "norm256": np.float32, "codes": np.uint8, "quant_scale": np.float32,
          "centroids": np.float32, "block_off": np.uint64, "ids": np.uint32, "blocks": np.uint8,
          "factors": np.float32, "rotation": np.float32, "tier2_sigma": np.float32,
          "tier2_codes": np.uint8, "tier2_norm": np.float32}
    out = {}
    for key, name in CORPUS_FILES.items():
        out[key] = np.fromfile(os.path.join(ingest_dir, name), dtype=dt[key])
    for key, name in INDEX_FILES.items():
        p = os.path.join(index_dir, name)
        out[key] = np.fromfile(p, dtype=dt[key]) if os.path.exists(p) else None
    out["n"] = out["norm256"].size
    out["k"] = out["centroids"].size // PDIM
    out["rerank"] = out["rerank"].reshape(out["n"], DIM)
    return out
