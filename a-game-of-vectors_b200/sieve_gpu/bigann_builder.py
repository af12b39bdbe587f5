"""bigann index build (src/bigann.rs:120-466) in torch, on the GPU when one is present, and the
reference's bigann file formats.

A base is int8 rows of 100 dims searched by L2 (score 2<q,x> - |x|^2). The build trains K1 coarse
cells and K2 leaves inside each (two-level k-means in L2, as bigann::train), assigns every row to
the best leaf among the children of its TOP_COARSE nearest cells (Model::assign), codes the
rotated residual of its padded 128-d row against the leaf (a 16-byte sign code with
[mul, |x|^2]) and, for bits > 1, the low planes and scale f of a uniform bits-bit code
(refine_encode), then packs each leaf's rows by id into 32-slot blocks (bigann::pack). The query
path reads only the packed arrays, so the build's float order need not follow the reference's.

Files (index dir): coarse.f32, centroids.f32 (leaves), rotation.f32, k2.u64, bits.u64,
postings.bin + postings.off (records, src/postings.rs:9-34), block_off.u64; base dir: base.NN
(100M int8 rows each) with base.NN.done.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from .builder import Rng, fwht, pack_bits, pack_blocks, rotation_signs

D, PD, CODE, G, BLOCK_BYTES, MAX_BITS = 100, 128, 16, 32, 512, 3
BLOCK = 32
PAD = 0xFFFFFFFF
TOP_COARSE = 4
CHUNK_ROWS = 100_000_000
ALIGN = 4096


# ---- synthetic SPACEV-like bases ---------------------------------------------------------------
class Spacev:
    """Seeded int8 rows: centre[U(n_centers)] + N(0, sigma^2) per dim, rounded and clipped to
    [-127, 127]; centres N(0, spread^2) per dim. Rows are generated in chunks, each from its own
    seed, so any range can be regenerated."""

    def __init__(self, n: int, n_centers: int, spread: float = 40.0, sigma: float = 12.0,
                 seed: int = 1, device: str | None = None):
        self.n, self.n_centers, self.sigma, self.seed = n, n_centers, sigma, seed
        self.device = device or ("cuda" if torch.cuda.is_available() else "cpu")
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.centers = (torch.randn((n_centers, D), generator=g) * spread).to(self.device)

    CHUNK = 1 << 20

    def _chunk(self, c: int, salt: int = 0) -> torch.Tensor:
        n = min(self.CHUNK, self.n - c * self.CHUNK) if salt == 0 else self.CHUNK
        g = torch.Generator(device=self.device).manual_seed(self.seed * 1_000_003 + c * 7919 + salt)
        lab = torch.randint(0, self.n_centers, (n,), generator=g, device=self.device)
        x = self.centers[lab] + torch.randn((n, D), generator=g, device=self.device) * self.sigma
        return torch.clamp(torch.round(x), -127, 127).to(torch.int8)

    def rows(self, start: int, count: int) -> torch.Tensor:
        out = []
        c0, c1 = start // self.CHUNK, (start + count - 1) // self.CHUNK
        for c in range(c0, c1 + 1):
            x = self._chunk(c)
            lo = max(start - c * self.CHUNK, 0)
            hi = min(start + count - c * self.CHUNK, x.shape[0])
            out.append(x[lo:hi])
        return torch.cat(out) if out else torch.zeros((0, D), dtype=torch.int8, device=self.device)

    def queries(self, nq: int) -> torch.Tensor:
        """Queries from the same mixture (a separate seed stream)."""
        return self._chunk(0, salt=977)[:nq]


# ---- k-means in L2 (src/bigann.rs:138-161) ------------------------------------------------------
def _nearest(x: torch.Tensor, cents: torch.Tensor, m: int = 1, chunk: int = 65536):
    cn = (cents * cents).sum(1)
    out_i, out_s = [], []
    for s in range(0, x.shape[0], chunk):
        sc = 2.0 * (x[s:s + chunk] @ cents.T) - cn
        v, i = torch.topk(sc, m, dim=1)
        out_i.append(i)
        out_s.append(v)
    return torch.cat(out_i), torch.cat(out_s)


def kmeans_l2(sample: torch.Tensor, k: int, iters: int, seed: int) -> torch.Tensor:
    n = sample.shape[0]
    rng = Rng(seed)
    cents = sample[torch.as_tensor(rng.below_many(n, k), device=sample.device)].clone()
    for _ in range(iters):
        a = _nearest(sample, cents)[0][:, 0]
        counts = torch.bincount(a, minlength=k)
        sums = torch.zeros_like(cents, dtype=torch.float64).index_add_(0, a, sample.double())
        cnt = counts.cpu().numpy()
        for c in np.nonzero(cnt == 0)[0]:
            cents[c] = sample[rng.below(n)]
        nz = torch.as_tensor(np.nonzero(cnt)[0], device=sample.device)
        cents[nz] = (sums[nz] / counts[nz, None].double()).float()
    return cents


def train(base: torch.Tensor, k1: int, k2: int, sample_n: int, iters: int = 8) -> dict:
    """bigann::train (src/bigann.rs:173-222): coarse cells, then k2 leaves per cell."""
    dev = base.device
    n = base.shape[0]
    rng = Rng(42)
    idx = np.sort(rng.below_many(n, min(sample_n, n)))
    sample = base[torch.as_tensor(idx, device=dev)].float()
    coarse_n = min(sample.shape[0], k1 * 512)
    stride = max(sample.shape[0] // coarse_n, 1)
    coarse = kmeans_l2(sample[::stride][:coarse_n], k1, iters, 7)
    a = _nearest(sample, coarse)[0][:, 0]
    leaves = []
    for c in range(k1):
        m = sample[a == c]
        rows = coarse[c:c + 1] if m.shape[0] == 0 else m
        if rows.shape[0] < k2:  # too few rows: repeat them (the duplicates stay empty)
            rows = rows[torch.arange(k2, device=dev) % rows.shape[0]]
        leaves.append(kmeans_l2(rows, k2, iters, c))
    return {"coarse": coarse, "leaves": torch.cat(leaves), "k2": k2}


def assign(model: dict, x: torch.Tensor) -> torch.Tensor:
    """Model::assign (src/bigann.rs:263-290): best leaf among the children of the row's
    TOP_COARSE nearest coarse cells, one dense product per (coarse cell, rows choosing it)."""
    k2 = model["k2"]
    leaves = model["leaves"]
    ln = (leaves * leaves).sum(1)
    top = _nearest(x, model["coarse"], min(TOP_COARSE, model["coarse"].shape[0]))[0]  # [n, T]
    n = x.shape[0]
    best_s = torch.full((n,), -float("inf"), device=x.device)
    best_l = torch.zeros(n, dtype=torch.int64, device=x.device)
    for t in range(top.shape[1]):
        cell = top[:, t]
        order = torch.argsort(cell)
        counts = torch.bincount(cell, minlength=model["coarse"].shape[0]).cpu().numpy()
        start = 0
        for c in np.nonzero(counts)[0]:
            rows = order[start:start + counts[c]]
            start += counts[c]
            lv = leaves[c * k2:(c + 1) * k2]
            sc = 2.0 * (x[rows] @ lv.T) - ln[c * k2:(c + 1) * k2]
            v, j = sc.max(1)
            better = v > best_s[rows]
            best_s[rows] = torch.where(better, v, best_s[rows])
            best_l[rows] = torch.where(better, j + c * k2, best_l[rows])
    return best_l


def rotate128(signs: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """pad_rotate (src/bigann.rs:243-248): pad 100 -> 128 with zeros, then Rotation::apply."""
    v = torch.zeros((x.shape[0], PD), dtype=torch.float32, device=x.device)
    v[:, :D] = x
    for r in range(3):
        v = fwht(v * signs[r * PD:(r + 1) * PD])
    norm = np.float32(np.power(np.float32(PD), np.float32(-1.5)))
    return v * float(norm)


def refine_encode(r: torch.Tensor, bits: int):
    """refine_encode (src/bigann.rs:65-108) on every row: (planes [n, (MAX_BITS-1)*16] u8, f)."""
    n = r.shape[0]
    top = 1 << (bits - 1)
    h = (2 * top - 1) / 2.0
    amax = r.abs().amax(1)
    planes = torch.zeros((n, (MAX_BITS - 1) * CODE), dtype=torch.uint8, device=r.device)

    def level(v, delta):
        u = torch.clamp(torch.floor(v / delta[:, None] + h + 0.5), 0, 2 * top - 1).to(torch.int64)
        return torch.where(v > 0, u | top, u & (top - 1))

    best = torch.full((n,), -float("inf"), device=r.device)
    best_delta = amax / h
    for s in range(24):
        delta = amax / h * (0.3 + 0.035 * s)
        w = level(r, delta).float() - h
        cos = (r * w).sum(1) / torch.sqrt((w * w).sum(1))
        take = cos > best
        best = torch.where(take, cos, best)
        best_delta = torch.where(take, delta, best_delta)
    u = level(r, best_delta)
    for p in range(bits - 1):
        planes[:, p * CODE:(p + 1) * CODE] = pack_bits(((u >> p) & 1).bool())
    rr = (r * r).sum(1)
    dot = (r * (u.float() - h)).sum(1)
    f = torch.where(dot > 0, rr / dot, torch.zeros_like(rr))
    zero = amax < 1e-12
    f = torch.where(zero, torch.zeros_like(f), f)
    planes[zero] = 0
    return planes, f


def build_bigann(base: torch.Tensor, k1: int, k2: int, bits: int = 2, sample_n: int = 262144,
                 iters: int = 8, batch: int = 1 << 18) -> dict:
    """train + add + pack (src/bigann.rs:173-466) into the arrays a bigann index opens."""
    dev = base.device
    n = base.shape[0]
    model = train(base, k1, k2, sample_n, iters)
    signs = torch.as_tensor(rotation_signs(11, PD), device=dev)
    leaves = model["leaves"]
    k = leaves.shape[0]
    leaves_rot = rotate128(signs, leaves)
    leaf_of = torch.empty(n, dtype=torch.int64, device=dev)
    codes = torch.empty((n, CODE), dtype=torch.uint8, device=dev)
    mul = torch.empty(n, dtype=torch.float32, device=dev)
    nx = torch.empty(n, dtype=torch.float32, device=dev)
    extra = (bits - 1) * CODE + 4 if bits > 1 else 0
    ext = torch.zeros((n, max(extra, 1)), dtype=torch.uint8, device=dev)
    for s in range(0, n, batch):
        x = base[s:s + batch].float()
        lf = assign(model, x)
        xr = rotate128(signs, x)
        r = xr - leaves_rot[lf]
        nr2 = (r * r).sum(1)
        l1 = r.abs().sum(1)
        m = torch.where(l1 < 1e-12, torch.zeros_like(nr2), nr2 / l1)
        leaf_of[s:s + batch] = lf
        codes[s:s + batch] = pack_bits(r > 0)
        mul[s:s + batch] = m
        nx[s:s + batch] = (x * x).sum(1)
        if bits > 1:
            planes, f = refine_encode(r, bits)
            np_ = (bits - 1) * CODE
            ext[s:s + batch, :np_] = planes[:, :np_]
            ext[s:s + batch, np_:np_ + 4] = f.view(torch.uint8).reshape(-1, 4)
    # pack: leaf-major, ids ascending inside a leaf
    order = torch.argsort(leaf_of * n + torch.arange(n, device=dev))
    leaf_sorted = leaf_of[order]
    sizes = torch.bincount(leaf_of, minlength=k).cpu().numpy().astype(np.int64)
    nb = (sizes + BLOCK - 1) // BLOCK
    block_off = np.zeros(k + 1, np.uint64)
    block_off[1:] = np.cumsum(nb)
    nblocks = int(block_off[-1])
    # slot of each sorted row: its leaf's first slot + rank inside the leaf
    first_row = np.zeros(k + 1, np.int64)
    first_row[1:] = np.cumsum(sizes)
    rank = torch.arange(n, device=dev) - torch.as_tensor(first_row[:-1], device=dev)[leaf_sorted]
    slot = torch.as_tensor(block_off[:-1].astype(np.int64) * BLOCK, device=dev)[leaf_sorted] + rank
    ids = torch.full((nblocks * BLOCK,), PAD, dtype=torch.int64, device=dev)
    ids[slot] = order
    raw = torch.zeros((nblocks * BLOCK, CODE), dtype=torch.uint8, device=dev)
    raw[slot] = codes[order]
    factors = torch.zeros((nblocks * BLOCK, 2), dtype=torch.float32, device=dev)
    factors[slot, 0] = mul[order]
    factors[slot, 1] = nx[order]
    ext_s = torch.zeros((nblocks * BLOCK, max(extra, 1)), dtype=torch.uint8, device=dev)
    ext_s[slot] = ext[order]
    blocks = pack_blocks(raw.reshape(nblocks, BLOCK, CODE)) if nblocks else raw.reshape(0, BLOCK_BYTES)
    return {
        "n": n, "k": k, "bits": bits, "k2": k2,
        "coarse": model["coarse"].cpu().numpy(),
        "leaves": leaves.cpu().numpy(),
        "block_off": block_off,
        "ids": ids.to(torch.int64).cpu().numpy().astype(np.uint32),
        "blocks": blocks.cpu().numpy().reshape(-1),
        "factors": factors.cpu().numpy().reshape(-1),
        "ext": ext_s[:, :extra].cpu().numpy().reshape(-1) if extra else np.zeros(0, np.uint8),
        "rotation": rotation_signs(11, PD),
        "base": base.cpu().numpy(),
        "sizes": sizes,
    }


def ground_truth(base: torch.Tensor, queries: torch.Tensor, k: int = 10, chunk: int = 1 << 20):
    """Exact top-k rows by 2<q,x> - |x|^2, ties by ascending row: (ids [nq, k], scores [nq, k]).
    Products and sums of int8 values stay below 2^24, so f32 (TF32 off) computes them exactly."""
    q = queries.float()
    best_v = torch.full((q.shape[0], k), -float("inf"), device=q.device)
    best_i = torch.zeros((q.shape[0], k), dtype=torch.int64, device=q.device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, base.shape[0], chunk):
            x = base[s:s + chunk].to(q.device).float()
            sc = 2.0 * (q @ x.T) - (x * x).sum(1)[None, :]
            v, i = torch.topk(sc, min(k, sc.shape[1]), dim=1)
            allv = torch.cat((best_v, v), 1)
            alli = torch.cat((best_i, i + s), 1)
            order = torch.argsort(alli, dim=1, stable=True)
            allv, alli = allv.gather(1, order), alli.gather(1, order)
            tv, ti = torch.sort(allv, dim=1, descending=True, stable=True)
            best_v, best_i = tv[:, :k], alli.gather(1, ti[:, :k])
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return best_i.cpu().numpy().astype(np.uint32), best_v.cpu().numpy()


# ---- the reference's bigann files ---------------------------------------------------------------
def write_files(index: dict, index_dir: str, base_dir: str) -> None:
    """Writes the bigann files: the leaf records of postings.bin (src/postings.rs:9-34, blocks,
    factors, ids, extra, each record 4 KiB aligned), postings.off, block_off.u64, the model
    files and the base chunks."""
    os.makedirs(index_dir, exist_ok=True)
    os.makedirs(base_dir, exist_ok=True)
    k, bits = int(index["k"]), int(index["bits"])
    extra = (bits - 1) * CODE + 4 if bits > 1 else 0
    bo = index["block_off"].astype(np.int64)
    blocks = index["blocks"].reshape(-1, BLOCK_BYTES)
    factors = index["factors"].reshape(-1, BLOCK * 2)
    ids = index["ids"].reshape(-1, BLOCK)
    ext = index["ext"].reshape(-1, BLOCK * extra) if extra else None
    off = np.zeros(k + 1, np.uint64)
    pos = 0
    with open(os.path.join(index_dir, "postings.bin"), "wb") as f:
        for c in range(k):
            b0, b1 = bo[c], bo[c + 1]
            off[c] = pos
            parts = [blocks[b0:b1].tobytes(), factors[b0:b1].astype(np.float32).tobytes(),
                     ids[b0:b1].astype(np.uint32).tobytes()]
            if extra:
                parts.append(ext[b0:b1].tobytes())
            rec = b"".join(parts)
            f.write(rec)
            pos += len(rec)
            pad = (-pos) % ALIGN
            f.write(b"\0" * pad)
            pos += pad
    off[k] = pos
    off.tofile(os.path.join(index_dir, "postings.off"))
    index["block_off"].astype(np.uint64).tofile(os.path.join(index_dir, "block_off.u64"))
    np.ascontiguousarray(index["coarse"], np.float32).tofile(os.path.join(index_dir, "coarse.f32"))
    np.ascontiguousarray(index["leaves"], np.float32).tofile(os.path.join(index_dir, "centroids.f32"))
    np.ascontiguousarray(index["rotation"], np.float32).tofile(os.path.join(index_dir, "rotation.f32"))
    np.array([index["k2"]], np.uint64).tofile(os.path.join(index_dir, "k2.u64"))
    np.array([bits], np.uint64).tofile(os.path.join(index_dir, "bits.u64"))
    base = np.ascontiguousarray(index["base"], np.int8).reshape(-1)
    n = int(index["n"])
    for c in range((n + CHUNK_ROWS - 1) // CHUNK_ROWS):
        name = os.path.join(base_dir, f"base.{c:02d}")
        base[c * CHUNK_ROWS * D:min(n, (c + 1) * CHUNK_ROWS) * D].tofile(name)
        open(name + ".done", "w").close()


def read_files(index_dir: str, base_dir: str) -> dict:
    """Reads the bigann files back into the arrays dict (records de-interleaved)."""
    bits_p = os.path.join(index_dir, "bits.u64")
    bits = int(np.fromfile(bits_p, np.uint64)[0]) if os.path.exists(bits_p) else 1
    extra = (bits - 1) * CODE + 4 if bits > 1 else 0
    bo = np.fromfile(os.path.join(index_dir, "block_off.u64"), np.uint64)
    off = np.fromfile(os.path.join(index_dir, "postings.off"), np.uint64)
    raw = np.fromfile(os.path.join(index_dir, "postings.bin"), np.uint8)
    k = bo.size - 1
    blocks, factors, ids, ext = [], [], [], []
    for c in range(k):
        nb = int(bo[c + 1] - bo[c])
        p = int(off[c])
        blocks.append(raw[p:p + nb * BLOCK_BYTES])
        p += nb * BLOCK_BYTES
        factors.append(raw[p:p + nb * BLOCK * 8].view(np.float32))
        p += nb * BLOCK * 8
        ids.append(raw[p:p + nb * BLOCK * 4].view(np.uint32))
        p += nb * BLOCK * 4
        if extra:
            ext.append(raw[p:p + nb * BLOCK * extra])
    chunks = []
    c = 0
    while os.path.exists(os.path.join(base_dir, f"base.{c:02d}.done")):
        chunks.append(np.fromfile(os.path.join(base_dir, f"base.{c:02d}"), np.int8))
        c += 1
    base = np.concatenate(chunks).reshape(-1, D)
    leaves = np.fromfile(os.path.join(index_dir, "centroids.f32"), np.float32)
    return {
        "n": base.shape[0], "k": k, "bits": bits,
        "k2": int(np.fromfile(os.path.join(index_dir, "k2.u64"), np.uint64)[0]),
        "coarse": np.fromfile(os.path.join(index_dir, "coarse.f32"), np.float32),
        "leaves": leaves,
        "block_off": bo,
        "ids": np.concatenate(ids) if ids else np.zeros(0, np.uint32),
        "blocks": np.concatenate(blocks) if blocks else np.zeros(0, np.uint8),
        "factors": np.concatenate(factors) if factors else np.zeros(0, np.float32),
        "ext": np.concatenate(ext) if ext else np.zeros(0, np.uint8),
        "rotation": np.fromfile(os.path.join(index_dir, "rotation.f32"), np.float32),
        "base": base,
    }
