"""Seeded synthetic corpora standing in for the reference's datasets (MS MARCO Arctic-Embed
768-d and MS SPACEV-1B), which are not available: Gaussian mixtures with the shapes, sizes and
value distributions the workloads name. Nothing from those datasets is reproduced.

A mixture has `n_centers` centres drawn N(0, spread^2) per dimension; a point is a uniformly
chosen centre plus N(0, sigma^2) noise per dimension, L2-normalised (cosine workloads) or rounded
and clipped to int8 (the L2 workload). Rows are generated in fixed chunks of CHUNK rows, each
from its own generator seeded by (seed, chunk), so any row range is reproducible on its own and
the corpus never has to exist as float32 in memory at once.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

CHUNK = 65536


def _gen(device: torch.device, seed: int) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(seed & ((1 << 63) - 1))
    return g


@dataclass
class Mixture:
    """A seeded Gaussian mixture of `n` rows in `dim` dimensions."""

    n: int
    n_centers: int
    dim: int = 768
    spread: float = 1.0
    sigma: float = 0.3
    seed: int = 1
    normalise: bool = True
    device: str = "cpu"

    def __post_init__(self):
        dev = torch.device(self.device)
        g = _gen(dev, self.seed * 7919 + 17)
        self.centers = torch.randn(self.n_centers, self.dim, generator=g, device=dev) * self.spread

    def _chunk(self, c: int, sigma: float, salt: int) -> torch.Tensor:
        dev = self.centers.device
        rows = min(CHUNK, self.n - c * CHUNK) if salt == 0 else CHUNK
        g = _gen(dev, (self.seed * 1_000_003 + c) * 31 + salt)
        which = torch.randint(0, self.n_centers, (rows,), generator=g, device=dev)
        x = self.centers[which] + sigma * torch.randn(rows, self.dim, generator=g, device=dev)
        if self.normalise:
            x = x / x.norm(dim=1, keepdim=True).clamp_min(1e-30)
        return x

    def rows(self, start: int, count: int) -> torch.Tensor:
        """Rows [start, start + count) as float32 (unit length for cosine mixtures)."""
        out = []
        c0, c1 = start // CHUNK, (start + count - 1) // CHUNK
        for c in range(c0, c1 + 1):
            x = self._chunk(c, self.sigma, 0)
            lo = max(start - c * CHUNK, 0)
            hi = min(start + count - c * CHUNK, x.shape[0])
            out.append(x[lo:hi])
        return torch.cat(out) if len(out) > 1 else out[0]

    def centres_of(self, start: int, count: int) -> torch.Tensor:
        """The mixture centre of rows [start, start + count): the first draw of each chunk's
        generator, so regenerating it alone gives the same centres as rows()."""
        out = []
        dev = self.centers.device
        c0, c1 = start // CHUNK, (start + count - 1) // CHUNK
        for c in range(c0, c1 + 1):
            rows = min(CHUNK, self.n - c * CHUNK)
            g = _gen(dev, (self.seed * 1_000_003 + c) * 31)
            which = torch.randint(0, self.n_centers, (rows,), generator=g, device=dev)
            lo = max(start - c * CHUNK, 0)
            hi = min(start + count - c * CHUNK, rows)
            out.append(which[lo:hi])
        return torch.cat(out) if len(out) > 1 else out[0]

    def queries(self, nq: int, sigma: float, seed: int = 99) -> torch.Tensor:
        """nq query vectors from the same centres with noise sigma (salted stream)."""
        out = []
        for c in range((nq + CHUNK - 1) // CHUNK):
            out.append(self._chunk(c, sigma, salt=1 + seed))
        return torch.cat(out)[:nq]
