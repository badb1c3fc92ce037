"""Whole k points owned by ranks: the k-point pools of an SCF map split over GPUs.

Restates the reference's pool layout with one rank per pool
(crates/dft-engine/src/refscf/k_pool.rs:76-330; the `auto` rule there picks one rank per
pool whenever there are at least as many k points as ranks): rank r owns the contiguous
block of k points given by block_counts(nk, world) (crates/dft-mpi/src/lib.rs:207-223).
A map then needs two exchanges, both from the reference's pool collectives:

- the eigenvalues of every k point (allgatherv) for the occupations, the Fermi level and
  the band energy, which every rank then computes identically;
- the density, the sum over k of the band densities, as a sum whose order does not depend
  on which rank computes it (the reference's ordered tree sum): every rank's partial sum
  is gathered and the partials are added pairwise in a fixed binary tree over the ranks,
  so every rank holds the same bits and the rest of the map (fields, mixer) is replicated.

The collectives run through torch.distributed on whatever group it was initialised with:
gloo with CPU tensors, NCCL with CUDA tensors (plain all_gather: no multicast, no library
kernel on a peer's memory).  With world size 1 every method is the identity.
"""
from __future__ import annotations

import numpy as np


def block_counts(total: int, parts: int) -> list[int]:
    """k points per rank: `total` split into `parts` blocks, the first total % parts one larger."""
    parts = max(parts, 1)
    base, extra = divmod(total, parts)
    return [base + (1 if r < extra else 0) for r in range(parts)]


def block_first(counts: list[int]) -> list[int]:
    out, at = [], 0
    for c in counts:
        out.append(at)
        at += c
    return out


def tree_sum(parts: list):
    """Sum of the items of `parts` in a fixed binary tree (pairs of neighbours, level by
    level): the result depends only on the list, not on who evaluates it."""
    level = list(parts)
    if not level:
        raise ValueError("nothing to sum")
    while len(level) > 1:
        nxt = [level[i] + level[i + 1] for i in range(0, len(level) - 1, 2)]
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    return level[0]


class KPool:
    """k points nk over the ranks of a torch.distributed group (or a single process)."""

    def __init__(self, nk: int, rank: int = 0, world: int = 1, dist=None, device=None):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("rank outside the world")
        if nk < world:
            raise ValueError("a pool of one rank per k point needs at least as many k points as ranks")
        self.nk, self.rank, self.world = nk, rank, world
        self.dist = dist if world > 1 else None
        self.device = device
        self.counts = block_counts(nk, world)
        self.first = block_first(self.counts)

    @classmethod
    def from_env(cls, nk: int, device=None):
        """The pool of the initialised default torch.distributed group, else one rank."""
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return cls(nk, dist.get_rank(), dist.get_world_size(), dist, device)
        return cls(nk, device=device)

    @property
    def local(self) -> range:
        return range(self.first[self.rank], self.first[self.rank] + self.counts[self.rank])

    def owner(self, k: int) -> int:
        for r in range(self.world):
            if self.first[r] <= k < self.first[r] + self.counts[r]:
                return r
        raise IndexError(k)

    def _tensor(self, a):
        import torch
        t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64))
        return t.to(self.device) if self.device is not None else t

    def gather_eigenvalues(self, local: list) -> list:
        """Eigenvalues (one array of `bands` per local k point) -> every k point's, in k order."""
        local = [np.asarray(v, dtype=np.float64) for v in local]
        if len(local) != self.counts[self.rank]:
            raise ValueError("one eigenvalue array per local k point")
        if self.dist is None:
            return local
        import torch
        bands = local[0].size if local else 0
        width = max(self.counts)
        buf = np.zeros((width, bands))
        for i, v in enumerate(local):
            buf[i] = v
        mine = self._tensor(buf)
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        self.dist.all_gather(parts, mine)
        out = []
        for r in range(self.world):
            p = parts[r].cpu().numpy()
            out.extend(p[i].copy() for i in range(self.counts[r]))
        return out

    def sum_partials(self, partial):
        """Sum over ranks of a partial (numpy array or torch tensor of one shape), in the
        fixed tree order over ranks; every rank gets the same result, as the same type."""
        if self.dist is None:
            return partial
        import torch
        is_np = isinstance(partial, np.ndarray)
        mine = self._tensor(partial) if is_np else partial.contiguous()
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        self.dist.all_gather(parts, mine)
        total = tree_sum(parts)
        return total.cpu().numpy() if is_np else total
