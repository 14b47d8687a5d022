"""Synthetic Poisson problems of the benchmark configurations.

Every problem is a block-AMR forest refined near disks and the divergence
of a seeded random Fourier velocity field as right-hand side (projected to
zero entry-sum for the Neumann walls).  Sizes follow the configurations the
solver is measured on:

  small   [0,2]x[0,1], bpdx=4, bpdy=2, levelMax=4, one disk r=0.1 at
          (0.6,0.5), band 0.15                     -> 128 blocks, 8k cells
  large   bpdx=8, bpdy=4, levelMax=7, 3 seeded disks r in [0.05,0.1],
          band 0.12                                -> ~20k blocks, ~1.3M cells
  batch   levelMax in {3..6}, 1-3 disks, sizes log-uniform 50..6000 blocks
  serve   sizes log-uniform 64..20k blocks
"""
from __future__ import annotations

import math

import numpy as np

from .mesh import Mesh

EXTENT = 2.0


def small_mesh() -> Mesh:
    return Mesh.disks(4, 2, 4, EXTENT, [(0.6, 0.5, 0.1)], 0.15)


def quoted_small_mesh() -> Mesh:
    """The small configuration at its quoted size (~300 blocks, ~19k cells):
    the same domain, level count and disk with the refinement band widened
    to 0.43, which gives 302 blocks / 19,328 cells (band 0.15 gives 128)."""
    return Mesh.disks(4, 2, 4, EXTENT, [(0.6, 0.5, 0.1)], 0.43)


def seeded_disks(rng: np.random.Generator, count: int, rmin: float = 0.05, rmax: float = 0.1):
    return [(float(rng.uniform(0.3, 1.7)), float(rng.uniform(0.25, 0.75)), float(rng.uniform(rmin, rmax)))
            for _ in range(count)]


def large_mesh(seed: int = 1, band: float = 0.12, shift_x: float = 0.0) -> Mesh:
    disks = seeded_disks(np.random.default_rng(seed), 3)
    disks = [(cx + shift_x, cy, r) for cx, cy, r in disks]
    return Mesh.disks(8, 4, 7, EXTENT, disks, band)


def sized_mesh(rng: np.random.Generator, target_blocks: int, level_max: int | None = None) -> Mesh:
    """A disk-refined mesh with roughly `target_blocks` blocks: picks the
    level count, disk count and band from the generator, then bisects the
    band toward the target size."""
    L = int(rng.integers(3, 7)) if level_max is None else level_max
    nd = int(rng.integers(1, 4))
    disks = seeded_disks(rng, nd)
    # root grid: grow the roots until the finest level can hold the target
    bpdx, bpdy = 2, 1
    while bpdx * bpdy * 4 ** (L - 1) < target_blocks and bpdx < 64:
        bpdx, bpdy = 2 * bpdx, 2 * bpdy
    lo, hi = 0.0, 1.0
    best = None
    for _ in range(14):
        band = 0.5 * (lo + hi)
        m = Mesh.disks(bpdx, bpdy, L, EXTENT, disks, band)
        if best is None or abs(math.log(m.nblocks / target_blocks)) < abs(math.log(best.nblocks / target_blocks)):
            best = m
        if m.nblocks < target_blocks:
            lo = band
        else:
            hi = band
    return best


def loguniform_sizes(rng: np.random.Generator, count: int, lo: int, hi: int) -> np.ndarray:
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(np.int64)


def batch_problems(count: int = 512, seed: int = 3, lo: int = 50, hi: int = 6000) -> list[Mesh]:
    """The batched workload: `count` disk-refined meshes with sizes drawn
    log-uniform in [lo, hi] blocks (levelMax 3..6, 1-3 disks each)."""
    rng = np.random.default_rng(seed)
    sizes = loguniform_sizes(rng, count, lo, hi)
    return [sized_mesh(rng, int(s)) for s in sizes]
