"""The pressure-transfer rule across a change of forest, restated in
Python for the tests (the device kernel `k_transfer` must match it bit for
bit), and the two-disk forests the time-stepping tests move.

Rule: positions in cells of level G = max(levelMax) + 1; a target cell at
the same level as, or finer than, the source leaf holding its centre takes
that source cell's value; a coarser target cell takes the mean of the source
cells at the centres of its four quadrants (summed in quadrant order)."""
import numpy as np

from cup2d_b200 import Mesh
from cup2d_b200.problems import EXTENT


def disk_mesh(shift: float, level_max: int = 5, band: float = 0.1) -> Mesh:
    return Mesh.disks(8, 4, level_max, EXTENT, [(0.6 + shift, 0.5, 0.1), (1.3 - shift, 0.4, 0.07)], band)


def transfer_restated(src: Mesh, xs: np.ndarray, dst: Mesh) -> np.ndarray:
    G = max(src.level_max, dst.level_max) + 1
    leaf = {(int(l), int(i), int(j)): k for k, (l, i, j) in enumerate(zip(src.level, src.bx, src.by))}

    def locate(px, py):
        for l in range(src.level_max):
            ci, cj = px >> (G - l), py >> (G - l)
            k = leaf.get((l, ci >> 3, cj >> 3))
            if k is not None:
                return k, (cj & 7) * 8 + (ci & 7)
        raise AssertionError("point outside the forest")

    out = np.empty(dst.ncells)
    for b, (l, bi, bj) in enumerate(zip(dst.level, dst.bx, dst.by)):
        sh = G - int(l)
        for c in range(64):
            ix, iy = c & 7, c >> 3
            px = ((int(bi) * 8 + ix) << sh) + (1 << (sh - 1))
            py = ((int(bj) * 8 + iy) << sh) + (1 << (sh - 1))
            k, sc = locate(px, py)
            if src.level[k] <= l:
                out[b * 64 + c] = xs[k * 64 + sc]
                continue
            q = 1 << (sh - 2)
            acc = 0.0
            for t in range(4):
                k2, c2 = locate(px + (q if t & 1 else -q), py + (q if t & 2 else -q))
                acc += xs[k2 * 64 + c2]
            out[b * 64 + c] = 0.25 * acc
    return out
