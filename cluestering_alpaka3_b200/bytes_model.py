"""Algorithmic HBM bytes of one CLUE pass over an input (the roofline numerator).

B_alg = n * (24 N + 124)                                      compulsory per-stage traffic
      + sum over stage s in {density: r = dc, nearest higher: r = dm}
          sum over non-empty cells c of an accounting grid of edge r
            sum over cells c' in the 3^N neighbourhood of c:  |c'| * (4 N + 4)

Term 1, per point: tile build 16N + 20 (bounding box 4N; bin 4N + 4; scatter 4N + 8 read,
4N + 8 written), density 4N + 8, nearest higher 4N + 12, seeds 16, follower CSR + labels 24,
un-permute of 5 outputs 44.  Term 2 is the neighbour staging traffic a tile-blocked scan needs
when a cell's 3^N neighbourhood is read once per cell; it is computed on a fixed grid of edge
r from the actual occupancy, so it does not depend on the implementation's own tile choice.
"""
from __future__ import annotations

import numpy as np


def term1(n: int, ndim: int) -> dict:
    return {
        "tiles": n * (16 * ndim + 20),
        "density": n * (4 * ndim + 8),
        "nearest_higher": n * (4 * ndim + 12),
        "seeds_labels": n * (16 + 24 + 44),
    }


def neighbour_traffic(coords: np.ndarray, r: float, offsets=None) -> int:
    """sum_c sum_{c' in 3^N(c)} |c'| * (4N + 4) on a grid of edge r (0 when it cannot be keyed).
    With `offsets` (event boundaries) every event has its own grid and cells never span events."""
    ndim, n = coords.shape
    if offsets is None:
        offsets = np.array([0, n])
    offsets = np.asarray(offsets, np.int64)
    E = len(offsets) - 1
    ev = np.repeat(np.arange(E, dtype=np.int64), np.diff(offsets))
    mn = np.minimum.reduceat(coords.astype(np.float64), offsets[:-1], axis=1)
    cells = np.floor((coords.astype(np.float64) - mn[:, ev]) / r).astype(np.int64) + 1
    extent = cells.max(axis=1) + 2
    if float(np.prod(extent.astype(np.float64))) * E > 2.0 ** 62:
        return 0
    mult = np.ones(ndim, np.int64)
    for d in range(ndim - 2, -1, -1):
        mult[d] = mult[d + 1] * extent[d + 1]
    keys = (cells * mult[:, None]).sum(axis=0) + ev * int(mult[0] * extent[0])
    uk, cnt = np.unique(keys, return_counts=True)
    offs = np.array(np.meshgrid(*[[-1, 0, 1]] * ndim, indexing="ij")).reshape(ndim, -1)
    total = 0
    for o in offs.T:
        nk = uk + int((o * mult).sum())
        pos = np.searchsorted(uk, nk)
        pos = np.minimum(pos, len(uk) - 1)
        hit = uk[pos] == nk
        total += int(cnt[pos[hit]].sum())
    return total * (4 * ndim + 4)


def algorithmic_bytes(coords: np.ndarray, dc: float, dm: float, offsets=None) -> dict:
    ndim, n = coords.shape
    t1 = term1(n, ndim)
    rho2 = neighbour_traffic(coords, dc, offsets)
    nh2 = neighbour_traffic(coords, dm, offsets)
    out = dict(t1)
    out["density_neighbours"] = rho2
    out["nearest_higher_neighbours"] = nh2
    out["term1"] = sum(t1.values())
    out["term2"] = rho2 + nh2
    out["total"] = out["term1"] + out["term2"]
    out["density_kernel"] = t1["density"] + rho2
    out["nearest_higher_kernel"] = t1["nearest_higher"] + nh2
    return out
