"""Seeded synthetic workloads with the shapes and distributions of the benchmark configs.

The reference measures on its own generated blob sets (data/generate_data.py:7-33,
benchmark/utils/generation.hpp:94-115); these generators produce the same family at the
requested sizes.  RNG: numpy PCG64, seed = config id * 1000 + replicate.  Points are
blobs concatenated, then noise (the reference generator's order); ``shuffle=True``
permutes them.  Coordinates are SoA float32 arrays of shape (ndim, n).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Workload:
    name: str
    coords: np.ndarray  # (ndim, n) float32
    weight: np.ndarray  # (n,) float32
    dc: float
    rhoc: float
    dm: float
    kernel: tuple       # ("flat", (0.5,)) / ("exp", (avg, amp)) / ("gaus", (avg, std, amp))


def _finish(blobs, noise, w, shuffle, rng):
    c = np.concatenate([blobs, noise], axis=1).astype(np.float32)
    if shuffle:
        p = rng.permutation(c.shape[1])
        c = c[:, p]
        w = w[p]
    return np.ascontiguousarray(c), np.ascontiguousarray(w.astype(np.float32))


def blobs_2d_16k(n: int = 16384, seed: int = 1000, shuffle: bool = False) -> Workload:
    """Plain 2-D: 20 isotropic blobs (sigma 1) in [5,95]^2, 10% uniform noise in [0,100]^2."""
    rng = np.random.default_rng(seed)
    nb = 20
    per = int(0.9 * n) // nb
    centres = rng.uniform(5, 95, size=(nb, 2))
    blobs = np.concatenate([rng.normal(centres[b], 1.0, size=(per, 2)) for b in range(nb)]).T
    noise = rng.uniform(0, 100, size=(2, n - per * nb))
    w = rng.uniform(0.5, 1.5, size=n)
    c, w = _finish(blobs, noise, w, shuffle, rng)
    return Workload("blobs2d_16k", c, w, 1.5, 5.0, 1.5, ("flat", (0.5,)))


def blobs_2d_1m(n: int = 1 << 20, seed: int = 2000, shuffle: bool = False) -> Workload:
    """Plain 2-D: 1000 blobs (sigma 0.3) in [0,1000]^2, 10% noise."""
    rng = np.random.default_rng(seed)
    nb = 1000
    per = int(0.9 * n) // nb
    centres = rng.uniform(0, 1000, size=(nb, 2))
    blobs = (centres[:, None, :] + rng.normal(0, 0.3, size=(nb, per, 2))).reshape(-1, 2).T
    noise = rng.uniform(0, 1000, size=(2, n - per * nb))
    w = rng.uniform(0.5, 1.5, size=n)
    c, w = _finish(blobs, noise, w, shuffle, rng)
    return Workload("blobs2d_1m", c, w, 1.0, 5.0, 1.5, ("flat", (0.5,)))


def blobs_3d_4m(n: int = 1 << 22, seed: int = 3000, shuffle: bool = False) -> Workload:
    """Plain 3-D: 5000 anisotropic blobs (per-axis sigma U[0.2,1]) in [0,500]^3, 15% noise,
    lognormal(0, 0.5) weights, Gaussian kernel (mean 0, std 0.5, amplitude 1)."""
    rng = np.random.default_rng(seed)
    nb = 5000
    per = int(0.85 * n) // nb
    centres = rng.uniform(0, 500, size=(nb, 3))
    sig = rng.uniform(0.2, 1.0, size=(nb, 3))
    blobs = (centres[:, None, :] + rng.normal(0, 1, size=(nb, per, 3)) * sig[:, None, :]).reshape(-1, 3).T
    noise = rng.uniform(0, 500, size=(3, n - per * nb))
    w = rng.lognormal(0.0, 0.5, size=n)
    c, w = _finish(blobs, noise, w, shuffle, rng)
    return Workload("blobs3d_4m", c, w, 1.2, 8.0, 2.0, ("gaus", (0.0, 0.5, 1.0)))


def calo_event(rng: np.random.Generator, n: int) -> tuple[np.ndarray, np.ndarray]:
    """One 2-D calorimeter-like event: 3-30 energy-weighted showers + 20% noise in [0,200]^2."""
    ns = int(rng.integers(3, 31))
    centres = rng.uniform(0, 200, size=(ns, 2))
    sig = rng.uniform(0.5, 3.0, size=ns)
    energy = rng.exponential(1.0, size=ns)
    n_sh = int(round(0.8 * n))
    counts = np.floor(energy / energy.sum() * n_sh).astype(np.int64)
    counts[np.argmax(energy)] += n_sh - counts.sum()
    parts = [centres[s] + rng.normal(0, sig[s], size=(counts[s], 2)) for s in range(ns)]
    parts.append(rng.uniform(0, 200, size=(n - n_sh, 2)))
    c = np.concatenate(parts).T.astype(np.float32)
    w = rng.exponential(1.0, size=n).astype(np.float32)
    return np.ascontiguousarray(c), w


def calo_events(n_events: int = 4096, seed: int = 4000, lo: int = 100, hi: int = 60000):
    """Batched 2-D events: sizes lognormal(median 2000, sigma 1) clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.round(rng.lognormal(np.log(2000), 1.0, size=n_events)), lo, hi).astype(np.int64)
    events = [calo_event(rng, int(s)) for s in sizes]
    return events, dict(dc=2.0, rhoc=4.0, dm=3.0, kernel=("exp", (1.0, 1.0)))


def blobs_4d_event(rng: np.random.Generator, n: int) -> tuple[np.ndarray, np.ndarray]:
    """One 4-D serving event: 5-50 blobs (sigma 1) in [0,100]^4 plus 10% noise."""
    nb = int(rng.integers(5, 51))
    per = int(0.9 * n) // nb
    centres = rng.uniform(0, 100, size=(nb, 4))
    blobs = (centres[:, None, :] + rng.normal(0, 1.0, size=(nb, per, 4))).reshape(-1, 4)
    noise = rng.uniform(0, 100, size=(n - per * nb, 4))
    c = np.concatenate([blobs, noise]).T.astype(np.float32)
    w = rng.uniform(0.5, 1.5, size=n).astype(np.float32)
    return np.ascontiguousarray(c), w


def serving_events(n_events: int, seed: int = 5000, lo: int = 100, hi: int = 200000):
    """4-D serving events: sizes lognormal(median 2000, sigma 1) clipped to [lo, hi]; returns
    the events concatenated (coords (4, n_total), weight, event offsets) and the parameters."""
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.round(rng.lognormal(np.log(2000), 1.0, size=n_events)), lo, hi).astype(np.int64)
    evs = [blobs_4d_event(rng, int(s)) for s in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    coords = np.ascontiguousarray(np.concatenate([e[0] for e in evs], axis=1))
    weight = np.ascontiguousarray(np.concatenate([e[1] for e in evs]))
    return coords, weight, off, dict(dc=2.5, rhoc=6.0, dm=2.5, kernel=("flat", (0.5,)))


def poisson_arrivals(rate: float, n: int, seed: int = 0) -> np.ndarray:
    """Arrival times (seconds) of a Poisson stream of `rate` events/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


CONFIGS = {
    "blobs2d_16k": blobs_2d_16k,
    "blobs2d_1m": blobs_2d_1m,
    "blobs3d_4m": blobs_3d_4m,
}
