"""Helpers shared by the parity tests: run the GPU library and the CPU oracle on one input."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

KERNEL_NAMES = {"flat": 0, "exp": 1, "gaus": 2}
METRIC_NAMES = list(O.METRICS.keys())


def oracle_cfg(dc, rhoc, dm=None, seed_dc=None, ppbin=128, kernel=("flat", (0.5,)),
               metric=("euclidean", ()), wrapped=(), seed_capacity=0, tiebreak="reference"):
    return O.Config(dc=dc, rhoc=rhoc, dm=dm, seed_dc=seed_dc, ppbin=ppbin, kernel=kernel[0],
                    kernel_par=tuple(kernel[1]), metric=metric[0], metric_par=tuple(metric[1]),
                    wrapped=tuple(wrapped), seed_capacity=seed_capacity, tiebreak=tiebreak)


def gpu_args(dc, rhoc, dm=None, seed_dc=None, ppbin=128, kernel=("flat", (0.5,)),
             metric=("euclidean", ()), wrapped=(), seed_capacity=0, tiebreak="reference", flags=0):
    from cluestering_alpaka3_b200 import capi
    params = capi.Params(dc=dc, rhoc=rhoc, dm=dm, seed_dc=seed_dc, points_per_tile=ppbin,
                         wrapped=tuple(wrapped), seed_capacity=seed_capacity,
                         tiebreak=capi.TIE_REFERENCE if tiebreak == "reference" else capi.TIE_RHO_INDEX,
                         flags=flags)
    k = capi.Kernel(KERNEL_NAMES[kernel[0]], tuple(kernel[1]))
    m = capi.Metric(METRIC_NAMES.index(metric[0]), tuple(metric[1]))
    return params, k, m


def run_both(ctx, coords, weight, **kw):
    cfg = oracle_cfg(**{k: v for k, v in kw.items() if k != "flags"})
    ref = O.run(coords, weight, cfg)
    params, k, m = gpu_args(**kw)
    got = ctx.make_clusters_host(coords, weight, params, k, m)
    return ref, got


def assert_exact(ref, got, check_rho=True):
    """Bit-exact comparison of every output of the pipeline."""
    np.testing.assert_array_equal(got.is_seed, ref.is_seed, err_msg="is_seed")
    np.testing.assert_array_equal(got.nearest_higher, ref.nearest_higher, err_msg="nearest_higher")
    np.testing.assert_array_equal(got.cluster_index, ref.cluster_index, err_msg="cluster_index")
    if check_rho:
        np.testing.assert_array_equal(got.rho.view(np.uint32), ref.rho.view(np.uint32), err_msg="rho bits")
        np.testing.assert_array_equal(got.delta.view(np.uint32), ref.delta.view(np.uint32),
                                      err_msg="delta bits")
    assert got.info.n_clusters == ref.stats["n_clusters"]
    assert got.info.n_seeds == ref.stats["n_seeds"]
    assert got.info.dropped_seeds == ref.stats["dropped_seeds"]


def random_blobs(rng, n, ndim, nblobs=8, extent=100.0, sigma=1.0, noise=0.1, weights="uniform"):
    per = int(n * (1 - noise)) // nblobs
    lo, hi = sorted((0.0, float(extent)))
    centres = rng.uniform(lo + 0.1 * (hi - lo), hi - 0.1 * (hi - lo), size=(nblobs, ndim))
    blobs = (centres[:, None, :] + rng.normal(0, sigma, size=(nblobs, per, ndim))).reshape(-1, ndim)
    rest = rng.uniform(lo, hi, size=(n - per * nblobs, ndim))
    c = np.concatenate([blobs, rest]).T.astype(np.float32)
    if weights == "ones":
        w = np.ones(n, np.float32)
    else:
        w = rng.uniform(0.5, 1.5, size=n).astype(np.float32)
    return np.ascontiguousarray(c), w


# ---- tolerance parity for kernels whose densities are not bit-exact (exponential, Gaussian) ----
#
# The device sums rho in another order than the reference and evaluates exp on the GPU, so rho
# differs from the restatement's FP32 rho in the last bits.  The rule checked here:
#   1. rho is within rtol relative of the FP64 oracle (points with a candidate within rtol of dc
#      are counted and excluded: their candidate set itself is on a threshold);
#   2. given the device's own densities, every later stage is exact: nearest highers and delta
#      bits equal the restatement's nearest-higher stage run on those densities, seed flags equal
#      the reference's rule on them, and labels equal the seed-rank numbering of the device's
#      own nearest-higher forest;
#   3. against the restatement run end to end on its own FP32 densities, every point whose
#      nearest higher or seed flag differs is a counted near-threshold point (its density within
#      rtol of rhoc, or a candidate whose higher-than relation flips between the two density
#      vectors, each flip a near-tie), and every point whose cluster (identified by its seed)
#      differs has such a point on its chain in one of the two forests.

def _forest_roots(parent):
    """Root of every point in a forest given as parent indices (-1 at roots), by pointer jumping."""
    n = len(parent)
    par = np.where(parent >= 0, parent, np.arange(n)).astype(np.int64)
    while True:
        nxt = par[par]
        if np.array_equal(nxt, par):
            return par
        par = nxt


def _forest_taint(parent, bad):
    """bad OR-ed down the forest: a point is tainted when it or an ancestor is bad."""
    n = len(parent)
    par = np.where(parent >= 0, parent, np.arange(n)).astype(np.int64)
    t = bad.copy()
    while True:
        t2 = t | t[par]
        nxt = par[par]
        if np.array_equal(nxt, par) and np.array_equal(t2, t):
            return t2
        t, par = t2, nxt


def expected_labels(nh_final, is_seed, offsets, seed_capacity, nh_none_count):
    """Labels of the seed-rank numbering (ClusteringKernels.hpp:246-281 with the serial seed
    order) on a given forest: the seed at position c of its event's index-ordered seed list gets
    c when c < the event's SeedArray capacity, every follower its root's label, the rest -1."""
    n = len(nh_final)
    roots = _forest_roots(nh_final)
    lab_root = np.full(n, -1, np.int64)
    for e in range(len(offsets) - 1):
        a, b = int(offsets[e]), int(offsets[e + 1])
        seeds = a + np.nonzero(is_seed[a:b])[0]
        cap = len(seeds) if seed_capacity < 0 else max(seed_capacity, int(nh_none_count[e]))
        kept = seeds[:cap]
        lab_root[kept] = np.arange(len(kept))
    return lab_root[roots].astype(np.int32), roots


def cluster_seed(labels, nh_final):
    """The seed index each point is clustered with (-1 for outliers): its forest root when the
    root carries a label."""
    roots = _forest_roots(nh_final)
    return np.where(labels[roots] >= 0, roots, -1)


def check_tolerant(coords, weight, cfg, got, offsets=None, ref=None, rtol=1e-5, near_counts=None, tag=""):
    """Checks `got` (device outputs: rho, delta, nearest_higher, is_seed, cluster_index; nearest
    highers batch-global) against the restatement by the rule above and returns the counts."""
    c = np.ascontiguousarray(coords, np.float32)
    n = c.shape[1]
    off = np.array([0, n], np.int32) if offsets is None else np.asarray(offsets, np.int32)
    E = len(off) - 1
    # 1. rho against FP64
    rho64, near_dc = O.rho_f64_events(c, weight, off, cfg, rtol)
    rel = np.abs(got.rho.astype(np.float64) - rho64) / np.maximum(np.abs(rho64), 1e-30)
    far = ~near_dc
    max_rel = float(rel[far].max()) if far.any() else 0.0
    assert max_rel <= rtol, (tag, "rho vs FP64", max_rel)
    # 2. later stages exact on the device's own densities
    nh_o, delta_o = O.nearest_higher_events(c, got.rho, off, cfg)
    seed_dc = cfg.dc if cfg.seed_dc is None else cfg.seed_dc
    seeds_exp = ((delta_o > np.float32(seed_dc)) & (got.rho >= np.float32(cfg.rhoc))).astype(np.int32)
    np.testing.assert_array_equal(got.is_seed, seeds_exp, err_msg=f"{tag}: seed rule on device rho")
    np.testing.assert_array_equal(got.nearest_higher, np.where(seeds_exp == 1, -1, nh_o),
                                  err_msg=f"{tag}: nearest higher on device rho")
    np.testing.assert_array_equal(got.delta.view(np.uint32), delta_o.view(np.uint32),
                                  err_msg=f"{tag}: delta on device rho")
    none = np.add.reduceat((nh_o < 0).astype(np.int64), off[:-1]) if n else np.zeros(E, np.int64)
    none[np.diff(off) == 0] = 0
    lab_exp, _ = expected_labels(got.nearest_higher, got.is_seed, off, cfg.seed_capacity, none)
    np.testing.assert_array_equal(got.cluster_index, lab_exp, err_msg=f"{tag}: labels on the device forest")
    # the device's near-threshold counts are the same tests on its own outputs
    if near_counts is not None:
        f32 = np.float32
        has = nh_o >= 0
        assert near_counts["rho_near_rhoc"] == int((np.abs(got.rho - f32(cfg.rhoc)) <= f32(1e-5) * f32(cfg.rhoc)).sum())
        assert near_counts["delta_near_seed_dc"] == int(
            (has & (np.abs(delta_o - f32(seed_dc)) <= f32(1e-5) * f32(seed_dc))).sum())
        dm = cfg.dc if cfg.dm is None else cfg.dm
        assert near_counts["delta_near_dm"] == int((has & (np.abs(delta_o - f32(dm)) <= f32(1e-5) * f32(dm))).sum())
    # 3. against the restatement end to end
    if ref is None:
        ref = O.run_events(c, weight, off, cfg)
    flags, worst = O.near_flags(c, ref.rho, got.rho, ref.delta, cfg, rtol, off)
    decide = (got.nearest_higher != ref.nearest_higher) | (got.is_seed != ref.is_seed)
    explained = (flags & (O.NEAR_RHOC | O.NEAR_FLIP)) != 0
    assert not (decide & ~explained).any(), (tag, "unexplained decision mismatches",
                                            np.nonzero(decide & ~explained)[0][:10])
    assert worst <= 4 * rtol, (tag, "a higher-than flip between densities that are not near-tied", worst)
    seed_got = cluster_seed(got.cluster_index, got.nearest_higher)
    seed_ref = cluster_seed(ref.cluster_index, ref.nearest_higher)
    moved = seed_got != seed_ref
    tainted = _forest_taint(got.nearest_higher, decide) | _forest_taint(ref.nearest_higher, decide)
    assert not (moved & ~tainted).any(), (tag, "cluster changes without a near-threshold cause")
    rep = {"n": int(n), "events": int(E), "max_rel_rho_vs_f64": max_rel, "near_dc": int(near_dc.sum()),
           "near_rhoc": int(((flags & O.NEAR_RHOC) != 0).sum()), "near_flip": int(((flags & O.NEAR_FLIP) != 0).sum()),
           "near_tie": int(((flags & O.NEAR_TIE) != 0).sum()),
           "near_seed_dc": int(((flags & O.NEAR_SEED_DC) != 0).sum()),
           "near_dm": int(((flags & O.NEAR_DM) != 0).sum()), "max_flip_rel_gap": worst,
           "decision_mismatch": int(decide.sum()), "cluster_mismatch": int(moved.sum()),
           "label_mismatch": int((got.cluster_index != ref.cluster_index).sum()),
           "rho_not_bitexact": int((got.rho.view(np.uint32) != ref.rho.view(np.uint32)).sum()),
           "clusters_gpu": int((got.cluster_index.max(initial=-1) + 1) if E == 1 else -1),
           "clusters_ref": int(ref.stats["n_clusters"])}
    print(f"tolerance parity {tag}: {rep}")
    return rep
