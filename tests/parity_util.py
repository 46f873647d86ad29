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


def tolerance_report(rho_gpu, rho_ref32, coords, weight, cfg, labels_gpu, labels_ref, rtol=1e-5):
    """rho within rtol of FP64 except at points whose candidates sit within rtol of dc (counted);
    returns a dict with the counts the tests assert on and report."""
    rho64, near = O.rho_f64(coords, weight, cfg, rel_tol=rtol, with_near=True)
    rel = np.abs(rho_gpu.astype(np.float64) - rho64) / np.maximum(np.abs(rho64), 1e-30)
    rel32 = np.abs(rho_ref32.astype(np.float64) - rho64) / np.maximum(np.abs(rho64), 1e-30)
    rhoc = cfg.rhoc
    near_rhoc = np.abs(rho64 - rhoc) <= rtol * max(rhoc, 1e-30)
    mism = labels_gpu != labels_ref
    return {"max_rel_far": float(rel[~near].max()) if (~near).any() else 0.0,
            "max_rel_far_oracle32": float(rel32[~near].max()) if (~near).any() else 0.0,
            "near_dc": int(near.sum()), "near_rhoc": int(near_rhoc.sum()),
            "rho_not_bitexact": int((rho_gpu.view(np.uint32) != rho_ref32.view(np.uint32)).sum()),
            "label_mismatch": int(mism.sum()), "n": len(rho_gpu)}
