"""The tolerance-parity rule itself, on the CPU: a stand-in for the device built from the
restatement with densities rounded from FP64 (another summation order, as the device's), and the
same stand-in with a planted wrong nearest higher, which the rule must reject."""
import copy
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import oracle as O
from parity_util import check_tolerant, expected_labels, random_blobs


def _stand_in(c, w, cfg, off):
    """Outputs of a pipeline whose densities are the FP64 sums rounded to FP32: every later
    stage is the restatement's on those densities."""
    rho64, _ = O.rho_f64_events(c, w, off, cfg)
    rho = rho64.astype(np.float32)
    nh, delta = O.nearest_higher_events(c, rho, off, cfg)
    seed_dc = cfg.dc if cfg.seed_dc is None else cfg.seed_dc
    is_seed = ((delta > np.float32(seed_dc)) & (rho >= np.float32(cfg.rhoc))).astype(np.int32)
    nh_final = np.where(is_seed == 1, -1, nh).astype(np.int32)
    none = np.array([(nh[off[e]:off[e + 1]] < 0).sum() for e in range(len(off) - 1)])
    lab, _ = expected_labels(nh_final, is_seed, off, cfg.seed_capacity, none)
    return SimpleNamespace(rho=rho, delta=delta, nearest_higher=nh_final, is_seed=is_seed, cluster_index=lab)


@pytest.mark.parametrize("kernel", [("exp", (1.0, 1.0)), ("gaus", (0.0, 0.5, 1.0))])
def test_rule_accepts_rounding_differences(kernel):
    rng = np.random.default_rng(3)
    c, w = random_blobs(rng, 6000, 2, nblobs=10, extent=60.0, sigma=1.0, weights="ones")
    cfg = O.Config(dc=2.0, rhoc=4.0, dm=3.0, kernel=kernel[0], kernel_par=kernel[1], nthreads=4)
    off = np.array([0, 2500, 6000], np.int32)
    got = _stand_in(c, w, cfg, off)
    rep = check_tolerant(c, w, cfg, got, offsets=off, tag="stand-in")
    assert rep["rho_not_bitexact"] > 0  # the stand-in really differs from the FP32 sums


def test_rule_rejects_a_wrong_nearest_higher():
    rng = np.random.default_rng(4)
    c, w = random_blobs(rng, 4000, 2, nblobs=8, extent=50.0, sigma=1.0)
    cfg = O.Config(dc=2.0, rhoc=4.0, dm=3.0, kernel="exp", kernel_par=(1.0, 1.0), nthreads=4)
    off = np.array([0, 4000], np.int32)
    got = _stand_in(c, w, cfg, off)
    bad = copy.deepcopy(got)
    i = int(np.nonzero(bad.nearest_higher >= 0)[0][100])
    bad.nearest_higher[i] = int(np.nonzero(bad.is_seed)[0][0]) if bad.nearest_higher[i] != np.nonzero(bad.is_seed)[0][0] else -1
    with pytest.raises(AssertionError):
        check_tolerant(c, w, cfg, bad, offsets=off, tag="planted")
