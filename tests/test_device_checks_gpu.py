"""The build with device bounds checks (libclue_b200_checked.so, CLUE_DEVICE_CHECKS): every
index the pipeline reads from its own data is tested before it addresses memory, a bad one is
recorded (no trap) and reported as an error after the run.  On valid inputs no check may fire,
and the checked build must give the default build's outputs bit for bit: the flat-kernel plain
path, an exponential-kernel batch through the overlapped host path, a 1-D density ramp whose
label chains outlast the enqueued pointer-jumping rounds, and the 3-D Gaussian symmetric sweep.
The checked library is loaded in a child process (CLUE_B200_LIB)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "cluestering_alpaka3_b200", "libclue_b200_checked.so")

CASES = r'''
import sys, numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/tests")
from cluestering_alpaka3_b200 import capi, synthetic
from parity_util import gpu_args, random_blobs
ctx = capi.Context(0)
out = {}
g = np.load(ROOT + "/tests/golden/data_4096.npz")
dc, rhoc, dm = (float(v) for v in g["params"])
r = ctx.make_clusters_host(g["coords"], g["weight"], *gpu_args(dc=dc, rhoc=rhoc, dm=dm))
out["flat"] = r
evs, p = synthetic.calo_events(1400, seed=4321)
off = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in evs])]).astype(np.int32)
c = np.ascontiguousarray(np.concatenate([e[0] for e in evs], axis=1))
w = np.ascontiguousarray(np.concatenate([e[1] for e in evs]))
ctx.set_tuning(overlap_chunk_points=400000)
r, _ = ctx.batch_host(c, w, off, *gpu_args(dc=p["dc"], rhoc=p["rhoc"], dm=p["dm"], kernel=p["kernel"]))
out["batch_exp"] = r
x = (np.sqrt(np.linspace(0.0, 1.0, 30000)) * 800.0).astype(np.float32)[None, :].copy()
r = ctx.make_clusters_host(x, np.ones(30000, np.float32), *gpu_args(dc=0.2, rhoc=1.0, dm=0.5))
out["deep"] = r
rng = np.random.default_rng(8)
c3, w3 = random_blobs(rng, 20000, 3, nblobs=10, extent=40.0)
r = ctx.make_clusters_host(c3, w3, *gpu_args(dc=1.2, rhoc=4.0, dm=2.0, kernel=("gaus", (0.0, 0.5, 1.0))))
out["gauss3d"] = r
arrays = {f"{k}.{f}": getattr(v, f) for k, v in out.items()
          for f in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta")}
np.savez(OUT, **arrays)
ctx.close()
'''


def _run(lib, path):
    env = dict(os.environ)
    if lib:
        env["CLUE_B200_LIB"] = lib
    else:
        env.pop("CLUE_B200_LIB", None)
    code = f"ROOT = {ROOT!r}\nOUT = {path!r}\n" + CASES
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(path)


def test_checked_build_matches_default_build(gpu_context, tmp_path):
    assert os.path.exists(CHECKED), "libclue_b200_checked.so is not built (make -C cluestering_alpaka3_b200)"
    checked = _run(CHECKED, str(tmp_path / "checked.npz"))
    default = _run(None, str(tmp_path / "default.npz"))
    assert sorted(checked.files) == sorted(default.files)
    for k in checked.files:
        np.testing.assert_array_equal(checked[k].view(np.uint32), default[k].view(np.uint32), err_msg=k)
