"""Regenerate the golden fixtures of tests/golden/ from the reference's own data files.

Reads the reference's data/*.csv inputs and data/truth_files/*_truth.csv outputs
(cluster_ids, is_seed per point) and stores them as compact .npz files, float32
coordinates parsed like the reference's read_csv (utils/detail/read_csv.hpp:18-49).
Run from the repository root with REFERENCE_ROOT naming the reference checkout:
  REFERENCE_ROOT=<path to CLUEstering_alpaka3> python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np
import pandas as pd

REF = os.environ.get("REFERENCE_ROOT")
if not REF:
    sys.exit("set REFERENCE_ROOT to the reference checkout (the directory holding data/)")
OUT = os.path.dirname(os.path.abspath(__file__))

# (input csv, truth csv, ndim, parameters used by the reference's own tests for that file)
CASES = [
    ("data_1024.csv", "data_1024_truth.csv", 2, (1.5, 10.0, 1.5)),
    ("data_2048.csv", "data_2048_truth.csv", 2, (1.5, 10.0, 1.5)),
    ("data_4096.csv", "data_4096_truth.csv", 2, (1.5, 10.0, 1.5)),
    ("data_8192.csv", "data_8192_truth.csv", 2, (1.5, 10.0, 1.5)),
    ("data_16384.csv", "data_16384_truth.csv", 2, (1.5, 10.0, 1.5)),
    ("data_32768.csv", "data_32768_truth.csv", 2, (1.3, 10.0, 1.3)),
    ("blob.csv", "blobs_truth.csv", 3, (1.0, 5.0, 2.0)),
    ("sissa_1000.csv", "sissa_1000_truth.csv", 2, (20.0, 10.0, 20.0)),
    ("toyDetector_1000.csv", "toy_det_1000_truth.csv", 2, (4.0, 2.5, 4.0)),
    ("aniso_1000.csv", "aniso_1000_truth.csv", 2, (28.0, 5.0, 28.0)),
]


def main():
    for inp, truth, ndim, (dc, rhoc, dm) in CASES:
        df = pd.read_csv(os.path.join(REF, "data", inp), dtype=str)
        coords = np.stack([np.array(df.iloc[:, d].tolist(), dtype=np.float32) for d in range(ndim)])
        weight = np.array(df.iloc[:, ndim].tolist(), dtype=np.float32)
        t = pd.read_csv(os.path.join(REF, "data", "truth_files", truth))
        name = os.path.splitext(inp)[0]
        np.savez_compressed(os.path.join(OUT, name + ".npz"), coords=coords, weight=weight,
                            truth_cluster_ids=t["cluster_ids"].to_numpy(np.int32),
                            truth_is_seed=t["is_seed"].to_numpy(np.int8),
                            params=np.array([dc, rhoc, dm], np.float32))
        print("wrote", name, coords.shape)


if __name__ == "__main__":
    sys.exit(main())
