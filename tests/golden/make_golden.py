"""Extracts the fixtures the reference's own tests read, as compact .npz files.

Run in a checkout that has the reference tree next to it:

    python tests/golden/make_golden.py /path/to/CLUEstering

Coordinates and weights are parsed to float32 as the reference's read_csv does
(std::stof, utils/detail/read_csv.hpp:21-66). Truth files keep their
`cluster_ids`/`is_seed` columns. The tests read only these .npz files.
"""

import os
import sys

import numpy as np
import pandas as pd

FILES = {
    # name: (csv relative to the reference's data/, ndim)
    "data_1024": ("data_1024.csv", 2),
    "data_4096": ("data_4096.csv", 2),
    "data_16384": ("data_16384.csv", 2),
    "data_32768": ("data_32768.csv", 2),
    "batched_data_1024": ("batched_data_1024.csv", 2),
    "opposite_angles": ("opposite_angles.csv", 2),
    "toyDetector_1000": ("toyDetector_1000.csv", 2),
    "sissa_1000": ("sissa_1000.csv", 2),
    "blob": ("blob.csv", 3),
}
TRUTH = ["data_1024", "data_2048", "data_4096", "data_8192", "data_16384", "data_32768", "data_65536"]


def load(path, ndim):
    df = pd.read_csv(path)
    cols = list(df.columns[:ndim])  # read_csv takes the first ndim columns
    coords = np.stack([df[c].to_numpy(np.float64).astype(np.float32) for c in cols])
    return coords, df["weight"].to_numpy(np.float64).astype(np.float32)


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    data = os.path.join(ref, "data")
    for name, (csv, ndim) in FILES.items():
        c, w = load(os.path.join(data, csv), ndim)
        np.savez_compressed(os.path.join(here, name + ".npz"), coords=c, weights=w)
    counts = {}
    for name in TRUTH:
        t = pd.read_csv(os.path.join(data, "truth_files", name + "_truth.csv"))
        counts[name] = int(t["cluster_ids"].max()) + 1
    t = pd.read_csv(os.path.join(data, "truth_files", "data_1024_truth.csv"))
    np.savez_compressed(os.path.join(here, "truth_data_1024.npz"),
                        cluster_ids=t["cluster_ids"].to_numpy(np.int32),
                        is_seed=t["is_seed"].to_numpy(np.int32))
    np.savez(os.path.join(here, "truth_counts.npz"), names=np.array(list(counts)),
             counts=np.array(list(counts.values()), np.int32))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/CLUEstering")
    main(sys.argv[1])
