"""Shared test helpers: fixture loading and the reference's silhouette score."""

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z["coords"], z["weights"]


def truth_count(name):
    z = np.load(os.path.join(GOLDEN, "truth_counts.npz"))
    return int(dict(zip(z["names"].tolist(), z["counts"].tolist()))[name])


def silhouette(coords, labels):
    """utils/detail/scores.hpp:33-100: mean over clustered points of clusters
    with >= 2 points of (b - a) / max(a, b), a = mean intra-cluster distance
    (excluding the point), b = smallest mean distance to another cluster."""
    X = np.asarray(coords, np.float64).T
    lab = np.asarray(labels)
    ids = np.unique(lab[lab >= 0])
    sizes = {c: int((lab == c).sum()) for c in ids}
    members = {c: X[lab == c] for c in ids}
    scores = []
    for i in np.nonzero(lab >= 0)[0]:
        c = lab[i]
        if sizes[c] < 2:
            continue
        d_own = np.sqrt(((members[c] - X[i]) ** 2).sum(1))
        a = d_own.sum() / (sizes[c] - 1)
        b = min(np.sqrt(((members[o] - X[i]) ** 2).sum(1)).mean() for o in ids if o != c) \
            if len(ids) > 1 else np.finfo(np.float32).max
        scores.append((b - a) / max(a, b))
    return float(np.mean(scores))


def same_partition(a, b):
    """Identical up to relabelling, with outliers (-1) fixed."""
    a, b = np.asarray(a), np.asarray(b)
    if ((a == -1) != (b == -1)).any():
        return False
    m = a >= 0
    pairs = set(zip(a[m].tolist(), b[m].tolist()))
    return len(pairs) == len(set(a[m].tolist())) == len(set(b[m].tolist()))
