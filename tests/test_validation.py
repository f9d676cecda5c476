"""Cluster centroids and silhouette scores (utils/detail/cluster_centroid.hpp,
utils/detail/scores.hpp).

The device functions add in the reference's order (points of a cluster in
ascending index order), so centroids and per-point silhouettes must equal the
CPU checker's bit for bit. The mean silhouette is the reference's std::reduce
over the per-point scores, whose grouping of the additions is the standard
library's; it is compared within 1e-6 relative.
"""

import numpy as np
import pytest

import cluestering_b200 as clue
from cluestering_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import fixture, silhouette as silhouette_f64

MEAN_RTOL = 1e-6


def _labels(coords, weights, prm, **kw):
    r = O.make_clusters(coords, weights, *prm, **kw)
    return r.cluster_index, int(r.cluster_index.max()) + 1


# ---- the checker against plain float64 definitions (no GPU) -----------------------------------

@pytest.mark.parametrize("name,prm", [("data_1024", (1.3, 10.0, 1.3)), ("blob", (1.5, 3.0, 2.0))])
def test_checker_silhouette_matches_the_float64_definition(name, prm):
    c, w = fixture(name)
    lab, k = _labels(c, w, prm)
    s = O.silhouette(c, lab, k)
    keep = ~np.isnan(s)
    # points skipped: outliers and clusters of one point (scores.hpp:83-88)
    sizes = np.bincount(lab[lab >= 0], minlength=k)
    assert np.array_equal(keep, (lab >= 0) & (sizes[np.maximum(lab, 0)] >= 2))
    assert np.mean(s[keep].astype(np.float64)) == pytest.approx(silhouette_f64(c, lab), rel=1e-5)


def test_checker_centroids_match_float64_means():
    c, w = fixture("data_1024")
    lab, k = _labels(c, w, (1.3, 10.0, 1.3))
    cen = O.centroids(c, w, lab, k)
    wcen = O.centroids(c, w, lab, k, weighted=True)
    for j in range(k):
        m = lab == j
        ref = c[:, m].astype(np.float64).mean(axis=1)
        wref = (c[:, m].astype(np.float64) * w[m]).sum(axis=1) / w[m].astype(np.float64).sum()
        assert np.allclose(cen[j], ref, rtol=1e-5, atol=1e-4)
        assert np.allclose(wcen[j], wref, rtol=1e-5, atol=1e-4)


# ---- the device functions against the checker ---------------------------------------------------

def _device_case(ev, prm, kernel=None):
    import torch
    dev = torch.device("cuda", 0)
    pts = clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev))
    algo = clue.Clusterer(*prm)
    algo.make_clusters(pts, clue.EuclideanMetric(), kernel or clue.FlatKernel(0.5))
    lab = pts.cluster_index.cpu().numpy()
    return pts, algo, lab, algo.n_clusters()


CASES = [
    ("single_2d", lambda: W.single_2d(4096, seed=81), (1.5, 5.0, 1.5), None),
    ("exp_weights", lambda: W.blobs(6000, 8, 0.0, 60.0, 1.0, 0.1, seed=82, weights="exponential"),
     (1.5, 3.0, 2.0), None),
    ("layered_3d", lambda: W.layered_3d(5000, seed=83), (3.0, 10.0, 4.0), "gauss"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,prm,kern", CASES)
def test_device_centroids_equal_the_checker(name, make, prm, kern):
    ev = make()
    pts, algo, lab, k = _device_case(ev, prm, clue.GaussianKernel(1.0, 1.0) if kern else None)
    assert k >= 2
    for weighted in (False, True):
        got = clue.cluster_centroids(pts, algo, weighted=weighted)
        ref = O.centroids(ev.coords, ev.weights, lab, k, weighted=weighted)
        assert got.shape == (k, ev.ndim)
        assert np.array_equal(got.view(np.int32), ref.view(np.int32)), (name, weighted)


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,prm,kern", CASES)
def test_device_silhouette_equals_the_checker(name, make, prm, kern):
    ev = make()
    pts, algo, lab, k = _device_case(ev, prm, clue.GaussianKernel(1.0, 1.0) if kern else None)
    got = clue.silhouette_scores(pts, algo)
    ref = O.silhouette(ev.coords, lab, k)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    keep = ~np.isnan(ref)
    assert np.array_equal(got[keep].view(np.int32), ref[keep].view(np.int32)), name
    mean = clue.silhouette(pts, algo)
    assert mean == pytest.approx(float(np.mean(ref[keep].astype(np.float64))), rel=MEAN_RTOL)
    i = int(np.nonzero(keep)[0][0])
    assert clue.silhouette(pts, algo, i) == float(ref[i])


@pytest.mark.gpu
def test_reference_silhouette_threshold_on_data_1024():
    # tests/test_clustering.cpp:14-36 asks for a silhouette of at least 0.9 on data_1024
    import torch
    c, w = fixture("data_1024")
    dev = torch.device("cuda", 0)
    pts = clue.PointsDevice(torch.from_numpy(c).to(dev), torch.from_numpy(w).to(dev))
    algo = clue.Clusterer(1.3, 10.0, 1.3)
    algo.make_clusters(pts)
    assert clue.silhouette(pts, algo) >= 0.9


def test_device_utilities_need_clustered_device_points():
    c, w = fixture("data_1024")
    with pytest.raises(TypeError):
        clue.cluster_centroids(clue.PointsHost(c, w), clue.Clusterer(1.3, 10.0, 1.3))
