"""Pins the CPU checker (oracle/) to the reference's own tests and fixtures.

Each case restates a CLUEstering test (file:line in the CLUEstering tree) on
the fixtures extracted into tests/golden/.
"""

import math
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import fixture, same_partition, silhouette, truth_count


def test_tag_tie_break_without_tags():
    # tests/test_clustering.cpp:541-551: two coincident unit-weight points;
    # on equal density the higher index is "higher".
    coords = np.array([[0.0, 0.0], [0.0, 0.0]], np.float32)
    r = O.make_clusters(coords, np.ones(2, np.float32), 1.0, 0.0, 1.0)
    assert r.nearest_higher.tolist() == [1, -1]
    assert r.is_seed.tolist() == [0, 1]


def test_tag_tie_break_with_tags():
    # tests/test_clustering.cpp:553-566: tags {100, 1} reverse the order.
    coords = np.array([[0.0, 0.0], [0.0, 0.0]], np.float32)
    r = O.make_clusters(coords, np.ones(2, np.float32), 1.0, 0.0, 1.0, tags=np.array([100, 1]))
    assert r.nearest_higher.tolist() == [-1, 0]
    assert r.is_seed.tolist() == [1, 0]


def test_mahalanobis_sigma_merges():
    # tests/test_mahalanobis.cpp:11-43
    coords = np.array([[2.0, 4.0]], np.float32)
    w = np.ones(2, np.float32)
    assert O.make_clusters(coords, w, 1.0, 0.3).n_clusters == 2
    sig = [np.array([2.0, 2.0], np.float32)]
    assert O.make_clusters(coords, w, 1.0, 0.3, sigma=sig, metric="mahalanobis").n_clusters == 1


def test_periodic_coordinates_single_cluster():
    # tests/test_clustering.cpp:237-253
    c, w = fixture("opposite_angles")
    two_pi = np.float32(2.0) * np.float32(math.pi)
    r = O.make_clusters(c, w, 0.2, 5.0, 0.2, wrapped=[0, 1], metric="periodic_euclidean",
                        metric_params=[0.0, float(two_pi)])
    assert r.n_clusters == 1


def test_batched_fixed_batch_size():
    # tests/test_batched_clustering.cpp:51-77: 10 copies of data_1024 in one
    # batch give 10x the truth's cluster count; the sample associator has 10 keys.
    c, w = fixture("batched_data_1024")
    r = O.make_clusters_batched(c, w, [1024] * 10, 1.3, 10.0, 1.3)
    assert r.n_clusters == 10 * truth_count("data_1024")
    assert int(r.event_associations.max()) + 1 == 10


@pytest.mark.parametrize("name", ["data_1024", "data_4096", "data_16384", "data_32768"])
def test_benchmark_datasets_silhouette(name):
    # tests/test_clustering.cpp:14-38 (dc=1.5, rhoc=10, dm=1.5, silhouette >= 0.9)
    c, w = fixture(name)
    r = O.make_clusters(c, w, 1.5, 10.0, 1.5, n_threads=4)
    assert silhouette(c, r.cluster_index) >= 0.9


def test_clusterer_overload_dataset_silhouette():
    # tests/test_clusterer.cpp:13-44 (data_32768, dc=1.3, rhoc=10, dm=1.3)
    c, w = fixture("data_32768")
    r = O.make_clusters(c, w, 1.3, 10.0, 1.3, n_threads=4)
    assert silhouette(c, r.cluster_index) >= 0.9


@pytest.mark.parametrize("name,params,threshold,ndim", [
    ("toyDetector_1000", (4.0, 2.5, 4.0), 0.8, 2),   # tests/test_clustering.cpp:167-200
    ("sissa_1000", (20.0, 10.0, 20.0), 0.5, 2),      # :97-113
    ("blob", (1.0, 5.0, 2.0), 0.8, 3),               # :202-235
])
def test_named_datasets_silhouette(name, params, threshold, ndim):
    c, w = fixture(name)
    assert c.shape[0] == ndim
    r = O.make_clusters(c, w, *params)
    assert silhouette(c, r.cluster_index) >= threshold


@pytest.mark.parametrize("name", ["data_1024", "data_4096", "data_16384", "data_32768"])
def test_truth_file_cluster_counts(name):
    # data/truth_files/*_truth.csv: their generating parameters are not recorded;
    # the cluster count is what they pin (tests/check_result.py:5-25 compares counts
    # and sizes; per-point labels differ from every current parameter set).
    c, w = fixture(name)
    assert O.make_clusters(c, w, 1.3, 10.0, 1.3).n_clusters == truth_count(name)
    assert O.make_clusters(c, w, 1.5, 10.0, 1.5).n_clusters == truth_count(name)


def test_invalid_parameters_rejected():
    # tests/test_clusterer.cpp:46-56
    c = np.zeros((2, 4), np.float32)
    w = np.ones(4, np.float32)
    for dc, rhoc in [(-1.0, 10.0), (1.0, -10.0)]:
        with pytest.raises(ValueError):
            O.make_clusters(c, w, dc, rhoc)


def _f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def _ulps(a, b):
    ia = struct.unpack("i", struct.pack("f", a))[0]
    ib = struct.unpack("i", struct.pack("f", b))[0]
    return abs(ia - ib)


def test_clue_expf_error_at_most_one_ulp():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-87.0, 88.0, 20000), rng.uniform(-1.0, 1.0, 5000),
                         np.linspace(-20, 0, 2001)]).astype(np.float32)
    worst = 0
    for x in xs.tolist():
        exact = _f32(math.exp(x))
        got = O.expf(x)
        worst = max(worst, _ulps(got, exact))
    assert worst <= 1


def test_clue_expf_special_values():
    assert O.expf(0.0) == 1.0
    assert O.expf(float("inf")) == float("inf")
    assert O.expf(-float("inf")) == 0.0
    assert math.isnan(O.expf(float("nan")))
    assert O.expf(89.0) == float("inf")
    assert O.expf(-110.0) == 0.0
    # subnormal results are rounded once
    assert abs(O.expf(-100.0) - _f32(math.exp(-100.0))) <= 2 ** -149


def _exp_cases():
    from cluestering_b200 import workloads as W
    gauss = dict(dc=3.0, rhoc=10.0, dm=4.0, kernel="gaussian", kernel_params=(1.0, 1.0))
    yield "layered_3d_10000", W.layered_3d(), gauss
    yield "layered_3d_262144", W.layered_3d(262144, seed=11), gauss
    yield "blobs_2d_exponential_kernel", \
        W.blobs(1 << 15, 40, 0.0, 100.0, 1.0, 0.1, seed=4, weights="exponential"), \
        dict(dc=1.5, rhoc=5.0, dm=1.5, kernel="exponential", kernel_params=(1.0, 1.0))


@pytest.mark.parametrize("case", ["layered_3d_10000", "layered_3d_262144", "blobs_2d_exponential_kernel"])
def test_exp_choice_keeps_nearest_higher_and_partitions(case):
    # The GPU path and this checker evaluate the Gaussian and exponential
    # kernels with clue_expf; the reference's serial backend calls libm's
    # std::exp (internal/math/exp/exp.hpp:19-29). The two differ in the last
    # bit of some exponentials, so densities may differ within the 1e-5
    # relative tolerance, while nearest-higher indices, seed flags and the
    # partition must come out identical.
    ev, prm = next((e, p) for name, e, p in _exp_cases() if name == case)
    threads = min(8, os.cpu_count() or 1)
    a = O.make_clusters(ev.coords, ev.weights, exp_mode=O.EXP_CLUE, n_threads=threads, **prm)
    b = O.make_clusters(ev.coords, ev.weights, exp_mode=O.EXP_LIBM, n_threads=threads, **prm)
    np.testing.assert_allclose(a.rho, b.rho, rtol=1e-5)
    assert np.array_equal(a.nearest_higher, b.nearest_higher)
    assert np.array_equal(a.is_seed, b.is_seed)
    assert same_partition(a.cluster_index, b.cluster_index)
    assert a.n_clusters > 0


def test_shared_and_per_event_grids_agree_on_exact_sums():
    # Unit weights with the flat kernel: every partial density is a multiple of
    # 0.5, so the summation order (the grid) cannot change any result.
    c, w = fixture("batched_data_1024")
    a = O.make_clusters_batched(c, w, [1024] * 10, 1.3, 10.0, 1.3, shared_grid=True)
    b = O.make_clusters_batched(c, w, [1024] * 10, 1.3, 10.0, 1.3, shared_grid=False)
    assert np.array_equal(a.rho, b.rho)
    assert np.array_equal(a.nearest_higher, b.nearest_higher)
    assert np.array_equal(a.cluster_index, b.cluster_index)


def test_per_event_grid_equals_events_alone():
    from cluestering_b200 import workloads as W
    ev, sizes = W.batch_2d(6, 256, 3000, seed=11)
    r = O.make_clusters_batched(ev.coords, ev.weights, sizes, 1.5, 5.0, 1.5, shared_grid=False)
    begin, label0 = 0, 0
    for s in sizes.tolist():
        one = O.make_clusters(ev.coords[:, begin:begin + s], ev.weights[begin:begin + s], 1.5, 5.0, 1.5)
        assert np.array_equal(r.rho[begin:begin + s], one.rho)
        nh = one.nearest_higher
        assert np.array_equal(r.nearest_higher[begin:begin + s], np.where(nh >= 0, nh + begin, -1))
        ci = one.cluster_index
        assert np.array_equal(r.cluster_index[begin:begin + s], np.where(ci >= 0, ci + label0, -1))
        begin += s
        label0 += one.n_clusters


def test_threads_do_not_change_results():
    c, w = fixture("data_16384")
    a = O.make_clusters(c, w, 1.5, 10.0, 1.5, n_threads=1)
    b = O.make_clusters(c, w, 1.5, 10.0, 1.5, n_threads=4)
    assert np.array_equal(a.rho, b.rho) and np.array_equal(a.cluster_index, b.cluster_index)
    assert same_partition(a.cluster_index, b.cluster_index)
