"""The checker against the reference itself.

oracle/_ref/libclue_ref.so is CLUEstering's unmodified make_clusters compiled
on its serial CPU backend (`make -C oracle ref`; oracle/ref.py). Every output of
the C restatement (oracle.py) must equal it bit for bit on the same inputs:
densities as bits, nearest-higher indices, seed flags and cluster ids. The
restatement evaluates the exponential with libm here (EXP_LIBM), as the
reference's serial backend does (std::exp, internal/math/exp/exp.hpp:19-29).
"""

import math

import numpy as np
import pytest

from cluestering_b200 import workloads as W
from oracle import oracle as O
from oracle import ref as R
from tests.helpers import fixture

pytestmark = pytest.mark.skipif(not R.available(),
                                reason="the reference build (make -C oracle ref) is not present")


def same(coords, weights, *args, sizes=None, shared_grid=True, **kw):
    if sizes is None:
        r = R.make_clusters(coords, weights, *args, **kw)
        o = O.make_clusters(coords, weights, *args, exp_mode=O.EXP_LIBM, n_threads=4, **kw)
    else:
        r = R.make_clusters_batched(coords, weights, sizes, *args, **kw)
        o = O.make_clusters_batched(coords, weights, sizes, *args, shared_grid=shared_grid,
                                    exp_mode=O.EXP_LIBM, n_threads=4, **kw)
    assert np.array_equal(r.rho.view(np.int32), o.rho.view(np.int32)), \
        f"rho differs at {np.nonzero(r.rho.view(np.int32) != o.rho.view(np.int32))[0][:10]}"
    assert np.array_equal(r.nearest_higher, o.nearest_higher), \
        f"nearest higher differs at {np.nonzero(r.nearest_higher != o.nearest_higher)[0][:10]}"
    assert np.array_equal(r.is_seed, o.is_seed)
    assert np.array_equal(r.cluster_index, o.cluster_index)
    return r


def test_single_2d_event():
    ev = W.single_2d()
    assert same(ev.coords, ev.weights, 1.5, 5.0, 1.5).n_clusters >= 15


def test_large_2d_event_exponential_weights_reduced():
    ev = W.blobs(1 << 17, 250, 0.0, 353.0, 1.0, 0.1, seed=9, weights="exponential")
    same(ev.coords, ev.weights, 1.5, 8.0, 2.0)


def test_layered_3d_gaussian_kernel():
    ev = W.layered_3d()
    same(ev.coords, ev.weights, 3.0, 10.0, 4.0, kernel="gaussian", kernel_params=(1.0, 1.0))


def test_exponential_kernel():
    ev = W.blobs(20000, 24, 0.0, 100.0, 1.0, 0.1, seed=4, weights="exponential")
    same(ev.coords, ev.weights, 1.5, 5.0, 1.5, kernel="exponential", kernel_params=(1.0, 1.0))


def test_batched_form_one_grid_for_the_batch():
    ev, sizes = W.batch_2d(48, 256, 8192, seed=5)
    w = np.random.default_rng(7).exponential(1.0, ev.n).astype(np.float32)
    same(ev.coords, w, 1.5, 5.0, 1.5, sizes=sizes)


def test_reference_datasets():
    for name in ("data_4096", "data_32768"):
        c, w = fixture(name)
        same(c, w, 1.5, 10.0, 1.5)
    c, w = fixture("batched_data_1024")
    same(c, w, 1.3, 10.0, 1.3, sizes=[1024] * 10)


@pytest.mark.parametrize("metric,params", [
    ("weighted_euclidean", (1.0, 2.0)), ("manhattan", ()), ("chebyshev", ()),
    ("weighted_chebyshev", (0.5, 1.5)),
])
def test_metrics(metric, params):
    ev = W.blobs(8000, 12, 0.0, 60.0, 1.0, 0.1, seed=13, weights="exponential")
    same(ev.coords, ev.weights, 1.5, 4.0, 2.0, metric=metric, metric_params=params)


def test_periodic_coordinates():
    c, w = fixture("opposite_angles")
    two_pi = float(np.float32(2.0) * np.float32(math.pi))
    r = same(c, w, 0.2, 5.0, 0.2, wrapped=[0, 1], metric="periodic_euclidean", metric_params=(0.0, two_pi))
    assert r.n_clusters == 1


def test_sigma_uncertainty_and_tags():
    rng = np.random.default_rng(17)
    ev = W.blobs(6000, 10, 0.0, 50.0, 1.0, 0.1, seed=17, weights="exponential")
    sig = [rng.uniform(0.1, 0.8, ev.n).astype(np.float32), rng.uniform(0.1, 0.8, ev.n).astype(np.float32)]
    same(ev.coords, ev.weights, 1.0, 3.0, 1.5, sigma=sig)
    same(ev.coords, ev.weights, 1.0, 3.0, 1.5, sigma=sig, metric="mahalanobis")
    same(ev.coords, ev.weights, 1.0, 3.0, 1.5, unc=rng.uniform(0.5, 1.5, ev.n).astype(np.float32))
    same(ev.coords, ev.weights, 1.0, 3.0, 1.5, tags=rng.permutation(ev.n))


def test_tag_tie_break():
    coords = np.array([[0.0, 0.0], [0.0, 0.0]], np.float32)
    r = same(coords, np.ones(2, np.float32), 1.0, 0.0, 1.0)
    assert r.nearest_higher.tolist() == [1, -1]
    r = same(coords, np.ones(2, np.float32), 1.0, 0.0, 1.0, tags=np.array([100, 1]))
    assert r.nearest_higher.tolist() == [-1, 0]


def test_seeding_distance_differs_from_outlier_distance():
    ev = W.single_2d(6000, seed=19)
    same(ev.coords, ev.weights, 1.5, 5.0, 3.0, 0.7)


@pytest.mark.parametrize("ndim", [1, 3, 4])
def test_dimensions(ndim):
    rng = np.random.default_rng(20 + ndim)
    coords = rng.normal(0.0, 2.0, (ndim, 3000)).astype(np.float32)
    w = rng.exponential(1.0, 3000).astype(np.float32)
    same(coords, w, 0.8, 2.0, 1.0)


def test_lattice_ties():
    g = np.arange(60, dtype=np.float32) * np.float32(0.1)
    xx, yy = np.meshgrid(g, g, indexing="ij")
    coords = np.stack([xx.ravel(), yy.ravel()]).astype(np.float32)
    same(coords, np.ones(coords.shape[1], np.float32), 0.15, 3.0, 0.15)
    g3 = np.arange(14, dtype=np.float32) * np.float32(0.1)
    xx, yy, zz = np.meshgrid(g3, g3, g3, indexing="ij")
    c3 = np.stack([xx.ravel(), yy.ravel(), zz.ravel()]).astype(np.float32)
    c3 = np.concatenate([c3, c3[:, ::7]], axis=1)
    same(c3, np.ones(c3.shape[1], np.float32), 0.15, 4.0, 0.25)
