"""The drop-in modules for CLUEstering's Python wrapper (cluestering_b200/compat).

mainRun must take the wrapper's arguments as CLUEstering.py passes them
(CLUEstering.py:640-659: dc, rhoc, dm, seed_dc, wrapped, the (Ndim + 1, n)
data array, the int32 results array, kernel, Ndim, batch sizes, n_points,
device id, metric descriptor) and fill `results` with the cluster ids the
reference computes; the GPU cases compare against the CPU checker bit for bit.
"""

import math
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import fixture

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "cluestering_b200", "compat"))
import CLUE_Convolutional_Kernels as clue_kernels  # noqa: E402
import CLUE_GPU_CUDA as gpu_cuda  # noqa: E402


def _wrapper_arrays(coords, weights):
    # CLUEstering.py:297-309: coordinates stacked over the weights, float32 SoA
    data = np.ascontiguousarray(np.vstack([coords, weights[None, :]]), dtype=np.float32)
    return data, np.zeros(coords.shape[1], np.int32)


# ---- host-side behaviour (no GPU) ---------------------------------------------------------------

def test_kernel_constructors_throw_like_the_binding():
    for bad in (lambda: clue_kernels.FlatKernel(0.0), lambda: clue_kernels.GaussianKernel(-1.0, 1.0),
                lambda: clue_kernels.GaussianKernel(1.0, 0.0), lambda: clue_kernels.ExponentialKernel(0.0, 1.0)):
        with pytest.raises(ValueError):
            bad()
    clue_kernels.FlatKernel(0.5)
    clue_kernels.GaussianKernel(1.0, 1.0)
    clue_kernels.ExponentialKernel(1.0, 1.0)


def test_metric_descriptors_check_their_size_against_ndim():
    data, res = _wrapper_arrays(np.zeros((2, 4), np.float32), np.ones(4, np.float32))
    k = clue_kernels.FlatKernel(0.5)
    for desc, msg in [(clue_kernels.EuclideanMetric([1.0, 2.0, 3.0]), "EuclideanMetric requires exactly 2"),
                      (clue_kernels.ChebyshevMetric([1.0]), "ChebyshevMetric requires exactly 2"),
                      (clue_kernels.PeriodicEuclideanMetric([]), "PeriodicEuclideanMetric requires exactly 2")]:
        with pytest.raises(ValueError, match=msg):
            gpu_cuda.mainRun(1.0, 1.0, 1.0, 1.0, [0, 0], data, res, k, 2, None, 4, 0, desc)


def test_mainrun_rejects_what_the_reference_cannot_bind():
    k = clue_kernels.FlatKernel(0.5)
    m = clue_kernels.EuclideanMetric()
    data, res = _wrapper_arrays(np.zeros((2, 4), np.float32), np.ones(4, np.float32))
    with pytest.raises(TypeError):
        gpu_cuda.mainRun(1.0, 1.0, 1.0, 1.0, [0, 0], data.astype(np.float64), res, k, 2, None, 4, 0, m)
    with pytest.raises(ValueError):
        gpu_cuda.mainRun(1.0, 1.0, 1.0, 1.0, [0, 0], data, res, k, 2, None, 5, 0, m)


def test_mainrun_prints_for_more_than_ten_dimensions(capsys):
    data, res = _wrapper_arrays(np.zeros((11, 4), np.float32), np.ones(4, np.float32))
    out = gpu_cuda.mainRun(1.0, 1.0, 1.0, 1.0, [0] * 11, data, res, clue_kernels.FlatKernel(0.5), 11,
                           None, 4, 0, clue_kernels.EuclideanMetric())
    assert out is None
    assert "only works up to 10 dimensions" in capsys.readouterr().out


# ---- on the GPU: the wrapper's calls against the checker ----------------------------------------

@pytest.mark.gpu
def test_mainrun_2d_flat_kernel_matches_the_checker():
    c, w = fixture("data_1024")
    data, res = _wrapper_arrays(c, w)
    gpu_cuda.mainRun(1.3, 10.0, 1.3, 1.3, [0, 0], data, res, clue_kernels.FlatKernel(0.5), 2, None,
                     c.shape[1], 0, clue_kernels.EuclideanMetric())
    o = O.make_clusters(c, w, 1.3, 10.0, 1.3, 1.3)
    assert np.array_equal(res, o.cluster_index)
    assert res.max() + 1 == 20


@pytest.mark.gpu
def test_mainrun_3d_gaussian_and_weighted_metrics_match_the_checker():
    c, w = fixture("blob")
    for desc, metric, mp in [(clue_kernels.EuclideanMetric(), "euclidean", ()),
                             (clue_kernels.EuclideanMetric([1.0, 2.0, 0.5]), "weighted_euclidean", (1.0, 2.0, 0.5)),
                             (clue_kernels.ManhattanMetric(), "manhattan", ()),
                             (clue_kernels.ChebyshevMetric([1.0, 1.5, 1.0]), "weighted_chebyshev", (1.0, 1.5, 1.0))]:
        data, res = _wrapper_arrays(c, w)
        gpu_cuda.mainRun(1.5, 3.0, 2.0, 1.5, [0, 0, 0], data, res, clue_kernels.GaussianKernel(1.0, 1.0), 3,
                         None, c.shape[1], 0, desc)
        o = O.make_clusters(c, w, 1.5, 3.0, 2.0, 1.5, kernel="gaussian", kernel_params=(1.0, 1.0),
                            metric=metric, metric_params=list(mp), exp_mode=O.EXP_CLUE)
        assert np.array_equal(res, o.cluster_index), metric


@pytest.mark.gpu
def test_mainrun_periodic_metric_with_wrapped_coordinates():
    c, w = fixture("opposite_angles")
    two_pi = float(np.float32(2.0) * np.float32(math.pi))
    data, res = _wrapper_arrays(c, w)
    gpu_cuda.mainRun(0.2, 5.0, 0.2, 0.2, [0, 1], data, res, clue_kernels.FlatKernel(0.5), 2, None,
                     c.shape[1], 0, clue_kernels.PeriodicEuclideanMetric([0.0, two_pi]))
    assert res.max() + 1 == 1  # tests/test_clustering.cpp:237-270


@pytest.mark.gpu
def test_mainrun_batched_matches_the_checker():
    c, w = fixture("batched_data_1024")
    sizes = np.full(10, 1024, np.uint32)
    data, res = _wrapper_arrays(c, w)
    gpu_cuda.mainRun(1.3, 10.0, 1.3, 1.3, [0, 0], data, res, clue_kernels.FlatKernel(0.5), 2, sizes,
                     c.shape[1], 0, clue_kernels.EuclideanMetric())
    o = O.make_clusters_batched(c, w, sizes, 1.3, 10.0, 1.3, 1.3, shared_grid=True)
    assert np.array_equal(res, o.cluster_index)
    assert res.max() + 1 == 200  # tests/test_batched_clustering.cpp:51-108
