"""CLUE_GPU_CUDA: the "gpu cuda" backend module of CLUEstering's Python wrapper,
rebuilt over libclue_sm100.so.

mainRun keeps the signature of the nanobind function it replaces
(CLUEstering/BindingModules/Run.hpp:67-131): `data` is the wrapper's
(Ndim + 1, n_points) float32 array — one row per coordinate, then the weights
(CLUEstering.py:297-309) — and `results` its int32 array of n_points cluster
ids, written in place. With `batch_sample_sizes` the points are a batch of
events clustered in one call with the reference's batch-wide tile grid
(Clusterer::make_clusters with batch sizes, core/Clusterer.hpp:62-68).
Parameter errors raise ValueError, as std::invalid_argument does through
nanobind. The reference also binds float64 overloads; this backend computes in
float32 only and raises TypeError for other input types.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from cluestering_b200 import _lib as L
from cluestering_b200.api import ExponentialKernel, FlatKernel, GaussianKernel

from cluestering_b200.compat.descriptor import MetricDescriptor

_workspaces: dict[int, C.c_void_p] = {}


def _workspace(device_id: int) -> C.c_void_p:
    """One workspace per device, reused across calls (buffers grow, never shrink)."""
    ws = _workspaces.get(device_id)
    if ws is None:
        ws = C.c_void_p()
        L.check(L.load().clue_workspace_create(C.byref(ws), int(device_id)))
        _workspaces[device_id] = ws
    return ws


def listDevices(backend: str) -> None:  # noqa: N802 - the binding's name
    """Run.hpp:56-67: prints the devices of this backend."""
    import torch

    n = torch.cuda.device_count() if torch.cuda.is_available() else 0
    if n == 0:
        print(f"No devices found for the {backend} backend.")
        return
    print(f"{backend} devices found: ")
    for i in range(n):
        print(f"\tdevice {i}: {torch.cuda.get_device_name(i)}")


def _metric_fields(desc: MetricDescriptor, ndim: int):
    """MetricDescriptor.hpp:28-93: the metric a descriptor names for ndim
    dimensions, as (metric_kind, params); unit weights are the unweighted metric
    (w * d * d and w * |d| with w = 1 round to d * d and |d|)."""
    tag, params = desc.tag, list(desc.params)
    if tag == MetricDescriptor.WEIGHTED_EUCLIDEAN:
        if not params:
            return L.METRIC_EUCLIDEAN, []
        if len(params) != ndim:
            raise ValueError(f"EuclideanMetric requires exactly {ndim} weight(s), got {len(params)}")
        return L.METRIC_WEIGHTED_EUCLIDEAN, params
    if tag == MetricDescriptor.MANHATTAN:
        return L.METRIC_MANHATTAN, []
    if tag == MetricDescriptor.PERIODIC_EUCLIDEAN:
        if len(params) != ndim:
            raise ValueError(f"PeriodicEuclideanMetric requires exactly {ndim} period(s), got {len(params)}")
        return L.METRIC_PERIODIC_EUCLIDEAN, params
    if tag == MetricDescriptor.WEIGHTED_CHEBYSHEV:
        if not params:
            return L.METRIC_CHEBYSHEV, []
        if len(params) != ndim:
            raise ValueError(f"ChebyshevMetric requires exactly {ndim} weight(s), got {len(params)}")
        return L.METRIC_WEIGHTED_CHEBYSHEV, params
    raise ValueError("unknown metric descriptor")


def mainRun(dc, rhoc, dm, seed_dc, wrapped, data, results, kernel, Ndim, batch_sample_sizes,  # noqa: N802,N803
            n_points, device_id, metric_desc):
    """Clusters `data` into `results` on GPU `device_id` (Run.hpp:76-131)."""
    if not 1 <= Ndim <= L.MAX_DIM:
        print("This library only works up to 10 dimensions")
        return None
    if not isinstance(data, np.ndarray) or data.dtype != np.float32:
        raise TypeError("mainRun: data must be a float32 numpy array (this backend computes in float32)")
    if not isinstance(results, np.ndarray) or results.dtype != np.int32:
        raise TypeError("mainRun: results must be an int32 numpy array")
    if not isinstance(kernel, (FlatKernel, GaussianKernel, ExponentialKernel)):
        raise TypeError("mainRun: kernel must be a FlatKernel, GaussianKernel or ExponentialKernel")
    if not isinstance(metric_desc, MetricDescriptor):
        raise TypeError("mainRun: metric must be a MetricDescriptor")
    n = int(n_points)
    if n <= 0:
        raise ValueError("Number of points passed to PointsHost constructor must be positive.")
    if not (data.flags.c_contiguous and data.size == (Ndim + 1) * n):
        raise ValueError("mainRun: data must be a contiguous (Ndim + 1, n_points) array")
    if not (results.flags.c_contiguous and results.size == n):
        raise ValueError("mainRun: results must hold n_points cluster ids")
    metric_kind, metric_params = _metric_fields(metric_desc, Ndim)

    prm = L.Params()
    prm.dc, prm.rhoc, prm.dm, prm.seed_dc = float(dc), float(rhoc), float(dm), float(seed_dc)
    for d, w in enumerate(list(wrapped)[:L.MAX_DIM]):
        prm.wrapped[d] = 1 if w else 0
    prm.kernel_kind = kernel.kind
    prm.kernel_params[0], prm.kernel_params[1] = kernel.params
    prm.metric_kind = metric_kind
    for d, v in enumerate(metric_params):
        prm.metric_params[d] = v
    prm.points_per_tile = 0

    pts = L.Points()
    pts.ndim, pts.n = Ndim, n
    base = data.ctypes.data
    for d in range(Ndim):
        pts.coords[d] = base + 4 * d * n
    pts.weight = base + 4 * Ndim * n
    pts.cluster_index = results.ctypes.data

    lib = L.load()
    ws = _workspace(int(device_id))
    if batch_sample_sizes is None:
        L.check(lib.clue_make_clusters_host(ws, C.byref(prm), C.byref(pts), None))
    else:
        sizes = np.ascontiguousarray(batch_sample_sizes, dtype=np.uint32)
        if int(sizes.sum()) != n:
            raise ValueError("mainRun: the batch sizes do not add up to n_points")
        L.check(lib.clue_make_clusters_batched_host(ws, C.byref(prm), C.byref(pts), sizes.ctypes.data,
                                                    len(sizes), L.GRID_SHARED, None))
    return None
