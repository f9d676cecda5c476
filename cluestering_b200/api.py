"""Python mirror of CLUEstering's C++ clustering API over the C ABI.

Names follow the reference (include/CLUEstering/core/Clusterer.hpp,
ConvolutionalKernel.hpp, DistanceMetrics.hpp, data_structures/PointsHost.hpp,
PointsDevice.hpp). Exceptions follow it too: std::invalid_argument ->
ValueError, std::out_of_range -> IndexError, std::runtime_error -> RuntimeError.

Host point sets are numpy arrays; device point sets are CUDA tensors (torch is
used only to hold device memory and streams).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib as L

# ---------------------------------------------------------------------------
# Convolutional kernels (core/ConvolutionalKernel.hpp, detail/ConvolutionalKernel.hpp:13-50)
# ---------------------------------------------------------------------------


class FlatKernel:
    kind = L.KERNEL_FLAT

    def __init__(self, flat: float = 0.5):
        if not flat > 0:
            raise ValueError("Flat kernel parameter must be positive.")
        self.params = (float(flat), 0.0)


class GaussianKernel:
    kind = L.KERNEL_GAUSSIAN

    def __init__(self, gaus_std: float, gaus_amplitude: float):
        if not (gaus_std > 0 and gaus_amplitude > 0):
            raise ValueError("Gaussian kernel parameters must be positive.")
        self.params = (float(gaus_std), float(gaus_amplitude))


class ExponentialKernel:
    kind = L.KERNEL_EXPONENTIAL

    def __init__(self, exp_avg: float, exp_amplitude: float):
        if not (exp_avg > 0 and exp_amplitude > 0):
            raise ValueError("Exponential kernel parameters must be positive.")
        self.params = (float(exp_avg), float(exp_amplitude))


# ---------------------------------------------------------------------------
# Distance metrics (core/DistanceMetrics.hpp:63-371)
# ---------------------------------------------------------------------------


class _Metric:
    kind = L.METRIC_EUCLIDEAN
    params: tuple = ()


class EuclideanMetric(_Metric):
    kind = L.METRIC_EUCLIDEAN


class WeightedEuclideanMetric(_Metric):
    kind = L.METRIC_WEIGHTED_EUCLIDEAN

    def __init__(self, *weights):
        self.params = tuple(float(w) for w in (weights[0] if len(weights) == 1 and
                                                 hasattr(weights[0], "__len__") else weights))


class PeriodicEuclideanMetric(_Metric):
    kind = L.METRIC_PERIODIC_EUCLIDEAN

    def __init__(self, *periods):
        self.params = tuple(float(p) for p in (periods[0] if len(periods) == 1 and
                                                 hasattr(periods[0], "__len__") else periods))


class ManhattanMetric(_Metric):
    kind = L.METRIC_MANHATTAN


class ChebyshevMetric(_Metric):
    kind = L.METRIC_CHEBYSHEV


class WeightedChebyshevMetric(WeightedEuclideanMetric):
    kind = L.METRIC_WEIGHTED_CHEBYSHEV


class MahalanobisMetric(_Metric):
    kind = L.METRIC_MAHALANOBIS


class metrics:  # noqa: N801 - mirrors clue::metrics
    Euclidean = EuclideanMetric
    WeightedEuclidean = WeightedEuclideanMetric
    PeriodicEuclidean = PeriodicEuclideanMetric
    Manhattan = ManhattanMetric
    Chebyshev = ChebyshevMetric
    WeightedChebyshev = WeightedChebyshevMetric
    Mahalanobis = MahalanobisMetric


# ---------------------------------------------------------------------------
# Point sets
# ---------------------------------------------------------------------------


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


@dataclass
class PointsHost:
    """SoA points in host memory (data_structures/PointsHost.hpp:28-254).

    coords is (ndim, n). Outputs are filled by Clusterer.make_clusters.
    """

    coords: np.ndarray
    weights: np.ndarray
    sigma: list = field(default_factory=list)
    density_uncertainty: np.ndarray | None = None
    tags: np.ndarray | None = None
    cluster_index: np.ndarray | None = None
    is_seed: np.ndarray | None = None
    rho: np.ndarray | None = None
    nearest_higher: np.ndarray | None = None
    clustered: bool = False

    def __post_init__(self):
        c = _f32(self.coords)
        if c.ndim == 1:
            c = c[None, :]
        self.coords = c
        self.weights = _f32(self.weights)
        if c.shape[1] <= 0:
            raise ValueError("Number of points passed to PointsHost constructor must be positive.")
        if self.weights.shape != (c.shape[1],):
            raise ValueError("weights must have one entry per point")
        if self.cluster_index is None:
            self.cluster_index = np.full(c.shape[1], -1, np.int32)
        if not self.sigma:
            self.sigma = [None] * c.shape[0]

    @property
    def ndim(self) -> int:
        return self.coords.shape[0]

    def size(self) -> int:
        return self.coords.shape[1]

    def set_sigma(self, dim: int, sigma) -> None:
        if dim >= self.ndim:
            raise IndexError("Dimension out of range in set_sigma")
        s = _f32(sigma)
        if s.shape != (self.size(),):
            raise ValueError("Size of sigma does not match the number of points")
        self.sigma[dim] = s

    def set_density_uncertainty(self, unc) -> None:
        u = _f32(unc)
        if u.shape != (self.size(),):
            raise ValueError("Size of density_uncertainty does not match the number of points")
        self.density_uncertainty = u

    def set_tags(self, tags) -> None:
        t = np.ascontiguousarray(tags, dtype=np.uint32)
        if t.shape != (self.size(),):
            raise ValueError("Size of tags does not match the number of points")
        self.tags = t

    def clusterIndexes(self) -> np.ndarray:  # noqa: N802
        return self.cluster_index

    def n_clusters(self) -> int:
        # detail::compute_nclusters: max label + 1
        return int(self.cluster_index.max()) + 1 if self.size() else 0

    def clusters(self):
        """Cluster -> points map (utils/detail/get_clusters.hpp:24-49): (offsets, points)."""
        return clusters_csr(self.cluster_index)

    def cluster_sizes(self) -> np.ndarray:
        offs, _ = self.clusters()
        return np.diff(offs)


def clusters_csr(labels: np.ndarray):
    """Counting sort of point ids by label, ids ascending within a cluster."""
    labels = np.asarray(labels)
    n_clusters = int(labels.max()) + 1 if labels.size else 0
    keep = np.nonzero(labels >= 0)[0]
    order = keep[np.argsort(labels[keep], kind="stable")]
    counts = np.bincount(labels[keep], minlength=n_clusters)
    offsets = np.zeros(n_clusters + 1, np.int32)
    np.cumsum(counts, out=offsets[1:])
    return offsets, order.astype(np.int32)


class PointsDevice:
    """SoA points in device memory (data_structures/PointsDevice.hpp:31-216).

    Holds CUDA tensors; coords is (ndim, n) float32 contiguous.
    """

    def __init__(self, coords, weights, *, sigma=None, density_uncertainty=None, tags=None,
                 outputs=("cluster_index", "is_seed", "rho", "nearest_higher")):
        import torch

        self.coords = coords.contiguous().float()
        if self.coords.dim() == 1:
            self.coords = self.coords[None, :]
        n = self.coords.shape[1]
        if n <= 0:
            raise ValueError("Number of points passed to PointsDevice constructor must be positive.")
        dev = self.coords.device
        self.weights = weights.contiguous().float()
        self.sigma = list(sigma) if sigma is not None else [None] * self.coords.shape[0]
        self.density_uncertainty = density_uncertainty
        self.tags = tags
        self.cluster_index = torch.empty(n, dtype=torch.int32, device=dev)
        self.is_seed = torch.empty(n, dtype=torch.int32, device=dev) if "is_seed" in outputs else None
        self.rho = torch.empty(n, dtype=torch.float32, device=dev) if "rho" in outputs else None
        self.nearest_higher = (torch.empty(n, dtype=torch.int32, device=dev)
                               if "nearest_higher" in outputs else None)
        self.clustered = False

    @property
    def ndim(self) -> int:
        return self.coords.shape[0]

    def size(self) -> int:
        return self.coords.shape[1]

    def clusterIndexes(self):  # noqa: N802
        return self.cluster_index

    def n_clusters(self) -> int:
        return int(self.cluster_index.max().item()) + 1


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _points_struct(p) -> L.Points:
    s = L.Points()
    s.ndim = p.ndim
    s.n = p.size()
    for d in range(p.ndim):
        s.coords[d] = _ptr(p.coords[d])
        if p.sigma[d] is not None:
            s.sigma[d] = _ptr(p.sigma[d])
    s.weight = _ptr(p.weights)
    s.density_uncertainty = _ptr(p.density_uncertainty)
    s.tags = _ptr(p.tags)
    s.cluster_index = _ptr(p.cluster_index)
    s.is_seed = _ptr(p.is_seed)
    s.rho = _ptr(p.rho)
    s.nearest_higher = _ptr(p.nearest_higher)
    return s


# ---------------------------------------------------------------------------
# Clusterer (core/Clusterer.hpp:37-312)
# ---------------------------------------------------------------------------


class Clusterer:
    def __init__(self, density_radius: float, min_density: float, outlier_distance: float | None = None,
                 seeding_distance: float | None = None, *, device: int = 0, points_per_tile: int = 0):
        self._device = device
        self._ws = None
        self._wrapped = [0] * L.MAX_DIM
        self._ppt = points_per_tile
        self.setParameters(density_radius, min_density, outlier_distance, seeding_distance)

    def __del__(self):
        ws = getattr(self, "_ws", None)
        lib = getattr(L, "_lib", None) if L is not None else None
        if ws is not None and lib is not None:  # at interpreter exit the module may be gone
            lib.clue_workspace_destroy(ws)
            self._ws = None

    # -- parameters -----------------------------------------------------
    def setParameters(self, density_radius, min_density, outlier_distance=None,  # noqa: N802
                      seeding_distance=None):
        dc = float(density_radius)
        dm = dc if outlier_distance is None else float(outlier_distance)
        sd = dc if seeding_distance is None else float(seeding_distance)
        rhoc = float(min_density)
        if not (dc > 0 and rhoc >= 0 and dm > 0 and sd > 0):
            raise ValueError("Invalid clustering parameters. The parameters must be positive.")
        self.dc, self.rhoc, self.dm, self.seed_dc = dc, rhoc, dm, sd

    def setWrappedCoordinates(self, *wrapped):  # noqa: N802
        vals = wrapped[0] if len(wrapped) == 1 and hasattr(wrapped[0], "__len__") else wrapped
        self._wrapped = [int(v) for v in vals] + [0] * (L.MAX_DIM - len(vals))

    def params(self, metric=None, kernel=None) -> L.Params:
        metric = metric or EuclideanMetric()
        kernel = kernel or FlatKernel(0.5)
        p = L.Params()
        p.dc, p.rhoc, p.dm, p.seed_dc = self.dc, self.rhoc, self.dm, self.seed_dc
        for d in range(L.MAX_DIM):
            p.wrapped[d] = self._wrapped[d]
        p.kernel_kind = kernel.kind
        p.kernel_params[0], p.kernel_params[1] = kernel.params
        p.metric_kind = metric.kind
        for d, v in enumerate(metric.params):
            p.metric_params[d] = v
        p.points_per_tile = self._ppt
        return p

    def _workspace(self):
        if self._ws is None:
            ws = C.c_void_p()
            L.check(L.load().clue_workspace_create(C.byref(ws), self._device))
            self._ws = ws
        return self._ws

    # -- clustering -----------------------------------------------------
    def make_clusters(self, points, metric=None, kernel=None, *, batch_item_sizes: Sequence[int] | None = None,
                      grid_mode: int = L.GRID_SHARED, stream=None, synchronize: bool = True):
        """Clusters `points` (PointsHost or PointsDevice), optionally as a batch.

        Host points return synchronised (core/detail/Clusterer.hpp:90-138). Device
        points run on `stream` (a torch stream or raw handle; default: torch's
        current stream) and, like the reference, synchronise unless told not to.
        """
        lib = L.load()
        prm = self.params(metric, kernel)
        if metric is not None and metric.kind in (L.METRIC_WEIGHTED_EUCLIDEAN, L.METRIC_PERIODIC_EUCLIDEAN,
                                                   L.METRIC_WEIGHTED_CHEBYSHEV):
            if len(metric.params) != points.ndim:
                raise ValueError("the metric needs one parameter per dimension")
        pts = _points_struct(points)
        ws = self._workspace()
        host = isinstance(points, PointsHost)
        st = self._stream_handle(stream, host)
        if batch_item_sizes is None:
            fn = lib.clue_make_clusters_host if host else lib.clue_make_clusters_device
            L.check(fn(ws, C.byref(prm), C.byref(pts), st))
            self._last_events = 1
        else:
            sizes = np.ascontiguousarray(batch_item_sizes, dtype=np.uint32)
            fn = lib.clue_make_clusters_batched_host if host else lib.clue_make_clusters_batched_device
            L.check(fn(ws, C.byref(prm), C.byref(pts), sizes.ctypes.data, len(sizes), grid_mode, st))
            self._last_events = len(sizes)
        if not host and synchronize:
            L.check(lib.clue_stream_synchronize(st))
        points.clustered = True
        self._last_n = points.size()
        return points

    @staticmethod
    def _stream_handle(stream, host: bool):
        if stream is None:
            if host:
                return None
            import torch
            return torch.cuda.current_stream().cuda_stream
        return getattr(stream, "cuda_stream", stream)

    # -- results --------------------------------------------------------
    def getSeeds(self) -> np.ndarray:  # noqa: N802
        if self._ws is None:
            raise RuntimeError("Seeds are not available. Please run make_clusters first.")
        n = C.c_int32()
        lib = L.load()
        L.check(lib.clue_get_seeds(self._ws, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.int32)
        L.check(lib.clue_get_seeds(self._ws, out.ctypes.data, n.value, C.byref(n)))
        return out[: n.value]

    def n_clusters(self) -> int:
        n = C.c_int32()
        L.check(L.load().clue_n_clusters(self._ws, C.byref(n)))
        return n.value

    def getSampleAssociations(self):  # noqa: N802
        """(offsets, n_keys): cluster ids of event e are offsets[e]..offsets[e+1]-1."""
        if self._ws is None:
            raise RuntimeError("Seeds are not available. Please run make_clusters first.")
        B = getattr(self, "_last_events", 1)
        offs = np.zeros(B + 1, np.int32)
        nk = C.c_int32()
        L.check(L.load().clue_sample_associations(self._ws, offs.ctypes.data, B + 1, C.byref(nk)))
        return offs, nk.value

    def getClustersDevice(self, stream=None):  # noqa: N802
        """Cluster -> points map of the last run built on the device:
        (offsets, points) CUDA tensors, ids ascending within a cluster."""
        import torch
        k = self.n_clusters()
        dev = torch.device("cuda", self._device)
        offsets = torch.empty(k + 1, dtype=torch.int32, device=dev)
        pts = torch.empty(max(1, self._last_n), dtype=torch.int32, device=dev)
        st = self._stream_handle(stream, False)
        L.check(L.load().clue_get_clusters_device(self._ws, offsets.data_ptr(), pts.data_ptr(), st))
        L.check(L.load().clue_stream_synchronize(st))
        return offsets, pts[: int(offsets[-1].item())]

    def set_graphs(self, enable: bool = True) -> None:
        """CUDA-graph replay of repeated identical runs (clue_workspace_set_graphs)."""
        L.check(L.load().clue_workspace_set_graphs(self._workspace(), int(enable)))

    def graph_replayed(self) -> bool:
        """Whether the last run replayed a captured graph."""
        r = C.c_int32()
        L.check(L.load().clue_workspace_graph_replayed(self._workspace(), C.byref(r)))
        return bool(r.value)

    def host_pieces(self) -> int:
        """Pieces the last host-buffer run was pipelined in (1: one piece)."""
        r = C.c_int32()
        L.check(L.load().clue_workspace_host_pieces(self._workspace(), C.byref(r)))
        return int(r.value)

    def set_profiling(self, enable: bool = True) -> None:
        L.check(L.load().clue_workspace_set_profiling(self._workspace(), int(enable)))

    def stage_ms(self) -> dict:
        """Device time of each stage of the last run (needs set_profiling)."""
        ms = (C.c_float * len(L.STAGES))()
        L.check(L.load().clue_workspace_stage_ms(self._ws, ms, len(L.STAGES)))
        return dict(zip(L.STAGES, list(ms)))

    def sweep_stats(self) -> dict:
        """Candidate counts of the sweeps in the last run (needs set_profiling):
        density candidate tests and work items, nearest-higher members tested,
        cells checked and cells entered (clue_workspace_sweep_stats)."""
        n = 5
        v = (C.c_int64 * n)()
        L.check(L.load().clue_workspace_sweep_stats(self._ws, v, n))
        keys = ["density_tests", "density_items", "nh_members_tested", "nh_cells_checked", "nh_cells_entered"]
        return dict(zip(keys, list(v)))

    def workspace_bytes(self) -> int:
        b = C.c_size_t()
        L.check(L.load().clue_workspace_bytes(self._workspace(), C.byref(b)))
        return b.value

    def get_tuning(self) -> dict:
        """Launch choices of this clusterer's workspace (see clue_tuning)."""
        t = L.Tuning()
        L.check(L.load().clue_workspace_get_tuning(self._workspace(), C.byref(t)))
        return {name: getattr(t, name) for name, _ in L.Tuning._fields_}

    def set_tuning(self, **fields) -> None:
        """Changes launch choices; results do not depend on them."""
        t = L.Tuning()
        lib = L.load()
        L.check(lib.clue_workspace_get_tuning(self._workspace(), C.byref(t)))
        for name, value in fields.items():
            if name not in dict(L.Tuning._fields_):
                raise KeyError(name)
            setattr(t, name, int(value))
        L.check(lib.clue_workspace_set_tuning(self._workspace(), C.byref(t)))

    def autotune(self, points, metric=None, kernel=None, *, batch_item_sizes: Sequence[int] | None = None,
                 grid_mode: int = L.GRID_SHARED, stream=None, reps: int = 3) -> dict:
        """Times make_clusters on these device points under candidate launch
        choices and keeps the fastest for this clusterer (clue_workspace_autotune);
        results are the same under every choice. Returns the chosen tuning."""
        if not isinstance(points, PointsDevice):
            raise TypeError("autotune runs on device points")
        lib = L.load()
        prm = self.params(metric, kernel)
        pts = _points_struct(points)
        st = self._stream_handle(stream, False)
        t = L.Tuning()
        if batch_item_sizes is None:
            L.check(lib.clue_workspace_autotune(self._workspace(), C.byref(prm), C.byref(pts), None, 0, 0, st,
                                                int(reps), C.byref(t)))
        else:
            sizes = np.ascontiguousarray(batch_item_sizes, dtype=np.uint32)
            L.check(lib.clue_workspace_autotune(self._workspace(), C.byref(prm), C.byref(pts), sizes.ctypes.data,
                                                len(sizes), grid_mode, st, int(reps), C.byref(t)))
        points.clustered = True
        return {name: getattr(t, name) for name, _ in L.Tuning._fields_}

    def kernel_launches(self) -> int:
        """CUDA kernels the last make_clusters enqueued."""
        k = C.c_int64()
        L.check(L.load().clue_workspace_kernel_launches(self._workspace(), C.byref(k)))
        return k.value


# ---------------------------------------------------------------------------
# Validation utilities on the device (utils/cluster_centroid.hpp, utils/scores.hpp)
# ---------------------------------------------------------------------------


def _device_map(points, clusterer, stream):
    if not isinstance(points, PointsDevice):
        raise TypeError("the device utilities take the PointsDevice the clusterer last clustered")
    if not getattr(points, "clustered", False):
        raise RuntimeError("the points have not been clustered")
    offsets, members = clusterer.getClustersDevice(stream)
    return offsets, members, len(offsets) - 1


def cluster_centroids(points, clusterer, *, weighted: bool = False, stream=None) -> np.ndarray:
    """clue::cluster_centroids / weighted_cluster_centroids
    (utils/detail/cluster_centroid.hpp:86-140) of `clusterer`'s last run on
    `points`, computed on the device: (n_clusters, ndim) float32, the reference's
    values bit for bit."""
    import torch
    offsets, members, k = _device_map(points, clusterer, stream)
    out = torch.zeros((max(k, 1), points.ndim), dtype=torch.float32, device=points.coords.device)
    st = Clusterer._stream_handle(stream, False)
    L.check(L.load().clue_cluster_centroids_device(C.byref(_points_struct(points)), offsets.data_ptr(),
                                                   members.data_ptr(), k, int(weighted), out.data_ptr(), st))
    L.check(L.load().clue_stream_synchronize(st))
    return out[:k].cpu().numpy()


def weighted_cluster_centroids(points, clusterer, *, stream=None) -> np.ndarray:
    return cluster_centroids(points, clusterer, weighted=True, stream=stream)


def silhouette_scores(points, clusterer, *, stream=None) -> np.ndarray:
    """clue::silhouette(points, point) for every point (utils/detail/scores.hpp:33-73),
    on the device; NaN for the points the reference's mean skips."""
    import torch
    offsets, members, k = _device_map(points, clusterer, stream)
    scores = torch.empty(points.size(), dtype=torch.float32, device=points.coords.device)
    st = Clusterer._stream_handle(stream, False)
    L.check(L.load().clue_silhouette_device(C.byref(_points_struct(points)), offsets.data_ptr(),
                                            members.data_ptr(), k, scores.data_ptr(), st))
    L.check(L.load().clue_stream_synchronize(st))
    return scores.cpu().numpy()


def silhouette(points, clusterer, point: int | None = None, *, stream=None) -> float:
    """clue::silhouette(points) (the mean over the points of clusters with at
    least two points, utils/detail/scores.hpp:76-100) or, with `point`,
    clue::silhouette(points, point)."""
    s = silhouette_scores(points, clusterer, stream=stream)
    if point is not None:
        return float(s[point])
    keep = s[~np.isnan(s)]
    return float(np.mean(keep.astype(np.float64))) if keep.size else float("nan")


# ---------------------------------------------------------------------------
# Serving (continuous batching; no counterpart in the reference)
# ---------------------------------------------------------------------------


class Server:
    """Request loop over clue_server_*: submit events as they arrive, poll or drain.

    `profiles` is a list of (ndim, Clusterer, metric, kernel) describing the
    kinds of events the server accepts; submit() names the profile by index.
    The host arrays of a submitted event must stay alive and unmodified until
    it completes (pinned arrays are copied by DMA).
    """

    def __init__(self, profiles, *, device: int = 0, budget_bytes: int = 8 << 30, max_inflight: int = 4,
                 max_batch_events: int = 1024, max_batch_points: int = 0, linger_us: int = 200,
                 max_batch_ms: float = 0.0, priority_ms: float = 0.0):
        lib = L.load()
        arr = (L.ServerProfile * len(profiles))()
        for i, (ndim, clusterer, metric, kernel) in enumerate(profiles):
            arr[i].ndim = ndim
            arr[i].params = clusterer.params(metric, kernel)
        cfg = L.ServerConfig(device=device, budget_bytes=budget_bytes, max_inflight=max_inflight,
                             max_batch_events=max_batch_events, max_batch_points=max_batch_points,
                             linger_us=linger_us, max_batch_ms=max_batch_ms, priority_ms=priority_ms)
        h = C.c_void_p()
        L.check(lib.clue_server_create(C.byref(h), C.byref(cfg), arr, len(profiles)))
        self._h = h
        self._keep = {}

    def submit(self, profile: int, points: PointsHost) -> int:
        s = _points_struct(points)
        t = C.c_uint64()
        L.check(L.load().clue_server_submit(self._h, profile, C.byref(s), C.byref(t)))
        self._keep[t.value] = points
        return t.value

    def done(self, ticket: int) -> bool:
        st = L.load().clue_server_poll(self._h, ticket)
        if st == L.ERR_NOT_READY:
            return False
        L.check(st)
        self._keep.pop(ticket, None)
        return True

    def drain(self) -> None:
        L.check(L.load().clue_server_drain(self._h))
        self._keep.clear()

    def stats(self) -> dict:
        s = L.ServerStats()
        L.check(L.load().clue_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in L.ServerStats._fields_}

    def latencies_ms(self) -> np.ndarray:
        n = C.c_int64()
        L.check(L.load().clue_server_latencies(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        L.check(L.load().clue_server_latencies(self._h, out.ctypes.data, n.value, C.byref(n)))
        return out[: n.value]

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            L.load().clue_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
