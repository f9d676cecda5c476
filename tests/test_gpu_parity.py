"""GPU parity: libclue_sm100.so (through the C ABI) against the CPU checker.

The bar is bit-exact equality of every output — density (compared as bits),
nearest higher, seed flags and cluster ids — on the same seeded inputs. The
checker evaluates the Gaussian/exponential kernels with the library-owned
exponential (clue_expf) that the GPU path uses.
"""

import math

import numpy as np
import pytest

import cluestering_b200 as clue
from cluestering_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import fixture, same_partition, truth_count

pytestmark = pytest.mark.gpu

METRIC_CLASSES = {
    "euclidean": lambda p: clue.EuclideanMetric(),
    "weighted_euclidean": lambda p: clue.WeightedEuclideanMetric(*p),
    "periodic_euclidean": lambda p: clue.PeriodicEuclideanMetric(*p),
    "manhattan": lambda p: clue.ManhattanMetric(),
    "chebyshev": lambda p: clue.ChebyshevMetric(),
    "weighted_chebyshev": lambda p: clue.WeightedChebyshevMetric(*p),
    "mahalanobis": lambda p: clue.MahalanobisMetric(),
}
KERNEL_CLASSES = {
    "flat": lambda p: clue.FlatKernel(*p),
    "gaussian": lambda p: clue.GaussianKernel(*p),
    "exponential": lambda p: clue.ExponentialKernel(*p),
}


def run_gpu(coords, weights, dc, rhoc, dm=None, seed_dc=None, *, metric="euclidean", metric_params=(),
            kernel="flat", kernel_params=(0.5,), sigma=None, unc=None, tags=None, wrapped=None,
            sizes=None, grid_mode=clue.GRID_SHARED, path="host", clusterer=None):
    c = clusterer or clue.Clusterer(dc, rhoc, dm, seed_dc)
    if clusterer is not None:
        c.setParameters(dc, rhoc, dm, seed_dc)
    if wrapped is not None:
        c.setWrappedCoordinates(*wrapped)
    m = METRIC_CLASSES[metric](metric_params)
    k = KERNEL_CLASSES[kernel](kernel_params)
    coords = np.ascontiguousarray(coords, np.float32)
    if coords.ndim == 1:
        coords = coords[None]
    D, n = coords.shape
    if path == "host":
        pts = clue.PointsHost(coords, weights)
        pts.is_seed = np.zeros(n, np.int32)
        pts.rho = np.zeros(n, np.float32)
        pts.nearest_higher = np.zeros(n, np.int32)
        if sigma is not None:
            for d, s in enumerate(sigma):
                if s is not None:
                    pts.set_sigma(d, s)
        if unc is not None:
            pts.set_density_uncertainty(unc)
        if tags is not None:
            pts.set_tags(tags)
        c.make_clusters(pts, m, k, batch_item_sizes=sizes, grid_mode=grid_mode)
        out = dict(rho=pts.rho, nh=pts.nearest_higher, seed=pts.is_seed, ci=pts.cluster_index)
    else:
        import torch
        dev = torch.device("cuda:0")
        t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
        pts = clue.PointsDevice(
            t(coords), t(weights),
            sigma=None if sigma is None else [None if s is None else t(s) for s in sigma],
            density_uncertainty=None if unc is None else t(unc),
            tags=None if tags is None else t(np.asarray(tags, np.int64).astype(np.int32), torch.int32))
        c.make_clusters(pts, m, k, batch_item_sizes=sizes, grid_mode=grid_mode)
        out = dict(rho=pts.rho.cpu().numpy(), nh=pts.nearest_higher.cpu().numpy(),
                   seed=pts.is_seed.cpu().numpy(), ci=pts.cluster_index.cpu().numpy())
    out["clusterer"] = c
    return out


def run_oracle(coords, weights, dc, rhoc, dm=None, seed_dc=None, *, metric="euclidean", metric_params=(),
               kernel="flat", kernel_params=(0.5,), sigma=None, unc=None, tags=None, wrapped=None,
               sizes=None, grid_mode=clue.GRID_SHARED, threads=8):
    kw = dict(metric=metric, metric_params=list(metric_params), kernel=kernel,
              kernel_params=tuple(kernel_params), sigma=sigma, unc=unc, tags=tags, wrapped=wrapped,
              exp_mode=O.EXP_CLUE, n_threads=threads)
    if sizes is None:
        return O.make_clusters(coords, weights, dc, rhoc, dm, seed_dc, **kw)
    return O.make_clusters_batched(coords, weights, sizes, dc, rhoc, dm, seed_dc,
                                   shared_grid=(grid_mode == clue.GRID_SHARED), **kw)


def assert_identical(g, o):
    assert np.array_equal(g["rho"].view(np.int32), o.rho.view(np.int32)), \
        f"rho differs at {np.nonzero(g['rho'].view(np.int32) != o.rho.view(np.int32))[0][:10]}"
    assert np.array_equal(g["nh"], o.nearest_higher), \
        f"nearest higher differs at {np.nonzero(g['nh'] != o.nearest_higher)[0][:10]}"
    assert np.array_equal(g["seed"], o.is_seed)
    assert np.array_equal(g["ci"], o.cluster_index)


def check(coords, weights, *args, **kw):
    g = run_gpu(coords, weights, *args, **kw)
    kw.pop("path", None)
    kw.pop("clusterer", None)
    o = run_oracle(coords, weights, *args, **kw)
    assert_identical(g, o)
    return g, o


# ---- the benchmark configurations -------------------------------------------------------------

@pytest.mark.parametrize("path", ["host", "device"])
def test_single_2d_event(path):
    ev = W.single_2d()
    g, o = check(ev.coords, ev.weights, 1.5, 5.0, 1.5, path=path)
    assert o.n_clusters >= 15


def test_layered_3d_event_gaussian_kernel():
    ev = W.layered_3d()
    check(ev.coords, ev.weights, 3.0, 10.0, 4.0, kernel="gaussian", kernel_params=(1.0, 1.0))


def test_large_2d_event_exponential_weights_reduced():
    ev = W.blobs(1 << 17, 250, 0.0, 353.0, 1.0, 0.1, seed=9, weights="exponential")
    check(ev.coords, ev.weights, 1.5, 8.0, 2.0)


def test_large_2d_event_full_size():
    ev = W.large_2d()
    check(ev.coords, ev.weights, 1.5, 8.0, 2.0, path="device")


def test_full_benchmark_batch_against_checker():
    # The benchmark's own batch: 4,096 events of log-uniform size in
    # [256, 65,536] (46.5 M points), one grid per event, through the device and
    # the host entry points (the latter pipelined in pieces), against the
    # checker on all host cores.
    import os
    ev, sizes = W.batch_2d()
    o = run_oracle(ev.coords, ev.weights, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_PER_EVENT,
                   threads=os.cpu_count() or 1)
    for path in ("device", "host"):
        g = run_gpu(ev.coords, ev.weights, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_PER_EVENT,
                    path=path)
        assert_identical(g, o)
        offsets, n_keys = g["clusterer"].getSampleAssociations()
        assert n_keys == len(sizes)
        assert np.array_equal(offsets, expected_sample_offsets(o, len(sizes)))
        assert np.array_equal(g["clusterer"].getSeeds(), o.seeds)
        del g


def test_batch_of_mixed_size_events_per_event_grid():
    ev, sizes = W.batch_2d(64, 256, 8192, seed=21)
    w = np.random.default_rng(3).exponential(1.0, ev.n).astype(np.float32)
    check(ev.coords, w, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_PER_EVENT)


def test_batch_of_mixed_size_events_shared_grid():
    ev, sizes = W.batch_2d(16, 256, 4096, seed=22)
    w = np.random.default_rng(4).exponential(1.0, ev.n).astype(np.float32)
    check(ev.coords, w, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_SHARED)


def test_batch_events_alone_and_in_the_mix():
    ev, sizes = W.batch_2d(12, 256, 6000, seed=23)
    w = np.random.default_rng(5).exponential(1.0, ev.n).astype(np.float32)
    mix = run_gpu(ev.coords, w, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_PER_EVENT)
    begin, label0 = 0, 0
    for s in sizes.tolist():
        one = run_gpu(ev.coords[:, begin:begin + s], w[begin:begin + s], 1.5, 5.0, 1.5)
        sl = slice(begin, begin + s)
        assert np.array_equal(mix["rho"][sl].view(np.int32), one["rho"].view(np.int32))
        assert np.array_equal(mix["nh"][sl], np.where(one["nh"] >= 0, one["nh"] + begin, -1))
        assert np.array_equal(mix["ci"][sl], np.where(one["ci"] >= 0, one["ci"] + label0, -1))
        begin += s
        label0 += int(one["ci"].max()) + 1


# ---- metrics, kernels and per-point options ---------------------------------------------------

@pytest.mark.parametrize("metric,params", [
    ("euclidean", ()), ("weighted_euclidean", (0.5, 2.0)), ("periodic_euclidean", (0.0, 100.0)),
    ("manhattan", ()), ("chebyshev", ()), ("weighted_chebyshev", (0.7, 1.3)), ("mahalanobis", ()),
])
def test_every_metric(metric, params):
    ev = W.blobs(6000, 12, 0.0, 100.0, 1.0, 0.1, seed=31)
    sigma = None
    if metric == "mahalanobis":
        rng = np.random.default_rng(7)
        sigma = [rng.uniform(0.5, 1.5, ev.n).astype(np.float32) for _ in range(2)]
    check(ev.coords, ev.weights, 1.5, 5.0, 1.5, metric=metric, metric_params=params, sigma=sigma)


@pytest.mark.parametrize("kernel,params", [("flat", (0.5,)), ("flat", (1.0,)), ("gaussian", (0.8, 2.0)),
                                           ("exponential", (1.2, 0.7))])
def test_every_kernel_with_real_weights(kernel, params):
    ev = W.blobs(5000, 10, 0.0, 60.0, 1.0, 0.1, seed=32, weights="exponential")
    check(ev.coords, ev.weights, 1.5, 3.0, 2.0, kernel=kernel, kernel_params=params)


def test_wrapped_coordinates_with_periodic_metric():
    rng = np.random.default_rng(8)
    ang = np.concatenate([rng.normal(0.05, 0.05, 400), rng.normal(2 * np.pi - 0.05, 0.05, 400)])
    ang = np.mod(ang, 2 * np.pi)
    r = rng.uniform(0, 1, ang.size)
    coords = np.stack([r, ang]).astype(np.float32)
    w = np.ones(ang.size, np.float32)
    check(coords, w, 0.2, 5.0, 0.2, metric="periodic_euclidean", metric_params=(0.0, 2 * np.pi),
          wrapped=[0, 1])


def test_sigma_widens_the_search_box():
    ev = W.blobs(4000, 8, 0.0, 50.0, 1.0, 0.1, seed=33, weights="exponential")
    rng = np.random.default_rng(9)
    sigma = [rng.uniform(0.0, 3.0, ev.n).astype(np.float32), None]
    check(ev.coords, ev.weights, 1.0, 3.0, 1.5, sigma=sigma)


def test_density_uncertainty_and_tags():
    ev = W.blobs(5000, 10, 0.0, 80.0, 1.0, 0.1, seed=34)
    rng = np.random.default_rng(10)
    unc = (1.0 + rng.normal(0, 0.3, ev.n)).astype(np.float32)
    tags = rng.permutation(ev.n).astype(np.uint32)
    check(ev.coords, ev.weights, 1.5, 5.0, 1.5, unc=unc, tags=tags)


def test_seeding_distance_differs_from_outlier_distance():
    ev = W.blobs(5000, 10, 0.0, 80.0, 1.0, 0.1, seed=35, weights="exponential")
    check(ev.coords, ev.weights, 1.0, 4.0, 1.5, 3.0)
    check(ev.coords, ev.weights, 1.0, 4.0, 3.0, 1.2)


@pytest.mark.parametrize("D", [1, 3, 4, 7, 10])
def test_dimensions(D):
    ev = W.blobs(3000 if D < 7 else 2000, 6, 0.0, 30.0, 1.0, 0.1, seed=40 + D, ndim=D,
                 weights="exponential")
    check(ev.coords, ev.weights, 1.5 if D < 4 else 3.0, 2.0, 2.0)


# ---- the reference's known-answer tests through the GPU path ----------------------------------

def test_tag_tie_break():
    coords = np.zeros((2, 2), np.float32)
    w = np.ones(2, np.float32)
    g = run_gpu(coords, w, 1.0, 0.0, 1.0)
    assert g["nh"].tolist() == [1, -1] and g["seed"].tolist() == [0, 1]
    g = run_gpu(coords, w, 1.0, 0.0, 1.0, tags=np.array([100, 1], np.uint32))
    assert g["nh"].tolist() == [-1, 0] and g["seed"].tolist() == [1, 0]


def test_mahalanobis_merge():
    coords = np.array([[2.0, 4.0]], np.float32)
    w = np.ones(2, np.float32)
    assert run_gpu(coords, w, 1.0, 0.3)["ci"].max() + 1 == 2
    g = run_gpu(coords, w, 1.0, 0.3, metric="mahalanobis", sigma=[np.array([2.0, 2.0], np.float32)])
    assert g["ci"].max() + 1 == 1


def test_opposite_angles_single_cluster():
    c, w = fixture("opposite_angles")
    two_pi = float(np.float32(2.0) * np.float32(math.pi))
    g, o = check(c, w, 0.2, 5.0, 0.2, wrapped=[0, 1], metric="periodic_euclidean",
                 metric_params=(0.0, two_pi))
    assert g["ci"].max() + 1 == 1


def test_batched_fixed_batch_size_counts():
    c, w = fixture("batched_data_1024")
    g, o = check(c, w, 1.3, 10.0, 1.3, sizes=[1024] * 10)
    assert g["ci"].max() + 1 == 10 * truth_count("data_1024")
    offsets, n_keys = g["clusterer"].getSampleAssociations()
    assert n_keys == 10
    assert np.array_equal(offsets, expected_sample_offsets(o, 10))
    seeds = g["clusterer"].getSeeds()
    assert np.array_equal(seeds, o.seeds)


def expected_sample_offsets(o, n_events):
    """The checker's seed -> event associations (core/detail/Clusterer.hpp:221-242)
    as the event -> cluster-id CSR offsets that getSampleAssociations returns:
    cluster k is seed k, so the clusters of event e are a contiguous id range."""
    ea = np.asarray(o.event_associations)
    assert np.all(np.diff(ea) >= 0)
    return np.concatenate([[0], np.cumsum(np.bincount(ea, minlength=n_events))]).astype(np.int32)


def test_sample_associations_full_csr_mixed_batch():
    ev, sizes = W.batch_2d(48, 256, 8192, seed=5)
    for mode in (clue.GRID_PER_EVENT, clue.GRID_SHARED):
        g, o = check(ev.coords, ev.weights, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=mode)
        offsets, n_keys = g["clusterer"].getSampleAssociations()
        assert n_keys == len(sizes)
        assert np.array_equal(offsets, expected_sample_offsets(o, len(sizes)))


@pytest.mark.parametrize("ordered_events", ["half", "one"])
def test_batch_mixing_exact_and_ordered_sums(ordered_events):
    # Events whose sums are exact in any order (unit weights) beside events
    # whose sums keep the reference's order (exponential weights): the tile
    # sort must still order the tiles of the latter, with counting-sort
    # binning, whether half the events or a single one need it.
    ev, sizes = W.batch_2d(32, 256, 8192, seed=41)
    offs = np.concatenate([[0], np.cumsum(sizes.astype(np.int64))])
    w = np.ones(ev.n, np.float32)
    rng = np.random.default_rng(42)
    pick = range(0, len(sizes), 2) if ordered_events == "half" else [len(sizes) // 2]
    for e in pick:
        w[offs[e]:offs[e + 1]] = rng.exponential(1.0, int(sizes[e])).astype(np.float32)
    for mode in (clue.GRID_PER_EVENT, clue.GRID_SHARED):
        c = clue.Clusterer(1.5, 5.0, 1.5)
        c.set_tuning(tile_binning=0)
        for path in ("host", "device"):
            check(ev.coords, w, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=mode, path=path, clusterer=c)


def with_empty_events(sizes, where):
    """`sizes` with a batch item of size 0 inserted before each position in
    `where` (len(sizes) appends one at the end)."""
    out = [int(s) for s in sizes]
    for pos in sorted(where, reverse=True):
        out.insert(pos, 0)
    return np.array(out, np.uint32)


@pytest.mark.parametrize("mode", [clue.GRID_PER_EVENT, clue.GRID_SHARED])
@pytest.mark.parametrize("binning", [0, 1])
def test_batch_with_empty_events(mode, binning):
    # Batch items of size 0 at the start, inside and at the end: the reference
    # scans the sizes as given (core/detail/Clusterer.hpp:293-300), so such an
    # item holds no points and no clusters, and the associator's key count
    # stops at the last event with a cluster (MakeAssociator.hpp:32-43).
    ev, sizes = W.batch_2d(24, 256, 8192, seed=31)
    sizes = with_empty_events(sizes, [0, 0, 5, 12, 12, 12, len(sizes), len(sizes)])
    w = np.random.default_rng(32).exponential(1.0, ev.n).astype(np.float32)
    for weights in (ev.weights, w):  # exact-sum and ordered density sums
        c = clue.Clusterer(1.5, 5.0, 1.5)
        c.set_tuning(tile_binning=binning)
        for path in ("host", "device"):
            g, o = check(ev.coords, weights, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=mode, path=path,
                         clusterer=c)
            offsets, n_keys = g["clusterer"].getSampleAssociations()
            ea = np.asarray(o.event_associations)
            assert n_keys == (int(ea[-1]) + 1 if len(ea) else 0) < len(sizes)
            assert np.array_equal(offsets, expected_sample_offsets(o, len(sizes)))


@pytest.mark.parametrize("name", ["data_4096", "data_32768"])
def test_reference_datasets(name):
    c, w = fixture(name)
    check(c, w, 1.5, 10.0, 1.5)


# ---- ties ---------------------------------------------------------------------------------------

@pytest.mark.parametrize("spacing", [1.0, 0.1, 0.3])
def test_lattice_ties_2d(spacing):
    # Equal densities and equal distances everywhere: the tag tie-break and the
    # equal-distance rule decide; with spacing 0.1 or 0.3 squared distances of
    # equal true length differ only by rounding.
    g = np.arange(70, dtype=np.float32) * np.float32(spacing)
    xx, yy = np.meshgrid(g, g, indexing="ij")
    coords = np.stack([xx.ravel(), yy.ravel()]).astype(np.float32)
    w = np.ones(coords.shape[1], np.float32)
    check(coords, w, 1.5 * spacing, 3.0, 1.5 * spacing)
    check(coords, w, 1.01 * spacing, 2.0, 2.9 * spacing)


def test_lattice_ties_3d_with_duplicates():
    g = np.arange(18, dtype=np.float32) * np.float32(0.1)
    xx, yy, zz = np.meshgrid(g, g, g, indexing="ij")
    coords = np.stack([xx.ravel(), yy.ravel(), zz.ravel()]).astype(np.float32)
    coords = np.concatenate([coords, coords[:, ::7]], axis=1)  # coincident copies
    w = np.ones(coords.shape[1], np.float32)
    check(coords, w, 0.15, 4.0, 0.25)


# ---- edge cases ---------------------------------------------------------------------------------

def test_single_point():
    g, o = check(np.array([[3.0], [4.0]], np.float32), np.ones(1, np.float32), 1.0, 0.5)
    assert g["ci"].tolist() == [0]


def test_all_points_identical_oversize_tile():
    # Zero extent in every dimension: every point falls in tile 0, a tile
    # larger than one shared-memory sort pass.
    n = 9000
    coords = np.full((2, n), 7.0, np.float32)
    w = np.random.default_rng(11).exponential(1.0, n).astype(np.float32)
    check(coords, w, 1.0, 2.0)


def test_dense_blob_in_one_tile():
    rng = np.random.default_rng(12)
    coords = np.concatenate([rng.normal(50, 0.05, (2, 12000)), rng.uniform(0, 100, (2, 2000))],
                            axis=1).astype(np.float32)
    w = rng.exponential(1.0, coords.shape[1]).astype(np.float32)
    check(coords, w, 0.05, 1.0, 0.1)


def test_dense_blob_in_one_tile_3d():
    # One tile holds most points: the nearest-higher search splits it into the
    # most cells a 3-D tile gets.
    rng = np.random.default_rng(13)
    coords = np.concatenate([rng.normal(20, 0.1, (3, 9000)), rng.uniform(0, 40, (3, 1500))],
                            axis=1).astype(np.float32)
    w = rng.exponential(1.0, coords.shape[1]).astype(np.float32)
    check(coords, w, 0.08, 2.0, 0.2, kernel="gaussian", kernel_params=(1.0, 0.05))


def test_infinite_outlier_distance_with_far_points():
    # dm = inf: the search box is the whole grid. Squared distances to the far
    # points overflow to inf; a candidate at infinite distance never becomes
    # the nearest higher (the search starts from delta = FLT_MAX).
    ev = W.single_2d(2000, seed=11)
    far = np.array([[3e19, -3e19, 3e19], [3e19, 3e19, -3e19]], np.float32)
    coords = np.concatenate([ev.coords, far], axis=1)
    w = np.concatenate([ev.weights, np.array([1.0, 1.0, 9.0], np.float32)])
    g, o = check(coords, w, 1.5, 5.0, np.inf, 1.5)
    assert (g["nh"][-3:] == -1).all()


def test_no_seeds_when_rhoc_is_unreachable():
    ev = W.single_2d(3000, seed=5)
    g, o = check(ev.coords, ev.weights, 1.5, 1e9, 1.5)
    assert (g["ci"] == -1).all()


def test_zero_rhoc():
    ev = W.single_2d(3000, seed=6)
    check(ev.coords, ev.weights, 1.5, 0.0, 1.5)


def test_workspace_reuse_across_sizes():
    c = clue.Clusterer(1.5, 5.0, 1.5)
    for n, seed in [(20000, 1), (2000, 2), (50000, 3), (100, 4)]:
        ev = W.single_2d(n, seed=seed)
        g = run_gpu(ev.coords, ev.weights, 1.5, 5.0, 1.5, clusterer=c)
        assert_identical(g, run_oracle(ev.coords, ev.weights, 1.5, 5.0, 1.5))


@pytest.mark.parametrize("host", [True, False])
def test_cluster_map_built_on_the_device(host):
    # utils/detail/get_clusters.hpp:24-49: cluster -> points, ids ascending.
    ev = W.blobs(30000, 5, 0.0, 30.0, 1.0, 0.1, seed=50)  # clusters larger than one sort pass
    g = run_gpu(ev.coords, ev.weights, 1.5, 5.0, 1.5, path="host" if host else "device")
    offsets, pts = g["clusterer"].getClustersDevice()
    ref_off, ref_pts = clue.clusters_csr(g["ci"])
    assert np.array_equal(offsets.cpu().numpy(), ref_off)
    assert np.array_equal(pts.cpu().numpy(), ref_pts)


def test_host_and_device_entry_points_agree():
    ev = W.single_2d(8000, seed=7)
    a = run_gpu(ev.coords, ev.weights, 1.5, 5.0, 1.5, path="host")
    b = run_gpu(ev.coords, ev.weights, 1.5, 5.0, 1.5, path="device")
    for k in ("rho", "nh", "seed", "ci"):
        assert np.array_equal(a[k], b[k])
    assert same_partition(a["ci"], b["ci"])


def _pipelined_against_device(ev, sizes, prm, kernel, unc=None, tags=None):
    import torch
    n = ev.n
    h = clue.PointsHost(ev.coords, ev.weights)
    h.is_seed = np.zeros(n, np.int32)
    h.rho = np.zeros(n, np.float32)
    h.nearest_higher = np.zeros(n, np.int32)
    if unc is not None:
        h.set_density_uncertainty(unc)
    if tags is not None:
        h.set_tags(tags)
    ch = clue.Clusterer(*prm)
    ch.make_clusters(h, clue.EuclideanMetric(), kernel, batch_item_sizes=sizes,
                     grid_mode=clue.GRID_PER_EVENT)
    dev = torch.device("cuda", 0)
    on_dev = lambda a, t: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev, t)
    d = clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev),
                          density_uncertainty=on_dev(unc, torch.float32),
                          tags=None if tags is None else on_dev(np.asarray(tags, np.int64).astype(np.int32),
                                                                torch.int32),
                          outputs=("cluster_index", "is_seed", "rho", "nearest_higher"))
    cd = clue.Clusterer(*prm)
    cd.make_clusters(d, clue.EuclideanMetric(), kernel, batch_item_sizes=sizes,
                     grid_mode=clue.GRID_PER_EVENT)
    assert np.array_equal(h.cluster_index, d.cluster_index.cpu().numpy())
    assert np.array_equal(h.is_seed, d.is_seed.cpu().numpy())
    assert np.array_equal(h.rho.view(np.int32), d.rho.cpu().numpy().view(np.int32))
    assert np.array_equal(h.nearest_higher, d.nearest_higher.cpu().numpy())
    assert ch.n_clusters() == cd.n_clusters()
    assert np.array_equal(ch.getSeeds(), cd.getSeeds())
    oh, kh = ch.getSampleAssociations()
    od, kd = cd.getSampleAssociations()
    assert kh == kd and np.array_equal(oh, od)
    for a, b in zip(ch.getClustersDevice(), cd.getClustersDevice()):
        assert torch.equal(a, b)
    return ch.host_pieces()


def test_pipelined_host_batch_equals_the_device_batch():
    # 2^23 points or more with one grid per event: the host entry point runs the
    # batch in pieces of whole events; ids, seeds and nearest-higher indices keep
    # their whole-batch numbering
    ev, sizes = W.batch_2d(640, 4096, 32768, seed=61)
    assert ev.n >= 1 << 23
    assert _pipelined_against_device(ev, sizes, (1.5, 5.0, 1.5), clue.FlatKernel(0.5)) >= 2


def test_pipelined_host_batch_with_empty_events():
    # items of size 0 among and after the events: every piece still holds
    # points (a piece of empty items alone would launch empty grids)
    ev, sizes = W.batch_2d(640, 4096, 32768, seed=61)
    sizes = with_empty_events(sizes, [0, 1, 64, 64, 200, 320, 321, 500] + [len(sizes)] * 3)
    assert _pipelined_against_device(ev, sizes, (1.5, 5.0, 1.5), clue.FlatKernel(0.5)) >= 2


def test_reused_tables_follow_the_batch_shape():
    # One clusterer keeps the tables (and the pipelined split) of the last batch
    # shape; a call with other event sizes over the same points must rebuild
    # them, and a return to the first shape must give the first results again.
    ev, sizes = W.batch_2d(640, 4096, 32768, seed=65)
    merged = np.concatenate([[sizes[0] + sizes[1]], sizes[2:]]).astype(np.uint32)
    n = ev.n

    def run(c, sz):
        h = clue.PointsHost(ev.coords, ev.weights)
        h.is_seed = np.zeros(n, np.int32)
        h.rho = np.zeros(n, np.float32)
        h.nearest_higher = np.zeros(n, np.int32)
        c.make_clusters(h, batch_item_sizes=sz, grid_mode=clue.GRID_PER_EVENT)
        return dict(ci=h.cluster_index.copy(), rho=h.rho.view(np.int32).copy(), nh=h.nearest_higher.copy(),
                    seed=h.is_seed.copy(), assoc=c.getSampleAssociations()[0], pieces=c.host_pieces())

    fresh = {k: run(clue.Clusterer(1.5, 5.0, 1.5), sz) for k, sz in (("a", sizes), ("b", merged))}
    reused = clue.Clusterer(1.5, 5.0, 1.5)
    for k in ("a", "b", "a", "a", "b"):
        got = run(reused, sizes if k == "a" else merged)
        for f in ("ci", "rho", "nh", "seed", "assoc"):
            assert np.array_equal(got[f], fresh[k][f]), (k, f)
        assert got["pieces"] == fresh[k]["pieces"] >= 2
    assert not np.array_equal(fresh["a"]["assoc"][:3], fresh["b"]["assoc"][:3])


def test_pipelined_host_batch_equals_the_device_batch_3d_gaussian():
    evs = [W.layered_3d(int(m), seed=70 + i) for i, m in
           enumerate(W.log_uniform_sizes(160, 16384, 131072, seed=71))]
    sizes = np.array([e.n for e in evs], np.uint32)
    ev = W.Event(np.ascontiguousarray(np.concatenate([e.coords for e in evs], axis=1)),
                 np.concatenate([e.weights for e in evs]))
    if ev.n < 1 << 23:
        pytest.skip("the 3-D batch came out below the pipelining size")
    assert _pipelined_against_device(ev, sizes, (3.0, 10.0, 4.0), clue.GaussianKernel(1.0, 1.0)) >= 2


def test_pipelined_host_batch_with_uncertainty_and_tags():
    # the tagged nearest-higher path and per-point uncertainties, staged piece by piece
    ev, sizes = W.batch_2d(640, 4096, 32768, seed=63)
    rng = np.random.default_rng(64)
    unc = rng.uniform(0.5, 1.5, ev.n).astype(np.float32)
    tags = rng.permutation(ev.n).astype(np.uint32)
    assert _pipelined_against_device(ev, sizes, (1.5, 5.0, 1.5), clue.FlatKernel(0.5), unc=unc,
                                     tags=tags) >= 2


def test_small_host_batch_runs_in_one_piece():
    ev, sizes = W.batch_2d(16, 256, 4096, seed=62)
    assert _pipelined_against_device(ev, sizes, (1.5, 5.0, 1.5), clue.FlatKernel(0.5)) == 1


# ---- launch tuning: results must not depend on it ---------------------------------------------

TUNINGS = [
    dict(density_union_x16_2d=0, density_union_x16_3d=0, label_jump_rounds=0, cell_points=1,
         density_shape=1, nh_shape=2, tile_binning=0),
    dict(density_union_x16_2d=1 << 20, density_union_x16_3d=1 << 20, label_jump_rounds=4, cell_points=8,
         density_shape=2, nh_shape=1, tile_binning=1),
    dict(density_union_x16_2d=16, density_union_x16_3d=24, label_jump_rounds=1, cell_points=3,
         density_shape=0, nh_shape=0, tile_binning=0),
]


@pytest.mark.parametrize("tuning", TUNINGS)
def test_results_do_not_depend_on_tuning_2d(tuning):
    ev, sizes = W.batch_2d(48, 256, 16384, seed=31)
    w = np.random.default_rng(5).exponential(1.0, ev.n).astype(np.float32)
    c = clue.Clusterer(1.5, 5.0, 1.5)
    c.set_tuning(**tuning)
    assert c.get_tuning() == tuning
    check(ev.coords, w, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_PER_EVENT, clusterer=c)


@pytest.mark.parametrize("tuning", TUNINGS)
def test_results_do_not_depend_on_tuning_exact_sums(tuning):
    # unit weights: every event takes the exact-sum density over the cells
    ev, sizes = W.batch_2d(48, 256, 32768, seed=33)
    c = clue.Clusterer(1.5, 5.0, 1.5)
    c.set_tuning(**tuning)
    check(ev.coords, ev.weights, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_PER_EVENT, clusterer=c,
          path="device")


@pytest.mark.parametrize("tuning", TUNINGS)
def test_results_do_not_depend_on_tuning_3d_showers(tuning):
    # dense showers: most density warps mix search boxes and stream their union
    ev = W.layered_3d(40000, seed=12)
    c = clue.Clusterer(3.0, 10.0, 4.0)
    c.set_tuning(**tuning)
    check(ev.coords, ev.weights, 3.0, 10.0, 4.0, kernel="gaussian", kernel_params=(1.0, 1.0),
          clusterer=c, path="device")


def test_set_tuning_rejects_out_of_range():
    c = clue.Clusterer(1.5, 5.0, 1.5)
    with pytest.raises(ValueError):
        c.set_tuning(density_union_x16_2d=-1)
    with pytest.raises(ValueError):
        c.set_tuning(label_jump_rounds=5)
    with pytest.raises(ValueError):
        c.set_tuning(cell_points=0)
    with pytest.raises(ValueError):
        c.set_tuning(density_shape=3)
    with pytest.raises(ValueError):
        c.set_tuning(nh_shape=-1)
    with pytest.raises(ValueError):
        c.set_tuning(tile_binning=2)
    with pytest.raises(KeyError):
        c.set_tuning(points_per_tile=64)


@pytest.mark.parametrize("batched", [False, True])
def test_autotune_keeps_results(batched):
    import torch
    dev = torch.device("cuda:0")
    if batched:
        ev, sizes = W.batch_2d(64, 256, 8192, seed=41)
        prm = (1.5, 5.0, 1.5)
        kern = clue.FlatKernel(0.5)
    else:
        ev, sizes = W.layered_3d(20000, seed=13), None
        prm = (3.0, 10.0, 4.0)
        kern = clue.GaussianKernel(1.0, 1.0)
    pts = clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev))
    c = clue.Clusterer(*prm)
    chosen = c.autotune(pts, clue.EuclideanMetric(), kern, batch_item_sizes=sizes,
                        grid_mode=clue.GRID_PER_EVENT, reps=1)
    assert c.get_tuning() == chosen
    o = run_oracle(ev.coords, ev.weights, *prm, kernel="flat" if batched else "gaussian",
                   kernel_params=(0.5,) if batched else (1.0, 1.0), sizes=sizes,
                   grid_mode=clue.GRID_PER_EVENT)
    assert_identical(dict(rho=pts.rho.cpu().numpy(), nh=pts.nearest_higher.cpu().numpy(),
                          seed=pts.is_seed.cpu().numpy(), ci=pts.cluster_index.cpu().numpy()), o)


# ---- CUDA-graph replay -------------------------------------------------------------------------

def _device_outputs(pts):
    return dict(rho=pts.rho.cpu().numpy(), nh=pts.nearest_higher.cpu().numpy(),
                seed=pts.is_seed.cpu().numpy(), ci=pts.cluster_index.cpu().numpy())


def test_graph_replay_reads_new_contents_and_recaptures_on_new_shapes():
    import torch
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream()
    ev, sizes = W.batch_2d(32, 256, 8192, seed=51)
    pts = clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev))
    c = clue.Clusterer(1.5, 5.0, 1.5)
    c.set_graphs(True)
    kw = dict(batch_item_sizes=sizes, grid_mode=clue.GRID_PER_EVENT, stream=stream)
    c.make_clusters(pts, **kw)
    assert not c.graph_replayed()
    first = _device_outputs(pts)
    assert_identical(first, run_oracle(ev.coords, ev.weights, 1.5, 5.0, 1.5, sizes=sizes,
                                       grid_mode=clue.GRID_PER_EVENT))
    c.make_clusters(pts, **kw)
    assert c.graph_replayed()
    assert_identical(_device_outputs(pts), run_oracle(ev.coords, ev.weights, 1.5, 5.0, 1.5, sizes=sizes,
                                                      grid_mode=clue.GRID_PER_EVENT))
    # new weights in the same buffer (the events stop being exact-sum ones): the replay reads them
    w2 = np.random.default_rng(52).exponential(1.0, ev.n).astype(np.float32)
    pts.weights.copy_(torch.from_numpy(w2).to(dev))
    c.make_clusters(pts, **kw)
    assert c.graph_replayed()
    assert_identical(_device_outputs(pts), run_oracle(ev.coords, w2, 1.5, 5.0, 1.5, sizes=sizes,
                                                      grid_mode=clue.GRID_PER_EVENT))
    # other event sizes over the same points: captured again
    sizes2 = np.array([ev.n // 2, ev.n - ev.n // 2], np.uint32)
    c.make_clusters(pts, batch_item_sizes=sizes2, grid_mode=clue.GRID_PER_EVENT, stream=stream)
    assert not c.graph_replayed()
    assert_identical(_device_outputs(pts), run_oracle(ev.coords, w2, 1.5, 5.0, 1.5, sizes=sizes2,
                                                      grid_mode=clue.GRID_PER_EVENT))
    c.set_graphs(False)
    c.make_clusters(pts, batch_item_sizes=sizes2, grid_mode=clue.GRID_PER_EVENT, stream=stream)
    assert not c.graph_replayed()


def test_sweep_statistics_of_a_profiled_run():
    # Profiling counts the sweeps' candidate tests without changing a result.
    ev = W.single_2d()
    c = clue.Clusterer(1.5, 5.0, 1.5)
    c.set_profiling(True)
    g, o = check(ev.coords, ev.weights, 1.5, 5.0, 1.5, clusterer=c, path="device")
    st = c.sweep_stats()
    assert st["density_items"] == (ev.n + 31) // 32
    # every point tests at least the candidates in range of it (unit weights:
    # rho = 1 + 0.5 (in range - 1))
    in_range = int((2.0 * (o.rho.astype(np.float64) - 1.0) + 1.0).sum())
    assert st["density_tests"] >= in_range > 0
    assert st["nh_cells_checked"] >= st["nh_cells_entered"] > 0
    assert st["nh_members_tested"] > 0
    c.set_profiling(False)
    with pytest.raises(RuntimeError):
        c.sweep_stats()


# ---- against the reference itself ---------------------------------------------------------------

def test_gpu_equals_the_reference_build():
    # The reference's own make_clusters (oracle/_ref, its serial CPU backend
    # compiled from its unmodified headers) on the same inputs: flat-kernel
    # results are identical bit for bit, single-event and batched (one grid for
    # the batch); with the Gaussian kernel the reference's std::exp differs
    # from clue_expf in the last bit of some densities, within 1e-5 relative,
    # and nearest-higher indices, seeds and clusters are identical.
    from oracle import ref as R
    if not R.available():
        pytest.skip("the reference build (make -C oracle ref) is not present")
    ev = W.blobs(1 << 17, 250, 0.0, 353.0, 1.0, 0.1, seed=9, weights="exponential")
    r = R.make_clusters(ev.coords, ev.weights, 1.5, 8.0, 2.0)
    assert_identical(run_gpu(ev.coords, ev.weights, 1.5, 8.0, 2.0, path="device"), r)
    evb, sizes = W.batch_2d(48, 256, 8192, seed=5)
    w = np.random.default_rng(7).exponential(1.0, evb.n).astype(np.float32)
    r = R.make_clusters_batched(evb.coords, w, sizes, 1.5, 5.0, 1.5)
    assert_identical(run_gpu(evb.coords, w, 1.5, 5.0, 1.5, sizes=sizes, grid_mode=clue.GRID_SHARED), r)
    l3 = W.layered_3d()
    r = R.make_clusters(l3.coords, l3.weights, 3.0, 10.0, 4.0, kernel="gaussian", kernel_params=(1.0, 1.0))
    g = run_gpu(l3.coords, l3.weights, 3.0, 10.0, 4.0, kernel="gaussian", kernel_params=(1.0, 1.0))
    np.testing.assert_allclose(g["rho"], r.rho, rtol=1e-5)
    assert np.array_equal(g["nh"], r.nearest_higher)
    assert np.array_equal(g["seed"], r.is_seed)
    assert np.array_equal(g["ci"], r.cluster_index)
