"""The entry point that allocates nothing, checked against the regular one.

clue_make_clusters_device_noalloc is for callers that may not allocate device
memory while they cluster (a framework whose caching allocator owns all device
memory, a real-time loop with a fixed reservation). It takes its scratch from
one array the library reserves on each GPU, so two calls in a row must not see
each other's leftovers. This file is collected last so that a failure here
leaves every other test already run.
"""

import ctypes as C

import numpy as np
import pytest

import cluestering_b200 as clue
from cluestering_b200 import _lib as L
from cluestering_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_POINTS = 16384


def _device_points(ev, torch):
    dev = torch.device("cuda", 0)
    return clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev))


def _outputs(p):
    return [p.rho.cpu().numpy().view(np.int32), p.nearest_higher.cpu().numpy(),
            p.is_seed.cpu().numpy(), p.cluster_index.cpu().numpy()]


def _noalloc(algo, p, stream, status):
    prm = algo.params()
    pts = clue.api._points_struct(p)
    return L.load().clue_make_clusters_device_noalloc(C.byref(prm), C.byref(pts),
                                                      None if status is None else status.data_ptr(),
                                                      stream.cuda_stream)


def test_noalloc_matches_the_workspace_path_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    stream = torch.cuda.Stream()
    status = torch.full((1,), 123, dtype=torch.int32, device="cuda")
    # Two different events, the second smaller: stale scratch from the first
    # call would show up in the second.
    events = [(W.single_2d(MAX_POINTS, seed=71), (1.5, 5.0, 1.5)),
              (W.blobs(5000, 8, 0.0, 60.0, 1.0, 0.1, seed=72, weights="exponential"), (1.5, 3.0, 2.0))]
    for ev, prm in events:
        ref = _device_points(ev, torch)
        algo = clue.Clusterer(*prm)
        algo.make_clusters(ref)
        got = _device_points(ev, torch)
        rc = _noalloc(algo, got, stream, status)
        assert rc == L.OK, L.load().clue_last_error()
        stream.synchronize()
        assert int(status.item()) == 0
        for a, b in zip(_outputs(got), _outputs(ref)):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("ndim", [3, 10])
def test_noalloc_takes_events_with_every_option_at_the_limit(ndim):
    # the largest scratch the entry point carves: sigma, density uncertainty
    # and tags on top of the coordinates, at the point limit (3-D adds the cell
    # layout, 10-D the most coordinate planes)
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(74 + ndim)
    if ndim == 3:
        ev = W.layered_3d(MAX_POINTS, seed=74)
        coords, weights, prm = ev.coords, ev.weights, (3.0, 10.0, 4.0)
    else:
        coords = rng.uniform(0.0, 4.0, (ndim, MAX_POINTS)).astype(np.float32)
        weights = np.ones(MAX_POINTS, np.float32)
        prm = (1.0, 2.0, 1.0)
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    sig = [rng.uniform(0.1, 0.5, MAX_POINTS).astype(np.float32) for _ in range(ndim)]
    unc = rng.uniform(0.5, 1.5, MAX_POINTS).astype(np.float32)
    tags = rng.permutation(MAX_POINTS).astype(np.int32)
    mk = lambda: clue.PointsDevice(t(coords), t(weights), sigma=[t(x) for x in sig],
                                   density_uncertainty=t(unc), tags=t(tags, torch.int32))
    algo = clue.Clusterer(*prm)
    ref = mk()
    algo.make_clusters(ref)
    got = mk()
    stream = torch.cuda.Stream()
    status = torch.full((1,), 123, dtype=torch.int32, device="cuda")
    rc = _noalloc(algo, got, stream, status)
    assert rc == L.OK, L.load().clue_last_error()
    stream.synchronize()
    assert int(status.item()) == 0
    for a, b in zip(_outputs(got), _outputs(ref)):
        assert np.array_equal(a, b)


def test_noalloc_rejects_events_above_the_limit():
    torch = pytest.importorskip("torch")
    ev = W.single_2d(MAX_POINTS + 1, seed=73)
    p = _device_points(ev, torch)
    algo = clue.Clusterer(1.5, 5.0, 1.5)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _noalloc(algo, p, torch.cuda.current_stream(), status)
    assert rc == L.ERR_INVALID_ARGUMENT
    assert b"at most 16384 points" in L.load().clue_last_error()


def test_noalloc_leaves_free_device_memory_unchanged():
    # The defining property: once the library's device code is loaded (the
    # first call), further calls take no device memory at all.
    torch = pytest.importorskip("torch")
    ev = W.single_2d(12000, seed=75)
    algo = clue.Clusterer(1.5, 5.0, 1.5)
    pts = [_device_points(ev, torch) for _ in range(4)]
    stream = torch.cuda.Stream()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert _noalloc(algo, pts[0], stream, status) == L.OK, L.load().clue_last_error()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for p in pts:
        assert _noalloc(algo, p, stream, status) == L.OK, L.load().clue_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    ref = _outputs(pts[0])
    for p in pts[1:]:
        for a, b in zip(_outputs(p), ref):
            assert np.array_equal(a, b)


def test_noalloc_without_status_and_in_one_dimension():
    # device_status may be NULL; a 1-D event takes the path without the cell
    # layout. Both match the workspace path.
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(76)
    x = np.concatenate([rng.normal(c, 0.5, 900) for c in (5.0, 20.0, 40.0)] +
                       [rng.uniform(0.0, 50.0, 300)]).astype(np.float32)[None, :]
    w = rng.exponential(1.0, x.shape[1]).astype(np.float32)
    for coords, weights, prm in [(x, w, (1.0, 4.0, 1.5)),
                                 (W.single_2d(8000, seed=77).coords, np.ones(8000, np.float32), (1.5, 5.0, 1.5))]:
        ev = W.Event(coords, weights)
        algo = clue.Clusterer(*prm)
        ref = _device_points(ev, torch)
        algo.make_clusters(ref)
        got = _device_points(ev, torch)
        stream = torch.cuda.Stream()
        assert _noalloc(algo, got, stream, None) == L.OK, L.load().clue_last_error()
        stream.synchronize()
        for a, b in zip(_outputs(got), _outputs(ref)):
            assert np.array_equal(a, b)
