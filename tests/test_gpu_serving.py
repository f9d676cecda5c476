"""The serving loop: every event's result is the same alone and in the mix.

Events of two profiles (2-D flat kernel, 3-D Gaussian kernel) and many sizes
are submitted while earlier batches run; each result must equal, bit for bit,
the single-event call on that event alone.
"""

import os
import threading
import time

import numpy as np
import pytest

import cluestering_b200 as clue
from cluestering_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P2 = (2, clue.Clusterer(1.5, 5.0, 1.5), clue.EuclideanMetric(), clue.FlatKernel(0.5))
P3 = (3, clue.Clusterer(3.0, 10.0, 4.0), clue.EuclideanMetric(), clue.GaussianKernel(1.0, 1.0))


def _events(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for e in range(n):
        size = int(np.exp(rng.uniform(np.log(300), np.log(30000))))
        if rng.uniform() < 0.75:
            out.append((0, W.blobs(size, max(1, round(20 * size / 16384)), 0, 100, 1.0, 0.1, seed * 1000 + e)))
        else:
            out.append((1, W.layered_3d(size, seed=seed * 1000 + e)))
    return out


def _alone(profile, ev):
    ndim, algo, metric, kernel = (P2, P3)[profile]
    p = clue.PointsHost(ev.coords, ev.weights)
    p.is_seed = np.zeros(ev.n, np.int32)
    p.rho = np.zeros(ev.n, np.float32)
    p.nearest_higher = np.zeros(ev.n, np.int32)
    algo.make_clusters(p, metric, kernel)
    return p


def _host_points(ev, pinned=False):
    if pinned:
        import torch
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        p = clue.PointsHost(pin(ev.coords), pin(ev.weights))
        p.cluster_index = pin(np.full(ev.n, -7, np.int32))
        p.is_seed = pin(np.zeros(ev.n, np.int32))
        p.rho = pin(np.zeros(ev.n, np.float32))
        p.nearest_higher = pin(np.zeros(ev.n, np.int32))
        return p
    p = clue.PointsHost(ev.coords, ev.weights)
    p.is_seed = np.zeros(ev.n, np.int32)
    p.rho = np.zeros(ev.n, np.float32)
    p.nearest_higher = np.zeros(ev.n, np.int32)
    return p


@pytest.mark.parametrize("pinned,timed", [(False, False), (True, False), (True, True)])
def test_results_are_the_same_alone_and_in_the_mix(pinned, timed):
    # timed: batches capped by learned device time, long ones on the high-priority stream
    evs = _events(60, seed=(1 if pinned else 2) + (10 if timed else 0))
    extra = dict(max_batch_ms=0.3, priority_ms=0.2) if timed else {}
    with clue.Server([P2, P3], max_inflight=3, max_batch_events=16, budget_bytes=2 << 30,
                     linger_us=500, **extra) as srv:
        pts = [_host_points(ev, pinned) for _, ev in evs]
        tickets = [srv.submit(prof, p) for (prof, _), p in zip(evs, pts)]
        srv.drain()
        assert all(srv.done(t) for t in tickets)
        st = srv.stats()
        assert st["completed"] == len(evs) and st["batches"] >= 2
    for (prof, ev), p in zip(evs, pts):
        a = _alone(prof, ev)
        assert np.array_equal(p.rho.view(np.int32), a.rho.view(np.int32))
        assert np.array_equal(p.nearest_higher, a.nearest_higher)
        assert np.array_equal(p.is_seed, a.is_seed)
        assert np.array_equal(p.cluster_index, a.cluster_index)


def _checker(prof, ev, **extra):
    kw = dict(kernel="flat", kernel_params=(0.5,)) if prof == 0 else \
        dict(kernel="gaussian", kernel_params=(1.0, 1.0))
    prm = (1.5, 5.0, 1.5) if prof == 0 else (3.0, 10.0, 4.0)
    return O.make_clusters(ev.coords, ev.weights, *prm, exp_mode=O.EXP_CLUE,
                           n_threads=os.cpu_count() or 1, **kw, **extra)


def _assert_checker(p, o):
    assert np.array_equal(p.rho.view(np.int32), o.rho.view(np.int32))
    assert np.array_equal(p.nearest_higher, o.nearest_higher)
    assert np.array_equal(p.is_seed, o.is_seed)
    assert np.array_equal(p.cluster_index, o.cluster_index)


def test_served_mix_matches_the_checker():
    # 200 events of the serving mix itself (80 % 2-D flat, 20 % 3-D Gaussian,
    # sizes log-uniform in [1,024, 262,144]), submitted at once so that they
    # share batches, each compared with the checker on that event alone.
    evs = list(W.serving_mix(200, seed=17))
    prof_of = [0 if ev.ndim == 2 else 1 for ev in evs]
    pts = [_host_points(ev, pinned=True) for ev in evs]
    with clue.Server([P2, P3], budget_bytes=8 << 30, max_inflight=4, max_batch_events=64,
                     max_batch_points=2_000_000) as srv:
        for prof, p in zip(prof_of, pts):
            srv.submit(prof, p)
        srv.drain()
        assert srv.stats()["batches"] < len(evs)
    for prof, ev, p in zip(prof_of, evs, pts):
        _assert_checker(p, _checker(prof, ev))


def test_arrivals_while_batches_run():
    evs = _events(80, seed=4)
    pts = [_host_points(ev, pinned=True) for _, ev in evs]
    with clue.Server([P2, P3], max_inflight=2, max_batch_events=8, linger_us=100) as srv:
        tickets = []

        def client():
            rng = np.random.default_rng(0)
            for (prof, _), p in zip(evs, pts):
                tickets.append(srv.submit(prof, p))
                time.sleep(rng.exponential(0.0005))

        th = threading.Thread(target=client)
        th.start()
        th.join()
        srv.drain()
        lat = srv.latencies_ms()
        st = srv.stats()
    assert len(lat) == len(evs) and (lat > 0).all()
    assert st["latency_p99_ms"] >= st["latency_p50_ms"] > 0
    assert st["points_completed"] == sum(ev.n for _, ev in evs)
    for (prof, ev), p in zip(evs, pts):
        assert np.array_equal(p.cluster_index, _alone(prof, ev).cluster_index)


def test_submit_rejects_what_the_server_cannot_take():
    ev = W.single_2d(2000, seed=5)
    with clue.Server([P2], budget_bytes=64 << 20, max_inflight=1, max_batch_events=4) as srv:
        big = W.single_2d(3_000_000, seed=6)
        with pytest.raises(MemoryError):
            srv.submit(0, clue.PointsHost(big.coords, big.weights))
        with pytest.raises(ValueError):
            srv.submit(0, clue.PointsHost(np.vstack([ev.coords, ev.coords[:1]]), ev.weights))


def _with_options(ev, kind, rng):
    """Host points of `ev` carrying per-point options (PointsHost.hpp:217-244)."""
    p = _host_points(ev, pinned=kind % 2 == 0)
    if kind in (1, 3):
        p.set_density_uncertainty(rng.uniform(0.5, 1.5, ev.n).astype(np.float32))
    if kind in (2, 3):
        p.set_tags(rng.permutation(ev.n).astype(np.int64))
    if kind == 4:
        p.set_sigma(0, rng.uniform(0.1, 0.6, ev.n).astype(np.float32))
    return p


def test_served_events_with_sigma_uncertainty_and_tags():
    # Events carrying uncertainties, tags or sigma share batches only with
    # events that carry the same options; each equals the checker's result
    # on that event alone with the same options.
    rng = np.random.default_rng(41)
    evs = _events(40, seed=41)
    kinds = [k % 5 for k in range(len(evs))]
    pts = [_with_options(ev, kind, rng) for (_, ev), kind in zip(evs, kinds)]
    with clue.Server([P2, P3], max_inflight=3, max_batch_events=8, budget_bytes=2 << 30,
                     linger_us=300) as srv:
        for (prof, _), p in zip(evs, pts):
            srv.submit(prof, p)
        srv.drain()
    for (prof, ev), p, kind in zip(evs, pts, kinds):
        extra = {}
        if p.density_uncertainty is not None:
            extra["unc"] = p.density_uncertainty
        if p.tags is not None:
            extra["tags"] = p.tags
        if kind == 4:
            extra["sigma"] = [p.sigma[0]] + [None] * (ev.ndim - 1)
        _assert_checker(p, _checker(prof, ev, **extra))


def test_admission_by_device_memory_budget():
    # A budget whose resident pool holds only a few events at a time: events
    # wait on the host until earlier ones complete, and every one completes
    # with the single-event result.
    evs = _events(50, seed=43)
    pts = [_host_points(ev, pinned=True) for _, ev in evs]
    cfg = dict(max_inflight=2, max_batch_events=4, max_batch_points=65536)
    with clue.Server([P2, P3], budget_bytes=1 << 30, **cfg) as srv:
        slots = srv.stats()["slot_bytes"]
    budget = slots + (3 << 20)  # the slots, and a pool of 3 MiB for the events' points
    with clue.Server([P2, P3], budget_bytes=budget, **cfg) as srv:
        for (prof, _), p in zip(evs, pts):
            srv.submit(prof, p)
        srv.drain()
        st = srv.stats()
    assert st["completed"] == len(evs)
    assert sum(ev.n * 4 * (ev.ndim + 1) for _, ev in evs) > 3 << 20
    assert st["admission_waits"] > 0
    assert 0 < st["resident_bytes_peak"] <= st["resident_pool_bytes"]
    assert st["slot_bytes"] + st["resident_pool_bytes"] <= budget
    for (prof, ev), p in zip(evs, pts):
        a = _alone(prof, ev)
        assert np.array_equal(p.cluster_index, a.cluster_index)
        assert np.array_equal(p.rho.view(np.int32), a.rho.view(np.int32))


def test_server_rejects_negative_time_targets():
    with pytest.raises(ValueError):
        clue.Server([P2], max_batch_ms=-1.0)
    with pytest.raises(ValueError):
        clue.Server([P2], priority_ms=float("nan"))
