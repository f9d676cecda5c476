"""Benchmark of libclue_sm100.so on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one batched make_clusters over the batch_2d workload: 4,096 2-D
events of log-uniform size in [256, 65,536] (46.5 M points), unit weights,
dc = 1.5, rhoc = 5, dm = 1.5, flat kernel, one tile grid per event. Inputs are
larger than L2 (126 MB), so no flush is needed between steps.

`value` is points/s with the inputs resident in HBM (device entry point);
`e2e` is the same metric through the host entry point with pinned host buffers,
so every step includes the host->device copy of coordinates and weights and the
device->host copy of the cluster ids. Extra keys report the plain per-event GPU
form (one make_clusters call per event with a host sync per event, the
reference's usage pattern), the 1,048,576-point single event and the serving
loop. With --impl reference the reference's own make_clusters (oracle/_ref:
its serial CPU backend compiled from its unmodified headers; the CPU
restatement in oracle/ where that build is absent) runs a bounded sample of
the same workload on all host cores, one share of the events per thread.

Under torchrun every rank clusters its own batch (events are independent: no
collective on the data path); time is the max over ranks and `value` the points
of all ranks divided by it.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/s batched+served vs plain per-event on same GPU; p50/p99 event latency"
CONFIG = {
    "workload": "batch_2d: 4096 2-D events, sizes log-uniform [256, 65536], 20*n/16384 blobs "
                "(sigma 1) in [0,100]^2 + 10% noise, unit weights; dc=1.5 rhoc=5 dm=1.5 flat(0.5), "
                "Euclidean; one tile grid per event",
    "l2": "inputs (~0.58 GB) exceed L2; no flush",
}
# Algorithmic bytes per point (4-byte values), 2-D: density reads coordinates
# and weight and writes rho (4D + 8); nearest higher reads coordinates, rho and
# index and writes nh (4D + 12); the whole pipeline moves 20D + 64.
BYTES_PER_POINT = {"density": lambda D: 4 * D + 8, "nearest_higher": lambda D: 4 * D + 12,
                   "pipeline": lambda D: 20 * D + 64}
# DRAM bytes (read + write) per point of each sweep, from one ncu capture
# (--set full) of the 1,024-event batch (10,621,973 points): 922.2 MB for the
# density sweep, 738.3 MB for the nearest-higher search; a launch's traffic
# grows with the points it processes.
DRAM_BYTES_PER_POINT = {"density": 86.8, "nearest_higher": 69.5}
# Warp instructions per point of each sweep (smsp__inst_executed.sum / points),
# from the same capture: 2.653 G for density, 1.609 G for nearest higher. The
# sweeps are bound by instruction issue: the issue roofline is SMs x 4
# schedulers x one warp instruction per cycle at the SM clock sampled during
# the timed steps.
INST_PER_POINT = {"density": 249.8, "nearest_higher": 151.5}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    from cluestering_b200 import replicas as R
    r = R.from_env()
    R.init(r, backend="nccl")
    return r.world, r.rank, r.local


def barrier(world):
    from cluestering_b200 import replicas as R
    R.barrier(R.from_env())


def max_over_ranks(x: float, world: int) -> float:
    from cluestering_b200 import replicas as R
    return R.max_over_ranks(x, R.from_env())


def cpu_reference(ev, sizes, budget_points: int, threads: int):
    """Times the CPU restatement on the first events of the batch (bounded sample).
    Returns (points/s, sample description, points, events, checker result)."""
    from oracle import oracle as O
    total, k = 0, 0
    while k < len(sizes) and total + int(sizes[k]) <= budget_points:
        total += int(sizes[k])
        k += 1
    k = max(k, 1)
    total = int(sizes[:k].sum())
    t0 = time.perf_counter()
    res = O.make_clusters_batched(ev.coords[:, :total], ev.weights[:total], sizes[:k], 1.5, 5.0, 1.5,
                                  shared_grid=False, n_threads=threads)
    dt = time.perf_counter() - t0
    return (total / dt, f"first {k} events of the batch ({total} points), all events clustered", total, k,
            res)


def reference_cpu(ev, sizes, budget_points: int, threads: int):
    """Times the reference's own make_clusters (oracle/_ref: its serial CPU
    backend, compiled from its unmodified headers) on the first events of the
    batch, a bounded sample. Like the reference's multi-threaded throughput
    driver (benchmark/throughput/main.cpp), each of `threads` host threads
    clusters its own share of the events with its own Clusterer, here through
    the reference's batched make_clusters. Returns (points/s, sample
    description, points, events), or None when the build is absent."""
    from oracle import ref as Rf
    if not Rf.available():
        return None
    total, k = 0, 0
    while k < len(sizes) and total + int(sizes[k]) <= budget_points:
        total += int(sizes[k])
        k += 1
    k = max(k, 1)
    offs = np.concatenate([[0], np.cumsum(sizes[:k].astype(np.int64))])
    total = int(offs[-1])
    # contiguous shares of about equal points
    cuts = [0]
    for t in range(1, threads):
        cuts.append(int(np.searchsorted(offs, total * t / threads)))
    cuts.append(k)
    cuts = sorted(set(cuts))
    jobs = [(cuts[i], cuts[i + 1]) for i in range(len(cuts) - 1) if cuts[i + 1] > cuts[i]]

    def work(a, b):
        p0, p1 = int(offs[a]), int(offs[b])
        Rf.make_clusters_batched(ev.coords[:, p0:p1], ev.weights[p0:p1], sizes[a:b], 1.5, 5.0, 1.5)

    t0 = time.perf_counter()
    th = [threading.Thread(target=work, args=j) for j in jobs]
    for t in th:
        t.start()
    for t in th:
        t.join()
    dt = time.perf_counter() - t0
    return (total / dt, f"first {k} events of the batch ({total} points), {len(jobs)} threads, each "
                        f"clustering its share of the events with the reference's batched make_clusters",
            total, k)


def parity_sample(algo, coords_d, weights_d, sizes, stream, timed_labels, ref, n_points, n_events):
    """Clusters the benchmark batch once more with every output requested and
    compares the first `n_events` events (densities as bits, nearest higher,
    seed flags, cluster ids) with the checker's result `ref` on those events;
    the run's cluster ids must also equal those of the timed runs."""
    import cluestering_b200 as clue
    full = clue.PointsDevice(coords_d, weights_d)
    algo.make_clusters(full, batch_item_sizes=sizes, grid_mode=clue.GRID_PER_EVENT, stream=stream)
    rho_all = full.rho.cpu().numpy()
    rho = rho_all[:n_points]
    ci_all = full.cluster_index.cpu().numpy()
    # unit weights, flat kernel: rho_i = 1 + 0.5 (candidates in range - 1), exactly
    in_range = float((2.0 * (rho_all.astype(np.float64) - 1.0) + 1.0).sum())
    same = (np.array_equal(rho.view(np.int32), ref.rho.view(np.int32))
            and np.array_equal(full.nearest_higher[:n_points].cpu().numpy(), ref.nearest_higher)
            and np.array_equal(full.is_seed[:n_points].cpu().numpy(), ref.is_seed)
            and np.array_equal(ci_all[:n_points], ref.cluster_index))
    return ({"events": int(n_events), "points": int(n_points), "identical": bool(same),
             "timed_run_labels_identical": bool(np.array_equal(ci_all, timed_labels)),
             "compared": "rho bits, nearest_higher, is_seed, cluster_index against the CPU checker"},
            in_range)


def run_reference(args, world, rank):
    from cluestering_b200 import workloads as W
    if rank != 0:
        return 0
    ev, sizes = W.batch_2d(n_events=args.events)
    threads = os.cpu_count() or 1
    budget = args.cpu_sample_points
    from oracle import ref as Rf
    kind = "reference" if Rf.available() else "port"

    def one(budget_points):
        if kind == "reference":
            return reference_cpu(ev, sizes, budget_points, threads)[:3]
        return cpu_reference(ev, sizes, budget_points, threads)[:3]

    for _ in range(args.warmup):
        one(budget // 4)
    vals = []
    for _ in range(args.steps):
        v, sample, pts = one(budget)
        vals.append(v)
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": pts / value * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": CONFIG,
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import torch

    import cluestering_b200 as clue
    from cluestering_b200 import _lib as L
    from cluestering_b200 import workloads as W

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    hbm_peak, peak_kind = measured_peaks()

    # ---- workload, resident in HBM --------------------------------------------------------------
    from cluestering_b200 import replicas as R
    ev, sizes = W.batch_2d(n_events=args.events, seed=R.event_seed(rank))
    n_total = int(sizes.sum())
    coords_d = torch.from_numpy(ev.coords).to(dev)
    weights_d = torch.from_numpy(ev.weights).to(dev)
    pts = clue.PointsDevice(coords_d, weights_d, outputs=("cluster_index",))
    algo = clue.Clusterer(1.5, 5.0, 1.5, device=local)
    # launch choices picked by the library's autotuner on this batch (results do not depend on them)
    tuning = algo.autotune(pts, batch_item_sizes=sizes, grid_mode=clue.GRID_PER_EVENT, stream=stream, reps=1)
    # the batch is the same every step: the first run is captured as a CUDA graph, the rest replay it
    algo.set_graphs(True)

    def step():
        algo.make_clusters(pts, batch_item_sizes=sizes, grid_mode=clue.GRID_PER_EVENT, stream=stream,
                           synchronize=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.nvtx.range_push("timed")  # profilers select the timed steps by this range
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = start.elapsed_time(end) / args.steps
    replayed = algo.graph_replayed()
    barrier(world)
    ms_max = max_over_ranks(ms, world)
    points_all = R.sum_over_ranks(n_total, R.from_env())
    value = R.job_throughput(points_all, ms_max)
    n_clusters = algo.n_clusters()
    launches_per_run = algo.kernel_launches()  # counted by the library at each launch site

    # ---- stage times and sweep statistics of one profiled run (outside the timed region) ---------
    algo.set_profiling(True)
    step()
    stage = algo.stage_ms()
    sweeps = algo.sweep_stats()
    algo.set_profiling(False)
    dom = max(("density", "nearest_higher"), key=lambda k: stage[k])
    D = 2
    achieved = BYTES_PER_POINT[dom](D) * n_total / (stage[dom] * 1e-3) / 1e9
    n_sms = torch.cuda.get_device_properties(dev).multi_processor_count

    # ---- end to end through the host entry point ------------------------------------------------
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    h = clue.PointsHost(pin(ev.coords), pin(ev.weights))
    h.cluster_index = pin(np.zeros(n_total, np.int32))
    algo_h = clue.Clusterer(1.5, 5.0, 1.5, device=local)
    algo_h.set_tuning(**tuning)
    algo_h.set_graphs(True)
    hstream = torch.cuda.Stream(device=dev)
    for _ in range(max(1, args.warmup // 2)):
        algo_h.make_clusters(h, batch_item_sizes=sizes, grid_mode=clue.GRID_PER_EVENT, stream=hstream)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        algo_h.make_clusters(h, batch_item_sizes=sizes, grid_mode=clue.GRID_PER_EVENT, stream=hstream)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    e2e_ms = max_over_ranks(e2e_ms, world)
    e2e_value = R.job_throughput(points_all, e2e_ms)
    timed_labels = pts.cluster_index.cpu().numpy()
    same = bool(np.array_equal(h.cluster_index, timed_labels))
    in_range = None
    pieces = algo_h.host_pieces()  # uploads and downloads overlap the clustering of other pieces

    # ---- CPU checker on the batch's first events: baseline timing and parity sample -------------
    parity = None
    if rank == 0:
        threads = os.cpu_count() or 1
        cpu_val, cpu_sample, cpu_pts, cpu_k, cpu_res = cpu_reference(ev, sizes, args.cpu_sample_points,
                                                                     threads)
        parity, in_range = parity_sample(algo, coords_d, weights_d, sizes, stream, timed_labels, cpu_res,
                                         cpu_pts, cpu_k)
        del cpu_res
        # the reference's own code where it was built, else the restatement
        ref_all = reference_cpu(ev, sizes, args.cpu_sample_points, threads)
        cpu_kind = "port"
        if ref_all is not None:
            cpu_val, cpu_sample = ref_all[0], ref_all[1]
            cpu_kind = "reference"
            ser_val, ser_sample = reference_cpu(ev, sizes, args.cpu_serial_points, 1)[:2]
        else:
            ser_val, ser_sample, _, _, _ = cpu_reference(ev, sizes, args.cpu_serial_points, 1)

    extras = {}
    if rank == 0 and not args.skip_extras:
        extras = run_extras(args, ev, sizes, local, stream, hbm_peak)
        extras["configs"] = run_configs(args, local)
        del coords_d, weights_d, pts
        torch.cuda.empty_cache()
        extras["serving"] = run_serving(args, local)

    if rank != 0:
        return 0
    clk = clocks.summary()
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "traffic": DRAM_BYTES_PER_POINT[dom] * n_total,
            "peak_kind": peak_kind,
            "note": "the sweeps are instruction-issue bound, not HBM bound: each point tests hundreds "
                    "of candidate records read from shared memory; achieved counts algorithmic bytes, "
                    "traffic is ncu DRAM bytes per point scaled to this launch; `issue` is the bound "
                    "they hit"}
    f_hz = (clk["sm_mhz"] or 1965.0) * 1e6
    roof["issue"] = {
        k: {"warp_inst_per_point": INST_PER_POINT[k],
            "achieved_warp_inst_per_s": INST_PER_POINT[k] * n_total / (stage[k] * 1e-3),
            "peak_warp_inst_per_s": n_sms * 4 * f_hz,
            "frac": INST_PER_POINT[k] * n_total / (stage[k] * 1e-3) / (n_sms * 4 * f_hz)}
        for k in ("density", "nearest_higher")}
    roof["issue_frac"] = roof["issue"][dom]["frac"]
    roof["pairs"] = {
        "density_candidate_tests_per_point": sweeps["density_tests"] / n_total,
        "density_candidate_tests_per_s": sweeps["density_tests"] / (stage["density"] * 1e-3),
        "density_in_range_per_point": in_range / n_total if in_range else None,
        "density_in_range_pairs_per_s": in_range / (stage["density"] * 1e-3) if in_range else None,
        "nearest_higher_members_tested_per_point": sweeps["nh_members_tested"] / n_total,
        "nearest_higher_cells_checked_per_point": sweeps["nh_cells_checked"] / n_total,
        "nearest_higher_member_tests_per_s": sweeps["nh_members_tested"] / (stage["nearest_higher"] * 1e-3),
    }
    roof["pairs_per_s"] = roof["pairs"]["density_in_range_pairs_per_s"]
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(CONFIG, points_per_step=int(points_all), events_per_step=len(sizes) * world,
                       tuning=tuning, cuda_graph_replay=replayed,
                       parallelism=f"replicas x{world} (events sharded by rank, no collective)"),
        "e2e": {"value": e2e_value, "unit": "points/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(ev.coords.nbytes + ev.weights.nbytes),
                "d2h_bytes_per_step": int(n_total * 4), "matches_device_path": same,
                "pipelined_pieces": pieces},
        "gpu_launches": launches_per_run * args.steps,
        "n_clusters": n_clusters,
        "stage_ms": {k: round(v, 4) for k, v in stage.items()},
        "roofline": roof,
        "clocks": clk,
        "cpu_baseline": {"value": cpu_val, "unit": "points/s", "cores": threads,
                         "kind": cpu_kind, "sample": cpu_sample,
                         "serial_1_core": {"value": ser_val, "unit": "points/s", "cores": 1,
                                           "sample": ser_sample}},
        "parity_sample": parity,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)
    return 0


def run_extras(args, ev, sizes, local, stream, hbm_peak):
    """Plain per-event GPU form, the 1M-point single event and (when present) serving."""
    import torch

    import cluestering_b200 as clue
    from cluestering_b200 import workloads as W

    out = {}
    dev = torch.device("cuda", local)
    # plain per-event: one device call per event and a host sync after each
    offs = np.concatenate([[0], np.cumsum(sizes)])
    n_ev = min(len(sizes), args.plain_events)
    views = []
    coords_d = torch.from_numpy(ev.coords).to(dev)
    weights_d = torch.from_numpy(ev.weights).to(dev)
    for e in range(n_ev):
        a, b = int(offs[e]), int(offs[e + 1])
        views.append(clue.PointsDevice(coords_d[:, a:b], weights_d[a:b], outputs=("cluster_index",)))
    algo = clue.Clusterer(1.5, 5.0, 1.5, device=local)
    for v in views[:8]:
        algo.make_clusters(v, stream=stream)
    lat = []
    t0 = time.perf_counter()
    for v in views:
        t1 = time.perf_counter()
        algo.make_clusters(v, stream=stream)  # synchronises
        lat.append((time.perf_counter() - t1) * 1e3)
    dt = time.perf_counter() - t0
    pts_plain = int(offs[n_ev])
    out["plain_per_event"] = {"value": pts_plain / dt, "unit": "points/s", "events": n_ev,
                              "latency_p50_ms": float(np.percentile(lat, 50)),
                              "latency_p99_ms": float(np.percentile(lat, 99))}
    del views, coords_d, weights_d

    # single large event (1,048,576 points, exponential weights)
    big = W.large_2d()
    bc = torch.from_numpy(big.coords).to(dev)
    bw = torch.from_numpy(big.weights).to(dev)
    bp = clue.PointsDevice(bc, bw, outputs=("cluster_index",))
    algo1 = clue.Clusterer(1.5, 8.0, 2.0, device=local)
    algo1.autotune(bp, stream=stream, reps=1)
    for _ in range(3):
        algo1.make_clusters(bp, stream=stream)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    reps = 10
    for _ in range(reps):
        algo1.make_clusters(bp, stream=stream, synchronize=False)
    e.record(stream)
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    algo1.set_profiling(True)
    algo1.make_clusters(bp, stream=stream)
    st = algo1.stage_ms()
    sweeps1 = algo1.sweep_stats()
    nb = BYTES_PER_POINT["pipeline"](2) * big.n
    out["single_event_1M"] = {
        "ms": ms, "points_per_s": big.n / (ms * 1e-3),
        "hbm_frac_pipeline": nb / (ms * 1e-3) / 1e9 / hbm_peak,
        "stage_ms": {k: round(v, 4) for k, v in st.items()},
        "density_gbs": BYTES_PER_POINT["density"](2) * big.n / (st["density"] * 1e-3) / 1e9,
        "nearest_higher_gbs": BYTES_PER_POINT["nearest_higher"](2) * big.n / (st["nearest_higher"] * 1e-3) / 1e9,
        "density_candidate_tests_per_point": sweeps1["density_tests"] / big.n,
        "nearest_higher_members_tested_per_point": sweeps1["nh_members_tested"] / big.n,
    }
    return out


def run_configs(args, local):
    """The single-event configurations on the GPU (device-resident inputs, median
    of 20 calls with a sync each) and in the CPU checker on 1 core and on all
    host cores (median of 3): 16,384-point 2-D, 1,048,576-point 2-D and
    10,000-hit 3-D layered events."""
    import torch

    import cluestering_b200 as clue
    from cluestering_b200 import workloads as W
    from oracle import oracle as O
    dev = torch.device("cuda", local)
    cases = [("single_2d_16384", W.single_2d(), (1.5, 5.0, 1.5), "flat", (0.5,)),
             ("large_2d_1048576", W.large_2d(), (1.5, 8.0, 2.0), "flat", (0.5,)),
             ("layered_3d_10000", W.layered_3d(), (3.0, 10.0, 4.0), "gaussian", (1.0, 1.0))]
    out = {}
    for name, ev, prm, kern, kp in cases:
        pts = clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev),
                                outputs=("cluster_index",))
        algo = clue.Clusterer(*prm, device=local)
        k = clue.FlatKernel(*kp) if kern == "flat" else clue.GaussianKernel(*kp)
        for _ in range(3):
            algo.make_clusters(pts, clue.EuclideanMetric(), k)
        ts = []
        for _ in range(20):
            t0 = time.perf_counter()
            algo.make_clusters(pts, clue.EuclideanMetric(), k)
            ts.append((time.perf_counter() - t0) * 1e3)
        row = {"points": ev.n, "gpu_ms": float(np.median(ts))}
        for cores in (1, os.cpu_count() or 1):
            cs = []
            for _ in range(1 if (cores == 1 and ev.n > 100000) else 3):
                t0 = time.perf_counter()
                O.make_clusters(ev.coords, ev.weights, *prm, kernel=kern, kernel_params=kp, n_threads=cores)
                cs.append((time.perf_counter() - t0) * 1e3)
            row[f"cpu_ms_{cores}_cores" if cores > 1 else "cpu_ms_1_core"] = float(np.median(cs))
        out[name] = row
    return out


def run_serving(args, local):
    """Serving form on a mixed stream: saturated throughput, then Poisson
    arrivals at fractions of it, with per-event latency (completion - arrival),
    and the configured stream of `serve_stream_total` arrivals at half of the
    peak load. Arrivals cycle through a pool of `serve_events` distinct
    generated events. The plain per-event form (one synchronous call per event)
    runs on the same pool for comparison."""
    import torch

    import cluestering_b200 as clue
    from cluestering_b200 import workloads as W

    evs = list(W.serving_mix(args.serve_events))
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    pts = []
    for ev in evs:
        p = clue.PointsHost(pin(ev.coords), pin(ev.weights))
        p.cluster_index = pin(np.zeros(ev.n, np.int32))
        pts.append(p)
    profs = [(2, clue.Clusterer(1.5, 5.0, 1.5, device=local), clue.EuclideanMetric(), clue.FlatKernel(0.5)),
             (3, clue.Clusterer(3.0, 10.0, 4.0, device=local), clue.EuclideanMetric(),
              clue.GaussianKernel(1.0, 1.0))]
    prof_of = [0 if ev.ndim == 2 else 1 for ev in evs]
    total = sum(ev.n for ev in evs)
    mean_pts = total / len(evs)
    cfg = dict(device=local, budget_bytes=40 << 30, max_inflight=args.serve_inflight,
               max_batch_events=args.serve_batch_events, max_batch_points=args.serve_batch_points,
               linger_us=args.serve_linger_us, max_batch_ms=args.serve_batch_ms,
               priority_ms=args.serve_priority_ms)
    out = {"events": len(evs), "points": total, "mix": "80% 2-D single_2d-style, 20% 3-D layered_3d-style",
           "sizes": "log-uniform [1024, 262144]", "config": cfg,
           "method": "each server first clusters 64 events (not counted), which also seeds its cost "
                     "model; peak = all pool events submitted at once; loads = Poisson arrivals "
                     "cycling through the pool of distinct events; the configured stream is "
                     "`stream_total` arrivals at half of the peak load"}
    warm = min(64, len(evs))

    def warm_up(srv):
        for i in range(warm):
            srv.submit(prof_of[i], pts[i])
        srv.drain()

    with clue.Server(profs, **cfg) as srv:
        warm_up(srv)
        t0 = time.perf_counter()
        for i, p in enumerate(pts):
            srv.submit(prof_of[i], p)
        srv.drain()
        peak = total / (time.perf_counter() - t0)
        st = srv.stats()
    out["peak_points_per_s"] = peak
    out["budget"] = {"budget_bytes": cfg["budget_bytes"], "slot_bytes": st["slot_bytes"],
                     "resident_pool_bytes": st["resident_pool_bytes"],
                     "max_batch_points": st["max_batch_points"]}
    peak_events = peak / mean_pts
    rng = np.random.default_rng(0)

    def offered(f, arrivals):
        # arrival k is pool event k mod len(evs); repeats of one event are
        # len(evs) arrivals apart, long after the earlier one completed
        order = [k % len(evs) for k in range(arrivals)]
        points = sum(evs[i].n for i in order)
        with clue.Server(profs, **cfg) as srv:
            warm_up(srv)
            gaps = rng.exponential(1.0 / (f * peak_events), size=len(order))
            t_next = time.perf_counter()
            t0 = t_next
            for k, i in enumerate(order):
                t_next += gaps[k]
                while time.perf_counter() < t_next:
                    pass
                srv.submit(prof_of[i], pts[i])
            srv.drain()
            dt = time.perf_counter() - t0
            lat = srv.latencies_ms()[warm:]
            st = srv.stats()
        return {"load": f, "arrivals": arrivals, "points_per_s": points / dt,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "batches": st["batches"], "resident_bytes_peak": st["resident_bytes_peak"],
                "admission_waits": st["admission_waits"]}

    out["loads"] = [offered(f, args.serve_stream) for f in args.serve_loads]
    if args.serve_stream_total > 0:
        out["configured_stream"] = offered(0.5, args.serve_stream_total)
        half = out["configured_stream"]
    else:
        half = min(out["loads"], key=lambda r: abs(r["load"] - 0.5))
    out["p50_ms_at_half_load"], out["p99_ms_at_half_load"] = half["p50_ms"], half["p99_ms"]
    # plain per-event on the same pool
    algos = [profs[0][1], profs[1][1]]
    for i in range(min(16, len(evs))):
        algos[prof_of[i]].make_clusters(pts[i], profs[prof_of[i]][2], profs[prof_of[i]][3])
    t0 = time.perf_counter()
    for i, p in enumerate(pts):
        algos[prof_of[i]].make_clusters(p, profs[prof_of[i]][2], profs[prof_of[i]][3])
    plain = total / (time.perf_counter() - t0)
    out["plain_per_event_points_per_s"] = plain
    out["speedup_vs_plain"] = peak / plain
    return out


def run_layered_3d(args):
    """One layered 3-D event of 262,144 hits (lognormal energies, Gaussian kernel,
    dc = 3, rhoc = 10, dm = 4): the largest 3-D event of the serving mix, whose
    density keeps the reference's order. Two runs; profiles capture the second."""
    import torch

    import cluestering_b200 as clue
    from cluestering_b200 import workloads as W
    ev = W.layered_3d(262144, seed=11)
    dev = torch.device("cuda", 0)
    pts = clue.PointsDevice(torch.from_numpy(ev.coords).to(dev), torch.from_numpy(ev.weights).to(dev),
                            outputs=("cluster_index",))
    algo = clue.Clusterer(3.0, 10.0, 4.0)
    for _ in range(2):
        algo.make_clusters(pts, clue.EuclideanMetric(), clue.GaussianKernel(1.0, 1.0))
    algo.set_profiling(True)
    algo.make_clusters(pts, clue.EuclideanMetric(), clue.GaussianKernel(1.0, 1.0))
    st = algo.stage_ms()
    print(json.dumps({"case": "layered-3d", "points": ev.n, "n_clusters": algo.n_clusters(),
                      "stage_ms": {k: round(v, 4) for k, v in st.items()}}), flush=True)
    return 0


def run_large_2d(args):
    """The 1,048,576-point 2-D event (exponential weights, dc = 1.5, rhoc = 8,
    dm = 2): median of 10 device-timed runs after warm-up, then stage times and
    sweep statistics of one profiled run. Profiles capture its launches."""
    import torch

    import cluestering_b200 as clue
    from cluestering_b200 import workloads as W
    big = W.large_2d()
    dev = torch.device("cuda", 0)
    bp = clue.PointsDevice(torch.from_numpy(big.coords).to(dev), torch.from_numpy(big.weights).to(dev),
                           outputs=("cluster_index",))
    algo = clue.Clusterer(1.5, 8.0, 2.0)
    stream = torch.cuda.Stream(device=dev)
    for _ in range(max(3, args.warmup)):
        algo.make_clusters(bp, stream=stream)
    times = []
    for _ in range(10):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        algo.make_clusters(bp, stream=stream, synchronize=False)
        e.record(stream)
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    algo.set_profiling(True)
    algo.make_clusters(bp, stream=stream)
    print(json.dumps({"case": "large-2d", "points": big.n, "ms": float(np.median(times)),
                      "stage_ms": {k: round(v, 4) for k, v in algo.stage_ms().items()},
                      "sweeps": algo.sweep_stats(), "kernel_launches": algo.kernel_launches()}), flush=True)
    return 0


def run_one_tile(args):
    """One event of 16,384 points uniform in [0, 10]^2 with a single tile (dc = 0.3): every
    density warp streams the same 16,384 candidates, which isolates the per-candidate cost
    (instructions per candidate = warp instructions / (512 warps x 16,384))."""
    import torch

    import cluestering_b200 as clue
    n = 16384
    x = np.random.default_rng(0).uniform(0, 10, (2, n)).astype(np.float32)
    dev = torch.device("cuda", 0)
    pts = clue.PointsDevice(torch.from_numpy(x).to(dev), torch.ones(n, device=dev))
    algo = clue.Clusterer(0.3, 5.0, 0.3, points_per_tile=1 << 24)
    for _ in range(max(1, args.warmup)):
        algo.make_clusters(pts)
    algo.set_profiling(True)
    algo.make_clusters(pts)
    st = algo.stage_ms()
    print(json.dumps({"case": "one-tile", "points": n, "candidates_per_point": n,
                      "stage_ms": {k: round(v, 4) for k, v in st.items()},
                      "kernel_launches": algo.kernel_launches()}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-points", type=int, default=3_000_000)
    ap.add_argument("--cpu-serial-points", type=int, default=600_000,
                    help="sample of the one-core checker timing (the serial backend's setting)")
    ap.add_argument("--plain-events", type=int, default=4096)
    ap.add_argument("--events", type=int, default=4096,
                    help="events per batch (4096 is the benchmark; fewer only for profiling)")
    ap.add_argument("--serve-events", type=int, default=3000,
                    help="distinct generated events the serving arrivals cycle through")
    ap.add_argument("--serve-inflight", type=int, default=4)
    ap.add_argument("--serve-batch-events", type=int, default=64)
    ap.add_argument("--serve-batch-points", type=int, default=2_000_000)
    ap.add_argument("--serve-linger-us", type=int, default=200)
    ap.add_argument("--serve-batch-ms", type=float, default=2.0)
    ap.add_argument("--serve-priority-ms", type=float, default=1.5)
    ap.add_argument("--serve-stream", type=int, default=12000, help="arrivals per offered load")
    ap.add_argument("--serve-stream-total", type=int, default=200_000,
                    help="arrivals of the configured stream at half of the peak load (0: skip)")
    ap.add_argument("--serve-loads", type=float, nargs="*", default=[0.1, 0.25, 0.5, 0.75, 1.0])
    ap.add_argument("--skip-extras", action="store_true")
    ap.add_argument("--case", choices=["one-tile", "layered-3d", "large-2d"], default=None,
                    help="profiling case instead of the benchmark: 'one-tile' clusters one "
                         "16,384-point event whose points all share one tile, so every warp of "
                         "the density sweep streams the same box; 'layered-3d' clusters one "
                         "262,144-hit layered 3-D event (the serving mix's heaviest kind); "
                         "'large-2d' the 1,048,576-point event")
    args = ap.parse_args()
    if args.case == "one-tile":
        return run_one_tile(args)
    if args.case == "layered-3d":
        return run_layered_3d(args)
    if args.case == "large-2d":
        return run_large_2d(args)
    if args.impl == "reference":
        # CPU arm: rank 0 times the CPU restatement; other ranks have no work.
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")),
                             int(os.environ.get("RANK", "0")))
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
