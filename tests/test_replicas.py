"""The multi-GPU replica bookkeeping with two gloo ranks on CPU.

bench.py runs one process per GPU; each rank clusters its own shard of events
and the ranks only meet for a barrier and the max / sum of their numbers. The
same calls run here over gloo, in two spawned processes, together with a real
(CPU checker) clustering of each rank's shard so the per-rank work differs.
"""

import os
import socket

import numpy as np
import pytest

pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from cluestering_b200 import replicas as R
    from cluestering_b200 import workloads as W
    from oracle import oracle as O

    r = R.from_env()
    assert R.init(r, backend="gloo", timeout_s=60) == "gloo"
    try:
        # each rank's own shard: a few small events seeded by its rank
        ev, sizes = W.batch_2d(n_events=6, lo=256, hi=1024, seed=R.event_seed(rank))
        res = O.make_clusters_batched(ev.coords, ev.weights, sizes, 1.5, 5.0, 1.5, None,
                                      shared_grid=False, n_threads=2)
        n_local = int(sizes.sum())
        R.barrier(r)
        t_local = 10.0 + rank  # stand-in device time of this rank
        t_max = R.max_over_ranks(t_local, r)
        n_all = R.sum_over_ranks(n_local, r)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), n_local=n_local, t_max=t_max,
                 n_all=n_all, value=R.job_throughput(n_all, t_max),
                 clusters=int(res.cluster_index.max()) + 1, coords_sum=float(ev.coords.sum()))
    finally:
        R.finish(r)


def test_two_gloo_ranks_combine_like_the_bench(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    out = [np.load(tmp_path / f"rank{k}.npz") for k in range(world)]
    n_locals = [int(o["n_local"]) for o in out]
    for o in out:
        assert float(o["t_max"]) == 11.0                  # the slowest rank's time
        assert int(o["n_all"]) == sum(n_locals)           # every rank's points
        assert float(o["value"]) == pytest.approx(sum(n_locals) / 11.0e-3)
    # the shards are different events, each clustered on its own rank
    assert float(out[0]["coords_sum"]) != float(out[1]["coords_sum"])
    assert all(int(o["clusters"]) >= 1 for o in out)


def test_single_rank_needs_no_process_group():
    from cluestering_b200 import replicas as R
    r = R.Ranks(world=1, rank=0, local=0)
    assert R.init(r) is None
    assert R.max_over_ranks(3.5, r) == 3.5
    assert R.sum_over_ranks(7, r) == 7.0
    assert R.event_seed(0) != R.event_seed(1)
    R.barrier(r)
    R.finish(r)
