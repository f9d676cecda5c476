"""Failure detection without a GPU fault.

Every wait inside the library's kernels is bounded: after its limit the kernel
records a timeout in the run's status word and returns, and the host call that
reads the run reports CLUE_ERR_TIMEOUT. clue_selftest_bounded_wait runs the
tile scan's decoupled look-back wait on a flag that nothing sets; the wait must
give up, the status must say so, and the GPU must stay usable.
"""

import time

import numpy as np
import pytest

import cluestering_b200 as clue
from cluestering_b200 import _lib as L
from cluestering_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_reports():
    lib = L.load()
    t0 = time.perf_counter()
    rc = lib.clue_selftest_bounded_wait(0, None)
    elapsed = time.perf_counter() - t0
    assert rc == L.ERR_TIMEOUT, lib.clue_last_error()
    assert b"gave up" in lib.clue_last_error()
    assert elapsed < 10.0
    # the context is still usable: a run afterwards matches the checker
    ev = W.single_2d(2048, seed=91)
    pts = clue.PointsHost(ev.coords, ev.weights)
    clue.Clusterer(1.5, 5.0, 1.5).make_clusters(pts)
    assert np.array_equal(pts.cluster_index, O.make_clusters(ev.coords, ev.weights, 1.5, 5.0, 1.5).cluster_index)
