"""The C++20 drop-in header (include/clue_sm100.hpp via CLUEstering/CLUEstering.hpp).

A C++ program written like the reference's doctest cases is compiled with g++
against the header and the shared library; on a GPU it runs the reference's
known-answer checks and every make_clusters overload, whose cluster ids must
equal the CPU checker's.
"""

import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import fixture

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_cpp_api.cpp")
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_cpp_api")


def build_cpp():
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           SRC, "-L" + os.path.join(ROOT, "cluestering_b200"), "-lclue_sm100",
           "-Wl,-rpath,$ORIGIN/../../../cluestering_b200", "-o", BIN]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return BIN


def test_cpp_api_compiles_and_links():
    build_cpp()
    assert os.access(BIN, os.X_OK)


@pytest.mark.gpu
def test_cpp_api_known_answers_and_overloads(tmp_path):
    exe = build_cpp()
    files = []
    for name in ("batched_data_1024", "data_32768"):
        c, w = fixture(name)
        path = tmp_path / f"{name}.f32"
        np.concatenate([c.ravel(), w]).astype(np.float32).tofile(path)
        files.append(str(path))
    out = tmp_path / "ids.i32"
    res = subprocess.run([exe, *files, str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    c, w = fixture("data_32768")
    ref = O.make_clusters(c, w, 1.3, 10.0, 1.3).cluster_index
    ids = np.fromfile(out, np.int32).reshape(-1, c.shape[1])
    assert ids.shape[0] == 5
    for row in ids:
        assert np.array_equal(row, ref)
    # clue::cluster_centroids, weighted_cluster_centroids and silhouette on the last overload's result
    util = np.fromfile(str(out) + ".util", np.float32)
    k = int(util[0])
    assert k == int(ref.max()) + 1
    cen, wcen = util[1:1 + 2 * k].reshape(k, 2), util[1 + 2 * k:1 + 4 * k].reshape(k, 2)
    assert np.array_equal(cen.view(np.int32), O.centroids(c, w, ref, k).view(np.int32))
    assert np.array_equal(wcen.view(np.int32), O.centroids(c, w, ref, k, weighted=True).view(np.int32))
    sil, sil_first, first = util[1 + 4 * k:]
    scores = O.silhouette(c, ref, k)
    assert sil_first == scores[int(first)]
    # the mean is a float std::reduce over ~30,000 scores, as in the reference: float accuracy
    assert sil == pytest.approx(float(np.mean(scores[~np.isnan(scores)].astype(np.float64))), rel=1e-5)
