"""Python access to the CPU checker (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/libclue_oracle.so`` (built by ``oracle/Makefile``) and runs
the serial restatement of CLUEstering's clustering on numpy arrays. Only the test
suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module; the library under ``cluestering_b200/`` never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

MAX_DIM = 10
KERNELS = {"flat": 0, "exponential": 1, "gaussian": 2}
METRICS = {
    "euclidean": 0,
    "weighted_euclidean": 1,
    "periodic_euclidean": 2,
    "manhattan": 3,
    "chebyshev": 4,
    "weighted_chebyshev": 5,
    "mahalanobis": 6,
}
EXP_LIBM, EXP_CLUE = 0, 1

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libclue_oracle.so")


class _Params(C.Structure):
    _fields_ = [
        ("dc", C.c_float),
        ("rhoc", C.c_float),
        ("dm", C.c_float),
        ("seed_dc", C.c_float),
        ("wrapped", C.c_uint8 * MAX_DIM),
        ("kernel_kind", C.c_int32),
        ("kernel_params", C.c_float * 2),
        ("metric_kind", C.c_int32),
        ("metric_params", C.c_float * MAX_DIM),
        ("exp_mode", C.c_int32),
        ("points_per_tile", C.c_int32),
        ("n_threads", C.c_int32),
    ]


class _Points(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("n", C.c_int32),
        ("coords", C.c_void_p * MAX_DIM),
        ("weight", C.c_void_p),
        ("sigma", C.c_void_p * MAX_DIM),
        ("density_uncertainty", C.c_void_p),
        ("tags", C.c_void_p),
    ]


class _Out(C.Structure):
    _fields_ = [
        ("rho", C.c_void_p),
        ("nearest_higher", C.c_void_p),
        ("is_seed", C.c_void_p),
        ("cluster_index", C.c_void_p),
        ("seeds", C.c_void_p),
        ("n_seeds", C.c_int32),
        ("n_per_dim", C.c_int32),
        ("n_tiles", C.c_int32),
        ("min_coord", C.c_float * MAX_DIM),
        ("max_coord", C.c_float * MAX_DIM),
        ("tile_size", C.c_float * MAX_DIM),
    ]


_lib = None


def build() -> str:
    """Compile the checker with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = C.CDLL(_LIB_PATH)
        lib.clue_oracle_make_clusters.argtypes = [C.POINTER(_Params), C.POINTER(_Points), C.POINTER(_Out)]
        lib.clue_oracle_make_clusters.restype = C.c_int
        lib.clue_oracle_make_clusters_batched.argtypes = [
            C.POINTER(_Params),
            C.POINTER(_Points),
            C.c_void_p,
            C.c_int32,
            C.c_int32,
            C.POINTER(_Out),
            C.c_void_p,
        ]
        lib.clue_oracle_make_clusters_batched.restype = C.c_int
        lib.clue_oracle_expf.argtypes = [C.c_float]
        lib.clue_oracle_expf.restype = C.c_float
        lib.clue_oracle_centroids.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_int32, C.c_int32, C.c_void_p]
        lib.clue_oracle_centroids.restype = None
        lib.clue_oracle_silhouette.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                               C.c_void_p]
        lib.clue_oracle_silhouette.restype = None
        _lib = lib
    return _lib


@dataclass
class OracleResult:
    rho: np.ndarray
    nearest_higher: np.ndarray
    is_seed: np.ndarray
    cluster_index: np.ndarray
    seeds: np.ndarray
    n_per_dim: int
    n_tiles: int
    min_coord: np.ndarray
    max_coord: np.ndarray
    tile_size: np.ndarray
    event_associations: np.ndarray | None = field(default=None)

    @property
    def n_clusters(self) -> int:
        return int(self.cluster_index.max()) + 1 if self.cluster_index.size else 0


def _params(dc, rhoc, dm=None, seed_dc=None, wrapped=None, kernel="flat", kernel_params=(0.5, 0.0),
            metric="euclidean", metric_params=None, exp_mode=EXP_CLUE, points_per_tile=128, n_threads=1):
    p = _Params()
    p.dc = dc
    p.rhoc = rhoc
    p.dm = dc if dm is None else dm
    p.seed_dc = dc if seed_dc is None else seed_dc
    for d, w in enumerate(wrapped or []):
        p.wrapped[d] = int(w)
    p.kernel_kind = KERNELS[kernel]
    kp = list(kernel_params) + [0.0] * (2 - len(kernel_params))
    p.kernel_params[0], p.kernel_params[1] = kp[0], kp[1]
    p.metric_kind = METRICS[metric]
    for d, v in enumerate(metric_params or []):
        p.metric_params[d] = v
    p.exp_mode = exp_mode
    p.points_per_tile = points_per_tile
    p.n_threads = n_threads
    return p


def _points(coords, weights, sigma, unc, tags, keep):
    coords = np.ascontiguousarray(coords, dtype=np.float32)
    if coords.ndim == 1:
        coords = coords[None, :]
    D, N = coords.shape
    pts = _Points()
    pts.ndim = D
    pts.n = N
    keep.append(coords)
    for d in range(D):
        pts.coords[d] = coords[d].ctypes.data
    w = np.ascontiguousarray(weights, dtype=np.float32)
    keep.append(w)
    pts.weight = w.ctypes.data
    if sigma is not None:
        for d, s in enumerate(sigma):
            if s is not None:
                s = np.ascontiguousarray(s, dtype=np.float32)
                keep.append(s)
                pts.sigma[d] = s.ctypes.data
    if unc is not None:
        u = np.ascontiguousarray(unc, dtype=np.float32)
        keep.append(u)
        pts.density_uncertainty = u.ctypes.data
    if tags is not None:
        t = np.ascontiguousarray(tags, dtype=np.uint32)
        keep.append(t)
        pts.tags = t.ctypes.data
    return pts, N


def _outputs(N):
    arrs = dict(
        rho=np.zeros(N, np.float32),
        nearest_higher=np.zeros(N, np.int32),
        is_seed=np.zeros(N, np.int32),
        cluster_index=np.zeros(N, np.int32),
        seeds=np.zeros(max(N, 1), np.int32),
    )
    out = _Out()
    for k, a in arrs.items():
        setattr(out, k, a.ctypes.data)
    return out, arrs


def _result(out, arrs):
    return OracleResult(
        rho=arrs["rho"],
        nearest_higher=arrs["nearest_higher"],
        is_seed=arrs["is_seed"],
        cluster_index=arrs["cluster_index"],
        seeds=arrs["seeds"][: out.n_seeds].copy(),
        n_per_dim=out.n_per_dim,
        n_tiles=out.n_tiles,
        min_coord=np.array(out.min_coord[:], np.float32),
        max_coord=np.array(out.max_coord[:], np.float32),
        tile_size=np.array(out.tile_size[:], np.float32),
    )


def make_clusters(coords, weights, dc, rhoc, dm=None, seed_dc=None, *, sigma=None, unc=None, tags=None,
                  **kw) -> OracleResult:
    """Single event. ``coords`` is (D, N) float32 (SoA, as the reference stores it)."""
    keep = []
    pts, N = _points(coords, weights, sigma, unc, tags, keep)
    prm = _params(dc, rhoc, dm, seed_dc, **kw)
    out, arrs = _outputs(N)
    rc = _load().clue_oracle_make_clusters(C.byref(prm), C.byref(pts), C.byref(out))
    if rc != 0:
        raise ValueError(f"oracle rejected the input (code {rc})")
    return _result(out, arrs)


def make_clusters_batched(coords, weights, event_sizes, dc, rhoc, dm=None, seed_dc=None, *,
                          shared_grid=True, sigma=None, unc=None, tags=None, **kw) -> OracleResult:
    keep = []
    pts, N = _points(coords, weights, sigma, unc, tags, keep)
    prm = _params(dc, rhoc, dm, seed_dc, **kw)
    out, arrs = _outputs(N)
    sizes = np.ascontiguousarray(event_sizes, dtype=np.uint32)
    assoc = np.zeros(max(N, 1), np.int32)
    rc = _load().clue_oracle_make_clusters_batched(
        C.byref(prm), C.byref(pts), sizes.ctypes.data, len(sizes), int(shared_grid), C.byref(out),
        assoc.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle rejected the input (code {rc})")
    res = _result(out, arrs)
    res.event_associations = assoc[: out.n_seeds].copy()
    return res


def expf(x: float) -> float:
    return float(_load().clue_oracle_expf(float(x)))


def _coord_table(coords):
    coords = np.ascontiguousarray(coords, dtype=np.float32)
    if coords.ndim == 1:
        coords = coords[None, :]
    table = (C.c_void_p * coords.shape[0])(*[coords[d].ctypes.data for d in range(coords.shape[0])])
    return coords, table


def centroids(coords, weights, labels, n_clusters: int, weighted: bool = False) -> np.ndarray:
    """utils/detail/cluster_centroid.hpp:86-140: (n_clusters, D) float32 centroids."""
    coords, table = _coord_table(coords)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    out = np.zeros((max(n_clusters, 0), coords.shape[0]), np.float32)
    _load().clue_oracle_centroids(coords.shape[0], coords.shape[1], table, w.ctypes.data, lab.ctypes.data,
                                  n_clusters, int(weighted), out.ctypes.data)
    return out


def silhouette(coords, labels, n_clusters: int) -> np.ndarray:
    """utils/detail/scores.hpp:33-73 for every point (NaN where the reference skips it)."""
    coords, table = _coord_table(coords)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    out = np.zeros(coords.shape[1], np.float32)
    _load().clue_oracle_silhouette(coords.shape[0], coords.shape[1], table, lab.ctypes.data, n_clusters,
                                   out.ctypes.data)
    return out
