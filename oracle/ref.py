"""TEST INFRASTRUCTURE ONLY: the reference's own make_clusters from Python.

oracle/_ref/libclue_ref.so is CLUEstering's unmodified `Clusterer::make_clusters`
compiled on its serial CPU backend (`make -C oracle ref`, ref_driver.cpp against
the alpaka stand-in in alpaka_shim/). The tests check the C restatement
(oracle.py) and the GPU library against it; bench.py times it as the CPU
baseline. The product never loads it. `available()` is False when the library
was not built (no reference tree where it was built).
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libclue_ref.so")

KERNELS = {"flat": 0, "exponential": 1, "gaussian": 2}
METRICS = {"euclidean": 0, "weighted_euclidean": 1, "periodic_euclidean": 2, "manhattan": 3,
           "chebyshev": 4, "weighted_chebyshev": 5, "mahalanobis": 6}
MAX_NDIM = 4  # the dimensions ref_driver.cpp instantiates


class _Params(C.Structure):
    _fields_ = [("dc", C.c_float), ("rhoc", C.c_float), ("dm", C.c_float), ("seed_dc", C.c_float),
                ("kernel_kind", C.c_int32), ("kernel_params", C.c_float * 2), ("metric_kind", C.c_int32),
                ("metric_params", C.c_float * 10), ("wrapped", C.c_uint8 * 10)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(LIB_PATH)
        lib.ref_make_clusters.restype = C.c_int
        lib.ref_make_clusters.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
        lib.ref_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


@dataclass
class RefResult:
    rho: np.ndarray
    nearest_higher: np.ndarray
    is_seed: np.ndarray
    cluster_index: np.ndarray

    @property
    def n_clusters(self) -> int:
        return int(self.cluster_index.max()) + 1 if self.cluster_index.size else 0


def _run(coords, weights, dc, rhoc, dm, seed_dc, sizes, *, sigma=None, unc=None, tags=None, wrapped=None,
         kernel="flat", kernel_params=(0.5,), metric="euclidean", metric_params=None) -> RefResult:
    c = np.ascontiguousarray(coords, np.float32)
    if c.ndim == 1:
        c = c[None, :]
    D, n = c.shape
    if not 1 <= D <= MAX_NDIM:
        raise ValueError(f"the reference build takes 1..{MAX_NDIM} dimensions")
    w = np.ascontiguousarray(weights, np.float32)
    p = _Params()
    p.dc, p.rhoc = dc, rhoc
    p.dm = dc if dm is None else dm
    p.seed_dc = dc if seed_dc is None else seed_dc
    p.kernel_kind = KERNELS[kernel]
    kp = list(kernel_params) + [0.0] * (2 - len(kernel_params))
    p.kernel_params[0], p.kernel_params[1] = kp[0], kp[1]
    p.metric_kind = METRICS[metric]
    for d, v in enumerate(metric_params or []):
        p.metric_params[d] = v
    for d, v in enumerate(wrapped or []):
        p.wrapped[d] = int(v)
    keep = []

    def ptr(a, dt):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dt)
        keep.append(a)
        return a.ctypes.data

    sig = None
    if sigma is not None:
        sig = np.zeros((D, n), np.float32)
        for d, s in enumerate(sigma):
            if s is not None:
                sig[d] = s
    sz = None if sizes is None else np.ascontiguousarray(sizes, np.uint32)
    out = dict(ci=np.zeros(n, np.int32), seed=np.zeros(n, np.int32), rho=np.zeros(n, np.float32),
               nh=np.zeros(n, np.int32))
    rc = _load().ref_make_clusters(
        D, n, c.ctypes.data, w.ctypes.data, C.byref(p), ptr(sig, np.float32), ptr(unc, np.float32),
        ptr(None if tags is None else np.asarray(tags, np.int64).astype(np.uint32), np.uint32),
        None if sz is None else sz.ctypes.data, 0 if sz is None else len(sz),
        out["ci"].ctypes.data, out["seed"].ctypes.data, out["rho"].ctypes.data, out["nh"].ctypes.data)
    if rc != 0:
        raise ValueError(_load().ref_last_error().decode())
    return RefResult(rho=out["rho"], nearest_higher=out["nh"], is_seed=out["seed"], cluster_index=out["ci"])


def make_clusters(coords, weights, dc, rhoc, dm=None, seed_dc=None, **kw) -> RefResult:
    """Clusterer<D>::make_clusters(queue, h_points, d_points, metric, kernel) of the reference."""
    return _run(coords, weights, dc, rhoc, dm, seed_dc, None, **kw)


def make_clusters_batched(coords, weights, event_sizes, dc, rhoc, dm=None, seed_dc=None, **kw) -> RefResult:
    """The reference's batched make_clusters (one tile grid from all points of the batch)."""
    return _run(coords, weights, dc, rhoc, dm, seed_dc, event_sizes, **kw)
