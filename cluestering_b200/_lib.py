"""ctypes binding of libclue_sm100.so (include/clue_sm100.h).

Loading fails loudly when the library has not been built: there is no
fallback implementation of the clustering path.
"""

from __future__ import annotations

import ctypes as C
import os

MAX_DIM = 10

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_RANGE = 2
ERR_RUNTIME = 3
ERR_CUDA = 4
ERR_OUT_OF_MEMORY = 5
ERR_TIMEOUT = 6
ERR_NOT_READY = 7

KERNEL_FLAT, KERNEL_EXPONENTIAL, KERNEL_GAUSSIAN = 0, 1, 2
(METRIC_EUCLIDEAN, METRIC_WEIGHTED_EUCLIDEAN, METRIC_PERIODIC_EUCLIDEAN, METRIC_MANHATTAN,
 METRIC_CHEBYSHEV, METRIC_WEIGHTED_CHEBYSHEV, METRIC_MAHALANOBIS) = range(7)
GRID_SHARED, GRID_PER_EVENT = 0, 1
STAGES = ("extents", "tiles", "gather", "density", "nearest_higher", "labels")

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libclue_sm100.so")


class Params(C.Structure):
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
        ("points_per_tile", C.c_int32),
    ]


class Points(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("n", C.c_int32),
        ("coords", C.c_void_p * MAX_DIM),
        ("weight", C.c_void_p),
        ("sigma", C.c_void_p * MAX_DIM),
        ("density_uncertainty", C.c_void_p),
        ("tags", C.c_void_p),
        ("cluster_index", C.c_void_p),
        ("is_seed", C.c_void_p),
        ("rho", C.c_void_p),
        ("nearest_higher", C.c_void_p),
    ]


class Tuning(C.Structure):
    _fields_ = [("density_union_x16_2d", C.c_int32), ("density_union_x16_3d", C.c_int32),
                ("label_jump_rounds", C.c_int32), ("cell_points", C.c_int32),
                ("density_shape", C.c_int32), ("nh_shape", C.c_int32), ("tile_binning", C.c_int32)]


class ServerProfile(C.Structure):
    _fields_ = [("ndim", C.c_int32), ("params", Params)]


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("budget_bytes", C.c_size_t),
        ("max_inflight", C.c_int32),
        ("max_batch_events", C.c_int32),
        ("max_batch_points", C.c_int64),
        ("linger_us", C.c_int32),
        ("max_batch_ms", C.c_float),
        ("priority_ms", C.c_float),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("batches", C.c_int64),
        ("points_completed", C.c_int64),
        ("inflight_bytes_peak", C.c_int64),
        ("latency_p50_ms", C.c_double),
        ("latency_p99_ms", C.c_double),
        ("latency_max_ms", C.c_double),
        ("resident_bytes_peak", C.c_int64),
        ("resident_pool_bytes", C.c_int64),
        ("slot_bytes", C.c_int64),
        ("admission_waits", C.c_int64),
        ("max_batch_points", C.c_int64),
    ]


# Every symbol include/clue_sm100.h declares, with (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "clue_abi_version": (C.c_int32, []),
    "clue_status_string": (C.c_char_p, [C.c_int]),
    "clue_last_error": (C.c_char_p, []),
    "clue_validate_params": (C.c_int, [C.POINTER(Params)]),
    "clue_workspace_create": (C.c_int, [C.POINTER(_P), C.c_int32]),
    "clue_workspace_destroy": (C.c_int, [_P]),
    "clue_workspace_bytes": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "clue_workspace_bytes_for": (C.c_size_t, [C.c_int32, C.c_int64, C.c_int64, C.c_int32]),
    "clue_workspace_set_profiling": (C.c_int, [_P, C.c_int32]),
    "clue_workspace_stage_ms": (C.c_int, [_P, _P, C.c_int32]),
    "clue_workspace_kernel_launches": (C.c_int, [_P, _P]),
    "clue_workspace_set_graphs": (C.c_int, [_P, C.c_int32]),
    "clue_selftest_bounded_wait": (C.c_int, [C.c_int32, _P]),
    "clue_workspace_graph_replayed": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "clue_workspace_host_pieces": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "clue_tuning_defaults": (C.c_int, [C.POINTER(Tuning)]),
    "clue_workspace_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "clue_workspace_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "clue_workspace_autotune": (
        C.c_int, [_P, C.POINTER(Params), C.POINTER(Points), _P, C.c_int32, C.c_int32, _P, C.c_int32,
                  C.POINTER(Tuning)]),
    "clue_make_clusters_device": (C.c_int, [_P, C.POINTER(Params), C.POINTER(Points), _P]),
    "clue_make_clusters_host": (C.c_int, [_P, C.POINTER(Params), C.POINTER(Points), _P]),
    "clue_make_clusters_batched_device": (
        C.c_int, [_P, C.POINTER(Params), C.POINTER(Points), _P, C.c_int32, C.c_int32, _P]),
    "clue_make_clusters_batched_host": (
        C.c_int, [_P, C.POINTER(Params), C.POINTER(Points), _P, C.c_int32, C.c_int32, _P]),
    "clue_make_clusters_device_noalloc": (C.c_int, [C.POINTER(Params), C.POINTER(Points), _P, _P]),
    "clue_n_clusters": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "clue_get_seeds": (C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "clue_get_clusters_device": (C.c_int, [_P, _P, _P, _P]),
    "clue_sample_associations": (C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "clue_cluster_centroids_device": (C.c_int, [C.POINTER(Points), _P, _P, C.c_int32, C.c_int32, _P, _P]),
    "clue_silhouette_device": (C.c_int, [C.POINTER(Points), _P, _P, C.c_int32, _P, _P]),
    "clue_stream_create": (C.c_int, [C.POINTER(_P), C.c_int32]),
    "clue_stream_destroy": (C.c_int, [_P]),
    "clue_stream_synchronize": (C.c_int, [_P]),
    "clue_device_malloc": (C.c_int, [C.POINTER(_P), C.c_size_t, C.c_int32]),
    "clue_device_free": (C.c_int, [_P]),
    "clue_host_malloc_pinned": (C.c_int, [C.POINTER(_P), C.c_size_t]),
    "clue_host_free_pinned": (C.c_int, [_P]),
    "clue_memcpy_async": (C.c_int, [_P, _P, C.c_size_t, C.c_int32, _P]),
    "clue_server_create": (
        C.c_int, [C.POINTER(_P), C.POINTER(ServerConfig), C.POINTER(ServerProfile), C.c_int32]),
    "clue_server_submit": (C.c_int, [_P, C.c_int32, C.POINTER(Points), C.POINTER(C.c_uint64)]),
    "clue_server_poll": (C.c_int, [_P, C.c_uint64]),
    "clue_server_drain": (C.c_int, [_P]),
    "clue_server_stats_get": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "clue_server_latencies": (C.c_int, [_P, _P, C.c_int64, C.POINTER(C.c_int64)]),
    "clue_workspace_sweep_stats": (C.c_int, [_P, C.POINTER(C.c_int64), C.c_int32]),
    "clue_server_destroy": (C.c_int, [_P]),
}

_lib = None


class ClueError(RuntimeError):
    """A failed call into libclue_sm100.so."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cluestering_b200.build` "
                "(the clustering path has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    """Raises the Python counterpart of the reference's exception for a status."""
    if status == OK:
        return
    msg = load().clue_last_error().decode() or load().clue_status_string(status).decode()
    if status == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == ERR_OUT_OF_RANGE:
        raise IndexError(msg)
    if status == ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise ClueError(status, msg)
