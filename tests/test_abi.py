"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every symbol include/clue_sm100.h declares, and validates like the reference."""

import ctypes as C
import os
import re

import pytest

import cluestering_b200 as clue
from cluestering_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "clue_sm100.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(clue_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert set(declared_functions()) == set(L.SIGNATURES)


def test_abi_version_and_status_strings():
    lib = L.load()
    assert lib.clue_abi_version() == 1
    assert lib.clue_status_string(L.OK) == b"ok"
    assert lib.clue_status_string(L.ERR_TIMEOUT) == b"timeout"


def _params(**kw):
    c = clue.Clusterer(1.0, 1.0)
    p = c.params()
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("field,value", [("dc", -1.0), ("dc", 0.0), ("rhoc", -10.0), ("dm", 0.0),
                                         ("seed_dc", -1.0), ("dc", float("nan"))])
def test_validate_params_rejects_like_the_constructor(field, value):
    # core/detail/Clusterer.hpp:42-48
    lib = L.load()
    assert lib.clue_validate_params(C.byref(_params(**{field: value}))) == L.ERR_INVALID_ARGUMENT
    assert b"must be positive" in lib.clue_last_error()


def test_validate_params_accepts_defaults():
    assert L.load().clue_validate_params(C.byref(_params())) == L.OK
    assert L.load().clue_validate_params(C.byref(_params(rhoc=0.0))) == L.OK


@pytest.mark.parametrize("kind,params", [(L.KERNEL_FLAT, (0.0, 0.0)), (L.KERNEL_FLAT, (-1.0, 0.0)),
                                         (L.KERNEL_GAUSSIAN, (0.0, 1.0)), (L.KERNEL_GAUSSIAN, (1.0, -1.0)),
                                         (L.KERNEL_EXPONENTIAL, (-1.0, 1.0)),
                                         (L.KERNEL_EXPONENTIAL, (1.0, 0.0))])
def test_validate_kernel_parameters(kind, params):
    # core/detail/ConvolutionalKernel.hpp:13-50; tests/test_convolutional_kernels.cpp:7-24
    p = _params(kernel_kind=kind)
    p.kernel_params[0], p.kernel_params[1] = params
    assert L.load().clue_validate_params(C.byref(p)) == L.ERR_INVALID_ARGUMENT


def test_python_constructors_throw_like_the_reference():
    with pytest.raises(ValueError):
        clue.Clusterer(-1.0, 10.0)
    with pytest.raises(ValueError):
        clue.Clusterer(1.0, -10.0)
    for bad in [lambda: clue.FlatKernel(0.0), lambda: clue.FlatKernel(-1.0),
                lambda: clue.ExponentialKernel(0.0, 1.0), lambda: clue.ExponentialKernel(1.0, -1.0),
                lambda: clue.GaussianKernel(0.0, 1.0), lambda: clue.GaussianKernel(1.0, 0.0)]:
        with pytest.raises(ValueError):
            bad()


def test_points_host_validation():
    import numpy as np
    with pytest.raises(ValueError):
        clue.PointsHost(np.zeros((2, 0), np.float32), np.zeros(0, np.float32))
    p = clue.PointsHost(np.zeros((2, 4), np.float32), np.ones(4, np.float32))
    with pytest.raises(IndexError):
        p.set_sigma(2, np.ones(4))
    with pytest.raises(ValueError):
        p.set_tags(np.arange(3))
    with pytest.raises(ValueError):
        p.set_density_uncertainty(np.ones(5))


def test_getseeds_before_run_raises():
    with pytest.raises(RuntimeError):
        clue.Clusterer(1.0, 1.0).getSeeds()


def test_workspace_bytes_grow_with_the_problem():
    lib = L.load()
    small = lib.clue_workspace_bytes_for(2, 1000, 10, 1)
    big = lib.clue_workspace_bytes_for(2, 1000000, 8281, 1)
    assert 0 < small < big
    # about 43 4-byte words per point in 2-D (sorted copies, sweep records and
    # the nearest-higher cell layout) plus a few per tile
    assert big < 1000000 * 4 * 48


def test_clusters_csr_host():
    import numpy as np
    offs, pts = clue.clusters_csr(np.array([1, -1, 0, 1, 0, 2], np.int32))
    assert offs.tolist() == [0, 2, 4, 5]
    assert pts.tolist() == [2, 4, 0, 3, 5]


def test_tuning_defaults_and_struct_layout():
    t = L.Tuning()
    assert L.load().clue_tuning_defaults(C.byref(t)) == 0
    # 2-D mixed warps stream unions up to 1.25x; 3-D always streams; jump rounds by size
    assert (t.density_union_x16_2d, t.density_union_x16_3d, t.label_jump_rounds) == (20, 1 << 20, -1)
    # two points per cell on average, the default block shapes of both sweeps
    assert (t.cell_points, t.density_shape, t.nh_shape, t.tile_binning) == (2, 0, 0, 1)
    assert C.sizeof(L.Tuning) == 28
    assert L.load().clue_tuning_defaults(None) == L.ERR_INVALID_ARGUMENT


def test_host_pieces_query_checks_its_arguments():
    # a null workspace or output is rejected before any CUDA call
    lib = L.load()
    n = C.c_int32(-1)
    assert lib.clue_workspace_host_pieces(None, C.byref(n)) == L.ERR_INVALID_ARGUMENT
    assert n.value == -1
