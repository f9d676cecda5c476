"""CLUE_Convolutional_Kernels: the kernel classes and metric factories of
CLUEstering/BindingModules/binding_kernels.cpp:10-53, with the same names,
arguments and errors (ValueError where the C++ throws std::invalid_argument).
"""

from __future__ import annotations

from cluestering_b200.api import ExponentialKernel, FlatKernel, GaussianKernel  # noqa: F401
from cluestering_b200.compat.descriptor import MetricDescriptor


def EuclideanMetric(weights=()):  # noqa: N802 - the binding's name
    """Euclidean (L2) distance; optional per-dimension weights (empty: unweighted)."""
    return MetricDescriptor(MetricDescriptor.WEIGHTED_EUCLIDEAN, weights)


def ManhattanMetric():  # noqa: N802
    """Manhattan (L1) distance."""
    return MetricDescriptor(MetricDescriptor.MANHATTAN)


def ChebyshevMetric(weights=()):  # noqa: N802
    """Chebyshev (L-infinity) distance; optional per-dimension weights."""
    return MetricDescriptor(MetricDescriptor.WEIGHTED_CHEBYSHEV, weights)


def PeriodicEuclideanMetric(periods):  # noqa: N802
    """Periodic Euclidean distance; one period per dimension (0: not periodic)."""
    return MetricDescriptor(MetricDescriptor.PERIODIC_EUCLIDEAN, periods)
