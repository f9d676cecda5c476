"""The metric descriptor shared by the drop-in modules (one class, whichever way
they are imported)."""

from __future__ import annotations


class MetricDescriptor:
    """Opaque metric handle (BindingModules/MetricDescriptor.hpp:14-26): a tag and
    its parameters. Obtain it from the factory functions of
    CLUE_Convolutional_Kernels."""

    WEIGHTED_EUCLIDEAN, PERIODIC_EUCLIDEAN, MANHATTAN, WEIGHTED_CHEBYSHEV = range(4)

    def __init__(self, tag: int, params=()):
        self.tag = tag
        self.params = [float(p) for p in params]

    def __repr__(self):
        names = ("WeightedEuclidean", "PeriodicEuclidean", "Manhattan", "WeightedChebyshev")
        return f"MetricDescriptor({names[self.tag]}, {self.params})"
