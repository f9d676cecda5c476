"""B200 (sm_100a) implementation of CLUEstering's Clusterer::make_clusters.

The clustering runs in libclue_sm100.so (CUDA kernels behind a C ABI, see
include/clue_sm100.h). This package is its Python binding, mirroring the
reference's C++ names.
"""

from .api import (  # noqa: F401
    ChebyshevMetric,
    Clusterer,
    EuclideanMetric,
    ExponentialKernel,
    FlatKernel,
    GaussianKernel,
    MahalanobisMetric,
    ManhattanMetric,
    PeriodicEuclideanMetric,
    PointsDevice,
    PointsHost,
    Server,
    WeightedChebyshevMetric,
    WeightedEuclideanMetric,
    cluster_centroids,
    clusters_csr,
    metrics,
    silhouette,
    silhouette_scores,
    weighted_cluster_centroids,
)
from ._lib import GRID_PER_EVENT, GRID_SHARED, ClueError  # noqa: F401
