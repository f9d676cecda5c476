"""Seeded synthetic events with the shapes of the benchmark configurations.

No dataset from the reference's benchmarks is available (its large CSVs are
not in the tree), so these generators stand in for them. They follow the
reference's blob generator (benchmark/utils/generation.hpp:110-131): equal-size
isotropic Gaussian blobs with centres uniform in the domain, the remaining
points uniform noise.

    single_2d       16,384 points, 20 blobs in [0,100]^2, sigma 1, 10 % noise, w = 1
    large_2d        1,048,576 points, 2,000 blobs in [0,1000]^2, sigma 1, 10 % noise,
                    weights ~ Exponential(mean 1)
    layered_3d      10,000 hits on 50 layers z = 0..49; 30 showers per layer whose
                    centres (uniform in [-100,100]^2) are shared by all layers;
                    transverse sigma 2; hits per layer and hit energy fall
                    geometrically with depth (ratio 0.9); energies lognormal(0, 1);
                    15 % noise hits of weight 0.1 uniform over the detector
    batch_2d        4,096 events, sizes log-uniform in [256, 65,536], each a
                    single_2d-style event with round(20 n / 16384) blobs (>= 1), w = 1
    serving_mix     events, 80 % single_2d-style 2-D and 20 % layered_3d-style 3-D,
                    sizes log-uniform in [1,024, 262,144]
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Event:
    coords: np.ndarray  # (D, n) float32
    weights: np.ndarray  # (n,) float32

    @property
    def n(self) -> int:
        return self.coords.shape[1]

    @property
    def ndim(self) -> int:
        return self.coords.shape[0]


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.MT19937(seed))


def blobs(n: int, n_blobs: int, lo: float, hi: float, sigma: float, noise: float, seed: int,
          weights: str = "unit", ndim: int = 2) -> Event:
    rng = _rng(seed)
    per_blob = int(np.floor(n * (1.0 - noise) / n_blobs))
    centres = rng.uniform(lo, hi, size=(n_blobs, ndim))
    pts = np.empty((ndim, n), np.float32)
    k = 0
    for b in range(n_blobs):
        pts[:, k:k + per_blob] = rng.normal(centres[b][:, None], sigma, size=(ndim, per_blob))
        k += per_blob
    pts[:, k:] = rng.uniform(lo, hi, size=(ndim, n - k))
    if weights == "unit":
        w = np.ones(n, np.float32)
    elif weights == "exponential":
        w = rng.exponential(1.0, size=n).astype(np.float32)
    else:
        raise ValueError(weights)
    return Event(pts, w)


def single_2d(n: int = 16384, seed: int = 0) -> Event:
    return blobs(n, 20, 0.0, 100.0, 1.0, 0.1, seed)


def large_2d(n: int = 1 << 20, seed: int = 1) -> Event:
    return blobs(n, 2000, 0.0, 1000.0, 1.0, 0.1, seed, weights="exponential")


def layered_3d(n: int = 10000, seed: int = 2, layers: int = 50, showers: int = 30,
               ratio: float = 0.9, noise: float = 0.15) -> Event:
    rng = _rng(seed)
    n_noise = int(round(n * noise))
    n_sig = n - n_noise
    share = ratio ** np.arange(layers)
    per_layer = np.floor(n_sig * share / share.sum()).astype(int)
    per_layer[0] += n_sig - per_layer.sum()
    centres = rng.uniform(-100.0, 100.0, size=(showers, 2))
    xs, ys, zs, ws = [], [], [], []
    for z in range(layers):
        m = per_layer[z]
        which = rng.integers(0, showers, size=m)
        xs.append(rng.normal(centres[which, 0], 2.0))
        ys.append(rng.normal(centres[which, 1], 2.0))
        zs.append(np.full(m, float(z)))
        ws.append(rng.lognormal(0.0, 1.0, size=m) * ratio ** z)
    xs.append(rng.uniform(-100.0, 100.0, n_noise))
    ys.append(rng.uniform(-100.0, 100.0, n_noise))
    zs.append(rng.integers(0, layers, n_noise).astype(float))
    ws.append(np.full(n_noise, 0.1))
    coords = np.stack([np.concatenate(xs), np.concatenate(ys), np.concatenate(zs)]).astype(np.float32)
    return Event(coords, np.concatenate(ws).astype(np.float32))


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = _rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)


def batch_2d(n_events: int = 4096, lo: int = 256, hi: int = 65536, seed: int = 3):
    """Returns (concatenated Event, sizes)."""
    sizes = log_uniform_sizes(n_events, lo, hi, seed)
    evs = [blobs(int(s), max(1, int(round(20 * s / 16384))), 0.0, 100.0, 1.0, 0.1, seed * 100003 + e)
           for e, s in enumerate(sizes)]
    coords = np.concatenate([e.coords for e in evs], axis=1)
    weights = np.concatenate([e.weights for e in evs])
    return Event(coords, weights), sizes.astype(np.uint32)


def serving_mix(n_events: int, lo: int = 1024, hi: int = 262144, seed: int = 4):
    """Yields (ndim, Event) for a stream of mixed 2-D / 3-D events."""
    rng = _rng(seed)
    sizes = log_uniform_sizes(n_events, lo, hi, seed + 1)
    kinds = rng.uniform(size=n_events) < 0.8
    for e in range(n_events):
        n = int(sizes[e])
        if kinds[e]:
            yield blobs(n, max(1, int(round(20 * n / 16384))), 0.0, 100.0, 1.0, 0.1, seed * 7919 + e)
        else:
            yield layered_3d(n, seed=seed * 7919 + e)


# Clustering parameters of each configuration: (dc, rhoc, dm, kernel, kernel params).
PARAMS = {
    "single_2d": dict(dc=1.5, rhoc=5.0, dm=1.5, kernel="flat", kernel_params=(0.5,)),
    "large_2d": dict(dc=1.5, rhoc=8.0, dm=2.0, kernel="flat", kernel_params=(0.5,)),
    "layered_3d": dict(dc=3.0, rhoc=10.0, dm=4.0, kernel="gaussian", kernel_params=(1.0, 1.0)),
    "batch_2d": dict(dc=1.5, rhoc=5.0, dm=1.5, kernel="flat", kernel_params=(0.5,)),
}
