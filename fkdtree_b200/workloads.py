"""Deterministic synthetic point clouds and box-query sets.

One generator for every workload the benchmarks and the parity tests use, so
the GPU path, the C restatement and the reference CPU tree all see the same
float32 inputs.  Everything is drawn from numpy's PCG64 stream with a fixed
seed; boxes are computed once here in float32 (lo = p - hw, hi = p + hw) and
passed unchanged to every implementation.

Workloads (sizes as used by bench.py and the tests):

* ``uniform_event``   -- n i.i.d. U[0,1)^dim points, ids 0..n-1, one box per
  point with a fixed half-width (100,000 points / half-width 0.01 / seed 0 is
  the small single-event case).
* ``clustered_event`` -- 80% of the points from isotropic Gaussian clusters
  (centres U[0,1)^3, sigma 0.002, cluster weights Dirichlet(alpha=1)), 20%
  uniform background; boxes centred on randomly chosen points with per-dim
  half-widths U[0.001, 0.02] (16,777,216 points, 4,096 clusters, 1,048,576
  boxes, seed 1 is the large single-event case).
* ``event_batch``     -- many independent clustered events with log-normal
  sizes; every point queries its own event with a fixed half-width
  (4,096 events, median 20,000, sigma_log 1.0, sizes clipped to
  [1,000, 200,000], 50-500 clusters, half-width 0.01), optionally with a
  4-D share whose fourth coordinate is one of 16 discrete layers in [0,1).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Event:
    """One point cloud plus its box queries, all float32 SoA."""

    dim: int
    coords: np.ndarray  # (dim, n) float32
    ids: np.ndarray  # (n,) uint32
    mins: np.ndarray  # (dim, q) float32
    maxs: np.ndarray  # (dim, q) float32

    @property
    def n(self) -> int:
        return int(self.coords.shape[1])

    @property
    def q(self) -> int:
        return int(self.mins.shape[1])


def _boxes(centres: np.ndarray, hw) -> tuple[np.ndarray, np.ndarray]:
    c = np.ascontiguousarray(centres, dtype=np.float32)
    h = np.asarray(hw, dtype=np.float32)
    return (c - h).astype(np.float32), (c + h).astype(np.float32)


def uniform_event(n: int = 100_000, dim: int = 3, half_width: float = 0.01, seed: int = 0) -> Event:
    rng = np.random.Generator(np.random.PCG64(seed))
    coords = rng.random((dim, n), dtype=np.float32)
    ids = np.arange(n, dtype=np.uint32)
    mins, maxs = _boxes(coords, half_width)
    return Event(dim, coords, ids, mins, maxs)


def _cluster_cloud(rng: np.random.Generator, n: int, n_clusters: int, sigma: float, cluster_frac: float,
                   dim: int = 3) -> np.ndarray:
    """(dim, n) float32: cluster members first, then uniform background, then a
    random permutation so that no structure survives in the input order."""
    n_cl = int(round(n * cluster_frac))
    centres = rng.random((n_clusters, dim))
    weights = rng.dirichlet(np.ones(n_clusters))
    members = rng.multinomial(n_cl, weights)
    which = np.repeat(np.arange(n_clusters), members)
    pts = np.empty((n, dim), dtype=np.float64)
    pts[:n_cl] = centres[which] + sigma * rng.standard_normal((n_cl, dim))
    pts[n_cl:] = rng.random((n - n_cl, dim))
    pts = pts[rng.permutation(n)]
    return np.ascontiguousarray(pts.T.astype(np.float32))


def clustered_event(n: int = 1 << 24, n_queries: int = 1 << 20, n_clusters: int = 4096, sigma: float = 0.002,
                    cluster_frac: float = 0.8, hw_lo: float = 0.001, hw_hi: float = 0.02, seed: int = 1) -> Event:
    rng = np.random.Generator(np.random.PCG64(seed))
    coords = _cluster_cloud(rng, n, n_clusters, sigma, cluster_frac)
    ids = np.arange(n, dtype=np.uint32)
    pick = rng.integers(0, n, size=n_queries)
    centres = coords[:, pick]
    hw = rng.uniform(hw_lo, hw_hi, size=(3, n_queries)).astype(np.float32)
    mins, maxs = _boxes(centres, hw)
    return Event(3, coords, ids, mins, maxs)


@dataclass
class Batch:
    """Concatenated events.  Event e owns points [pt_off[e], pt_off[e+1]) and
    boxes [q_off[e], q_off[e+1]); its coordinates are stored SoA inside its own
    slice of ``coords`` starting at coord_off[e] (coords[coord_off[e] + c*n_e + i]),
    and likewise for the boxes at qcoord_off[e]."""

    dims: np.ndarray  # (E,) uint32
    pt_off: np.ndarray  # (E+1,) uint64
    coord_off: np.ndarray  # (E+1,) uint64
    q_off: np.ndarray  # (E+1,) uint64
    qcoord_off: np.ndarray  # (E+1,) uint64
    coords: np.ndarray  # float32 flat
    ids: np.ndarray  # uint32 flat
    mins: np.ndarray  # float32 flat
    maxs: np.ndarray  # float32 flat
    meta: dict = field(default_factory=dict)

    @property
    def n_events(self) -> int:
        return int(self.dims.shape[0])

    @property
    def n_points(self) -> int:
        return int(self.pt_off[-1])

    @property
    def n_queries(self) -> int:
        return int(self.q_off[-1])

    def event(self, e: int) -> Event:
        d = int(self.dims[e])
        n = int(self.pt_off[e + 1] - self.pt_off[e])
        q = int(self.q_off[e + 1] - self.q_off[e])
        c0 = int(self.coord_off[e])
        q0 = int(self.qcoord_off[e])
        return Event(d, self.coords[c0:c0 + d * n].reshape(d, n), self.ids[int(self.pt_off[e]):int(self.pt_off[e + 1])],
                     self.mins[q0:q0 + d * q].reshape(d, q), self.maxs[q0:q0 + d * q].reshape(d, q))


def event_sizes(rng: np.random.Generator, n_events: int, median: float, sigma_log: float, lo: int, hi: int,
                total: int | None = None) -> np.ndarray:
    s = np.exp(np.log(median) + sigma_log * rng.standard_normal(n_events))
    s = np.clip(np.rint(s), lo, hi).astype(np.int64)
    if total is not None:
        s = np.clip(np.rint(s * (total / s.sum())), lo, hi).astype(np.int64)
    return s


def event_batch(n_events: int = 4096, median: float = 20_000, sigma_log: float = 1.0, size_lo: int = 1_000,
                size_hi: int = 200_000, clusters_lo: int = 50, clusters_hi: int = 500, sigma: float = 0.002,
                cluster_frac: float = 0.8, half_width: float = 0.01, seed: int = 2, frac_4d: float = 0.0,
                total: int | None = None, queries: bool = True) -> Batch:
    """Independent clustered events; every point queries its own event.  With
    frac_4d > 0 the first round(frac_4d*E) events get a fourth coordinate that
    is one of 16 discrete layers, layer/16 in [0,1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = event_sizes(rng, n_events, median, sigma_log, size_lo, size_hi, total)
    n4 = int(round(frac_4d * n_events))
    dims = np.array([4 if e < n4 else 3 for e in range(n_events)], dtype=np.uint32)
    pt_off = np.zeros(n_events + 1, dtype=np.uint64)
    pt_off[1:] = np.cumsum(sizes)
    coord_off = np.zeros(n_events + 1, dtype=np.uint64)
    coord_off[1:] = np.cumsum(sizes * dims)
    coords = np.empty(int(coord_off[-1]), dtype=np.float32)
    ids = np.empty(int(pt_off[-1]), dtype=np.uint32)
    for e in range(n_events):
        n = int(sizes[e])
        k = int(rng.integers(clusters_lo, clusters_hi + 1))
        c3 = _cluster_cloud(rng, n, k, sigma, cluster_frac, 3)
        c0 = int(coord_off[e])
        coords[c0:c0 + 3 * n] = c3.reshape(-1)
        if dims[e] == 4:
            layer = rng.integers(0, 16, size=n).astype(np.float32) / np.float32(16.0)
            coords[c0 + 3 * n:c0 + 4 * n] = layer
        ids[int(pt_off[e]):int(pt_off[e + 1])] = np.arange(n, dtype=np.uint32)
    if queries:
        q_off = pt_off.copy()
        qcoord_off = coord_off.copy()
        hw = np.float32(half_width)
        mins = (coords - hw).astype(np.float32)
        maxs = (coords + hw).astype(np.float32)
    else:
        q_off = np.zeros(n_events + 1, dtype=np.uint64)
        qcoord_off = np.zeros(n_events + 1, dtype=np.uint64)
        mins = np.empty(0, dtype=np.float32)
        maxs = np.empty(0, dtype=np.float32)
    return Batch(dims, pt_off, coord_off, q_off, qcoord_off, coords, ids, mins, maxs,
                 meta=dict(seed=seed, median=median, sigma_log=sigma_log, half_width=half_width))


def mixed_events(seed: int = 5, total: int = 120_000_000, queries: bool = True) -> Batch:
    """Large mixed-dimension batch: 1,024 events totalling about 120M points,
    sizes log-normal (median 80,000, sigma_log 1.0) clipped to [5,000,
    2,000,000], half 3D and half 4D (the fourth coordinate one of 16 discrete
    layers), every point a box of half-width 0.005 on its own event."""
    return event_batch(n_events=1024, median=80_000, sigma_log=1.0, size_lo=5_000, size_hi=2_000_000,
                       half_width=0.005, seed=seed, frac_4d=0.5, total=total, queries=queries)
