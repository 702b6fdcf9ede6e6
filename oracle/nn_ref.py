"""CPU restatement of the radius and k-nearest-neighbour searches.

TEST INFRASTRUCTURE ONLY: the checker for fkdtree_b200/csrc/fkd_nn.cu (the
searches have no counterpart in the reference, which answers boxes only,
FKDTree_cpu.h:25-207).  Both are stated by their definitions, as brute force
over every point, in float32 numpy arithmetic that rounds each operation on
its own -- the same expression, in the same order, as the GPU kernels:

    d2(p, c) = (((0 + (p0-c0)^2) + (p1-c1)^2) + (p2-c2)^2) + (p3-c3)^2

* radius(c, r): the points with d2 <= fl(r*r), for r >= 0 and a centre without
  NaN coordinates (otherwise none), in ascending heap-index order of the
  tree's tables (the order of the reference's level-order search,
  FKDTree_cpu.h:123-169);
* knn(c, k): the k points smallest in (d2, id), ascending; points whose d2 is
  NaN never qualify; rows with fewer than k points end in id 0xffffffff and
  d2 = +inf.

The brute force does not depend on the tree, so it checks the GPU's pruning
as well as its arithmetic.  tests/test_nn.py pins the radius definition to
the reference's own box search (the points of the enclosing box, filtered by
d2), run from the unmodified reference headers.
"""
from __future__ import annotations

import numpy as np

NO_ID = np.uint32(0xFFFFFFFF)


def dist2(points: np.ndarray, centre: np.ndarray) -> np.ndarray:
    """points (dim, n) float32, centre (dim,) float32 -> (n,) float32."""
    points = np.asarray(points, dtype=np.float32)
    centre = np.asarray(centre, dtype=np.float32)
    acc = np.zeros(points.shape[1], dtype=np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        for c in range(points.shape[0]):
            t = points[c] - centre[c]
            acc = acc + t * t
    return acc


def radius(tab: np.ndarray, tab_ids: np.ndarray, centres: np.ndarray, radii: np.ndarray):
    """Brute-force radius search over the heap tables (dim, n) / (n,); returns
    (offsets (q+1,) uint64, ids) with query j's ids in ascending heap index."""
    tab = np.asarray(tab, dtype=np.float32)
    tab_ids = np.asarray(tab_ids, dtype=np.uint32)
    centres = np.asarray(centres, dtype=np.float32)
    radii = np.asarray(radii, dtype=np.float32)
    q = centres.shape[1]
    parts = []
    offsets = np.zeros(q + 1, dtype=np.uint64)
    for j in range(q):
        r = radii[j]
        c = centres[:, j]
        if not (r >= 0) or np.isnan(c).any() or tab.shape[1] == 0:
            hit = np.zeros(0, dtype=np.int64)
        else:
            with np.errstate(over="ignore"):
                r2 = np.float32(r * r)
            hit = np.nonzero(dist2(tab, c) <= r2)[0]
        parts.append(tab_ids[hit])
        offsets[j + 1] = offsets[j] + hit.size
    ids = np.concatenate(parts) if parts else np.zeros(0, dtype=np.uint32)
    return offsets, ids.astype(np.uint32)


def knn(coords: np.ndarray, ids: np.ndarray, centres: np.ndarray, k: int):
    """Brute-force k nearest points of every centre; returns (ids (q, k)
    uint32, d2 (q, k) float32)."""
    coords = np.asarray(coords, dtype=np.float32)
    ids = np.asarray(ids, dtype=np.uint32)
    centres = np.asarray(centres, dtype=np.float32)
    q = centres.shape[1]
    out_i = np.full((q, k), NO_ID, dtype=np.uint32)
    out_d = np.full((q, k), np.inf, dtype=np.float32)
    for j in range(q):
        c = centres[:, j]
        if np.isnan(c).any() or coords.shape[1] == 0:
            continue
        d2 = dist2(coords, c)
        ok = np.nonzero(~np.isnan(d2))[0]
        if ok.size > k:  # keep the candidates up to the k-th smallest d2 (ties included)
            kth = np.partition(d2[ok], k - 1)[k - 1]
            ok = ok[d2[ok] <= kth]
        sel = ok[np.lexsort((ids[ok], d2[ok]))][:k]
        out_i[j, :sel.size] = ids[sel]
        out_d[j, :sel.size] = d2[sel]
    return out_i, out_d
