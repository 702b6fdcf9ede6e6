"""Radius and k-nearest-neighbour search (fkd_nn.cu) and the FKDPoint-layout
build (fkd_build_points).

CPU tests pin the brute-force checker (oracle/nn_ref.py) to the unmodified
reference: a radius query's answer is the reference's own box search of the
enclosing box, filtered by the distance; a kNN row is the nearest k of the
reference's box search around the k-th distance.  GPU tests compare the CUDA
path with the checker: ordered id lists, ids and float32 distance bits equal.
"""
import ctypes as C

import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import _capi
from fkdtree_b200 import workloads as W
from oracle import nn_ref as NN
from oracle import oracle as O
from tests._fixtures import slices


def _cloud(n, dim, seed, grid=0):
    """Clustered points; grid > 0 snaps them to a grid so distances tie."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if n == 0:
        return np.zeros((dim, 0), dtype=np.float32), np.zeros(0, dtype=np.uint32)
    pts = W._cluster_cloud(rng, n, max(1, n // 200), 0.01, 0.7, dim=dim)
    if grid:
        pts = (np.round(pts * grid) / grid).astype(np.float32)
    ids = rng.permutation(n).astype(np.uint32)  # ids unrelated to positions
    return np.ascontiguousarray(pts), ids


def _centres(coords, q, seed, special=True):
    rng = np.random.Generator(np.random.PCG64(seed + 100))
    dim, n = coords.shape
    c = rng.random((dim, q), dtype=np.float32)
    if n:
        k = q // 2
        c[:, :k] = coords[:, rng.integers(0, n, size=k)]  # on tree points: distance 0 ties
    if special and q >= 4:
        c[0, 1] = np.nan
        c[:, 2] = 0.5
        c[-1, 3] = -3.0  # far outside
    return np.ascontiguousarray(c)


def _radii(q, seed, special=True):
    rng = np.random.Generator(np.random.PCG64(seed + 200))
    r = rng.uniform(0.0, 0.08, size=q).astype(np.float32)
    if special and q >= 8:
        r[4] = 0.0
        r[5] = -0.01
        r[6] = np.nan
        r[7] = np.inf
    return r


# ---------------------------------------------------------------- CPU: pins

def test_abi_arg_checks_without_gpu():
    L = _capi.lib()
    assert L.fkd_knn_max_k() == 64
    assert L.fkd_build_points(None, None, 0, 0) == 1
    assert L.fkd_search_radius_count(None, None, None, 0, None, 0) == 1
    tot = C.c_uint64(0)
    assert L.fkd_search_radius(None, None, None, 0, None, None, 0, C.byref(tot), 1, 0) == 1
    assert L.fkd_search_knn(None, None, 0, 1, None, None, 0) == 1


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_radius_checker_matches_reference_box_search(dim):
    coords, ids = _cloud(6000, dim, seed=dim)
    ref = O.RefTree(coords, ids)
    ref.build()
    tab, tid = ref.tables()
    q = 160
    ctr = _centres(coords, q, seed=dim, special=False)
    rad = _radii(q, seed=dim, special=False)
    # the enclosing box, a little wider than the ball
    pad = (rad * np.float32(1.001) + np.float32(1e-6)).astype(np.float32)
    mins = (ctr - pad).astype(np.float32)
    maxs = (ctr + pad).astype(np.float32)
    _, roff, rids, _ = ref.search(mins, maxs, variant=O.RECURSIVE)
    pos = np.empty(coords.shape[1], dtype=np.int64)
    pos[ids] = np.arange(coords.shape[1])  # id -> input column
    heap = np.empty(coords.shape[1], dtype=np.int64)
    heap[tid] = np.arange(coords.shape[1])  # id -> heap index
    noff, nids = NN.radius(tab, tid, ctr, rad)
    for j, (box, got) in enumerate(zip(slices(roff, rids), slices(noff, nids))):
        d2 = NN.dist2(coords[:, pos[box]], ctr[:, j])
        keep = box[d2 <= np.float32(rad[j] * rad[j])]
        want = keep[np.argsort(heap[keep])]
        assert np.array_equal(got, want), f"query {j}"
        assert np.all(np.diff(heap[got]) > 0)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_knn_checker_matches_reference_candidates():
    coords, ids = _cloud(5000, 3, seed=7, grid=64)
    ref = O.RefTree(coords, ids)
    ref.build()
    q, k = 120, 12
    ctr = _centres(coords, q, seed=7, special=False)
    ki, kd = NN.knn(coords, ids, ctr, k)
    pos = np.empty(coords.shape[1], dtype=np.int64)
    pos[ids] = np.arange(coords.shape[1])
    hw = (np.sqrt(kd[:, -1].astype(np.float64)) * 1.001 + 1e-6).astype(np.float32)
    mins = (ctr - hw).astype(np.float32)
    maxs = (ctr + hw).astype(np.float32)
    _, roff, rids, _ = ref.search(mins, maxs, variant=O.RECURSIVE)
    for j, box in enumerate(slices(roff, rids)):
        d2 = NN.dist2(coords[:, pos[box]], ctr[:, j])
        o = np.lexsort((box, d2))[:k]
        assert np.array_equal(box[o], ki[j]), f"query {j}"
        assert np.array_equal(d2[o].view(np.uint32), kd[j].view(np.uint32))


def test_checker_edge_semantics():
    coords = np.array([[0.0, 1.0, 1.0, np.inf], [0.0, 0.0, 0.0, 0.0]], dtype=np.float32)
    ids = np.array([5, 3, 9, 1], dtype=np.uint32)
    ctr = np.array([[1.0, np.nan, 1.0], [0.0, 0.0, 0.0]], dtype=np.float32)
    ki, kd = NN.knn(coords, ids, ctr, 3)
    assert list(ki[0]) == [3, 9, 5]  # equal distances: smaller id first
    assert list(ki[1]) == [0xFFFFFFFF] * 3 and np.all(np.isinf(kd[1]))
    off, got = NN.radius(coords, ids, ctr, np.array([1.0, 1.0, -1.0], dtype=np.float32))
    assert list(got[off[0]:off[1]]) == [5, 3, 9]  # heap order of the table given
    assert off[2] == off[1] and off[3] == off[2]


# ------------------------------------------------------------ GPU: parity

CASES = [(n, dim) for dim in (1, 2, 3, 4) for n in (1, 2, 3, 5, 17, 1000)] + [(20000, 3), (20000, 4), (30000, 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("n,dim", CASES)
@pytest.mark.parametrize("grid", [0, 32])
def test_radius_matches_checker(cuda, n, dim, grid):
    coords, ids = _cloud(n, dim, seed=n + dim, grid=grid)
    t = F.FKDTree(coords, ids).build()
    tab, tid = t.tables()
    q = 200
    ctr = _centres(coords, q, seed=n)
    rad = _radii(q, seed=n)
    woff, wids = NN.radius(tab, tid, ctr, rad)
    assert np.array_equal(t.count_radius(ctr, rad), np.diff(woff).astype(np.uint32))
    off, got = t.search_radius(ctr, rad)
    assert np.array_equal(off, woff)
    assert np.array_equal(got, wids)
    off, got = t.search_radius(ctr, rad, ordered=False)  # depth-first order: the same sets
    assert np.array_equal(off, woff)
    for a, b in zip(slices(off, got), slices(woff, wids)):
        assert np.array_equal(np.sort(a), np.sort(b))


@pytest.mark.gpu
@pytest.mark.parametrize("n,dim", CASES)
@pytest.mark.parametrize("k", [1, 5, 64])
def test_knn_matches_checker(cuda, n, dim, k):
    coords, ids = _cloud(n, dim, seed=n * 3 + dim, grid=16 if dim < 3 else 0)
    t = F.FKDTree(coords, ids).build()
    q = 150
    ctr = _centres(coords, q, seed=n + k)
    wi, wd = NN.knn(coords, ids, ctr, k)
    gi, gd = t.knn(ctr, k)
    assert np.array_equal(gi, wi)
    assert np.array_equal(gd.view(np.uint32), wd.view(np.uint32))


@pytest.mark.gpu
def test_infinite_coordinates_and_empty_tree(cuda):
    coords = np.array([[0.0, np.inf, -np.inf, 1.0, np.inf], [0.0, 1.0, 2.0, np.inf, np.inf]], dtype=np.float32)
    ids = np.arange(5, dtype=np.uint32)
    t = F.FKDTree(coords, ids).build()
    tab, tid = t.tables()
    ctr = np.array([[np.inf, 0.0, 1.0, np.inf], [1.0, 0.0, np.inf, np.inf]], dtype=np.float32)
    rad = np.array([np.inf, np.inf, 1.0, 0.0], dtype=np.float32)
    woff, wids = NN.radius(tab, tid, ctr, rad)
    off, got = t.search_radius(ctr, rad)
    assert np.array_equal(off, woff) and np.array_equal(got, wids)
    wi, wd = NN.knn(coords, ids, ctr, 5)
    gi, gd = t.knn(ctr, 5)
    assert np.array_equal(gi, wi) and np.array_equal(gd.view(np.uint32), wd.view(np.uint32))
    e = F.FKDTree(np.zeros((3, 0), dtype=np.float32), np.zeros(0, dtype=np.uint32)).build()
    c3 = np.zeros((3, 4), dtype=np.float32)
    off, got = e.search_radius(c3, np.ones(4, dtype=np.float32))
    assert got.size == 0 and np.all(off == 0)
    gi, gd = e.knn(c3, 3)
    assert np.all(gi == 0xFFFFFFFF) and np.all(np.isinf(gd))


@pytest.mark.gpu
def test_knn_rejects_bad_k(cuda):
    coords, ids = _cloud(100, 3, seed=1)
    t = F.FKDTree(coords, ids).build()
    with pytest.raises(F.FKDError):
        t.knn(coords[:, :4], 0)
    with pytest.raises(F.FKDError):
        t.knn(coords[:, :4], 65)


@pytest.mark.gpu
def test_radius_equals_filtered_box_search_at_scale(cuda):
    """2M clustered points: the radius answer is the ordered box search of the
    enclosing box filtered by distance (the box search is the one the golden
    fixtures pin)."""
    ev = W.clustered_event(n=1 << 21, n_queries=3000, seed=3)
    t = F.FKDTree(ev.coords, ev.ids).build()
    ctr = ((ev.mins + ev.maxs) * np.float32(0.5)).astype(np.float32)
    rad = ((ev.maxs[0] - ev.mins[0]) * np.float32(0.5)).astype(np.float32)
    pad = (rad * np.float32(1.001) + np.float32(1e-6)).astype(np.float32)
    boff, bids = t.search_boxes((ctr - pad).astype(np.float32), (ctr + pad).astype(np.float32), ordered=True)
    off, got = t.search_radius(ctr, rad)
    res = slices(off, got)
    for j, box in enumerate(slices(boff, bids)):
        d2 = NN.dist2(ev.coords[:, box], ctr[:, j])  # ids are 0..n-1
        assert np.array_equal(res[j], box[d2 <= np.float32(rad[j] * rad[j])]), f"query {j}"


@pytest.mark.gpu
def test_knn_at_scale(cuda):
    ev = W.clustered_event(n=1 << 20, n_queries=300, seed=4)
    t = F.FKDTree(ev.coords, ev.ids).build()
    ctr = ((ev.mins + ev.maxs) * np.float32(0.5)).astype(np.float32)
    wi, wd = NN.knn(ev.coords, ev.ids, ctr, 16)
    gi, gd = t.knn(ctr, 16)
    assert np.array_equal(gi, wi)
    assert np.array_equal(gd.view(np.uint32), wd.view(np.uint32))


@pytest.mark.gpu
def test_device_tensors(cuda):
    import torch
    coords, ids = _cloud(5000, 3, seed=11)
    t = F.FKDTree(torch.from_numpy(coords).to(cuda), torch.from_numpy(ids.view(np.int32)).to(cuda)).build()
    tab, tid = t.tables()
    ctr = _centres(coords, 100, seed=11, special=False)
    rad = _radii(100, seed=11, special=False)
    woff, wids = NN.radius(tab, tid, ctr, rad)
    off, got = t.search_radius(torch.from_numpy(ctr).to(cuda), torch.from_numpy(rad).to(cuda))
    assert np.array_equal(off.cpu().numpy().astype(np.uint64), woff)
    assert np.array_equal(got.cpu().numpy().view(np.uint32), wids)
    wi, wd = NN.knn(coords, ids, ctr, 8)
    gi, gd = t.knn(torch.from_numpy(ctr).to(cuda), 8)
    assert np.array_equal(gi.cpu().numpy().view(np.uint32), wi)
    assert np.array_equal(gd.cpu().numpy().view(np.uint32), wd.view(np.uint32))


# ------------------------------------------------ FKDPoint-layout build

def _aos(coords, ids):
    dim, n = coords.shape
    a = np.empty((n, dim + 1), dtype=np.uint32)
    a[:, :dim] = coords.T.view(np.uint32)
    a[:, dim] = ids
    return a


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [1, 2, 3, 4])
@pytest.mark.parametrize("n", [1, 7, 4096, 70000])
def test_build_points_equals_soa_build(cuda, dim, n):
    coords, ids = _cloud(n, dim, seed=dim * 10 + n)
    want = O.build(coords, ids)
    a = F.FKDTree.from_points(_aos(coords, ids), dim).build()
    tab, tid = a.tables()
    assert np.array_equal(tab.view(np.uint32), want[0].view(np.uint32))
    assert np.array_equal(tid, want[1])


@pytest.mark.gpu
def test_build_points_from_device(cuda):
    import torch
    coords, ids = _cloud(50000, 3, seed=5)
    want = O.build(coords, ids)
    dev = torch.from_numpy(_aos(coords, ids).view(np.int32)).to(cuda)
    a = F.FKDTree.from_points(dev, 3).build()
    tab, tid = a.tables()
    assert np.array_equal(tab.view(np.uint32), want[0].view(np.uint32))
    assert np.array_equal(tid, want[1])


@pytest.mark.gpu
def test_zero_queries(cuda):
    coords, ids = _cloud(1000, 3, seed=2)
    t = F.FKDTree(coords, ids).build()
    none = np.zeros((3, 0), dtype=np.float32)
    off, got = t.search_radius(none, np.zeros(0, dtype=np.float32))
    assert off.shape == (1,) and off[0] == 0 and got.size == 0
    assert t.count_radius(none, np.zeros(0, dtype=np.float32)).size == 0
    gi, gd = t.knn(none, 4)
    assert gi.shape == (0, 4) and gd.shape == (0, 4)
