"""GPU search parity through the C ABI: per-box id lists equal the
reference's (golden fixtures, in its emission order), sets equal the
recursive search and the brute-force scan, counts and digests agree."""
import hashlib

import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import workloads as W
from oracle import oracle as O
from tests._fixtures import GOLDEN, fixture_names, load, slices

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", fixture_names())
def test_ordered_results_match_reference_lists(cuda, name):
    f = load(name)
    t = F.FKDTree(f["coords"], f["ids"]).build()
    offs, ids = t.search_boxes(f["mins"], f["maxs"], ordered=True)
    got = slices(offs, ids)
    sel = f.get("lvl_sel")
    want = slices(f["lvl_offsets"], f["lvl_ids"])
    idx = range(len(got)) if sel is None else sel
    for k, j in enumerate(idx):
        assert np.array_equal(got[j], want[k]), f"box {j}"
    # the recursive variant: same set
    for a, b in zip(got, slices(f["rec_offsets"], f["rec_ids"])):
        assert np.array_equal(np.sort(a), np.sort(b))
    # per-box counts (search_in_the_box_multiple)
    assert np.array_equal(t.search_in_the_box_multiple(f["mins"], f["maxs"]), f["rec_counts"])


@pytest.mark.parametrize("name", ["uniform3d_n1000", "layers4d_n3000", "grid2d_n2000", "clustered3d_n20000"])
def test_unordered_sets_and_digests(cuda, name):
    f = load(name)
    t = F.FKDTree(f["coords"], f["ids"]).build()
    offs, ids = t.search_boxes(f["mins"], f["maxs"], ordered=False)
    for a, b in zip(slices(offs, ids), slices(f["rec_offsets"], f["rec_ids"])):
        assert np.array_equal(np.sort(a), np.sort(b))
    c, d = t.digest_boxes(f["mins"], f["maxs"])
    assert np.array_equal(c, f["rec_counts"])
    assert np.array_equal(d, O.digest_of(f["rec_ids"], f["rec_offsets"]))


def test_single_box_api(cuda):
    f = load("uniform3d_n1000")
    t = F.FKDTree(f["coords"], f["ids"]).build()
    want = slices(f["lvl_offsets"], f["lvl_ids"])
    for j in range(5):
        lo, hi = f["mins"][:, j], f["maxs"][:, j]
        assert np.array_equal(t.search_in_the_box(lo, hi), want[j])
        assert np.array_equal(t.search_in_the_box_BFS(lo, hi), want[j])
        assert np.array_equal(t.search_in_the_box_branchless(lo, hi), want[j])
        assert np.array_equal(np.sort(t.search_in_the_box_recursive(lo, hi)), np.sort(want[j]))


def test_small_single_event_against_reference_summary(cuda):
    """100,000 uniform points, one box per point, half-width 0.01, seed 0."""
    ev = W.uniform_event()
    t = F.FKDTree(ev.coords, ev.ids).build()
    tab, tid = t.tables()
    offs, ids = t.search_boxes(ev.mins, ev.maxs, ordered=True)
    with np.load(GOLDEN / "uniform3d_n100000_summary.npz") as z:
        assert hashlib.sha256(tab.tobytes()).hexdigest() == str(z["tab_sha"])
        assert hashlib.sha256(tid.tobytes()).hexdigest() == str(z["ids_sha"])
        assert np.array_equal(np.diff(offs.astype(np.int64)), z["counts"].astype(np.int64))
        assert hashlib.sha256(ids.tobytes()).hexdigest() == str(z["lvl_ids_sha"])


@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_search_vs_brute_force_random(cuda, dim):
    rng = np.random.default_rng(dim)
    n = 50_000
    c = rng.random((dim, n), dtype=np.float32)
    ids = rng.permutation(n).astype(np.uint32)
    q = 3000
    ctr = c[:, rng.integers(0, n, q)]
    hw = rng.uniform(0.0, 0.2, (dim, q)).astype(np.float32)
    mins, maxs = (ctr - hw).astype(np.float32), (ctr + hw).astype(np.float32)
    mins[:, :10] = -np.inf   # half-open and unbounded boxes
    maxs[:, 5:15] = np.inf
    mins[:, 20:25], maxs[:, 20:25] = maxs[:, 20:25].copy(), mins[:, 20:25].copy()  # empty boxes (lo > hi)
    t = F.FKDTree(c, ids).build()
    tab, tid = t.tables()
    cb, ob, ib, _ = O.search(tab, tid, mins, maxs, variant=O.BRUTE)
    offs, got = t.search_boxes(mins, maxs, ordered=True)
    assert np.array_equal(offs, ob)
    assert np.array_equal(got, ib)  # brute force scans in heap order too
    c2, d2 = t.digest_boxes(mins, maxs)
    assert np.array_equal(c2, cb) and np.array_equal(d2, O.digest_of(ib, ob))


def test_whole_tree_and_nan_boxes(cuda):
    rng = np.random.default_rng(3)
    n = 10_000
    c = rng.random((3, n), dtype=np.float32)
    t = F.FKDTree(c).build()
    mins = np.full((3, 3), -np.inf, np.float32)
    maxs = np.full((3, 3), np.inf, np.float32)
    mins[0, 1] = np.nan
    maxs[2, 2] = np.nan
    offs, got = t.search_boxes(mins, maxs, ordered=False)
    assert offs[1] - offs[0] == n and np.array_equal(np.sort(got[:n]), np.arange(n))
    assert offs[2] == offs[1] and offs[3] == offs[2]  # NaN bounds select nothing, like the reference


def test_clustered_large_boxes_vs_recursive(cuda):
    """Boxes containing whole dense clusters -- the regime where the
    reference's FQueue overflows (FQueue.h:158); the GPU frontier must not
    drop anything."""
    ev = W.clustered_event(n=1 << 20, n_queries=4096, n_clusters=64, hw_lo=0.001, hw_hi=0.05, seed=4)
    t = F.FKDTree(ev.coords, ev.ids).build()
    tab, tid = t.tables()
    cr, orr, ir, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.RECURSIVE)
    offs, got = t.search_boxes(ev.mins, ev.maxs, ordered=False)
    assert np.array_equal(offs, orr)
    ok = all(np.array_equal(np.sort(a), np.sort(b)) for a, b in zip(slices(offs, got), slices(orr, ir)))
    assert ok
    c, d = t.digest_boxes(ev.mins, ev.maxs)
    assert np.array_equal(c, cr) and np.array_equal(d, O.digest_of(ir, orr))


def test_device_memory_search_and_capacity_error(cuda):
    import torch
    ev = W.uniform_event(n=100_000, seed=8, half_width=0.02)
    t = F.FKDTree(torch.from_numpy(ev.coords).to(cuda)).build()
    mins = torch.from_numpy(ev.mins).to(cuda)
    maxs = torch.from_numpy(ev.maxs).to(cuda)
    offs, ids = t.search_boxes(mins, maxs, ordered=True)
    tab, tid = t.tables()
    cb, ob, ib, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.LEVEL_ORDER)
    assert np.array_equal(offs.cpu().numpy().astype(np.uint64), ob)
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), ib)
    with pytest.raises(F.FKDError) as e:
        t.search_boxes(ev.mins, ev.maxs, capacity=10)
    assert e.value.status == 6


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("dim", [1, 3, 4])
def test_search_lanes_per_box(cuda, dim, lanes):
    """Count and digest with several boxes per warp (search_lanes) equal the
    brute-force scan, unbounded, empty and whole-tree boxes included."""
    rng = np.random.default_rng(40 + dim)
    n = 30_000
    c = rng.random((dim, n), dtype=np.float32)
    ids = rng.permutation(n).astype(np.uint32)
    q = 2000
    ctr = c[:, rng.integers(0, n, q)]
    hw = rng.uniform(0.0, 0.15, (dim, q)).astype(np.float32)
    mins, maxs = (ctr - hw).astype(np.float32), (ctr + hw).astype(np.float32)
    mins[:, :10] = -np.inf
    maxs[:, 5:15] = np.inf
    mins[:, 20:25], maxs[:, 20:25] = maxs[:, 20:25].copy(), mins[:, 20:25].copy()
    t = F.FKDTree(c, ids).build()
    tab, tid = t.tables()
    cb, ob, ib, _ = O.search(tab, tid, mins, maxs, variant=O.BRUTE)
    t.set_param("search_lanes", lanes)
    assert np.array_equal(t.count_boxes(mins, maxs), cb)
    c2, d2 = t.digest_boxes(mins, maxs)
    assert np.array_equal(c2, cb) and np.array_equal(d2, O.digest_of(ib, ob))
    with pytest.raises(F.FKDError):
        t.set_param("search_lanes", 3)


@pytest.mark.parametrize("record,pool", [(0, 0), (1, 0), (1, 64), (1, 5000)])
def test_search_record_paths(cuda, record, pool):
    """fkd_search with and without the recording count pass, and with record
    pools so small that some or all boxes fall back to the traversing write
    pass: the same sets, equal to the recursive search, and the same ordered
    lists as the reference's level order."""
    ev = W.clustered_event(n=200_000, n_queries=3000, n_clusters=64, hw_lo=0.001, hw_hi=0.05, seed=12)
    t = F.FKDTree(ev.coords, ev.ids).build()
    t.set_param("search_record", record).set_param("search_pool", pool)
    tab, tid = t.tables()
    cr, orr, ir, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.RECURSIVE)
    for _ in range(2):  # the second call uses the pools sized by the first
        offs, got = t.search_boxes(ev.mins, ev.maxs, ordered=False)
        assert np.array_equal(offs, orr)
        assert all(np.array_equal(np.sort(a), np.sort(b)) for a, b in zip(slices(offs, got), slices(orr, ir)))
    offs, got = t.search_boxes(ev.mins, ev.maxs, ordered=True)
    cl, ol, il, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.BRUTE)
    assert np.array_equal(offs, ol) and np.array_equal(got, il)


@pytest.mark.parametrize("dim", [1, 2, 3, 4])
@pytest.mark.parametrize("n", [5, 40, 700, 60_001])
def test_leaf_buckets_equal_walk(cuda, dim, n):
    """The bottom subtrees scanned in in-order layout ("search_bucket" 1..6)
    give exactly the walk's results (bucket 0): counts, ordered lists,
    unordered sets, digests, recorded and traversing write passes."""
    rng = np.random.default_rng(100 + dim + n)
    c = rng.random((dim, n), dtype=np.float32)
    c[-1] = np.round(c[-1] * 16) / 16  # ties on the last coordinate
    ids = rng.permutation(n).astype(np.uint32) * 3 + 1
    q = 1500
    ctr = c[:, rng.integers(0, n, q)]
    hw = rng.uniform(0.0, 0.15, (dim, q)).astype(np.float32)
    mins, maxs = (ctr - hw).astype(np.float32), (ctr + hw).astype(np.float32)
    t = F.FKDTree(c, ids).build()
    tab, tid = t.tables()
    wc, wo, wids, _ = O.search(tab, tid, mins, maxs, variant=O.RECURSIVE)
    wd = O.digest_of(wids, wo)
    for b, runs in ((0, 0), (1, 0), (3, 1), (4, 0), (4, 1), (6, 0)):
        t.set_param("search_bucket", b)
        t.set_param("bucket_runs", runs)
        assert np.array_equal(t.count_boxes(mins, maxs), wc), f"bucket {b}: counts"
        offs, got = t.search_boxes(mins, maxs, ordered=False)
        assert np.array_equal(offs, wo) and np.array_equal(O.digest_of(got, offs), wd), f"bucket {b}: unordered"
        offs, got = t.search_boxes(mins, maxs, ordered=True)
        assert np.array_equal(offs, wo)
        for j in range(q):
            a = got[int(offs[j]):int(offs[j + 1])]
            assert np.array_equal(np.sort(a), np.sort(wids[int(wo[j]):int(wo[j + 1])])), f"bucket {b} box {j}"
        cc, dd = t.digest_boxes(mins, maxs)
        assert np.array_equal(cc, wc) and np.array_equal(dd, wd), f"bucket {b}: digests"
        # the traversing write pass alone (fkd_search_write)
        t.set_param("search_record", 0)
        offs, got = t.search_boxes(mins, maxs, ordered=False)
        assert np.array_equal(O.digest_of(got, offs), wd), f"bucket {b}: traversing write"
        t.set_param("search_record", 1)
    t.close()


@pytest.mark.parametrize("dim", [2, 3, 4])
def test_leaf_buckets_with_lanes_per_box_equal_walk(cuda, dim):
    """Count and digest with 1-16 lanes per box: leaf buckets of height
    1..3 scanned by one lane ("search_bucket_lanes") give the walk's result."""
    rng = np.random.default_rng(300 + dim)
    n = 40_000
    c = rng.random((dim, n), dtype=np.float32)
    ids = rng.permutation(n).astype(np.uint32)
    q = 2000
    ctr = c[:, rng.integers(0, n, q)]
    hw = rng.uniform(0.0, 0.08, (dim, q)).astype(np.float32)
    mins, maxs = (ctr - hw).astype(np.float32), (ctr + hw).astype(np.float32)
    t = F.FKDTree(c, ids).build()
    tab, tid = t.tables()
    wc, wo, wids, _ = O.search(tab, tid, mins, maxs, variant=O.RECURSIVE)
    wd = O.digest_of(wids, wo)
    for lanes in (1, 2, 8, 16):
        t.set_param("search_lanes", lanes)
        for b in (0, 1, 2, 3):
            t.set_param("search_bucket_lanes", b)
            assert np.array_equal(t.count_boxes(mins, maxs), wc), f"lanes {lanes} bucket {b}"
            cc, dd = t.digest_boxes(mins, maxs)
            assert np.array_equal(cc, wc) and np.array_equal(dd, wd), f"lanes {lanes} bucket {b}"
    t.close()


@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_single_box_fast_path(cuda, dim):
    """fkd_search of one host-memory box (the drop-in's search_in_the_box)
    runs one warp level by level ("search_one"); its lists equal the
    reference's level-order lists and the general count + write path's, for
    empty boxes, boxes past the 1,024 ids copied back with the count, boxes
    whose frontier outgrows the warp's buffer or whose results outgrow its
    65,536 ids (both answered by the general path), NaN bounds (general path)
    and a capacity too small (FKD_ERR_CAPACITY with the true total)."""
    import ctypes as C

    from fkdtree_b200 import _capi
    rng = np.random.default_rng(40 + dim)
    n = 100_000
    c = rng.random((dim, n), dtype=np.float32)
    c[-1] = np.round(c[-1] * 64) / 64  # ties
    ids = rng.permutation(n).astype(np.uint32) * 3 + 1
    t = F.FKDTree(c, ids).build()
    tab, tid = t.tables()
    q = 160
    ctr = rng.random((dim, q), dtype=np.float32)
    hw = np.exp(rng.uniform(np.log(0.002), np.log(0.4), (1, q))).astype(np.float32)
    mins, maxs = ctr - hw, ctr + hw
    mins[:, 0], maxs[:, 0] = -np.inf, np.inf  # the whole tree: more than 65,536 results
    mins[:, 1], maxs[:, 1] = 0.0, 1.0
    maxs[-1, 1] = 0.3  # about 30,000 results, a frontier far wider than 2,048 nodes
    mins[:, 2], maxs[:, 2] = 0.5, 0.4  # empty (min > max)
    mins[0, 3] = np.nan  # NaN bound
    mins, maxs = np.ascontiguousarray(mins), np.ascontiguousarray(maxs)
    _, wo, wi, _ = O.search(tab, tid, mins, maxs, variant=O.LEVEL_ORDER)
    want = slices(wo, wi)
    assert len(want[0]) == n and len(want[1]) > 1024
    for knob in (1, 0):
        t.set_param("search_one", knob)
        for j in range(q):
            got = t.search_in_the_box(mins[:, j], maxs[:, j])
            assert np.array_equal(got, want[j]), f"search_one={knob} box {j}"
            got_u = t._one(mins[:, j], maxs[:, j], ordered=False)
            assert np.array_equal(np.sort(got_u), np.sort(want[j])), f"unordered search_one={knob} box {j}"
    t.set_param("search_one", 1)
    L = _capi.lib()
    j = int(np.argmax([len(w) for w in want[2:]])) + 2
    lo = np.ascontiguousarray(mins[:, j])
    hi = np.ascontiguousarray(maxs[:, j])
    offs = np.zeros(2, dtype=np.uint64)
    buf = np.empty(1, dtype=np.uint32)
    tot = C.c_uint64(0)
    st = L.fkd_search(t._h, lo.ctypes.data_as(C.c_void_p), hi.ctypes.data_as(C.c_void_p), 1,
                      offs.ctypes.data_as(C.c_void_p), buf.ctypes.data_as(C.c_void_p), 1, C.byref(tot), 1,
                      _capi.MEM_HOST)
    assert st == _capi.ERR_CAPACITY and tot.value == len(want[j]) and offs[1] == len(want[j])
    t.close()
