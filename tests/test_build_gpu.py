"""GPU build parity: the tables built on the B200 through the C ABI are
bit-identical to the reference's (golden fixtures) and to the C restatement.
Split values and per-node ids equal => every subtree's membership is equal."""
import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import workloads as W
from oracle import oracle as O
from tests._fixtures import fixture_names, load

pytestmark = pytest.mark.gpu


def gpu_tables(coords, ids):
    t = F.FKDTree(coords, ids).build()
    tab, tid = t.tables()
    t.close()
    return tab, tid


def assert_same(t1, t2, what=""):
    assert np.array_equal(t1[0].view(np.uint32), t2[0].view(np.uint32)), f"theDimensions differ {what}"
    assert np.array_equal(t1[1], t2[1]), f"theIds differ {what}"


@pytest.mark.parametrize("name", fixture_names())
def test_build_matches_reference_fixture(cuda, name):
    f = load(name)
    assert_same(gpu_tables(f["coords"], f["ids"]), (f["tab"], f["tab_ids"]), name)


@pytest.mark.parametrize("n", [1, 2, 3, 4095, 4096, 4097, 8191, 8192, 8193, 12289, 65535, 65536, 65537, 300_001])
@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_build_matches_oracle_sizes(cuda, n, dim):
    rng = np.random.default_rng(n * 7 + dim)
    c = rng.random((dim, n), dtype=np.float32)
    ids = rng.permutation(n).astype(np.uint32)
    assert_same(gpu_tables(c, ids), O.build(c, ids), f"n={n} dim={dim}")


@pytest.mark.parametrize("kind", ["layers4d", "grid3d", "signed_zero", "inf", "clustered", "constant", "wide"])
def test_build_ties_and_special_values(cuda, kind):
    rng = np.random.default_rng(11)
    n = 70_000
    dim = 4 if kind == "layers4d" else 3
    c = rng.random((dim, n), dtype=np.float32)
    if kind == "layers4d":
        c[3] = rng.integers(0, 16, n).astype(np.float32) / np.float32(16)
    elif kind == "grid3d":
        c = rng.integers(0, 4, (3, n)).astype(np.float32)
    elif kind == "signed_zero":
        c[:, : n // 2] = np.where(rng.random((3, n // 2)) < 0.5, np.float32(-0.0), np.float32(0.0))
    elif kind == "inf":
        c[0, :1000] = np.inf
        c[1, 1000:2000] = -np.inf
    elif kind == "clustered":
        c = W.clustered_event(n=n, n_queries=1, n_clusters=16, seed=3).coords
    elif kind == "constant":
        c[:] = np.float32(0.25)
    elif kind == "wide":
        c = (rng.standard_normal((3, n)) * np.exp(rng.uniform(-30, 30, (3, n)))).astype(np.float32)
    ids = rng.permutation(n).astype(np.uint32)
    assert_same(gpu_tables(c, ids), O.build(c, ids), kind)


def test_build_from_device_memory(cuda):
    import torch
    ev = W.uniform_event(n=200_000, seed=5)
    c = torch.from_numpy(ev.coords).to(cuda)
    i = torch.from_numpy(ev.ids.view(np.int32)).to(cuda)
    t = F.FKDTree(c, i).build()
    assert_same(t.tables(), O.build(ev.coords, ev.ids))


def test_build_rejects_nan(cuda):
    rng = np.random.default_rng(0)
    for n in (100, 50_000):
        c = rng.random((3, n), dtype=np.float32)
        c[1, n // 2] = np.nan
        with pytest.raises(F.FKDError) as e:
            F.FKDTree(c).build()
        assert e.value.status == 4


def test_empty_build(cuda):
    t = F.FKDTree(np.zeros((3, 0), np.float32)).build()
    tab, tid = t.tables()
    assert tab.shape == (3, 0) and tid.shape == (0,)
    offs, ids = t.search_boxes(np.zeros((3, 2), np.float32), np.ones((3, 2), np.float32))
    assert ids.size == 0 and np.all(offs == 0)


def test_large_clustered_build_properties(cuda):
    """At 4M points: the tables are a permutation of the input and respect the
    kd order node-by-node against both children (a strong form of
    test_correct_build, FKDTree.h:24-51); full equality with the C
    restatement."""
    ev = W.clustered_event(n=1 << 22, n_queries=1, n_clusters=1024, seed=9)
    tab, tid = gpu_tables(ev.coords, ev.ids)
    assert np.array_equal(np.sort(tid), ev.ids)
    assert np.array_equal(tab[:, np.argsort(tid)], ev.coords[:, np.argsort(ev.ids)])
    n = tid.size
    i = np.arange(n)
    depth = np.floor(np.log2(i + 1)).astype(np.int64)
    c = depth % 3
    v = tab[c, i]
    for child, left in ((2 * i + 1, True), (2 * i + 2, False)):
        ok = child < n
        p, ch, cc = i[ok], child[ok], c[ok]
        pv, chv = tab[cc, p], tab[cc, ch]
        if left:
            assert np.all((chv < pv) | ((chv == pv) & (tid[ch] < tid[p])))
        else:
            assert np.all((chv > pv) | ((chv == pv) & (tid[ch] > tid[p])))
    assert_same((tab, tid), O.build(ev.coords, ev.ids))


@pytest.mark.parametrize("subtree", [1, 2])
@pytest.mark.parametrize("dim,kind", [(1, "uniform"), (2, "uniform"), (3, "uniform"), (3, "grid"), (2, "grid"),
                                      (3, "signed_zero"), (3, "sparse_ids")])
def test_subtree_kernels_agree(cuda, subtree, dim, kind):
    """Both shared-memory subtree kernels (radix select, presorted lists) give
    the oracle's tables, on ties, signed zeros, and ids far apart."""
    rng = np.random.default_rng(31 + dim)
    n = 50_000
    c = rng.random((dim, n), dtype=np.float32)
    ids = rng.permutation(n).astype(np.uint32)
    if kind == "grid":
        c = rng.integers(0, 3, (dim, n)).astype(np.float32)
    elif kind == "signed_zero":
        c[:, : n // 3] = np.where(rng.random((dim, n // 3)) < 0.5, np.float32(-0.0), np.float32(0.0))
    elif kind == "sparse_ids":
        ids = rng.choice(np.iinfo(np.uint32).max, n, replace=False).astype(np.uint32)
    t = F.FKDTree(c, ids).set_param("subtree", subtree).build()
    got = t.tables()
    t.close()
    assert_same(got, O.build(c, ids), f"subtree={subtree} dim={dim} {kind}")


@pytest.mark.parametrize("q", [1 << 21, 1 << 18, 1 << 15, 1 << 13, 1 << 11])
@pytest.mark.parametrize("dim", [2, 3, 4])
def test_build_pivot_ties_resolved_by_id(cuda, q, dim):
    """Coordinates on a grid of q steps: the points sharing a level's pivot
    value number from one to a few hundred, so some segments take the
    partition's tie resolution (up to 32 tied points, ordered by id) and
    others the id digit passes; both must give the reference's tables, with
    the tie resolution on and off."""
    rng = np.random.default_rng(q + dim)
    n = 300_000
    c = (np.floor(rng.random((dim, n)) * q) / q).astype(np.float32)
    ids = (rng.permutation(n).astype(np.uint64) * 2654435761 % (1 << 32)).astype(np.uint32)
    want = O.build(c, ids)
    for tf in (1, 0):
        t = F.FKDTree(c, ids)
        t.set_param("small_fix", tf)
        t.build()
        assert_same(t.tables(), want, f"q={q} dim={dim} small_fix={tf}")
        t.close()


@pytest.mark.parametrize("subn", [512, 1024])
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("n", [511, 512, 513, 1023, 1025, 70_001])
def test_build_presorted_subtree_sizes(cuda, subn, dim, n):
    """Both sizes of the presorted-list subtree kernel ("subtree_size") give
    the reference's tables; 512 takes one more global level."""
    rng = np.random.default_rng(n + 31 * dim + subn)
    c = rng.random((dim, n), dtype=np.float32)
    c[0, : n // 3] = np.round(c[0, : n // 3] * 64) / 64  # ties
    ids = rng.permutation(n).astype(np.uint32)
    t = F.FKDTree(c, ids)
    t.set_param("subtree_size", subn)
    t.build()
    assert_same(t.tables(), O.build(c, ids), f"subn={subn} dim={dim} n={n}")
    t.close()


@pytest.mark.parametrize("subn", [512, 1024])
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("kind", ["wide", "near_zero", "long_runs", "short_runs"])
def test_build_presorted_subtree_key_paths(cuda, subn, dim, kind):
    """The presorted-list kernel's sort keys: ranges of order bits far wider
    than a 32-bit key holds ("wide": magnitudes over 2^-40..2^40;
    "near_zero": cells that reach down to 0), where the keys drop low bits and
    runs of equal keys are re-ordered by (coordinate, id); runs of more than
    32 equal coordinates ("long_runs"), which take the exact 64-bit path; and
    runs of a few ("short_runs")."""
    rng = np.random.default_rng(7 * dim + subn + len(kind))
    n = 40_001
    c = rng.random((dim, n), dtype=np.float32)
    if kind == "wide":
        c = (rng.standard_normal((dim, n)) * np.exp2(rng.uniform(-40, 40, (dim, n)))).astype(np.float32)
    elif kind == "near_zero":
        c = (rng.random((dim, n)) ** 8).astype(np.float32)
    elif kind == "long_runs":
        c[-1] = np.floor(c[-1] * 400) / 400  # about 100 points per value
    else:
        c[-1] = np.floor(c[-1] * 8000) / 8000  # about 5 points per value
    ids = rng.permutation(n).astype(np.uint32)
    t = F.FKDTree(c, ids)
    t.set_param("subtree_size", subn)
    t.build()
    assert_same(t.tables(), O.build(c, ids), f"subn={subn} dim={dim} {kind}")
    t.close()
