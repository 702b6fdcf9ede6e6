"""The C restatement (oracle/fkd_oracle.c) against the golden fixtures that
the unmodified reference produced (tests/golden/make_golden.py).  CPU only."""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from fkdtree_b200 import workloads as W
from tests._fixtures import GOLDEN, fixture_names, load, slices


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.build_libs()


@pytest.mark.parametrize("name", fixture_names())
def test_oracle_build_matches_reference(name):
    f = load(name)
    tab, tid = O.build(f["coords"], f["ids"])
    assert np.array_equal(tab.view(np.uint32), f["tab"].view(np.uint32)), "theDimensions differ"
    assert np.array_equal(tid, f["tab_ids"]), "theIds differ"


@pytest.mark.parametrize("name", fixture_names())
def test_oracle_searches_match_reference(name):
    f = load(name)
    tab, tid = f["tab"], f["tab_ids"]
    c, o, i, _ = O.search(tab, tid, f["mins"], f["maxs"], variant=O.RECURSIVE)
    assert np.array_equal(c, f["rec_counts"]) and np.array_equal(i, f["rec_ids"])
    for v, key in [(O.LEVEL_ORDER, "lvl"), (O.BFS, "bfs"), (O.BRANCHLESS, "bl")]:
        mins, maxs = f["mins"], f["maxs"]
        if f"{key}_sel" in f:
            mins, maxs = mins[:, f[f"{key}_sel"]], maxs[:, f[f"{key}_sel"]]
        c, o, i, _ = O.search(tab, tid, mins, maxs, variant=v)
        assert np.array_equal(c, f[f"{key}_counts"]) and np.array_equal(i, f[f"{key}_ids"]), key


@pytest.mark.parametrize("name", fixture_names())
def test_every_variant_returns_the_brute_force_set(name):
    """FKDTree.h:54-86: each result set equals the brute-force scan."""
    f = load(name)
    cb, ob, ib, _ = O.search(f["tab"], f["tab_ids"], f["mins"], f["maxs"], variant=O.BRUTE)
    assert np.array_equal(cb, f["rec_counts"])
    for a, b in zip(slices(ob, ib), slices(f["rec_offsets"], f["rec_ids"])):
        assert np.array_equal(np.sort(a), np.sort(b))


def test_level_order_is_ascending_heap_order():
    """search_in_the_box emits in-box nodes sorted by heap index; the GPU's
    ordered output relies on it."""
    f = load("uniform3d_n1000")
    pos = np.empty(f["tab_ids"].max() + 1, dtype=np.int64)
    pos[f["tab_ids"]] = np.arange(f["tab_ids"].size)
    for s in slices(f["lvl_offsets"], f["lvl_ids"]):
        assert np.all(np.diff(pos[s]) > 0)


def test_oracle_small_single_event_summary():
    ev = W.uniform_event()
    with np.load(GOLDEN / "uniform3d_n100000_summary.npz") as z:
        tab, tid = O.build(ev.coords, ev.ids)
        assert hashlib.sha256(tab.tobytes()).hexdigest() == str(z["tab_sha"])
        assert hashlib.sha256(tid.tobytes()).hexdigest() == str(z["ids_sha"])
        c, o, i, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.LEVEL_ORDER)
        assert np.array_equal(c, z["counts"])
        assert hashlib.sha256(i.tobytes()).hexdigest() == str(z["lvl_ids_sha"])


def test_digest_definition():
    ids = np.array([0, 1, 2, 3, 0xFFFFFFFF], dtype=np.uint32)
    m = O.mix64(ids)
    for a, b in zip(ids, m):
        assert O.lib().fkd_oracle_mix64(int(a)) == int(b)
    f = load("uniform3d_n1000")
    c, d = O.search_digest(f["tab"], f["tab_ids"], f["mins"], f["maxs"])
    assert np.array_equal(c, f["rec_counts"])
    assert np.array_equal(d, O.digest_of(f["rec_ids"], f["rec_offsets"]))


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_oracle_matches_reference_on_random_inputs():
    rng = np.random.default_rng(99)
    for n in [10, 257, 4096, 30000]:
        for dim in (2, 3, 4):
            c = rng.random((dim, n), dtype=np.float32)
            c[0] = np.round(c[0] * 64) / 64
            ids = rng.permutation(n).astype(np.uint32)
            t1 = O.build(c, ids)
            r = O.RefTree(c, ids)
            r.build()
            t2 = r.tables()
            r.close()
            assert np.array_equal(t1[0].view(np.uint32), t2[0].view(np.uint32)) and np.array_equal(t1[1], t2[1])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_reference_batch_matches_restated_batch():
    """The unmodified reference over a batch of events (OpenMP over events,
    recursive search) gives the same per-box counts and digests as the C
    restatement -- the batched CPU baseline and the GPU parity target agree."""
    from fkdtree_b200 import workloads as W
    wb = W.event_batch(n_events=24, median=2000, size_lo=1, size_hi=12_000, clusters_lo=5, clusters_hi=30,
                       half_width=0.02, seed=8, frac_4d=0.3)
    c1, d1, _ = O.ref_batch(wb, threads=2)
    _, _, c2, d2 = O.batch(wb)
    assert np.array_equal(c1, c2) and np.array_equal(d1, d2)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_vanilla_cmssw_tree_counts_match_reference():
    """The reference's vanilla CMSSW tree (the extra CPU baseline column)
    finds the same number of points per box as FKDTree_CPU on boxes whose
    faces hold no point (it tests inner regions with strict inequalities)."""
    ev = W.clustered_event(n=50_000, n_queries=500, n_clusters=64, seed=12)
    counts, tb, ts = O.ref_cmssw(ev.coords, ev.mins, ev.maxs)
    r = O.RefTree(ev.coords, ev.ids)
    r.build()
    want, _, _, _ = r.search(ev.mins, ev.maxs, variant=O.RECURSIVE, want_ids=False)
    r.close()
    assert np.array_equal(counts, want)
    assert tb > 0 and ts > 0


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_oracle_matches_reference_at_edge_sizes_and_values(dim):
    """Sizes around powers of two (incomplete last levels, single-child
    nodes) and degenerate values -- all-equal coordinates, an integer grid,
    signed zeros and infinities -- built by the restatement and by the
    unmodified reference: identical tables; every search variant of the
    restatement equals brute force on them."""
    rng = np.random.default_rng(dim)
    sizes = [1, 2, 3, 4, 7, 8, 9, 15, 16, 17, 31, 32, 33, 1023, 1024, 1025, 4095, 4096, 4097]
    kinds = ["uniform", "equal", "grid", "signed_zero_inf"]
    for n in sizes:
        for kind in kinds:
            c = rng.random((dim, n), dtype=np.float32)
            if kind == "equal":
                c[:] = np.float32(0.25)
            elif kind == "grid":
                c = np.round(c * 4).astype(np.float32)
            elif kind == "signed_zero_inf":
                c = np.where(c < 0.3, np.float32(-0.0), np.where(c > 0.9, np.float32(np.inf), c)).astype(np.float32)
                c[:, ::5] = np.float32(0.0)
            ids = rng.permutation(n).astype(np.uint32)
            t1 = O.build(c, ids)
            r = O.RefTree(c, ids)
            r.build()
            t2 = r.tables()
            r.close()
            assert np.array_equal(t1[0].view(np.uint32), t2[0].view(np.uint32)), (n, kind)
            assert np.array_equal(t1[1], t2[1]), (n, kind)
            lo = (c[:, : min(n, 40)] - np.float32(0.3)).astype(np.float32)
            hi = (c[:, : min(n, 40)] + np.float32(0.3)).astype(np.float32)
            want = O.search(t1[0], t1[1], lo, hi, variant=O.BRUTE)[0]
            for v in (O.LEVEL_ORDER, O.BFS, O.BRANCHLESS, O.RECURSIVE):
                assert np.array_equal(O.search(t1[0], t1[1], lo, hi, variant=v)[0], want), (n, kind, v)


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_fixtures_reproduce_from_the_reference():
    """The committed fixtures are what tests/golden/make_golden.py gets from
    the unmodified reference today: same generator, same tables, same lists."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    checked = 0
    for name, coords, ids, boxes in mg.cases():
        if not (name.startswith("tiny3d") or name in ("layers4d_n3000", "grid2d_n2000", "zeros_inf3d_n600")):
            continue
        f = load(name)
        assert np.array_equal(f["coords"].view(np.uint32), coords.view(np.uint32)) and np.array_equal(f["ids"], ids)
        r = O.RefTree(coords, ids)
        r.build()
        tab, tid = r.tables()
        assert np.array_equal(tab.view(np.uint32), f["tab"].view(np.uint32)) and np.array_equal(tid, f["tab_ids"])
        rc, ro, ri, _ = r.search(f["mins"], f["maxs"], variant=O.RECURSIVE)
        assert np.array_equal(ro, f["rec_offsets"]) and np.array_equal(ri, f["rec_ids"])
        sel = f.get("lvl_sel")
        lo, hi = (f["mins"], f["maxs"]) if sel is None else (f["mins"][:, sel], f["maxs"][:, sel])
        _, lo_off, lo_ids, _ = r.search(lo, hi, variant=O.LEVEL_ORDER)
        assert np.array_equal(lo_off, f["lvl_offsets"]) and np.array_equal(lo_ids, f["lvl_ids"])
        r.close()
        checked += 1
    assert checked == 22
