"""Batched events through the C ABI: every event's tables equal the per-event
C restatement (one FKDTree_CPU::build per event), every box's count and
digest equal the per-event recursive search, for uneven sizes, mixed 3D/4D
events and the single CUDA-graph launch."""
import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def check_batch(wb, gpu_tab, gpu_tid, counts, digests):
    otab, otid, oc, od = O.batch(wb)
    assert np.array_equal(gpu_tab.view(np.uint32), otab.view(np.uint32)), "tables differ"
    assert np.array_equal(gpu_tid, otid), "ids differ"
    assert np.array_equal(np.asarray(counts).astype(np.uint32), oc), "counts differ"
    assert np.array_equal(np.asarray(digests).astype(np.uint64), od), "digests differ"


@pytest.mark.parametrize("frac_4d,lanes,big_n,lanes_big", [(0.0, 0, 0, 0), (0.5, 0, 0, 0), (0.5, 1, 0, 0),
                                                           (0.0, 2, 0, 0), (0.5, 4, 0, 0), (0.0, 8, 0, 0),
                                                           (0.5, 16, 0, 0), (0.0, 2, 6000, 32), (0.5, 1, 3000, 8),
                                                           (0.5, 4, 100_000, 32)])
def test_batch_matches_per_event_oracle(cuda, frac_4d, lanes, big_n, lanes_big):
    wb = W.event_batch(n_events=64, median=6000, size_lo=1, size_hi=60_000, clusters_lo=5, clusters_hi=50,
                       half_width=0.01, seed=21, frac_4d=frac_4d)
    b = F.Batch.of(wb)
    b.set_param("search_lanes", lanes)
    b.set_param("search_lanes_big", lanes_big)
    b.set_param("search_big_n", big_n)
    b.build(wb.coords, wb.ids)
    tab, tid = b.tables()
    c, d = b.search_digest(wb.mins, wb.maxs)
    check_batch(wb, tab, tid, c, d)


def test_batch_edge_sizes(cuda):
    """Events of 1, 2, 3 points, exactly the shared-memory capacity and one
    past it, and an event with no boxes."""
    rng = np.random.default_rng(5)
    sizes = [1, 2, 3, 4095, 4096, 4097, 8193, 17, 100_000]
    dims = np.array([3] * len(sizes), np.uint32)
    pt_off = np.zeros(len(sizes) + 1, np.uint64)
    pt_off[1:] = np.cumsum(sizes)
    coords = np.concatenate([rng.random((3, n), dtype=np.float32).reshape(-1) for n in sizes])
    ids = np.concatenate([rng.permutation(n).astype(np.uint32) for n in sizes])
    qn = [n if k != 7 else 0 for k, n in enumerate(sizes)]
    q_off = np.zeros(len(sizes) + 1, np.uint64)
    q_off[1:] = np.cumsum(qn)
    mins, maxs = [], []
    c0 = 0
    for k, n in enumerate(sizes):
        sl = coords[c0:c0 + 3 * n].reshape(3, n)
        c0 += 3 * n
        if qn[k]:
            mins.append((sl - np.float32(0.05)).reshape(-1))
            maxs.append((sl + np.float32(0.05)).reshape(-1))
    wb = W.Batch(dims, pt_off, pt_off.copy(), q_off, q_off.copy(), coords, ids,
                 np.concatenate(mins).astype(np.float32), np.concatenate(maxs).astype(np.float32))
    wb.coord_off = np.zeros(len(sizes) + 1, np.uint64)
    wb.coord_off[1:] = np.cumsum(np.array(sizes) * 3)
    wb.qcoord_off = np.zeros(len(sizes) + 1, np.uint64)
    wb.qcoord_off[1:] = np.cumsum(np.array(qn) * 3)
    b = F.Batch.of(wb)
    b.build(wb.coords, wb.ids)
    tab, tid = b.tables()
    c, d = b.search_digest(wb.mins, wb.maxs)
    check_batch(wb, tab, tid, c, d)


def test_batch_graph_run_device(cuda):
    import torch
    wb = W.event_batch(n_events=200, median=20_000, size_lo=1_000, size_hi=200_000, clusters_lo=50,
                       clusters_hi=500, half_width=0.01, seed=33, frac_4d=0.5)
    b = F.Batch.of(wb)
    dev = cuda
    coords = torch.from_numpy(wb.coords).to(dev)
    ids = torch.from_numpy(wb.ids.view(np.int32)).to(dev)
    mins = torch.from_numpy(wb.mins).to(dev)
    maxs = torch.from_numpy(wb.maxs).to(dev)
    counts = torch.empty(wb.n_queries, dtype=torch.int32, device=dev)
    dig = torch.empty(wb.n_queries, dtype=torch.int64, device=dev)
    for _ in range(2):  # capture, then replay
        counts.zero_()
        dig.zero_()
        b.run(coords, ids, mins, maxs, counts, dig)
    tab, tid = b.tables()
    check_batch(wb, tab, tid, counts.cpu().numpy().view(np.uint32), dig.cpu().numpy().view(np.uint64))


def test_autotuned_batch_graph(cuda, tmp_path):
    """The autotuner sweeps the knobs on the batch itself, caches the choice,
    and the graph launched with the chosen knobs still gives exact results."""
    import torch
    wb = W.event_batch(n_events=96, median=8_000, size_lo=500, size_hi=60_000, clusters_lo=20, clusters_hi=200,
                       half_width=0.01, seed=34, frac_4d=0.25)
    b = F.Batch.of(wb)
    dev = cuda
    coords = torch.from_numpy(wb.coords).to(dev)
    ids = torch.from_numpy(wb.ids.view(np.int32)).to(dev)
    mins = torch.from_numpy(wb.mins).to(dev)
    maxs = torch.from_numpy(wb.maxs).to(dev)
    cache = str(tmp_path / "tune.json")
    r = b.autotune(coords, ids, mins, maxs, cache_file=cache, reps=1, hist_ctas=[148, 592])
    assert not r["cached"] and r["search_lanes"] in (1, 2, 4, 8, 16, 32) and r["hist_ctas"] in (148, 592)
    b2 = F.Batch.of(wb)
    r2 = b2.autotune(coords, ids, mins, maxs, cache_file=cache)
    assert r2["cached"] and r2["search_lanes"] == r["search_lanes"]
    counts = torch.empty(wb.n_queries, dtype=torch.int32, device=dev)
    dig = torch.empty(wb.n_queries, dtype=torch.int64, device=dev)
    b2.run(coords, ids, mins, maxs, counts, dig)
    tab, tid = b2.tables()
    check_batch(wb, tab, tid, counts.cpu().numpy().view(np.uint32), dig.cpu().numpy().view(np.uint64))


@pytest.mark.parametrize("lanes", [2, 32])
def test_batch_leaf_buckets_equal_walk(cuda, lanes):
    """Batched digest search with and without leaf buckets, against the oracle."""
    import torch
    wb = W.event_batch(n_events=40, median=4000, size_lo=1, size_hi=50_000, clusters_lo=3, clusters_hi=40,
                       half_width=0.01, seed=41, frac_4d=0.3)
    _, _, oc, od = O.batch(wb)
    coords = torch.from_numpy(wb.coords).cuda()
    ids = torch.from_numpy(wb.ids.view(np.int32)).cuda()
    mins = torch.from_numpy(wb.mins).cuda()
    maxs = torch.from_numpy(wb.maxs).cuda()
    b = F.Batch.of(wb)
    b.set_param("search_lanes", lanes)
    b.build(coords, ids)
    for bk, bg in ((0, 0), (4, 2), (6, 3)):
        b.set_param("search_bucket", bk)
        b.set_param("search_bucket_lanes", bg)
        c, d = b.search_digest(mins, maxs)
        assert np.array_equal(c.cpu().numpy().view(np.uint32), oc), f"bucket {bk}/{bg}"
        assert np.array_equal(d.cpu().numpy().view(np.uint64), od), f"bucket {bk}/{bg}"
    b.close()
