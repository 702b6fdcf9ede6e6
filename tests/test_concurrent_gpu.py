"""Concurrent searches on one built tree (the reference's TBB loop over one
FKDTree_CPU, main.cpp:351-359): host threads call the C ABI's searches on
the same handle at once -- ctypes releases the GIL for the length of each
call, so the calls really overlap -- and every result must equal the
oracle's.  Mixes single-box and batched calls, host- and device-memory
buffers, box / radius / kNN / count / digest searches."""
import ctypes as C
import threading

import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import _capi
from fkdtree_b200 import workloads as W
from oracle import nn_ref as NN
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _run_threads(fn, n):
    errors = []

    def wrap(t):
        try:
            fn(t)
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append(f"thread {t}: {e!r}")

    th = [threading.Thread(target=wrap, args=(t,)) for t in range(n)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert not errors, errors


def test_threads_single_box_searches_equal_reference(cuda):
    ev = W.uniform_event(n=100_000, seed=11, half_width=0.02)
    t = F.FKDTree(ev.coords, ev.ids).build()
    tab, tid = t.tables()
    q = 4000
    _, want_off, want_ids, _ = O.search(tab, tid, ev.mins[:, :q], ev.maxs[:, :q], variant=O.LEVEL_ORDER)
    got = [None] * q
    L = _capi.lib()

    def work(k):
        buf = np.empty(4096, dtype=np.uint32)
        offs = np.zeros(2, dtype=np.uint64)
        tot = C.c_uint64(0)
        for j in range(k, q, 8):
            lo = np.ascontiguousarray(ev.mins[:, j])
            hi = np.ascontiguousarray(ev.maxs[:, j])
            _capi.check(L.fkd_search(t._h, lo.ctypes.data_as(C.c_void_p), hi.ctypes.data_as(C.c_void_p), 1,
                                     offs.ctypes.data_as(C.c_void_p), buf.ctypes.data_as(C.c_void_p), buf.size,
                                     C.byref(tot), 1, _capi.MEM_HOST))
            got[j] = buf[:tot.value].copy()

    _run_threads(work, 8)
    for j in range(q):
        assert np.array_equal(got[j], want_ids[int(want_off[j]):int(want_off[j + 1])]), f"box {j}"
    t.close()


def test_threads_mixed_searches_equal_oracle(cuda):
    import torch
    ev = W.clustered_event(n=300_000, n_queries=20_000, n_clusters=64)
    t = F.FKDTree(ev.coords, ev.ids).build()
    tab, tid = t.tables()
    wc, wo, wids, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.RECURSIVE)
    wdc, wdd = O.search_digest(tab, tid, ev.mins, ev.maxs)
    ctr = np.ascontiguousarray(ev.coords[:, :2000])
    rad = np.full(2000, 0.01, dtype=np.float32)
    woff_r, wids_r = NN.radius(tab, tid, ctr, rad)
    wk, wkd = NN.knn(ev.coords, ev.ids, ctr, 8)
    dmins = torch.from_numpy(ev.mins).cuda()
    dmaxs = torch.from_numpy(ev.maxs).cuda()
    results = {}

    def work(k):
        for rep in range(3):
            kind = (k + rep) % 5
            if kind == 0:
                offs, ids = t.search_boxes(ev.mins, ev.maxs, ordered=False)
                assert np.array_equal(offs, wo)
                assert np.array_equal(O.digest_lists(offs, ids), O.digest_lists(wo, wids))
            elif kind == 1:
                c, d = t.digest_boxes(ev.mins, ev.maxs)
                assert np.array_equal(c, wdc) and np.array_equal(d, wdd)
            elif kind == 2:
                c = t.count_boxes(dmins, dmaxs)  # device memory: the handle's stream
                assert np.array_equal(c.cpu().numpy().view(np.uint32), wc)
            elif kind == 3:
                ro, ri = t.search_radius(ctr, rad)
                assert np.array_equal(ro, woff_r) and np.array_equal(ri, wids_r)
            else:
                ki, kd = t.knn(ctr, 8)
                assert np.array_equal(ki, wk) and np.array_equal(kd.view(np.uint32), wkd.view(np.uint32))
            results[(k, rep)] = True

    _run_threads(work, 10)
    assert len(results) == 30
    t.close()
