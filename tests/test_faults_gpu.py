"""Failure detection without a GPU fault: device allocation failures are
injected on the host (fkd_debug_fail_alloc), the call reports FKD_ERR_NOMEM,
nothing is left half-done, and the same handle then builds and searches
correctly."""
import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import _capi
from fkdtree_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NOMEM = 3


@pytest.fixture
def inject():
    L = _capi.lib()
    yield L.fkd_debug_fail_alloc
    L.fkd_debug_fail_alloc(-1)


@pytest.mark.parametrize("after", [0, 1, 3, 5])
def test_build_reports_nomem_then_recovers(cuda, inject, after):
    ev = W.uniform_event(n=50_000, seed=4)
    t = F.FKDTree(ev.coords, ev.ids)
    inject(after)
    with pytest.raises(F.FKDError) as e:
        t.build()
    assert e.value.status == NOMEM
    inject(-1)
    t.build()
    tab, tid = t.tables()
    want = O.build(ev.coords, ev.ids)
    assert np.array_equal(tab.view(np.uint32), want[0].view(np.uint32)) and np.array_equal(tid, want[1])


def test_search_reports_nomem_then_recovers(cuda, inject):
    ev = W.uniform_event(n=20_000, seed=5, half_width=0.03)
    t = F.FKDTree(ev.coords, ev.ids).build()
    inject(0)
    with pytest.raises(F.FKDError) as e:
        t.search_boxes(ev.mins[:, :500], ev.maxs[:, :500])
    assert e.value.status == NOMEM
    inject(-1)
    offs, ids = t.search_boxes(ev.mins[:, :500], ev.maxs[:, :500])
    tab, tid = t.tables()
    _, o, want, _ = O.search(tab, tid, ev.mins[:, :500], ev.maxs[:, :500], variant=O.LEVEL_ORDER)
    assert np.array_equal(offs, o) and np.array_equal(ids, want)


def test_failed_replan_is_not_reused(cuda, inject):
    """A build of size B whose plan upload fails must not leave the handle
    believing it still holds a plan: building size A again afterwards plans
    again and gives the reference's tables."""
    import ctypes as C
    L = _capi.lib()
    a = W.uniform_event(n=30_000, seed=6)
    b = W.uniform_event(n=200_000, seed=7)
    t = F.FKDTree(a.coords, a.ids)

    def build(ev):
        return L.fkd_build(t._h, ev.coords.ctypes.data_as(C.c_void_p), ev.ids.ctypes.data_as(C.c_void_p),
                           ev.n, F.MEM_HOST)

    assert build(a) == 0
    inject(0)  # the larger plan's upload is the first allocation of this build
    assert build(b) == NOMEM
    inject(-1)
    assert build(a) == 0
    tab = np.empty((3, a.n), dtype=np.float32)
    tid = np.empty(a.n, dtype=np.uint32)
    assert L.fkd_get_tables(t._h, tab.ctypes.data_as(C.c_void_p), tid.ctypes.data_as(C.c_void_p), F.MEM_HOST) == 0
    want = O.build(a.coords, a.ids)
    assert np.array_equal(tab.view(np.uint32), want[0].view(np.uint32)) and np.array_equal(tid, want[1])
    assert build(b) == 0
    t.close()
