"""The 16M-point clustered workload itself (16,777,216 points: 80% in 4,096
Gaussian clusters, sigma 0.002, Dirichlet(1) weights, 20% uniform; seed 1),
built on the GPU through the C ABI and compared with the unmodified
reference FKDTree_CPU (oracle/_ref) built from the same points: the tables
bit for bit (FKDTree_cpu.h:221-277), and on 65,536 of its boxes every box's
count and order-independent digest against the reference's
search_in_the_box_recursive (FKDTree_cpu.h:171-207), through both the
written-id search and the digest search."""
import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2():
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    ev = W.clustered_event(n_queries=1 << 16)
    r = O.RefTree(ev.coords, ev.ids)
    r.build()
    tab, tid = r.tables()
    rc, rd, _ = r.search_digest(ev.mins, ev.maxs, threads=O.host_threads())
    r.close()
    return ev, tab, tid, rc, rd


def test_c2_tables_equal_reference(cuda, c2):
    ev, tab, tid, _, _ = c2
    t = F.FKDTree(ev.coords, ev.ids).build()
    gtab, gtid = t.tables()
    t.close()
    assert np.array_equal(gtab.view(np.uint32), tab.view(np.uint32))
    assert np.array_equal(gtid, tid)


def test_c2_box_results_equal_reference(cuda, c2):
    import torch
    ev, _, _, rc, rd = c2
    coords = torch.from_numpy(ev.coords).cuda()
    ids = torch.from_numpy(ev.ids.view(np.int32)).cuda()
    t = F.FKDTree(coords, ids).build()
    offs, out = t.search_boxes(ev.mins, ev.maxs, ordered=False)
    gd = O.digest_lists(offs, out, threads=O.host_threads())
    assert np.array_equal(np.diff(offs).astype(np.uint32), rc)
    assert np.array_equal(gd, rd)
    dc, dd = t.digest_boxes(ev.mins, ev.maxs)
    assert np.array_equal(dc, rc) and np.array_equal(dd, rd)
    t.close()
