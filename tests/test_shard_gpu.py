"""Event sharding through the CUDA library on one GPU: the events of a batch
split over two ranks' shares (shard.assign_events), each share re-packed and
run as its own batch graph (shard.run_share), the per-box counts and digests
scattered back by shard.box_index -- equal to the whole batch run as one
graph and to the oracle.  (The ranks run one after the other here; on
several GPUs each runs on its own device with no collective.)"""
import numpy as np
import pytest
import torch

import fkdtree_b200 as F
from fkdtree_b200 import shard as S
from fkdtree_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_shards_reassemble_the_whole_batch(cuda, world):
    wb = W.event_batch(n_events=60, median=3000, size_lo=1, size_hi=40_000, clusters_lo=3, clusters_hi=40,
                       half_width=0.01, seed=31, frac_4d=0.3)
    coords = torch.from_numpy(wb.coords).cuda()
    ids = torch.from_numpy(wb.ids.view(np.int32)).cuda()
    mins = torch.from_numpy(wb.mins).cuda()
    maxs = torch.from_numpy(wb.maxs).cuda()
    wc = torch.empty(wb.n_queries, dtype=torch.int32, device="cuda")
    wd = torch.empty(wb.n_queries, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    b = F.Batch.of(wb, stream=s)
    b.run(coords, ids, mins, maxs, wc, wd)
    b.close()
    whole_c = wc.cpu().numpy().view(np.uint32)
    whole_d = wd.cpu().numpy().view(np.uint64)
    sizes = np.diff(wb.pt_off.astype(np.int64))
    got_c = np.zeros(wb.n_queries, dtype=np.uint32)
    got_d = np.zeros(wb.n_queries, dtype=np.uint64)
    seen = np.zeros(wb.n_queries, dtype=bool)
    for share in S.assign_events(sizes, world):
        c, d, bi, ms = S.run_share(wb, share, "cuda:0")
        assert ms > 0
        got_c[bi] = c.cpu().numpy().view(np.uint32)
        got_d[bi] = d.cpu().numpy().view(np.uint64)
        seen[bi] = True
    assert seen.all()
    assert np.array_equal(got_c, whole_c) and np.array_equal(got_d, whole_d)
    _, _, oc, od = O.batch(wb)
    assert np.array_equal(whole_c, oc) and np.array_equal(whole_d, od)
