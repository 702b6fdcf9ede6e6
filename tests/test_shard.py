"""Event sharding for several GPUs, tested on the CPU: the balance of the
assignment, the re-packed sub-batches, and two gloo ranks that each run the
oracle on their own share and reassemble exactly the single-process result
(no collective on the data path; only the test gathers the results)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fkdtree_b200 import shard as S
from fkdtree_b200 import workloads as W


def small_batch(seed=7):
    return W.event_batch(n_events=24, median=800, size_lo=1, size_hi=5_000, clusters_lo=3, clusters_hi=20,
                         half_width=0.02, seed=seed, frac_4d=0.25)


def test_assign_events_balanced_and_disjoint():
    rng = np.random.default_rng(0)
    sizes = rng.integers(1, 200_000, 4096)
    for world in (1, 2, 3, 8):
        share = S.assign_events(sizes, world)
        allev = np.concatenate(share)
        assert np.array_equal(np.sort(allev), np.arange(len(sizes)))
        loads = np.array([sizes[s].sum() for s in share])
        assert loads.max() - loads.min() <= sizes.max()  # LPT bound
    with pytest.raises(ValueError):
        S.assign_events(sizes, 0)


def test_sub_batch_repacks_events():
    wb = small_batch()
    ev = [5, 0, 17]
    sb = S.sub_batch(wb, ev)
    for k, e in enumerate(ev):
        a, b = sb.event(k), wb.event(e)
        assert a.dim == b.dim
        for x, y in ((a.coords, b.coords), (a.ids, b.ids), (a.mins, b.mins), (a.maxs, b.maxs)):
            assert np.array_equal(x, y)
    idx = S.box_index(wb, ev)
    assert len(idx) == sb.n_queries and idx[0] == wb.q_off[5]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wb = small_batch()
        mine = S.assign_events(np.diff(wb.pt_off.astype(np.int64)), world)[rank]
        sb = S.sub_batch(wb, mine)
        _, _, c, d = O.batch(sb)
        got = [None] * world
        dist.all_gather_object(got, (mine.tolist(), c, d))
        if rank == 0:
            nq = wb.n_queries
            counts = np.zeros(nq, np.uint32)
            digests = np.zeros(nq, np.uint64)
            seen = np.zeros(nq, bool)
            for ev, cc, dd in got:
                idx = S.box_index(wb, ev)
                counts[idx], digests[idx] = cc, dd
                seen[idx] = True
            _, _, c0, d0 = O.batch(wb)
            out.put(bool(seen.all() and np.array_equal(counts, c0) and np.array_equal(digests, d0)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reassemble_single_process_result():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ok
