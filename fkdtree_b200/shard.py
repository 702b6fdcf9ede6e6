"""Sharding batched events over ranks (one process per GPU).

Events are independent trees, so a multi-GPU batch needs no collective on
the data path: each rank builds and searches its own share of the events and
the per-box results are gathered only where the caller wants them in one
place.  Shares are balanced by points (longest-processing-time greedy:
largest event first, onto the rank with the fewest points so far; ties go to
the lower rank), which keeps the slowest rank -- the one that sets the
job's time -- close to the mean.  No reference counterpart (the reference has
no multi-GPU path).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np

from .workloads import Batch


def assign_events(sizes: Sequence[int], world: int) -> List[np.ndarray]:
    """Event indices of every rank (ascending), balanced by size."""
    if world < 1:
        raise ValueError("world must be >= 1")
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    heap = [(0, r) for r in range(world)]
    share: List[List[int]] = [[] for _ in range(world)]
    for e in order:
        load, r = heapq.heappop(heap)
        share[r].append(int(e))
        heapq.heappush(heap, (load + int(sizes[e]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in share]


def sub_batch(wb: Batch, events: Sequence[int]) -> Batch:
    """The batch of the given events (in the given order), re-packed."""
    events = np.asarray(events, dtype=np.int64)
    dims = wb.dims[events].astype(np.uint32)
    n = (wb.pt_off[events + 1] - wb.pt_off[events]).astype(np.int64)
    q = (wb.q_off[events + 1] - wb.q_off[events]).astype(np.int64)

    def offs(x):
        o = np.zeros(len(events) + 1, dtype=np.uint64)
        o[1:] = np.cumsum(x)
        return o

    def gather(flat, off, width):
        parts = [flat[int(off[e]):int(off[e]) + int(w)] for e, w in zip(events, width)]
        return np.concatenate(parts) if parts else flat[:0].copy()

    coords = gather(wb.coords, wb.coord_off, n * dims)
    ids = gather(wb.ids, wb.pt_off, n)
    mins = gather(wb.mins, wb.qcoord_off, q * dims)
    maxs = gather(wb.maxs, wb.qcoord_off, q * dims)
    return Batch(dims, offs(n), offs(n * dims), offs(q), offs(q * dims), coords, ids, mins, maxs,
                 dict(wb.meta, events=events.tolist()))


def box_index(wb: Batch, events: Sequence[int]) -> np.ndarray:
    """Global box index of every box of sub_batch(wb, events), in its order:
    scatters per-shard counts / digests back into the full batch's order."""
    parts = [np.arange(int(wb.q_off[e]), int(wb.q_off[e + 1]), dtype=np.int64) for e in events]
    return np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)


def run_share(wb: Batch, events: Sequence[int], device, reps: int = 1, stream=None):
    """Builds and digest-searches one rank's share of the events on its own GPU
    through the batch C ABI (fkd_batch_run: gather, build and per-box count +
    digest in one CUDA graph), `reps` times after one warm-up run.  Returns
    (counts, digests, box_index, ms): counts / digests (CUDA tensors, the
    share's boxes in its order), box_index the global box index of each
    (box_index()), ms the CUDA-event time of the last run on the share's
    stream.  No collective: events are independent trees."""
    import torch

    from . import Batch as _Batch

    sb = sub_batch(wb, events)
    dev = torch.device(device)
    # the graph is captured on this stream (capture needs a stream other than the legacy default one)
    s = stream if stream is not None else torch.cuda.Stream(dev)
    coords = torch.from_numpy(sb.coords).to(dev)
    ids = torch.from_numpy(sb.ids.view(np.int32)).to(dev)
    mins = torch.from_numpy(sb.mins).to(dev)
    maxs = torch.from_numpy(sb.maxs).to(dev)
    counts = torch.empty(sb.n_queries, dtype=torch.int32, device=dev)
    digests = torch.empty(sb.n_queries, dtype=torch.int64, device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    b = _Batch.of(sb, stream=s)
    try:
        b.run(coords, ids, mins, maxs, counts, digests)
        ms = 0.0
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.run(coords, ids, mins, maxs, counts, digests)
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
    finally:
        b.close()
    return counts, digests, box_index(wb, events), ms
