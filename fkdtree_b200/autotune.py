"""Autotuner of the launch choices of batched builds and searches.

No reference counterpart: the reference has one fixed launch shape per
kernel.  The knobs are the ones `fkd_batch_set_param` / `fkd_set_param`
expose (include/fkdtree_b200.h):

* ``hist_ctas``     CTAs of each global digit pass and partition of the build
                    (the tile count of the segmented radix select);
* ``subtree_size``  the largest subtree the presorted-list kernel finishes in
                    shared memory (512 or 1,024 points: one global level more
                    against a cheaper subtree kernel);
* ``search_lanes``  lanes that share one box in the count / digest search
                    (32 = a warp per box; 1 = a thread per box).
* ``search_big_n``, ``search_lanes_big``  a size split of the digest search:
                    events of at least big_n points search in a launch of
                    their own with their own lanes per box (large events fill
                    a warp per box, small ones do not).

The build and the search are independent, so each knob is swept on its own
phase: every candidate is timed (best of ``reps`` runs after one warm-up),
the fastest wins, ties go to the earlier candidate.  Results are cached in a
JSON file keyed by the device name and a coarse shape of the workload (event
dimensions, log2 buckets of the event count, the median event size and the
boxes per point), so a later batch of the same shape skips the sweep.
The cache file is ``$FKD_AUTOTUNE_CACHE`` or
``~/.cache/fkdtree_b200/autotune.json``.
"""
from __future__ import annotations

import json
import math
import os
import time
from typing import Callable, Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

SEARCH_LANES = (32, 16, 8, 4, 2, 1)
HIST_CTAS_PER_SM = (1, 2, 4, 8)
SUBTREE_SIZES = (1024, 512)
# size split of the digest search: events of at least big_n points get their
# own launch with big_lanes lanes per box ((0, 0): no split)
SPLITS = ((0, 0), (32768, 32), (65536, 32), (131072, 32), (65536, 16))


def cache_path() -> str:
    p = os.environ.get("FKD_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "fkdtree_b200", "autotune.json")


def _bucket(x: float) -> int:
    return int(math.floor(math.log2(x))) if x >= 1 else 0


def shape_key(device: str, dims: Sequence[int], pt_off: Sequence[int], q_off: Sequence[int]) -> str:
    """Cache key of a batch: device, dims present, log2 buckets of the event
    count, the median event size and the boxes per point."""
    dims = np.asarray(dims)
    sizes = np.diff(np.asarray(pt_off, dtype=np.int64))
    nq = int(np.asarray(q_off, dtype=np.int64)[-1])
    npts = int(sizes.sum())
    med = float(np.median(sizes)) if sizes.size else 0.0
    qpp = nq / npts if npts else 0.0
    return (f"{device}|dims={','.join(str(int(d)) for d in sorted(set(dims.tolist())))}"
            f"|ev=2^{_bucket(len(sizes))}|med=2^{_bucket(med)}|qpp=2^{_bucket(qpp * 16) - 4}")


def load_cache(path: Optional[str] = None) -> Dict[str, dict]:
    path = path or cache_path()
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(entries: Dict[str, dict], path: Optional[str] = None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(entries, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def sweep(candidates: Iterable, apply: Callable[[object], None], run: Callable[[], None],
          sync: Callable[[], None], reps: int = 2,
          clock: Callable[[], float] = time.perf_counter) -> Tuple[object, List[Tuple[object, float]]]:
    """Times run() under every candidate (after apply(candidate)); returns the
    fastest candidate and the (candidate, seconds) table."""
    table: List[Tuple[object, float]] = []
    for c in candidates:
        apply(c)
        run()  # warm-up (re-plans, re-captures, first-touch allocations)
        sync()
        best = float("inf")
        for _ in range(max(1, reps)):
            t0 = clock()
            run()
            sync()
            best = min(best, clock() - t0)
        table.append((c, best))
    winner = min(table, key=lambda cs: cs[1])[0] if table else None
    return winner, table


def _device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name()
    except Exception:  # pragma: no cover - torch without CUDA
        pass
    return "unknown"


def _sms() -> int:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_properties(0).multi_processor_count
    except Exception:  # pragma: no cover
        pass
    return 148


def tune_batch(batch, coords, ids, mins, maxs, *, device: Optional[str] = None, use_cache: bool = True,
               cache_file: Optional[str] = None, reps: int = 2, lanes: Sequence[int] = SEARCH_LANES,
               splits: Sequence[Tuple[int, int]] = SPLITS,
               hist_ctas: Optional[Sequence[int]] = None, subtree_sizes: Sequence[int] = SUBTREE_SIZES,
               sync: Optional[Callable[[], None]] = None,
               clock: Callable[[], float] = time.perf_counter) -> dict:
    """Chooses hist_ctas and subtree_size (build) and search_lanes (digest
    search) for `batch` (a fkdtree_b200.Batch) on its own inputs, applies them
    and returns {"hist_ctas", "subtree_size", "search_lanes", "search_big_n",
    "search_lanes_big", "cached", "key", "build_s", "subtree_s", "search_s",
    "split_s"}.
    Inputs may be host arrays or CUDA tensors (device tensors keep the copies
    out of the timing)."""
    if sync is None:
        def sync():
            try:
                import torch
                if torch.cuda.is_available():
                    torch.cuda.synchronize()
            except Exception:  # pragma: no cover
                pass
    device = device or _device_name()
    key = shape_key(device, batch.dims, batch.pt_off, batch.q_off)
    entries = load_cache(cache_file) if use_cache else {}
    hit = entries.get(key)
    if hit is not None and "hist_ctas" in hit and "search_lanes" in hit:
        batch.set_param("hist_ctas", int(hit["hist_ctas"]))
        batch.set_param("subtree_size", int(hit.get("subtree_size", 0)))
        batch.set_param("search_lanes", int(hit["search_lanes"]))
        batch.set_param("search_lanes_big", int(hit.get("search_lanes_big", 0)))
        batch.set_param("search_big_n", int(hit.get("search_big_n", 0)))
        return dict(hit, cached=True, key=key)
    if hist_ctas is None:
        hist_ctas = [k * _sms() for k in HIST_CTAS_PER_SM]
    hc, build_table = sweep(hist_ctas, lambda v: batch.set_param("hist_ctas", int(v)),
                            lambda: batch.build(coords, ids), sync, reps=reps, clock=clock)
    batch.set_param("hist_ctas", int(hc))
    ss, subtree_table = sweep(subtree_sizes, lambda v: batch.set_param("subtree_size", int(v)),
                              lambda: batch.build(coords, ids), sync, reps=reps, clock=clock)
    batch.set_param("subtree_size", int(ss))
    batch.build(coords, ids)
    ln, search_table = sweep(lanes, lambda v: batch.set_param("search_lanes", int(v)),
                             lambda: batch.search_digest(mins, maxs), sync, reps=reps, clock=clock)
    batch.set_param("search_lanes", int(ln))

    def apply_split(v):
        batch.set_param("search_lanes_big", int(v[1]))
        batch.set_param("search_big_n", int(v[0]))

    sp, split_table = sweep(splits, apply_split, lambda: batch.search_digest(mins, maxs), sync, reps=reps,
                            clock=clock)
    apply_split(sp)
    result = {"hist_ctas": int(hc), "subtree_size": int(ss), "search_lanes": int(ln), "search_big_n": int(sp[0]),
              "search_lanes_big": int(sp[1]),
              "build_s": {str(k): v for k, v in build_table},
              "subtree_s": {str(k): v for k, v in subtree_table},
              "search_s": {str(k): v for k, v in search_table},
              "split_s": {f"{k[0]}:{k[1]}": v for k, v in split_table}}
    if use_cache:
        entries = load_cache(cache_file)
        entries[key] = result
        save_cache(entries, cache_file)
    return dict(result, cached=False, key=key)
