#!/usr/bin/env python
"""FKDTree build + box search benchmark (B200).

One step = build the flat kd-tree over the workload's points and answer all
of its box queries (count pass, prefix sum, write pass) -- the reference's
FKDTree_CPU::build (FKDTree_cpu.h:221-277) followed by search_in_the_box over
every box (main.cpp:369-381).

Default workload (single GPU): 16,777,216 float32 points in 3D, 80% from 4,096
Gaussian clusters (sigma 0.002, Dirichlet(1) weights) + 20% uniform
background, 1,048,576 boxes centred on random points with half-widths
U[0.001, 0.02] per dim, seed 1 -- seeded synthetic data of the shapes and
distributions the reference's benchmark description gives.  The point set
(268 MB) and the result ids (~18 GB) are far larger than the 126 MB L2, so no
L2 flush is needed between steps.

Printed JSON line (rank 0):
  value     build+search throughput over the whole job, Mpoints/s (points of
            the tree built and queried per second; N GPUs run N replicas)
  e2e       the same through the public C ABI with pinned host buffers:
            host->device copy of points and boxes, build, table download,
            search, device->host copy of offsets and every result id
  roofline  achieved algorithmic GB/s of the dominant phase vs measured HBM peak
  cpu_baseline  the reference CPU tree (oracle/_ref) on this host's cores

`--impl reference` times the reference's own CPU implementation (the
unmodified FKDTree_CPU compiled from its headers into oracle/_ref) on the
same workload: serial build (the reference build is serial by design) plus
search_in_the_box_recursive over a sample of the boxes on all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "build Mpoints/s + box queries/s, learned/batched vs plain GPU, exact results"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the recording
# count pass + k_expand, from ncu --set full captures of the same search with
# 65,536 boxes (2.84e8 results): the count pass reads 274.5 MB (the tree and
# the boxes, 83% L2 hits) and writes 138.9 MB (record pools); k_expand reads
# 601.2 MB and writes 1,087.4 MB.  A full search is modelled as that fixed
# read plus the rest per result id:
#   ncu --set full --clock-control none -k regex:k_expand -s 4 -c 1 python bench.py --steps 1 --warmup 4 \
#       --queries 65536 --no-e2e --no-cpu --no-batched --no-nn --no-c1   (and the same for k_search<3,0,1>)
SEARCH_DRAM_FIXED = 274.5e6
SEARCH_DRAM_BYTES_PER_RESULT = (138.9e6 + 601.2e6 + 1087.4e6) / 283829259
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="clustered16m", choices=["clustered16m", "uniform100k"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-queries", type=int, default=8192, help="box sample of the CPU baseline")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched / learned events report")
    ap.add_argument("--no-nn", action="store_true", help="skip the radius / kNN search report")
    ap.add_argument("--no-c1", action="store_true", help="skip the 100k-point sub-report (profiling runs)")
    ap.add_argument("--queries", type=int, default=0,
                    help="box count of the 16M-point workload (0: 1,048,576; smaller cases are for profiling)")
    ap.add_argument("--batched-events", type=int, default=4096)
    ap.add_argument("--level-times", action="store_true",
                    help="print the device time of every kernel of one build (CUDA activity records) and exit")
    ap.add_argument("--set", action="append", default=[], metavar="NAME=VALUE",
                    help="a fkd_set_param knob of the bench tree (repeatable); every value gives the same results")
    return ap.parse_args()


def make_workload(name, queries=None):
    from fkdtree_b200 import workloads as W
    if name == "uniform100k":
        ev = W.uniform_event(n=100_000, half_width=0.01, seed=0)
        cfg = {"workload": "uniform3d_100k", "n_points": ev.n, "n_boxes": ev.q, "dim": 3,
               "points": "U[0,1)^3", "half_width": 0.01, "seed": 0}
    else:
        ev = W.clustered_event() if not queries else W.clustered_event(n_queries=queries)
        cfg = {"workload": "clustered3d_16m_boxes1m" if not queries else f"clustered3d_16m_boxes{queries}", "n_points": ev.n, "n_boxes": ev.q, "dim": 3,
               "points": "80% of 4096 Gaussian clusters (sigma 0.002, Dirichlet(1)) + 20% U[0,1)^3",
               "half_width": "U[0.001,0.02] per dim", "seed": 1}
    cfg["l2"] = "inputs larger than L2 (no flush)" if ev.n * 16 > 126e6 else "inputs smaller than L2"
    return ev, cfg


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def build_bytes(n, dim):
    """Algorithmic bytes of one build: every record read and written once per
    partition level plus the final table write, N*(4*dim+4)*(2*floor(log2 N)+1)."""
    L = int(math.floor(math.log2(n))) if n > 0 else 0
    return n * (4 * dim + 4) * (2 * L + 1)


def search_bytes(n, dim, q, results):
    """Tree read once, boxes + count + offset per box, result ids written."""
    return n * (4 * dim + 4) + q * (8 * dim + 8) + 4 * results


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.lines = []

    def __enter__(self):
        # the timed region starts only once nvidia-smi has attached and printed
        # its first sample: a sampler starting up during a short timed step
        # was seen to stall it (a 7.5 ms step measured 1.1 s and 16 s)
        import threading
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
            return self
        first = threading.Event()

        def read():
            for line in self.p.stdout:
                self.lines.append(line)
                first.set()
            first.set()

        self.reader = threading.Thread(target=read, daemon=True)
        self.reader.start()
        first.wait(timeout=10.0)
        self.skip = len(self.lines)  # samples taken before the timed region
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.reader.join(timeout=5)
            self.out = "".join(self.lines[self.skip:])

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in rows)
        mx = max(float(r[2]) for r in rows)
        reasons = set()
        for r in rows:
            for name, col in (("hw_slowdown", 5), ("hw_thermal_slowdown", 6), ("sw_thermal_slowdown", 7),
                              ("sw_power_cap", 8)):
                if r[col].strip().lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------- batched events

def _timed(fn, k):
    import torch
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(k):
        a = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - a)
    return best


def _cpu_events(wb, n_sample, gpu_counts=None, gpu_digests=None):
    """The reference CPU path on n_sample events spread over the batch, scaled
    to the whole batch by points: the unmodified FKDTree_CPU (oracle/_ref) with
    OpenMP over events, each a serial build and a serial
    search_in_the_box_recursive of its boxes -- or, without oracle/_ref, the C
    restatement the same way."""
    from fkdtree_b200 import shard as S
    from oracle import oracle as O
    threads = O.host_threads()
    ev = np.linspace(0, wb.n_events - 1, min(n_sample, wb.n_events)).astype(np.int64)
    sb = S.sub_batch(wb, ev)
    kind = "reference" if O.ref_available() else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        rc, rd, _ = O.ref_batch(sb, threads=threads)
    else:
        _, _, rc, rd = O.batch(sb, threads=threads)
    sec = time.perf_counter() - t0
    scaled = sec * wb.n_points / max(1, sb.n_points)
    what = "FKDTree_CPU build + search_in_the_box_recursive" if kind == "reference" else "restated build + search"
    out = {"kind": kind, "cores": threads, "value": wb.n_points / scaled / 1e6, "unit": "Mpoints/s",
           "ms_scaled": 1e3 * scaled, "events_run_fraction": len(ev) / wb.n_events,
           "points_run_fraction": sb.n_points / wb.n_points,
           "sample": (f"{what} of {len(ev)} of {wb.n_events} events ({sb.n_points} points, "
                      f"{sb.n_queries} boxes) with {threads} threads over events, measured, then scaled to the "
                      "whole batch by points")}
    if gpu_counts is not None:
        # the same events' boxes in the GPU run, re-indexed into the sample's order
        bi = S.box_index(wb, ev)
        out["sample_counts_digests_equal_" + kind] = bool(np.array_equal(gpu_counts[bi].view(np.uint32), rc)
                                                         and np.array_equal(gpu_digests[bi].view(np.uint64), rd))
    return out


def _events_run(wb, mlp, dev, steps, plain_single, cpu_sample=0):
    """Batched graph run (autotuned) with and without the learned split, the
    plain single-event path (optional), exactness checks between them."""
    import torch

    import fkdtree_b200 as F
    from fkdtree_b200 import _capi

    L = _capi.lib()
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    coords = torch.from_numpy(wb.coords).to(dev)
    ids = torch.from_numpy(wb.ids.view(np.int32)).to(dev)
    mins = torch.from_numpy(wb.mins).to(dev)
    maxs = torch.from_numpy(wb.maxs).to(dev)
    nq = wb.n_queries
    out = {"events": wb.n_events, "points": wb.n_points, "boxes": nq,
           "dims": sorted(set(int(d) for d in wb.dims))}
    pc = pd = None
    if plain_single:
        pc = torch.empty(nq, dtype=torch.int32, device=dev)
        pd = torch.empty(nq, dtype=torch.int64, device=dev)
        hd = {}
        sh = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

        def plain():
            for e in range(wb.n_events):
                d = int(wb.dims[e])
                if d not in hd:
                    hh = C.c_void_p()
                    _capi.check(L.fkd_create(d, _capi.FLAG_ASYNC, sh, C.byref(hh)))
                    hd[d] = hh
                hh = hd[d]
                n = int(wb.pt_off[e + 1] - wb.pt_off[e])
                q = int(wb.q_off[e + 1] - wb.q_off[e])
                c0, p0 = int(wb.coord_off[e]), int(wb.pt_off[e])
                qc0, q0 = int(wb.qcoord_off[e]), int(wb.q_off[e])
                _capi.check(L.fkd_build(hh, P(coords[c0:c0 + d * n]), P(ids[p0:p0 + n]), n, _capi.MEM_DEVICE))
                if q:
                    _capi.check(L.fkd_search_digest(hh, P(mins[qc0:qc0 + d * q]), P(maxs[qc0:qc0 + d * q]), q,
                                                    P(pc[q0:q0 + q]), P(pd[q0:q0 + q]), _capi.MEM_DEVICE))
            for hh in hd.values():
                _capi.check(L.fkd_sync(hh))

        plain_s = _timed(plain, 1)
        for hh in hd.values():
            _capi.check(L.fkd_destroy(hh))
        out["plain_single_event_ms"] = 1e3 * plain_s

    b = F.Batch.of(wb)
    tune = b.autotune(coords, ids, mins, maxs, use_cache=False, reps=1)
    bc = torch.empty(nq, dtype=torch.int32, device=dev)
    bd = torch.empty(nq, dtype=torch.int64, device=dev)
    batched_s = _timed(lambda: b.run(coords, ids, mins, maxs, bc, bd), steps)
    out["results"] = int(bc.to(torch.int64).sum().item())
    tab0 = torch.empty(wb.coords.size, dtype=torch.float32, device=dev)
    tid0 = torch.empty(wb.n_points, dtype=torch.int32, device=dev)
    _capi.check(L.fkd_batch_get_tables(b._h, P(tab0), P(tid0), _capi.MEM_DEVICE))
    out["batched_graph_ms"] = 1e3 * batched_s
    out["batched_build_ms"] = 1e3 * _timed(lambda: b.build(coords, ids), steps)
    out["batched_digest_ms"] = 1e3 * _timed(lambda: b.search_digest(mins, maxs), 1)
    launches0 = L.fkd_kernel_launches()
    b.build(coords, ids)
    b.search_digest(mins, maxs)
    out["kernels_per_batched_run"] = int(L.fkd_kernel_launches() - launches0)
    # where one batched build's device time goes, against its CUDA-event time:
    # the gap is what launching level by level costs
    kt = _kernel_times(lambda: b.build(coords, ids))
    out["batched_build_device_ms"] = {"per_kernel": kt, "sum": round(sum(v["ms"] for v in kt.values()), 3),
                                      "launches": sum(v["launches"] for v in kt.values())}
    b.learn_stats(reset=True)
    b.build(coords, ids)
    plain_passes = b.learn_stats(reset=True)["passes"]
    out["autotune"] = {"hist_ctas": tune["hist_ctas"], "subtree_size": tune["subtree_size"],
                       "search_lanes": tune["search_lanes"],
                       "search_big_n": tune["search_big_n"], "search_lanes_big": tune["search_lanes_big"],
                       "build_s": tune["build_s"], "subtree_s": tune["subtree_s"], "search_s": tune["search_s"],
                       "split_s": tune["split_s"]}
    delta = 0.1
    b.set_mlp(mlp, delta=delta)
    lc = torch.empty(nq, dtype=torch.int32, device=dev)
    ld = torch.empty(nq, dtype=torch.int64, device=dev)
    learned_s = _timed(lambda: b.run(coords, ids, mins, maxs, lc, ld), steps)
    st = b.learn_stats(reset=True)
    tab1 = torch.empty_like(tab0)
    tid1 = torch.empty_like(tid0)
    _capi.check(L.fkd_batch_get_tables(b._h, P(tab1), P(tid1), _capi.MEM_DEVICE))
    out["learned_graph_ms"] = 1e3 * learned_s
    out["learned_build_ms"] = 1e3 * _timed(lambda: b.build(coords, ids), steps)
    kt = _kernel_times(lambda: b.build(coords, ids))
    out["learned_build_device_ms"] = {"per_kernel": kt, "sum": round(sum(v["ms"] for v in kt.values()), 3)}
    b.learn_stats(reset=True)
    b.build(coords, ids)
    learned_passes = b.learn_stats(reset=True)["passes"]
    b.set_mlp(None)
    runs = steps + 1
    hit = st["verified"] / st["brackets"] if st["brackets"] else 0.0
    out["learned"] = {"delta": delta, "brackets_per_run": st["brackets"] // runs, "hit_rate": hit,
                      "fallback_rate": 1.0 - hit if st["brackets"] else 0.0,
                      "fallbacks_per_run": st["fallbacks"] // runs,
                      "digit_passes_per_build_plain": plain_passes,
                      "digit_passes_per_build_learned": learned_passes,
                      "digit_passes_saved_per_build": plain_passes - learned_passes,
                      "speedup_build": out["batched_build_ms"] / out["learned_build_ms"]}
    exact = {"learned_tables_equal_plain_batched": bool(torch.equal(tab0.view(torch.int32), tab1.view(torch.int32))
                                                        and torch.equal(tid0, tid1)),
             "learned_counts_digests_equal_plain_batched": bool(torch.equal(lc, bc) and torch.equal(ld, bd))}
    if plain_single:
        exact["batched_counts_digests_equal_single_event"] = bool(torch.equal(bc, pc) and torch.equal(bd, pd))
        out["speedup_batched_vs_plain_single_event"] = plain_s / batched_s
        out["speedup_learned_batched_vs_plain_single_event"] = plain_s / learned_s
    out["speedup_learned_vs_plain_batched"] = batched_s / learned_s
    if cpu_sample:
        out["cpu_baseline"] = _cpu_events(wb, cpu_sample, bc.cpu().numpy(), bd.cpu().numpy())
        k = [x for x in out["cpu_baseline"] if x.startswith("sample_counts_digests_equal_")][0]
        exact[k] = out["cpu_baseline"][k]
    out["exact"] = exact
    out["batched_mpoints_per_s"] = wb.n_points / batched_s / 1e6
    out["learned_mpoints_per_s"] = wb.n_points / learned_s / 1e6
    out["mboxes_per_s"] = nq / batched_s / 1e6
    del coords, ids, mins, maxs, bc, bd, lc, ld, tab0, tid0, tab1, tid1, pc, pd
    b.close()
    torch.cuda.empty_cache()
    return out


def sharded_events(rank, world, dev, n_events=4096, reps=3):
    """The events4096 batch split over the ranks (one GPU each) by points
    (shard.assign_events); every rank builds and digest-searches its own share
    as one batch graph (shard.run_share), no collective on the data path.  The
    job's time is the slowest rank's CUDA-event time (max over ranks);
    value = all ranks' points / that time."""
    import torch
    import torch.distributed as dist

    from fkdtree_b200 import shard as S
    from fkdtree_b200 import workloads as W
    wb = W.event_batch(n_events=n_events, seed=20)
    share = S.assign_events(np.diff(wb.pt_off.astype(np.int64)), world)[rank]
    counts, _, _, ms = S.run_share(wb, share, dev, reps=reps)
    pts = int(sum(int(wb.pt_off[e + 1] - wb.pt_off[e]) for e in share))
    t = torch.tensor([ms, float(pts), float(counts.to(torch.int64).sum().item())], device=dev, dtype=torch.float64)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    del counts
    torch.cuda.empty_cache()
    return {"workload": f"events{n_events}: seed 20, every point a box of half-width 0.01 on its own event",
            "ranks": world, "points": int(sm[1].item()), "results": int(sm[2].item()),
            "slowest_rank_ms": float(mx[0].item()), "value": float(sm[1].item()) / float(mx[0].item()) / 1e3,
            "unit": "Mpoints/s", "scaling": "strong (the batch is fixed; ranks split its events)",
            "assignment": "largest event first onto the rank with the fewest points (shard.assign_events)"}


def batched_report(dev, n_events=4096, steps=3, train_events=2000, cpu=True):
    """The batched workloads, each a set of independent events in one CUDA graph
    launch (fkd_batch_run), launch knobs from the autotuner:

      events4096  4,096 3D events, sizes LogNormal(ln 20000, 1.0) clipped to
                  [1,000, 200,000], 50-500 clusters each, every point a box of
                  half-width 0.01 on its own event (eval seed 20); against the
                  plain single-event GPU path (one fkd_build +
                  fkd_search_digest per event, every event)
      mixed1024   1,024 events, ~120M points, half 3D / half 4D (16 discrete
                  layers), every point a box of half-width 0.005 (seed 5)

    each with and without the learned split (MLP trained on the GPU on splits
    recorded from 2,000 training events of the events4096 generator, seed 10),
    and the oracle on the host cores on a sample of events."""
    import fkdtree_b200 as F
    from fkdtree_b200 import workloads as W

    t0 = time.perf_counter()
    tr = W.event_batch(n_events=train_events, seed=10, queries=False)
    btr = F.Batch.of(tr)
    import torch
    trc = torch.from_numpy(tr.coords).to(dev)
    tri = torch.from_numpy(tr.ids.view(np.int32)).to(dev)
    x, t = btr.record(trc, tri)
    record_s = time.perf_counter() - t0
    mlp = F.MLP(seed=1)
    t0 = time.perf_counter()
    losses = mlp.train(x, t, epochs=60, batch=256, lr=2e-3)
    train_s = time.perf_counter() - t0
    btr.close()
    # (the MLP is tiny: its training is launch- and latency-bound, not a roofline concern)
    del trc, tri
    # 40 -> 64 -> 64 -> 1: 2 * (40*64 + 64*64 + 64) FLOPs per node forward, about 3x that per
    # training sample (forward, input and weight gradients)
    fwd = 2 * (40 * 64 + 64 * 64 + 64)
    epochs = 60
    train_flops = 3 * fwd * int(x.shape[0]) * epochs
    try:
        with open(PEAKS_FILE) as f:
            bf16 = float(json.load(f)["bf16_tflops_sustained"])
    except Exception:
        bf16 = 1400.0
    rep = {"training": {"events": train_events, "seed": 10, "rows": int(x.shape[0]), "epochs": epochs,
                        "record_s": record_s, "train_s": train_s, "loss_first": float(losses[0]),
                        "loss_last": float(losses[-1]), "flops_per_node_forward": fwd,
                        "train_tflops": train_flops / train_s / 1e12,
                        "train_frac_of_bf16_sustained": train_flops / train_s / 1e12 / bf16,
                        "kernels": "fkd_mlp_train: k_mlp_grad (bf16 mma.sync, fp32 accumulate) + k_mlp_adam"}}
    t0 = time.perf_counter()
    wb = W.event_batch(n_events=n_events, seed=20)
    gen = time.perf_counter() - t0
    r = _events_run(wb, mlp, dev, steps, plain_single=True, cpu_sample=64 if cpu else 0)
    r["workload"] = ("events4096: 4,096 3D events, LogNormal(ln 20000, 1.0) sizes in [1000, 200000], 50-500 "
                     "clusters, every point a box of half-width 0.01 on its own event, seed 20")
    r["generate_s"] = gen
    rep["events4096"] = r
    del wb
    t0 = time.perf_counter()
    wm = W.mixed_events()
    gen = time.perf_counter() - t0
    r = _events_run(wm, mlp, dev, steps, plain_single=False, cpu_sample=16 if cpu else 0)
    r["workload"] = ("mixed1024: 1,024 events, ~120M points, LogNormal(ln 80000, 1.0) sizes in [5000, 2000000], "
                     "half 3D / half 4D (16 discrete layers), every point a box of half-width 0.005, seed 5")
    r["generate_s"] = gen
    rep["mixed1024"] = r
    return rep


# ------------------------------------------------------------------ our arm

def run_ours(args):
    import torch
    import torch.distributed as dist

    from fkdtree_b200 import _capi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    ev, cfg = make_workload(args.workload, args.queries)
    n, q, dim = ev.n, ev.q, ev.dim
    L = _capi.lib()
    stream = torch.cuda.current_stream(dev)
    h = C.c_void_p()
    _capi.check(L.fkd_create(dim, _capi.FLAG_ASYNC, C.c_void_p(stream.cuda_stream), C.byref(h)))
    # CUDA events around the library's kernels (read back after the timed region)
    _capi.check(L.fkd_set_param(h, b"kernel_events", 1))
    apply_knobs(L, h, args.set)
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    coords = torch.from_numpy(ev.coords).to(dev)
    ids = torch.from_numpy(ev.ids.view(np.int32)).to(dev)
    mins = torch.from_numpy(ev.mins).to(dev)
    maxs = torch.from_numpy(ev.maxs).to(dev)
    offsets = torch.empty(q + 1, dtype=torch.int64, device=dev)
    counts = torch.empty(q, dtype=torch.int32, device=dev)
    # size the result buffer once
    _capi.check(L.fkd_build(h, P(coords), P(ids), n, _capi.MEM_DEVICE))
    _capi.check(L.fkd_search_count(h, P(mins), P(maxs), q, P(counts), _capi.MEM_DEVICE))
    _capi.check(L.fkd_sync(h))
    results = int(counts.to(torch.int64).sum().item())
    out = torch.empty(max(results, 1), dtype=torch.int32, device=dev)
    total = C.c_uint64(0)

    ev_b0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_b1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_s1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]

    def step(i=None):
        if i is not None:
            ev_b0[i].record(stream)
        _capi.check(L.fkd_build(h, P(coords), P(ids), n, _capi.MEM_DEVICE))
        if i is not None:
            ev_b1[i].record(stream)
        _capi.check(L.fkd_search(h, P(mins), P(maxs), q, P(offsets), P(out), results, C.byref(total), 0,
                                 _capi.MEM_DEVICE))
        if i is not None:
            ev_s1[i].record(stream)

    for _ in range(args.warmup):
        step()
    _capi.check(L.fkd_sync(h))
    launches0 = L.fkd_kernel_launches()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i in range(args.steps):
            step(i)
        t1.record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = L.fkd_kernel_launches() - launches0
    _capi.check(L.fkd_sync(h))
    assert total.value == results
    kt = np.zeros((min(args.steps, 63), 5), dtype=np.float32)
    for b in range(kt.shape[0]):
        _capi.check(L.fkd_kernel_times(h, b, kt[b].ctypes.data_as(C.c_void_p)))
    kms = [float(x) for x in kt.mean(axis=0)]  # count, write, build, global levels, subtree
    ms = t0.elapsed_time(t1)
    build_ms = float(np.mean([ev_b0[i].elapsed_time(ev_b1[i]) for i in range(args.steps)]))
    search_ms = float(np.mean([ev_b1[i].elapsed_time(ev_s1[i]) for i in range(args.steps)]))
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_step = ms / args.steps
    value = world * n / (ms_step / 1e3) / 1e6

    peak, peak_kind = hbm_peak()
    bb = build_bytes(n, dim)
    sb = search_bytes(n, dim, q, results)
    phases = {
        "build": {"ms": build_ms, "algorithmic_bytes": bb, "gbs": bb / build_ms / 1e6,
                  "kernels": ["k_sel_init", "k_hist", "k_partition", "k_subtree"]},
        "search": {"ms": search_ms, "algorithmic_bytes": sb, "gbs": sb / search_ms / 1e6,
                   "kernels": ["k_box_keys", "k_box_scatter", "k_inorder", "k_search<count> (recording)", "k_scan_*",
                               "k_expand", "k_search<write> (boxes the record pool missed)"]},
    }
    # per kernel (CUDA events inside the library, same stream, every timed step)
    kern = {
        "write pass (k_expand)": {"ms": float(kms[1]),
                                  "algorithmic_bytes": n * (4 * dim + 4) + q * (8 * dim + 8) + 4 * results,
                                  "bytes_rule": "tree once + boxes + offsets + 4 B per result id"},
        "count pass (k_search<count>, recording)": {"ms": float(kms[0]),
                                                    "algorithmic_bytes": n * (4 * dim + 4) + q * (8 * dim + 4),
                                                    "bytes_rule": "tree once + boxes + one count per box"},
        "build (k_hist + k_partition + k_subtree)": {"ms": float(kms[2]), "algorithmic_bytes": bb,
                                                     "bytes_rule": "N*(4*dim+4)*(2*floor(log2 N)+1)"},
        "global levels (k_sel_init + k_hist + k_partition)": {"ms": float(kms[3])},
        "k_subtree": {"ms": float(kms[4])},
    }
    # the search is one operation in two launches (the count pass records, the
    # write pass copies); its algorithmic bytes are the search_bytes() rule
    kern["search (count pass + write pass)"] = {"ms": float(kms[0] + kms[1]), "algorithmic_bytes": sb,
                                                "bytes_rule": "tree once + boxes + count + offset per box "
                                                              "+ 4 B per result id"}
    for v in kern.values():
        if "algorithmic_bytes" in v and v["ms"] > 0:
            v["gbs"] = v["algorithmic_bytes"] / v["ms"] / 1e6
    dom = max(("search (count pass + write pass)", "build (k_hist + k_partition + k_subtree)"),
              key=lambda k: kern[k]["ms"])
    roof = {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["gbs"], "peak": peak, "unit": "GB/s",
            "frac": kern[dom]["gbs"] / peak, "peak_kind": f"{peak_kind} (copy bandwidth, MEASURED_PEAKS.json)",
            "traffic": (SEARCH_DRAM_FIXED + SEARCH_DRAM_BYTES_PER_RESULT * results
                        if dom.startswith("search") and args.workload == "clustered16m" else None),
            "traffic_note": ("ncu DRAM bytes of a 65,536-box capture: the count pass's tree read once plus "
                             "6.44 B per result id (record pools written and read, ids gathered and written)"),
            "algorithmic_bytes_per_launch": kern[dom]["algorithmic_bytes"],
            "launch_ms": kern[dom]["ms"],
            "build_frac": bb / kms[2] / 1e6 / peak if kms[2] > 0 else None}

    line = {"metric": METRIC, "value": value, "unit": "Mpoints/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, fkdtree_b200/workloads.py)",
            "config": dict(cfg, parallelism=f"replicas{world}", results_per_step=results,
                           **({"knobs": args.set} if args.set else {})),
            "build_mpoints_per_s": n / build_ms / 1e3, "search_mboxes_per_s": q / search_ms / 1e3,
            "phases": phases, "kernels": kern, "roofline": roof, "gpu_launches": int(launches)}
    line["clocks"] = clk.summary()

    host = None
    if not args.no_e2e:
        line["e2e"], host = run_e2e(args, L, h, ev, results, stream, world, barrier, dev)
    check = rank == 0 and world == 1 and not args.no_cpu
    if check:
        # the device-timed output itself: offsets and a checksum of all ids
        if host is None:
            host = {"offsets": offsets.cpu().numpy().view(np.uint64), "ids": out[:results].cpu().numpy().view(np.uint32)}
            tab = np.empty((dim, n), dtype=np.float32)
            tid = np.empty(n, dtype=np.uint32)
            _capi.check(L.fkd_get_tables(h, tab.ctypes.data_as(C.c_void_p), tid.ctypes.data_as(C.c_void_p),
                                         _capi.MEM_HOST))
            host["tab"], host["tid"] = tab, tid
        host["device_offsets_equal"] = bool(np.array_equal(offsets.cpu().numpy().view(np.uint64), host["offsets"]))
        host["device_checksum"] = device_checksum(out[:results])
    if rank == 0 and world == 1 and not args.no_nn:
        line["radius_knn"] = nn_report(L, h, ev, dev, stream, out)
    _capi.check(L.fkd_destroy(h))
    del coords, ids, mins, maxs, offsets, counts, out
    torch.cuda.empty_cache()
    if world > 1 and not args.no_batched:
        line["sharded_events"] = sharded_events(rank, world, dev, args.batched_events)
    if rank == 0 and world == 1 and not args.no_c1:
        line["c1"] = c1_report(dev, cpu=not args.no_cpu)
    if rank == 0 and world == 1 and not args.no_batched:
        line["batched"] = batched_report(dev, n_events=args.batched_events, cpu=not args.no_cpu)
    if check:
        line["cpu_baseline"], line["exact"] = reference_check(ev, host, args.cpu_queries)
        del host
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def nn_report(L, h, ev, dev, stream, out, reps=3, k=16):
    """Radius and kNN search on the built tree (fkd_nn.cu; no reference
    counterpart): every box's inscribed ball (centre, smallest half-width) and
    the k nearest points of every box centre, device buffers, CUDA events on
    the library's stream, best of `reps` after one warm-up call."""
    import torch

    from fkdtree_b200 import _capi
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    n, q, dim = ev.n, ev.q, ev.dim
    ctr = torch.from_numpy(((ev.mins + ev.maxs) * np.float32(0.5)).astype(np.float32)).to(dev)
    rad = torch.from_numpy(((ev.maxs - ev.mins) * np.float32(0.5)).min(axis=0).astype(np.float32)).to(dev)
    offs = torch.empty(q + 1, dtype=torch.int64, device=dev)
    kids = torch.empty((q, k), dtype=torch.int32, device=dev)
    kd2 = torch.empty((q, k), dtype=torch.float32, device=dev)
    total = C.c_uint64(0)

    cnt = torch.empty(q, dtype=torch.int32, device=dev)

    def radius(ordered=0):
        _capi.check(L.fkd_search_radius(h, P(ctr), P(rad), q, P(offs), P(out), out.numel(), C.byref(total),
                                        ordered, _capi.MEM_DEVICE))

    def radius_count():
        _capi.check(L.fkd_search_radius_count(h, P(ctr), P(rad), q, P(cnt), _capi.MEM_DEVICE))

    def knn():
        _capi.check(L.fkd_search_knn(h, P(ctr), q, k, P(kids), P(kd2), _capi.MEM_DEVICE))

    def best_ms(fn):
        fn()
        _capi.check(L.fkd_sync(h))
        best = float("inf")
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        _capi.check(L.fkd_sync(h))
        return best

    peak, _ = hbm_peak()
    c_ms = best_ms(radius_count)
    o_ms = best_ms(lambda: radius(1))
    r_ms = best_ms(radius)
    res = int(total.value)
    r_bytes = n * (4 * dim + 4) + q * (4 * dim + 4 + 8 + 4) + 4 * res
    k_ms = best_ms(knn)
    k_bytes = n * (4 * dim + 4) + q * (4 * dim) + q * k * 8
    return {
        "radius": {"queries": q, "results": res, "ms": r_ms, "count_pass_ms": c_ms, "ordered_ms": o_ms,
                   "mqueries_per_s": q / r_ms / 1e3,
                   "algorithmic_bytes": r_bytes, "gbs": r_bytes / r_ms / 1e6, "frac_of_hbm": r_bytes / r_ms / 1e6 / peak,
                   "bytes_rule": "tree once + centre, radius, count, offset per query + 4 B per result id",
                   "kernels": ["k_radius (count)", "k_scan_*", "k_radius (write)"],
                   "note": "ms: depth-first order (like the box search line's unordered write); ordered_ms adds "
                           "the sort to ascending heap index (k_order)"},
        "knn": {"queries": q, "k": k, "ms": k_ms, "mqueries_per_s": q / k_ms / 1e3,
                "algorithmic_bytes": k_bytes, "gbs": k_bytes / k_ms / 1e6, "frac_of_hbm": k_bytes / k_ms / 1e6 / peak,
                "bytes_rule": "tree once + centre per query + (id, d2) per neighbour", "kernels": ["k_knn"]},
        "workload": "the bench tree; centres = box centres, radius = smallest box half-width, k = 16",
    }


def run_e2e(args, L, h, ev, results, stream, world, barrier, dev):
    """The public C ABI with pinned host buffers: every step copies the points
    and boxes in and the tables, offsets and every result id out."""
    import torch

    from fkdtree_b200 import _capi
    n, q, dim = ev.n, ev.q, ev.dim
    pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
    coords_h, ids_h = pin(ev.coords), pin(ev.ids.view(np.int32))
    mins_h, maxs_h = pin(ev.mins), pin(ev.maxs)
    tab_h = torch.empty((dim, n), dtype=torch.float32, pin_memory=True)
    tid_h = torch.empty(n, dtype=torch.int32, pin_memory=True)
    offs_h = torch.empty(q + 1, dtype=torch.int64, pin_memory=True)
    out_h = torch.empty(max(results, 1), dtype=torch.int32, pin_memory=True)
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    total = C.c_uint64(0)

    def step():
        _capi.check(L.fkd_build(h, P(coords_h), P(ids_h), n, _capi.MEM_HOST))
        _capi.check(L.fkd_get_tables(h, P(tab_h), P(tid_h), _capi.MEM_HOST))
        _capi.check(L.fkd_search(h, P(mins_h), P(maxs_h), q, P(offs_h), P(out_h), results, C.byref(total), 0,
                                 _capi.MEM_HOST))

    k = max(1, min(args.steps, 3))
    step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k):
        step()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    barrier()
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([sec], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        sec = float(tt.item())
    assert total.value == results
    h2d = n * 4 * dim + n * 4 + 2 * q * 4 * dim
    d2h = n * 4 * dim + n * 4 + (q + 1) * 8 + 4 * results
    line = {"value": world * n / (sec / k) / 1e6, "unit": "Mpoints/s", "steps": k, "ms_per_step": 1e3 * sec / k,
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "path": "fkd_build + fkd_get_tables + fkd_search, FKD_MEM_HOST (pinned)"}
    host = {"tab": tab_h.numpy(), "tid": tid_h.numpy().view(np.uint32), "offsets": offs_h.numpy().view(np.uint64),
            "ids": out_h.numpy().view(np.uint32)[:results]}
    return line, host


# ------------------------------------------------------------ reference arm

def ref_step(oracle_mod, ev, threads):
    """One reference step, measured in full: FKDTree_CPU construction + build
    of all points (serial by design) and search_in_the_box_recursive of every
    box on all threads (main.cpp:201-212, :369-381).  Returns (tree,
    build_s, search_s, counts); the caller closes the tree."""
    r = oracle_mod.RefTree(ev.coords, ev.ids)
    tb = r.build()
    counts, _, _, ts = r.search(ev.mins, ev.maxs, variant=oracle_mod.RECURSIVE, want_ids=False, threads=threads)
    return r, tb, ts, counts


MIX_C = (0x9E3779B97F4A7C15, 0xBF58476D1CE4E5B9, 0x94D049BB133111EB)


def device_checksum(ids_dev, chunk=1 << 27):
    """Wrap-around sum over all ids of the digest finaliser (the per-box digest
    summed over boxes), computed on the GPU from the search's own output
    buffer: checks the device-timed result against the reference's digests
    without copying it to the host."""
    import torch

    def s64(v):
        return v - (1 << 64) if v >= (1 << 63) else v

    def lsr(z, k):
        return (z >> k) & ((1 << (64 - k)) - 1)

    tot = torch.zeros((), dtype=torch.int64, device=ids_dev.device)
    for a in range(0, ids_dev.numel(), chunk):
        z = ids_dev[a:a + chunk].to(torch.int64) & 0xFFFFFFFF
        z = z + s64(MIX_C[0])
        z = (z ^ lsr(z, 30)) * s64(MIX_C[1])
        z = (z ^ lsr(z, 27)) * s64(MIX_C[2])
        z = z ^ lsr(z, 31)
        tot += z.sum()
    return int(tot.item()) & ((1 << 64) - 1)


def reference_check(ev, host, nq_sample):
    """The unmodified reference (oracle/_ref) on the bench workload, in full:
    its build and recursive search are timed (the cpu_baseline) and its output
    is compared with the GPU's -- tables bit for bit, every box's count and
    digest against the written result ids (copied out through the C ABI), a
    checksum of the device-timed output buffer, and full sorted id sets on a
    sample of boxes."""
    from oracle import oracle as O
    if not O.ref_available():
        return ({"value": None, "unit": "Mpoints/s", "kind": "reference", "cores": 0,
                 "sample": "reference CPU build unavailable (oracle/_ref not built)"}, {"checked": False})
    threads = O.host_threads()
    r, tb, ts, counts = ref_step(O, ev, threads)
    out = {"value": ev.n / (tb + ts) / 1e6, "unit": "Mpoints/s", "kind": "reference", "cores": threads,
           "build_s": tb, "search_s": ts,
           "sample": (f"the whole workload, measured: FKDTree_CPU::build of all {ev.n} points (serial, as in the "
                      f"reference) + search_in_the_box_recursive of all {ev.q} boxes with {threads} OpenMP threads")}
    tab, tid = r.tables()
    exact = {"c2_tables_equal_reference": bool(np.array_equal(tab.view(np.uint32), host["tab"].view(np.uint32))
                                               and np.array_equal(tid, host["tid"]))}
    rc, rd, tsd = r.search_digest(ev.mins, ev.maxs, threads=threads)
    gcounts = np.diff(host["offsets"]).astype(np.uint32)
    gd = O.digest_lists(host["offsets"], host["ids"], threads=threads)
    exact["c2_counts_equal_reference"] = bool(np.array_equal(gcounts, counts) and np.array_equal(rc, counts))
    exact["c2_digests_equal_reference"] = bool(np.array_equal(gd, rd))
    if "device_checksum" in host:
        want = int(np.sum(rd, dtype=np.uint64))
        exact["c2_device_output_checksum_equal_reference"] = bool(host["device_checksum"] == want
                                                                  and host["device_offsets_equal"])
    sel = np.linspace(0, ev.q - 1, min(nq_sample, ev.q)).astype(np.int64)
    sc, so, sids, _ = r.search(ev.mins[:, sel], ev.maxs[:, sel], variant=O.RECURSIVE, want_ids=True,
                               threads=threads)
    ok = True
    go = host["offsets"]
    for k, j in enumerate(sel):
        a = np.sort(host["ids"][int(go[j]):int(go[j + 1])])
        b = np.sort(sids[int(so[k]):int(so[k + 1])])
        if not np.array_equal(a, b):
            ok = False
            break
    exact["c2_sample_sets_equal_reference"] = ok
    exact["what"] = (f"{ev.n} points, {ev.q} boxes, {int(counts.sum(dtype=np.uint64))} result ids; sets on "
                     f"{len(sel)} sampled boxes; reference digest pass {tsd:.2f} s")
    r.close()
    if ev.dim == 3:
        # the reference's other CPU tree, an extra column (main.cpp:558-612)
        vc, vb, vs = O.ref_cmssw(ev.coords, ev.mins[:, sel], ev.maxs[:, sel])
        vs_all = vs * ev.q / len(sel)
        out["cmssw_vanilla"] = {
            "value": ev.n / (vb + vs_all) / 1e6, "unit": "Mpoints/s", "kind": "reference", "cores": 1,
            "build_s": vb, "search_s": vs_all,
            "counts_equal_fkdtree": float(np.mean(vc == counts[sel])),
            "sample": (f"KDTreeLinkerAlgo<unsigned, 3> (KDTreeLinkerAlgoT.h) build of all {ev.n} points + serial "
                       f"search of {len(sel)} of {ev.q} boxes, as main.cpp runs it; search time scaled to all "
                       "boxes")}
    return out, exact


def single_box_latency(L, h, ev, boxes=2000, threads=8):
    """The per-box path (search_in_the_box on one box, as main.cpp:351-359
    calls it): fkd_search with one box and host buffers, timed by the wall
    clock over `boxes` calls from one thread, then from `threads` host threads
    sharing the tree (ctypes releases the GIL inside each call).  Python's
    call overhead (a few microseconds) is included."""
    import threading

    from fkdtree_b200 import _capi

    def run(idx):
        buf = np.empty(1 << 16, dtype=np.uint32)
        offs = np.zeros(2, dtype=np.uint64)
        tot = C.c_uint64(0)
        lo = np.ascontiguousarray(ev.mins[:, idx].T)
        hi = np.ascontiguousarray(ev.maxs[:, idx].T)
        for k in range(len(idx)):
            _capi.check(L.fkd_search(h, lo[k].ctypes.data_as(C.c_void_p), hi[k].ctypes.data_as(C.c_void_p), 1,
                                     offs.ctypes.data_as(C.c_void_p), buf.ctypes.data_as(C.c_void_p), buf.size,
                                     C.byref(tot), 1, _capi.MEM_HOST))

    run(np.arange(50))
    t0 = time.perf_counter()
    run(np.arange(boxes))
    one = time.perf_counter() - t0
    parts = [np.arange(t, threads * boxes, threads) % ev.q for t in range(threads)]
    th = [threading.Thread(target=run, args=(p,)) for p in parts]
    t0 = time.perf_counter()
    for x in th:
        x.start()
    for x in th:
        x.join()
    many = time.perf_counter() - t0
    return {"us_per_box_one_thread": 1e6 * one / boxes, "boxes_per_s_one_thread": boxes / one,
            "threads": threads, "boxes_per_s_threads": threads * boxes / many,
            "what": "fkd_search(q=1, host buffers, ordered) per box through ctypes; wall clock"}


def c1_report(dev=None, cpu=True, reps=5):
    """The small single-event case: 100,000 U[0,1)^3 points (seed 0), one box of
    half-width 0.01 per point -- the reference's own CPU path (FKDTree_CPU
    build, level-order search_in_the_box and search_in_the_box_recursive of
    every box on all host threads, main.cpp:201-212, :369-381) and, with a
    device, the GPU (build + ordered search = the reference's level-order
    lists, device buffers, CUDA events), with exactness flags."""
    from fkdtree_b200 import workloads as W
    ev = W.uniform_event(n=100_000, half_width=0.01, seed=0)
    rep = {"workload": "uniform3d_100k: 100,000 U[0,1)^3 points, seed 0, one box of half-width 0.01 per point",
           "n_points": ev.n, "n_boxes": ev.q}
    gpu = None
    if dev is not None:
        import torch

        from fkdtree_b200 import _capi
        L = _capi.lib()
        P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        stream = torch.cuda.current_stream(dev)
        h = C.c_void_p()
        _capi.check(L.fkd_create(3, _capi.FLAG_ASYNC, C.c_void_p(stream.cuda_stream), C.byref(h)))
        coords = torch.from_numpy(ev.coords).to(dev)
        ids = torch.from_numpy(ev.ids.view(np.int32)).to(dev)
        mins = torch.from_numpy(ev.mins).to(dev)
        maxs = torch.from_numpy(ev.maxs).to(dev)
        cnt = torch.empty(ev.q, dtype=torch.int32, device=dev)
        _capi.check(L.fkd_build(h, P(coords), P(ids), ev.n, _capi.MEM_DEVICE))
        _capi.check(L.fkd_search_count(h, P(mins), P(maxs), ev.q, P(cnt), _capi.MEM_DEVICE))
        _capi.check(L.fkd_sync(h))
        res = int(cnt.to(torch.int64).sum().item())
        offs = torch.empty(ev.q + 1, dtype=torch.int64, device=dev)
        out = torch.empty(max(res, 1), dtype=torch.int32, device=dev)
        total = C.c_uint64(0)
        times = {"build": [], "search_ordered": [], "search": []}
        for it in range(reps + 2):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(stream)
            _capi.check(L.fkd_build(h, P(coords), P(ids), ev.n, _capi.MEM_DEVICE))
            e[1].record(stream)
            _capi.check(L.fkd_search(h, P(mins), P(maxs), ev.q, P(offs), P(out), res, C.byref(total), 0,
                                     _capi.MEM_DEVICE))
            e[2].record(stream)
            _capi.check(L.fkd_search(h, P(mins), P(maxs), ev.q, P(offs), P(out), res, C.byref(total), 1,
                                     _capi.MEM_DEVICE))
            e[3].record(stream)
            torch.cuda.synchronize()
            if it >= 2:
                times["build"].append(e[0].elapsed_time(e[1]))
                times["search"].append(e[1].elapsed_time(e[2]))
                times["search_ordered"].append(e[2].elapsed_time(e[3]))
        _capi.check(L.fkd_sync(h))
        tab = np.empty((3, ev.n), dtype=np.float32)
        tid = np.empty(ev.n, dtype=np.uint32)
        _capi.check(L.fkd_get_tables(h, tab.ctypes.data_as(C.c_void_p), tid.ctypes.data_as(C.c_void_p),
                                     _capi.MEM_HOST))
        gpu = {"tab": tab, "tid": tid, "offsets": offs.cpu().numpy().view(np.uint64),
               "ids": out[:res].cpu().numpy().view(np.uint32)}
        single = single_box_latency(L, h, ev)
        _capi.check(L.fkd_destroy(h))
        ms = {k: float(np.median(v)) for k, v in times.items()}
        rep["gpu"] = {"build_ms": ms["build"], "search_ms": ms["search"], "search_ordered_ms": ms["search_ordered"],
                      "value": ev.n / (ms["build"] + ms["search_ordered"]) / 1e3, "unit": "Mpoints/s",
                      "mboxes_per_s": ev.q / ms["search_ordered"] / 1e3, "results": res,
                      "timing": f"median of {reps} after 2 warm-up, CUDA events, device buffers; value = points / "
                                "(build + ordered search)",
                      "single_box": single}
    if cpu:
        from oracle import oracle as O
        if O.ref_available():
            threads = O.host_threads()
            r = O.RefTree(ev.coords, ev.ids)
            tb = r.build()
            lc, lo, lids, tl = r.search(ev.mins, ev.maxs, variant=O.LEVEL_ORDER, want_ids=True, threads=threads)
            rc, ro, rids, tr = r.search(ev.mins, ev.maxs, variant=O.RECURSIVE, want_ids=True, threads=threads)
            rtab, rtid = r.tables()
            r.close()
            rep["reference"] = {"build_ms": 1e3 * tb, "search_level_order_ms": 1e3 * tl,
                                "search_recursive_ms": 1e3 * tr, "cores": threads, "kind": "reference",
                                "value": ev.n / (tb + tl) / 1e6, "unit": "Mpoints/s",
                                "what": "FKDTree_CPU build (serial) + search_in_the_box (level order) of every box "
                                        f"on {threads} OpenMP threads; value = points / (build + level-order search)"}
            if gpu is not None:
                rep["exact"] = {
                    "tables_equal_reference": bool(np.array_equal(rtab.view(np.uint32), gpu["tab"].view(np.uint32))
                                                   and np.array_equal(rtid, gpu["tid"])),
                    "ordered_lists_equal_reference_level_order": bool(np.array_equal(lo, gpu["offsets"])
                                                                      and np.array_equal(lids, gpu["ids"])),
                    "sets_equal_reference_recursive": bool(
                        np.array_equal(ro, gpu["offsets"])
                        and np.array_equal(O.digest_lists(ro, rids), O.digest_lists(gpu["offsets"], gpu["ids"]))),
                }
                rep["speedup_gpu_vs_reference"] = rep["gpu"]["value"] / rep["reference"]["value"]
    return rep


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfkdref.so not built"}), flush=True)
        return
    ev, cfg = make_workload(args.workload, args.queries)
    threads = O.host_threads()
    # warm-up steps on a 1/16 sample of the points and boxes keep the run bounded
    from fkdtree_b200 import workloads as W
    m = max(1, ev.q // 16)
    sub = W.Event(ev.dim, np.ascontiguousarray(ev.coords[:, : ev.n // 16]), ev.ids[: ev.n // 16].copy(),
                  np.ascontiguousarray(ev.mins[:, :m]), np.ascontiguousarray(ev.maxs[:, :m]))
    for _ in range(args.warmup):
        r, _, _, _ = ref_step(O, sub, threads)
        r.close()
    tot_b = tot_s = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r, tb, ts, _ = ref_step(O, ev, threads)
        r.close()
        tot_b += tb
        tot_s += ts
    wall = time.perf_counter() - t0
    ms_step = 1e3 * (tot_b + tot_s) / args.steps
    value = ev.n / (ms_step / 1e3) / 1e6
    line = {"metric": METRIC, "value": value, "unit": "Mpoints/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, fkdtree_b200/workloads.py)",
            "config": dict(cfg, parallelism="cpu"), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Mpoints/s", "kind": "reference", "cores": threads,
                             "sample": (f"per step, the whole workload, measured: FKDTree_CPU::build of all {ev.n} "
                                        f"points (serial) + search_in_the_box_recursive of all {ev.q} boxes with "
                                        f"{threads} OpenMP threads; warm-up steps on 1/16 of the points and boxes"),
                             "build_s_per_step": tot_b / args.steps, "search_s_per_step": tot_s / args.steps,
                             "wall_s": wall},
            "e2e": {"value": value, "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "clustered16m":
        line["c1"] = c1_report(None, cpu=True)
    print(json.dumps(line), flush=True)


def apply_knobs(L, h, items):
    from fkdtree_b200 import _capi
    for it in items:
        name, _, val = it.partition("=")
        _capi.check(L.fkd_set_param(h, name.encode(), int(val)))


def _kernel_times(fn):
    """Device time of every kernel (and memset / copy) one call of fn
    launches, summed per name in ms (CUDA activity records through
    torch.profiler; outside every timed region)."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    tot, n = {}, {}
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA:
            k = e.name.split("(")[0].replace("void ", "").split("<")[0].replace("fkd::", "").strip() or "other"
            us = e.device_time_total if hasattr(e, "device_time_total") else e.cuda_time_total
            tot[k] = tot.get(k, 0.0) + float(us)
            n[k] = n.get(k, 0) + 1
    return {k: {"ms": round(v / 1e3, 3), "launches": n[k]} for k, v in sorted(tot.items(), key=lambda kv: -kv[1])}


def level_times(args):
    """Device time of every kernel launch of one build of the workload, in
    launch order (CUDA activity records through torch.profiler)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    from fkdtree_b200 import _capi
    ev, cfg = make_workload(args.workload, args.queries or 1)
    dev = torch.device("cuda", 0)
    L = _capi.lib()
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    coords = torch.from_numpy(ev.coords).to(dev)
    ids = torch.from_numpy(ev.ids.view(np.int32)).to(dev)
    h = C.c_void_p()
    _capi.check(L.fkd_create(ev.dim, 0, None, C.byref(h)))
    apply_knobs(L, h, args.set)
    for _ in range(3):
        _capi.check(L.fkd_build(h, P(coords), P(ids), ev.n, _capi.MEM_DEVICE))
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        _capi.check(L.fkd_build(h, P(coords), P(ids), ev.n, _capi.MEM_DEVICE))
        torch.cuda.synchronize()
    seq = []
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA:
            us = e.device_time_total if hasattr(e, "device_time_total") else e.cuda_time_total
            seq.append([e.name.split("(")[0].replace("void ", ""), round(float(us), 1)])
    _capi.check(L.fkd_destroy(h))
    print(json.dumps({"workload": cfg["workload"], "build_kernels_us": seq,
                      "total_us": round(sum(t for _, t in seq), 1)}), flush=True)


def main():
    args = parse_args()
    if args.level_times:
        level_times(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
