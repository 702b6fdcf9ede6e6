"""Generates the golden fixtures under tests/golden/ from the REFERENCE itself.

The reference (te42kyfo/FKDTree) ships no golden vectors or known-answer tests,
so the fixtures are outputs of the unmodified reference CPU tree, compiled from
its own headers into oracle/_ref/libfkdref.so by oracle/Makefile:

  * the build tables theDimensions / theIds (FKDTree_cpu.h:221-277, :209-213);
  * per-box result lists of search_in_the_box (level order, FKDTree_cpu.h:123-169),
    search_in_the_box_BFS (:72-121), search_in_the_box_branchless (:25-70) and
    search_in_the_box_recursive (:171-207), in the order the reference emits them.
    The level-order / BFS / branchless variants are only recorded for boxes whose
    frontier fits FQueue's 1024 slots (FQueue.h:158, :232) -- elsewhere the
    reference asserts -- which the C restatement measures first.

Run from the repository root, where the reference checkout is present:

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fkdtree_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    rng = np.random.Generator(np.random.PCG64(1234))
    # tiny trees: every shape of the last level
    for n in [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100]:
        c = rng.random((3, n), dtype=np.float32)
        yield f"tiny3d_n{n}", c, rng.permutation(n).astype(np.uint32), 0.2
    # uniform 3D, several dims
    yield "uniform3d_n1000", rng.random((3, 1000), dtype=np.float32), np.arange(1000, dtype=np.uint32), 0.05
    yield "uniform1d_n777", rng.random((1, 777), dtype=np.float32), rng.permutation(777).astype(np.uint32), 0.01
    yield "uniform2d_n5000", rng.random((2, 5000), dtype=np.float32), np.arange(5000, dtype=np.uint32), 0.02
    # heavy ties: 4th coordinate on 16 discrete layers, ids shuffled
    c = rng.random((4, 3000), dtype=np.float32)
    c[3] = rng.integers(0, 16, 3000).astype(np.float32) / np.float32(16)
    yield "layers4d_n3000", c, rng.permutation(3000).astype(np.uint32), 0.05
    # every coordinate drawn from 8 values: ties on all dims, decided by id
    c = (rng.integers(0, 8, (2, 2000)).astype(np.float32) / np.float32(8))
    yield "grid2d_n2000", c, rng.permutation(2000).astype(np.uint32), 0.1
    # signed zeros and infinities
    c = rng.standard_normal((3, 600)).astype(np.float32)
    c[0, :50] = -0.0
    c[0, 50:100] = 0.0
    c[1, 100:110] = np.inf
    c[2, 110:120] = -np.inf
    yield "zeros_inf3d_n600", c, rng.permutation(600).astype(np.uint32), 0.3
    # negative and positive values, wide dynamic range
    c = (rng.standard_normal((3, 4099)) * np.exp(rng.uniform(-20, 20, (3, 4099)))).astype(np.float32)
    yield "wide3d_n4099", c, np.arange(4099, dtype=np.uint32), 1.0
    # clustered: boxes that fully contain dense clusters (frontier overflow regime)
    ev = W.clustered_event(n=20_000, n_queries=64, n_clusters=8, sigma=0.002, seed=7)
    yield "clustered3d_n20000", ev.coords, ev.ids, (ev.mins, ev.maxs)


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libfkdref.so is missing: run `make -C oracle` with the reference present")
    manifest = []
    for name, coords, ids, boxes in cases():
        dim, n = coords.shape
        ref = O.RefTree(coords, ids)
        ref.build()
        tab, tid = ref.tables()
        if isinstance(boxes, tuple):
            mins, maxs = boxes
        else:
            q = min(n, 200)
            hw = np.float32(boxes)
            mins = (coords[:, :q] - hw).astype(np.float32)
            maxs = (coords[:, :q] + hw).astype(np.float32)
        # which boxes the FQueue-bound variants can run (C restatement measures the frontier)
        _, _, _, front = O.search(tab, tid, mins, maxs, variant=O.LEVEL_ORDER, want_ids=False)
        _, _, _, front_bfs = O.search(tab, tid, mins, maxs, variant=O.BFS, want_ids=False)
        _, _, _, front_bl = O.search(tab, tid, mins, maxs, variant=O.BRANCHLESS, want_ids=False)
        ok = (front < O.FQUEUE_SLOTS) & (front_bfs < O.FQUEUE_SLOTS) & (front_bl < O.FQUEUE_SLOTS)
        rec = dict(coords=coords, ids=ids, tab=tab, tab_ids=tid, mins=mins, maxs=maxs, fqueue_ok=ok)
        rc, ro, ri, _ = ref.search(mins, maxs, variant=O.RECURSIVE)
        rec.update(rec_counts=rc, rec_offsets=ro, rec_ids=ri)
        if ok.all():
            for v, key in [(O.LEVEL_ORDER, "lvl"), (O.BFS, "bfs"), (O.BRANCHLESS, "bl")]:
                c_, o_, i_, _ = ref.search(mins, maxs, variant=v)
                rec.update({f"{key}_counts": c_, f"{key}_offsets": o_, f"{key}_ids": i_})
        else:
            sel = np.nonzero(ok)[0]
            for v, key in [(O.LEVEL_ORDER, "lvl"), (O.BFS, "bfs"), (O.BRANCHLESS, "bl")]:
                c_, o_, i_, _ = ref.search(mins[:, sel], maxs[:, sel], variant=v)
                rec.update({f"{key}_counts": c_, f"{key}_offsets": o_, f"{key}_ids": i_, f"{key}_sel": sel})
        ref.close()
        np.savez_compressed(OUT / f"{name}.npz", **rec)
        manifest.append(f"{name} dim={dim} n={n} q={mins.shape[1]} fqueue_ok={int(ok.sum())}/{ok.size}")
    # the small single-event workload: 100,000 uniform points, half-width 0.01, seed 0
    ev = W.uniform_event()
    ref = O.RefTree(ev.coords, ev.ids)
    ref.build()
    tab, tid = ref.tables()
    c_, o_, i_, _ = ref.search(ev.mins, ev.maxs, variant=O.LEVEL_ORDER)
    np.savez_compressed(OUT / "uniform3d_n100000_summary.npz", tab_sha=sha(tab), ids_sha=sha(tid), counts=c_,
                        lvl_ids_sha=sha(i_), total=np.uint64(c_.sum(dtype=np.uint64)))
    ref.close()
    manifest.append(f"uniform3d_n100000_summary total={int(c_.sum())}")
    (OUT / "MANIFEST.txt").write_text("\n".join(manifest) + "\n")
    print("\n".join(manifest))


if __name__ == "__main__":
    main()
