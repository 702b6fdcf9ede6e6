"""The stack bounds the radius and kNN kernels (fkd_nn.cu) rely on, checked
by replaying their walks on the CPU over trees the oracle builds.  CPU only.

* k_radius: a warp pops up to 32 entries from the top of its shared-memory
  stack per round (lane k takes the k-th of them from below) and pushes the
  children back in lane order; the stack never holds more than
  1 + sum_{d=1..H} min(64, 2^d) entries.
* k_knn: one thread walks near children first and stacks the far ones; the
  stack never holds more than H + 1 <= 32 entries.
"""
import math

import numpy as np
import pytest

from fkdtree_b200 import workloads as W
from oracle import nn_ref as NN
from oracle import oracle as O


def radius_stack_words(H):
    return 1 + sum(min(64, 2 ** d) for d in range(1, H + 1))


def _split(tab, i, c):
    """(split value, diff) of node i for centre c: float32 as the kernel."""
    dim = tab.shape[0]
    a = int(math.floor(math.log2(i + 1))) % dim
    s = tab[a, i]
    return s, np.float32(c[a] - s)


def replay_radius(tab, c, r):
    """Replays k_radius for one query: returns (hits, max stack size)."""
    n = tab.shape[1]
    r2 = np.float32(np.float32(r) * np.float32(r))
    stk = [0]
    hits, peak = 0, 1
    while stk:
        cnt = min(len(stk), 32)
        b0 = len(stk) - cnt
        popped = stk[b0:]
        del stk[b0:]
        pushes = []
        hits += int(np.count_nonzero(NN.dist2(tab[:, popped], c) <= r2))
        for i in popped:  # lane order: the k-th popped entry from below
            _, diff = _split(tab, i, c)
            pd = np.float32(diff * diff)
            l = 2 * i + 1
            if l < n and not (diff > 0 and pd > r2):
                pushes.append(l)
            if l + 1 < n and not (diff < 0 and pd > r2):
                pushes.append(l + 1)
        stk.extend(pushes)
        peak = max(peak, len(stk))
    return hits, peak


def replay_knn(tab, c):
    """Replays k_knn's walk with an unbounded k (every subtree is visited):
    returns the largest number of pending far children."""
    n = tab.shape[1]
    stack, peak = [], 0
    i = 0
    while True:
        while True:
            _, diff = _split(tab, i, c)
            l = 2 * i + 1
            near, far = (l, l + 1) if not diff > 0 else (l + 1, l)
            if near < n:
                if far < n:
                    stack.append(far)
                    peak = max(peak, len(stack))
                i = near
            elif far < n:
                i = far
            else:
                break
        if not stack:
            return peak
        i = stack.pop()


@pytest.mark.parametrize("n,dim", [(1, 3), (2, 2), (1000, 3), (4097, 4), (30000, 3), (65535, 2)])
def test_radius_stack_stays_within_bound(n, dim):
    rng = np.random.default_rng(n + dim)
    coords = rng.random((dim, n), dtype=np.float32)
    coords[0] = np.round(coords[0] * 32) / 32  # ties on the first coordinate
    tab, tid = O.build(coords, np.arange(n, dtype=np.uint32))
    H = int(math.floor(math.log2(n)))
    cap = radius_stack_words(H)
    centres = [coords[:, 0], np.full(dim, 0.5, np.float32), np.full(dim, -1.0, np.float32)]
    radii = [0.05, 0.3, 10.0]  # small, wide, the whole tree
    for c in centres:
        for r in radii:
            hits, peak = replay_radius(tab, np.asarray(c, np.float32), r)
            assert peak <= cap, (n, dim, r, peak, cap)
            want = int(np.count_nonzero(NN.dist2(tab, c) <= np.float32(np.float32(r) * np.float32(r))))
            assert hits == want


def test_radius_bound_is_tight_enough_for_the_kernel():
    # the largest tree (H = 30) keeps four warps' stacks well inside 48 KB of shared memory
    assert radius_stack_words(30) * 4 * 4 <= 48 * 1024
    assert radius_stack_words(24) == 1279


@pytest.mark.parametrize("n,dim", [(3, 1), (1000, 3), (4097, 4), (65536, 3)])
def test_knn_stack_stays_within_depth(n, dim):
    ev = W.uniform_event(n=n, dim=dim, seed=n)
    tab, _ = O.build(ev.coords, ev.ids)
    H = int(math.floor(math.log2(n)))
    for j in range(0, n, max(1, n // 7)):
        assert replay_knn(tab, ev.coords[:, j]) <= H + 1 <= 32
