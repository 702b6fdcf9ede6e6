"""The synthetic workloads are what the benchmark says they are: shapes,
dtypes, seeds, size distributions, box half-widths, the 4-D layer
coordinate and the batch layout.  CPU only."""
import numpy as np
import pytest

from fkdtree_b200 import workloads as W


def test_uniform_event():
    ev = W.uniform_event(n=5000, dim=3, half_width=0.01, seed=0)
    assert ev.coords.shape == (3, 5000) and ev.coords.dtype == np.float32
    assert np.array_equal(ev.ids, np.arange(5000, dtype=np.uint32))
    assert ev.coords.min() >= 0.0 and ev.coords.max() < 1.0
    # one box per point, lo = p - hw and hi = p + hw in float32
    assert np.array_equal(ev.mins, (ev.coords - np.float32(0.01)).astype(np.float32))
    assert np.array_equal(ev.maxs, (ev.coords + np.float32(0.01)).astype(np.float32))
    again = W.uniform_event(n=5000, dim=3, half_width=0.01, seed=0)
    assert np.array_equal(ev.coords, again.coords)


def test_clustered_event_boxes_and_determinism():
    ev = W.clustered_event(n=40_000, n_queries=3000, n_clusters=64, seed=1)
    assert ev.coords.shape == (3, 40_000) and ev.mins.shape == (3, 3000)
    hw = (ev.maxs - ev.mins) * np.float32(0.5)
    assert hw.min() >= 0.001 * 0.999 and hw.max() <= 0.02 * 1.001
    # boxes are centred on points of the cloud
    ctr = (ev.mins + ev.maxs) * np.float32(0.5)
    pts = {tuple(p) for p in np.round(ev.coords.T.astype(np.float64), 5)}
    hits = sum(tuple(c) in pts for c in np.round(ctr.T.astype(np.float64), 5)[:200])
    assert hits >= 190
    # most points sit in clusters: the densest 5% of a 64^3 grid holds well over half
    cells = np.floor(ev.coords.T * 64).astype(np.int64)
    _, counts = np.unique(cells[:, 0] * 4096 + cells[:, 1] * 64 + cells[:, 2], return_counts=True)
    top = np.sort(counts)[::-1]
    assert top[: max(1, len(top) // 20)].sum() > 0.5 * ev.n
    assert np.array_equal(ev.coords, W.clustered_event(n=40_000, n_queries=3000, n_clusters=64, seed=1).coords)


def test_event_batch_layout():
    b = W.event_batch(n_events=40, median=2000, size_lo=500, size_hi=8000, clusters_lo=5, clusters_hi=20,
                      seed=3, frac_4d=0.25)
    sizes = np.diff(b.pt_off.astype(np.int64))
    assert b.n_events == 40 and sizes.min() >= 500 and sizes.max() <= 8000
    assert int((b.dims == 4).sum()) == 10 and np.all(b.dims[:10] == 4) and np.all(b.dims[10:] == 3)
    assert np.array_equal(np.diff(b.coord_off.astype(np.int64)), sizes * b.dims.astype(np.int64))
    assert b.coords.size == int(b.coord_off[-1]) and b.ids.size == int(b.pt_off[-1])
    for e in (0, 9, 10, 39):
        ev = b.event(e)
        assert ev.coords.shape == (int(b.dims[e]), int(sizes[e]))
        assert np.array_equal(ev.ids, np.arange(sizes[e], dtype=np.uint32))
        if b.dims[e] == 4:  # the fourth coordinate: one of 16 layers, layer / 16
            layers = np.unique(ev.coords[3])
            assert layers.size <= 16 and np.all(np.isin(layers, np.arange(16, dtype=np.float32) / 16))
        # every point is a box of the batch's half-width on its own event
        assert np.array_equal(ev.mins, (ev.coords - np.float32(0.01)).astype(np.float32))


@pytest.mark.parametrize("total", [400_000])
def test_mixed_events_shape(total):
    b = W.mixed_events(seed=5, total=total, queries=False)
    assert b.n_events == 1024
    assert int((b.dims == 4).sum()) == 512
    assert abs(b.n_points - total) < 0.2 * total or b.n_points >= 1024 * 5000  # the size floor dominates
    assert b.n_queries == 0
