"""Autotuner logic on the CPU: a fake batch whose phase times depend on the
knobs and a fake clock stand in for the GPU."""
import json

import numpy as np

from fkdtree_b200 import autotune as A


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeBatch:
    """Build time is minimal at hist_ctas=296, search time at lanes=4."""

    def __init__(self, clock, dims=(3,) * 8, sizes=(20_000,) * 8):
        self.clock = clock
        self.dims = np.array(dims, np.uint32)
        self.pt_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
        self.q_off = self.pt_off.copy()
        self.params = {"hist_ctas": 0, "subtree_size": 0, "search_lanes": 0, "search_lanes_big": 0, "search_big_n": 0}

    def set_param(self, name, value):
        self.params[name] = value

    def build(self, coords, ids):
        self.clock.t += 1.0 + abs(self.params["hist_ctas"] - 296) / 1000.0 - (0.1 if self.params["subtree_size"] == 512 else 0.0)

    def search_digest(self, mins, maxs):
        split_gain = 0.5 if (self.params["search_big_n"] == 65536 and self.params["search_lanes_big"] == 32) else 0.0
        self.clock.t += 2.0 + abs(self.params["search_lanes"] - 4) / 10.0 - split_gain


def test_sweep_picks_fastest_and_breaks_ties_by_order():
    clk = FakeClock()
    cost = {1: 3.0, 2: 1.0, 3: 1.0, 4: 2.0}
    state = {}
    best, table = A.sweep([1, 2, 3, 4], lambda v: state.update(v=v),
                          lambda: setattr(clk, "t", clk.t + cost[state["v"]]), lambda: None, reps=3, clock=clk)
    assert best == 2
    assert [c for c, _ in table] == [1, 2, 3, 4]
    assert dict(table) == cost


def test_tune_batch_sweeps_applies_and_caches(tmp_path):
    clk = FakeClock()
    b = FakeBatch(clk)
    cache = str(tmp_path / "tune.json")
    r = A.tune_batch(b, None, None, None, None, device="FakeGPU", cache_file=cache, reps=2,
                     hist_ctas=[148, 296, 592], sync=lambda: None, clock=clk)
    assert r["hist_ctas"] == 296 and r["subtree_size"] == 512 and r["search_lanes"] == 4 and not r["cached"]
    assert r["search_big_n"] == 65536 and r["search_lanes_big"] == 32
    assert b.params == {"hist_ctas": 296, "subtree_size": 512, "search_lanes": 4, "search_lanes_big": 32,
                        "search_big_n": 65536}
    data = json.load(open(cache))
    assert r["key"] in data and data[r["key"]]["search_lanes"] == 4
    # a second batch of the same shape takes the cached choice without timing anything
    clk2 = FakeClock()
    b2 = FakeBatch(clk2)
    r2 = A.tune_batch(b2, None, None, None, None, device="FakeGPU", cache_file=cache, sync=lambda: None, clock=clk2)
    assert r2["cached"] and clk2.t == 0.0
    assert b2.params == {"hist_ctas": 296, "subtree_size": 512, "search_lanes": 4, "search_lanes_big": 32,
                         "search_big_n": 65536}


def test_shape_key_buckets():
    k1 = A.shape_key("B200", [3, 3, 4], [0, 10_000, 30_000, 50_000], [0, 10_000, 30_000, 50_000])
    k2 = A.shape_key("B200", [4, 3, 3], [0, 11_000, 31_000, 52_000], [0, 11_000, 31_000, 52_000])
    k3 = A.shape_key("B200", [3, 3, 3], [0, 10_000, 30_000, 50_000], [0, 10_000, 30_000, 50_000])
    k4 = A.shape_key("H100", [3, 3, 4], [0, 10_000, 30_000, 50_000], [0, 10_000, 30_000, 50_000])
    assert k1 == k2 and k1 != k3 and k1 != k4


def test_unreadable_cache_is_empty(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("{not json")
    assert A.load_cache(str(p)) == {}
    A.save_cache({"k": {"hist_ctas": 1}}, str(p))
    assert A.load_cache(str(p)) == {"k": {"hist_ctas": 1}}
