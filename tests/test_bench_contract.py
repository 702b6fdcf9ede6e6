"""bench.py's host-side pieces that need no GPU: the algorithmic byte rules
behind `roofline`, the peak lookup and the clock sampler's summary (the
throttle reasons that reject a run).  CPU only."""
import json

import bench


def test_algorithmic_byte_rules():
    n, dim = 16_777_216, 3
    # N * (4*dim + 4) * (2*floor(log2 N) + 1): 16M points in 3D -> 13.15 GB
    assert bench.build_bytes(n, dim) == n * 16 * 49
    assert abs(bench.build_bytes(n, dim) / 1e9 - 13.15) < 0.01
    assert bench.build_bytes(0, 3) == 0
    q, results = 1_048_576, 4_544_080_537
    assert bench.search_bytes(n, dim, q, results) == n * 16 + q * 32 + 4 * results


def test_peak_lookup(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "PEAKS_FILE", str(tmp_path / "none.json"))
    assert bench.hbm_peak() == (bench.FALLBACK_HBM_GBS, "fallback")
    p = tmp_path / "peaks.json"
    p.write_text(json.dumps({"hbm_gbs": 6547.2, "bf16_tflops": 1675.0}))
    monkeypatch.setattr(bench, "PEAKS_FILE", str(p))
    assert bench.hbm_peak() == (6547.2, "measured")


def test_clock_summary_reasons():
    s = bench.ClockSampler(0)
    s.out = "\n".join([
        "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1965, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1950, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active",
    ])
    r = s.summary()
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"] and r["samples"] == 3
    s.out = "0, 1200, 1965, 900.0, 0x8, Active, Not Active, Not Active, Not Active"
    assert s.summary()["reasons"] == ["hw_slowdown"]
    s.out = ""
    assert s.summary()["reasons"] == ["unsampled"]
