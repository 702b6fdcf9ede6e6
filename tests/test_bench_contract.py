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


def test_device_checksum_matches_digest_sum():
    """The on-device checksum of a search's output equals the sum over boxes of
    the per-box digests (torch CPU tensors stand in for the device buffer)."""
    import numpy as np
    import torch

    from oracle import oracle as O
    rng = np.random.default_rng(3)
    ids = rng.integers(0, 2**32, size=100_003, dtype=np.uint64).astype(np.uint32)
    offs = np.array([0, 10, 10, 5000, 100_003], dtype=np.uint64)
    want = int(np.sum(O.digest_lists(offs, ids), dtype=np.uint64))
    got = bench.device_checksum(torch.from_numpy(ids.view(np.int32)), chunk=4096)
    assert got == want


def _fake_gpu_output(ev, tab, tid):
    """The host dict reference_check reads, filled from the C restatement."""
    import numpy as np

    from oracle import oracle as O
    _, offs, ids, _ = O.search(tab, tid, ev.mins, ev.maxs, variant=O.RECURSIVE)
    return {"tab": tab, "tid": tid, "offsets": offs, "ids": ids}


def test_reference_check_flags():
    """reference_check's exactness flags on a small clustered event: true for the
    restatement's output, false once one result id is changed."""
    import numpy as np
    import pytest

    from fkdtree_b200 import workloads as W
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    ev = W.clustered_event(n=50_000, n_queries=2_000, n_clusters=32)
    tab, tid = O.build(ev.coords, ev.ids)
    host = _fake_gpu_output(ev, tab, tid)
    cpu, exact = bench.reference_check(ev, host, 64)
    assert cpu["kind"] == "reference" and cpu["value"] > 0 and cpu["search_s"] > 0
    assert exact["c2_tables_equal_reference"] and exact["c2_counts_equal_reference"]
    assert exact["c2_digests_equal_reference"] and exact["c2_sample_sets_equal_reference"]
    k = int(np.argmax(np.diff(host["offsets"]) > 0))
    host["ids"] = host["ids"].copy()
    host["ids"][int(host["offsets"][k])] ^= 1
    _, bad = bench.reference_check(ev, host, ev.q)
    assert bad["c2_tables_equal_reference"] and bad["c2_counts_equal_reference"]
    assert not bad["c2_digests_equal_reference"] and not bad["c2_sample_sets_equal_reference"]


def test_c1_reference_block():
    """The config-1 block's reference part runs on the CPU alone."""
    import pytest

    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    rep = bench.c1_report(None, cpu=True)
    assert rep["n_points"] == 100_000 and rep["n_boxes"] == 100_000
    r = rep["reference"]
    assert r["kind"] == "reference" and r["value"] > 0 and r["build_ms"] > 0
    assert "gpu" not in rep and "exact" not in rep


def test_clock_sampler_waits_for_first_sample(tmp_path, monkeypatch):
    """The sampler's process is running and has printed before the timed
    region starts; samples printed before it are not counted (a fake
    nvidia-smi on PATH stands in for the real one)."""
    import os
    import time
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\nwhile true; do echo '0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, "
                    "Not Active, Not Active'; sleep 0.05; done\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    with bench.ClockSampler(0) as s:
        assert s.lines, "no sample before the timed region"
        t0 = time.time()
        time.sleep(0.3)
    assert time.time() - t0 < 10
    r = s.summary()
    assert r["sm_mhz"] == 1965.0 and r["reasons"] == [] and r["samples"] >= 2
