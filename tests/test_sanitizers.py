"""The CPU checkers under AddressSanitizer and UndefinedBehaviorSanitizer:
the C restatement (oracle/fkd_oracle.c) and the reference harness
(oracle/ref_harness.cpp over the unmodified reference headers), built by
`make -C oracle sanitize`, run builds and every search variant in a child
Python process with the ASan runtime preloaded.  CPU only."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SAN_ORACLE = ROOT / "oracle" / "_build" / "libfkdoracle_san.so"
SAN_REF = ROOT / "oracle" / "_ref" / "libfkdref_san.so"

CHILD = r"""
import numpy as np
from oracle import oracle as O
from fkdtree_b200 import workloads as W
rng = np.random.default_rng(5)
for dim in (1, 2, 3, 4):
    for n in (1, 2, 3, 7, 64, 1023, 1024, 1025, 5000):
        c = rng.random((dim, n), dtype=np.float32)
        c[0] = np.round(c[0] * 16) / 16                      # ties
        ids = rng.permutation(n).astype(np.uint32)
        tab, tid = O.build(c, ids)
        lo = (c[:, : min(n, 200)] - np.float32(0.1)).astype(np.float32)
        hi = (c[:, : min(n, 200)] + np.float32(0.1)).astype(np.float32)
        want = O.search(tab, tid, lo, hi, variant=O.BRUTE)[0]
        for v in (O.LEVEL_ORDER, O.BFS, O.BRANCHLESS, O.RECURSIVE):
            assert np.array_equal(O.search(tab, tid, lo, hi, variant=v)[0], want)
        cnt, dig = O.search_digest(tab, tid, lo, hi)
        assert np.array_equal(cnt, want)
        if O.ref_available():
            r = O.RefTree(c, ids)
            r.build()
            t2 = r.tables()
            assert np.array_equal(t2[0].view(np.uint32), tab.view(np.uint32)) and np.array_equal(t2[1], tid)
            assert np.array_equal(r.search(lo, hi, variant=O.RECURSIVE, threads=2)[0], want)
            r.close()
wb = W.event_batch(n_events=12, median=800, size_lo=1, size_hi=3000, clusters_lo=2, clusters_hi=8, seed=4,
                   frac_4d=0.3, half_width=0.02)
_, _, c1, d1 = O.batch(wb, threads=2)
if O.ref_available():
    c2, d2, _ = O.ref_batch(wb, threads=2)
    assert np.array_equal(c1, c2) and np.array_equal(d1, d2)
    ev = W.clustered_event(n=20_000, n_queries=300, n_clusters=16, seed=3)
    O.ref_cmssw(ev.coords, ev.mins, ev.maxs)
print("SANITIZED OK")
"""


def _libasan():
    try:
        p = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True, text=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    path = p.stdout.strip()
    return path if os.path.isabs(path) and os.path.exists(path) else None


def test_checkers_clean_under_asan_and_ubsan():
    asan = _libasan()
    if asan is None:
        pytest.skip("gcc's ASan runtime not found")
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "sanitize"], capture_output=True, text=True)
    if r.returncode != 0 or not SAN_ORACLE.exists():
        pytest.skip("sanitised oracle build unavailable: " + r.stderr[-300:])
    env = dict(os.environ)
    env.update(LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1", FKD_ORACLE_SO=str(SAN_ORACLE),
               PYTHONPATH=str(ROOT))
    if SAN_REF.exists():
        env["FKD_REF_SO"] = str(SAN_REF)
    p = subprocess.run([sys.executable, "-c", CHILD], capture_output=True, text=True, env=env, cwd=str(ROOT),
                       timeout=600)
    out = p.stdout + p.stderr
    assert p.returncode == 0 and "SANITIZED OK" in p.stdout, out[-3000:]
    assert "AddressSanitizer" not in out and "runtime error" not in out, out[-3000:]
