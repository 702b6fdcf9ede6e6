"""The C++ drop-in (include/FKDTree_CUDA.h) behind the reference's own
FKDTree<float, dim> interface, compared in one process with the reference's
FKDTree_CPU: tables, ordered search lists, per-box counts, test_correct_build
and test_correct_search.  The binary is built by oracle/Makefile where the
reference headers are present."""
import subprocess
from pathlib import Path

import pytest

BIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "test_dropin"

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not BIN.exists(), reason="drop-in test binary not built (needs the reference headers)")
def test_cpp_dropin_matches_reference_cpu_tree(cuda):
    """Includes main.cpp's threaded pattern: 8 std::threads searching one
    built tree at once, every list equal to FKDTree_CPU's."""
    r = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "DROPIN OK" in r.stdout, r.stdout + r.stderr
    assert "threads 8: 20000 boxes identical" in r.stdout
