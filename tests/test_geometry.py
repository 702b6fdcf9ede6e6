"""The closed-form interval geometry of fkd_common.cuh against the
reference's own interval recurrence (FKDTree_cpu.h:224-267).  The header's
host functions are compiled with g++ into a throwaway library; CPU only."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]

SRC = r'''
#include "fkd_common.cuh"
extern "C" void geom(unsigned n, unsigned* start, unsigned* len, unsigned* rank) {
  fkd::Geom g = fkd::make_geom(n);
  for (unsigned i = 0; i < n; ++i) {
    unsigned d = fkd::floor_log2_u32(i + 1), t = i + 1 - (1u << d);
    start[i] = fkd::seg_start(g, d, t);
    len[i] = fkd::seg_len(g, d, t);
    rank[i] = d < g.H ? fkd::seg_rank(g, d, t) : 0u;
  }
}
extern "C" unsigned subtree(unsigned n, unsigned i) { return fkd::subtree_size(fkd::make_geom(n), i); }
'''


@pytest.fixture(scope="module")
def geomlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("geom")
    (d / "g.cpp").write_text(SRC)
    so = d / "libg.so"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-x", "c++",
                    f"-I{ROOT / 'fkdtree_b200' / 'csrc'}", "-I/usr/local/cuda/include", str(d / "g.cpp"),
                    "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    u = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    L.geom.argtypes = [C.c_uint, u, u, u]
    L.subtree.argtypes = [C.c_uint, C.c_uint]
    L.subtree.restype = C.c_uint
    return L


def _partition_complete(length):  # FKDTree_cpu.h:287-296
    if length == 1:
        return 0
    index = 1 << (int(length).bit_length() - 1)
    return index - 1 if (index // 2) - 1 <= length - index else length - index // 2


@pytest.mark.parametrize("n", list(range(1, 70)) + [100, 1000, 4095, 4096, 4097, 12345, 65535, 65536, 100000])
def test_closed_form_intervals(geomlib, n):
    O.build_libs()
    imin, ilen = O.intervals(n)
    s = np.empty(n, np.uint32)
    l = np.empty(n, np.uint32)
    r = np.empty(n, np.uint32)
    geomlib.geom(n, s, l, r)
    assert np.array_equal(s, imin) and np.array_equal(l, ilen)
    depth = np.floor(np.log2(np.arange(1, n + 1))).astype(int)
    H = int(n).bit_length() - 1
    for i in np.nonzero(depth < H)[0][:2000]:
        assert r[i] == _partition_complete(int(ilen[i]))
    for i in [0, n // 3, n - 1]:
        assert geomlib.subtree(n, i) == ilen[i]
