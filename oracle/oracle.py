"""ctypes access to the CPU checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by bench.py's CPU-baseline leg and reference arm.  The
product package (fkdtree_b200) never imports this module.

Two libraries:

* ``C``   -- oracle/_build/libfkdoracle.so, the C restatement of the reference
  build and searches (fkd_oracle.c);
* ``Ref`` -- oracle/_ref/libfkdref.so, the unmodified reference FKDTree_CPU
  compiled from its own headers (ref_harness.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# FKD_ORACLE_SO / FKD_REF_SO select other builds of the same sources (the
# sanitised ones of `make -C oracle sanitize`)
ORACLE_SO = Path(os.environ.get("FKD_ORACLE_SO") or HERE / "_build" / "libfkdoracle.so")
REF_SO = Path(os.environ.get("FKD_REF_SO") or HERE / "_ref" / "libfkdref.so")

LEVEL_ORDER, BFS, BRANCHLESS, RECURSIVE, BRUTE = 0, 1, 2, 3, 4
FQUEUE_SLOTS = 1024  # FQueue.h:232 -- the reference frontier ring

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def build_libs() -> None:
    """Runs oracle/Makefile (the C restatement always; the reference harness
    only where the reference sources are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_c = None
_ref = None


def lib():
    global _c
    if _c is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} is missing: run `make -C oracle` (or __graft_entry__.build())")
        L = C.CDLL(str(ORACLE_SO))
        L.fkd_oracle_build.argtypes = [C.c_int, C.c_uint32, _f32p, _u32p, _f32p, _u32p]
        L.fkd_oracle_build.restype = C.c_int
        L.fkd_oracle_intervals.argtypes = [C.c_uint32, _u32p, _u32p]
        L.fkd_oracle_search.argtypes = [C.c_int, C.c_int, C.c_uint32, _f32p, _u32p, C.c_uint64, _f32p, _f32p, _u32p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.fkd_oracle_search.restype = C.c_int
        L.fkd_oracle_search_digest.argtypes = [C.c_int, C.c_uint32, _f32p, _u32p, C.c_uint64, _f32p, _f32p, _u32p,
                                               _u64p, C.c_int]
        L.fkd_oracle_mix64.argtypes = [C.c_uint32]
        L.fkd_oracle_mix64.restype = C.c_uint64
        L.fkd_oracle_batch.argtypes = [C.c_uint32, _u32p, _u64p, _u64p, _f32p, _u32p, _u64p, _u64p, _f32p, _f32p,
                                       _f32p, _u32p, _u32p, _u64p, C.c_int]
        L.fkd_oracle_batch.restype = C.c_int
        L.fkd_oracle_digest_lists.argtypes = [C.c_uint64, _u64p, _u32p, _u64p, C.c_int]
        L.fkd_oracle_digest_lists.restype = C.c_int
        _c = L
    return _c


def ref_available() -> bool:
    return REF_SO.exists()


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise RuntimeError(f"{REF_SO} is missing: it is built from the reference sources by `make -C oracle`")
        L = C.CDLL(str(REF_SO))
        L.fkdref_create.argtypes = [C.c_int, C.c_uint32, _f32p, _u32p]
        L.fkdref_create.restype = C.c_void_p
        L.fkdref_destroy.argtypes = [C.c_void_p]
        L.fkdref_build.argtypes = [C.c_void_p]
        L.fkdref_build.restype = C.c_double
        L.fkdref_tables.argtypes = [C.c_void_p, _f32p, _u32p]
        L.fkdref_search.argtypes = [C.c_void_p, C.c_int, C.c_uint64, _f32p, _f32p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int, C.POINTER(C.c_double)]
        L.fkdref_max_threads.restype = C.c_int
        L.fkdref_batch.argtypes = [C.c_uint32, _u32p, _u64p, _u64p, _f32p, _u32p, _u64p, _u64p, _f32p, _f32p, _u32p,
                                   _u64p, C.c_int]
        L.fkdref_batch.restype = C.c_double
        L.fkdref_search_digest.argtypes = [C.c_void_p, C.c_uint64, _f32p, _f32p, _u32p, _u64p, C.c_int]
        L.fkdref_search_digest.restype = C.c_double
        L.fkdref_cmssw.argtypes = [C.c_uint32, _f32p, C.c_uint64, _f32p, _f32p, _u32p, C.POINTER(C.c_double)]
        L.fkdref_cmssw.restype = C.c_double
        _ref = L
    return _ref


def _soa(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ C oracle

def build(coords: np.ndarray, ids: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Restated FKDTree_CPU::build (FKDTree_cpu.h:221-277): returns the heap
    tables (dim, n) float32 and (n,) uint32."""
    coords = _soa(coords, np.float32)
    ids = _soa(ids, np.uint32)
    dim, n = coords.shape
    tab = np.empty((dim, n), dtype=np.float32)
    tid = np.empty(n, dtype=np.uint32)
    rc = lib().fkd_oracle_build(dim, n, coords, ids, tab, tid)
    if rc != 0:
        raise RuntimeError(f"fkd_oracle_build failed ({rc})")
    return tab, tid


def intervals(n: int) -> tuple[np.ndarray, np.ndarray]:
    imin = np.zeros(max(n, 1), dtype=np.uint32)
    ilen = np.zeros(max(n, 1), dtype=np.uint32)
    lib().fkd_oracle_intervals(n, imin, ilen)
    return imin[:n], ilen[:n]


def search(tab: np.ndarray, tab_ids: np.ndarray, mins: np.ndarray, maxs: np.ndarray, variant: int = RECURSIVE,
           want_ids: bool = True, threads: int = 0):
    """Returns (counts, offsets, ids, max_frontier): offsets has q+1 entries and
    ids the concatenated per-box results in the variant's emission order."""
    tab = _soa(tab, np.float32)
    tab_ids = _soa(tab_ids, np.uint32)
    mins = _soa(mins, np.float32)
    maxs = _soa(maxs, np.float32)
    dim, n = tab.shape
    q = mins.shape[1]
    counts = np.empty(q, dtype=np.uint32)
    front = np.empty(q, dtype=np.uint32)
    L = lib()
    rc = L.fkd_oracle_search(variant, dim, n, tab, tab_ids, q, mins, maxs, counts, _ptr(front), None, None, threads)
    if rc != 0:
        raise RuntimeError(f"fkd_oracle_search failed ({rc})")
    offsets = np.zeros(q + 1, dtype=np.uint64)
    np.cumsum(counts, out=offsets[1:])
    ids = None
    if want_ids:
        ids = np.empty(int(offsets[-1]), dtype=np.uint32)
        L.fkd_oracle_search(variant, dim, n, tab, tab_ids, q, mins, maxs, counts, None, _ptr(offsets), _ptr(ids),
                            threads)
    return counts, offsets, ids, front


def search_digest(tab, tab_ids, mins, maxs, threads: int = 0):
    tab = _soa(tab, np.float32)
    tab_ids = _soa(tab_ids, np.uint32)
    mins = _soa(mins, np.float32)
    maxs = _soa(maxs, np.float32)
    dim, n = tab.shape
    q = mins.shape[1]
    counts = np.empty(q, dtype=np.uint32)
    dig = np.empty(q, dtype=np.uint64)
    rc = lib().fkd_oracle_search_digest(dim, n, tab, tab_ids, q, mins, maxs, counts, dig, threads)
    if rc != 0:
        raise RuntimeError("fkd_oracle_search_digest failed")
    return counts, dig


def digest_lists(offsets: np.ndarray, ids: np.ndarray, threads: int = 0) -> np.ndarray:
    """Per-box digest of result lists laid out as ids[offsets[j]:offsets[j+1]]
    (the C twin of digest_of, multi-threaded, for billions of ids)."""
    offsets = _soa(offsets, np.uint64)
    ids = _soa(ids, np.uint32)
    q = offsets.shape[0] - 1
    dig = np.empty(q, dtype=np.uint64)
    lib().fkd_oracle_digest_lists(q, offsets, ids, dig, threads)
    return dig


def batch(b, threads: int = 0):
    """Builds and searches every event of a workloads.Batch; returns
    (tab, tab_ids, counts, digests) in the batch's flat layouts."""
    tab = np.empty_like(b.coords)
    tid = np.empty_like(b.ids)
    counts = np.empty(b.n_queries, dtype=np.uint32)
    dig = np.empty(b.n_queries, dtype=np.uint64)
    rc = lib().fkd_oracle_batch(b.n_events, _soa(b.dims, np.uint32), _soa(b.pt_off, np.uint64),
                                _soa(b.coord_off, np.uint64), _soa(b.coords, np.float32), _soa(b.ids, np.uint32),
                                _soa(b.q_off, np.uint64), _soa(b.qcoord_off, np.uint64), _soa(b.mins, np.float32),
                                _soa(b.maxs, np.float32), tab, tid, counts, dig, threads)
    if rc != 0:
        raise RuntimeError("fkd_oracle_batch failed")
    return tab, tid, counts, dig


def ref_batch(b, threads: int = 0):
    """The unmodified reference over every event of a workloads.Batch (OpenMP
    over events, each a serial FKDTree_CPU build + search_in_the_box_recursive
    of its boxes): returns (counts, digests, seconds)."""
    counts = np.empty(b.n_queries, dtype=np.uint32)
    dig = np.empty(b.n_queries, dtype=np.uint64)
    sec = ref_lib().fkdref_batch(b.n_events, _soa(b.dims, np.uint32), _soa(b.pt_off, np.uint64),
                                 _soa(b.coord_off, np.uint64), _soa(b.coords, np.float32), _soa(b.ids, np.uint32),
                                 _soa(b.q_off, np.uint64), _soa(b.qcoord_off, np.uint64), _soa(b.mins, np.float32),
                                 _soa(b.maxs, np.float32), counts, dig, threads)
    return counts, dig, float(sec)


def ref_cmssw(coords, mins, maxs):
    """The reference's vanilla CMSSW tree (KDTreeLinkerAlgoT.h) over 3D points,
    built and searched serially as main.cpp:558-612 does: returns (counts,
    build_seconds, search_seconds).  Its search tests boxes with strict
    inequalities for inner regions (KDTreeLinkerAlgoT.h:186-207), so points
    lying exactly on a box face may be missed; counts equal FKDTree's
    otherwise."""
    coords = _soa(coords, np.float32)
    mins = _soa(mins, np.float32)
    maxs = _soa(maxs, np.float32)
    if coords.shape[0] != 3:
        raise ValueError("the vanilla CMSSW comparison is 3D (main.cpp:564)")
    q = mins.shape[1]
    counts = np.empty(q, dtype=np.uint32)
    ts = C.c_double(0.0)
    tb = ref_lib().fkdref_cmssw(coords.shape[1], coords, q, mins, maxs, counts, C.byref(ts))
    return counts, float(tb), float(ts.value)


def mix64(ids: np.ndarray) -> np.ndarray:
    """numpy copy of the digest finaliser in fkd_oracle.c (per-id 64-bit mix)."""
    z = ids.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def digest_of(ids_concat: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """Per-box wrap-around sum of mix64 over each box's ids."""
    m = mix64(ids_concat)
    cs = np.zeros(m.shape[0] + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        np.cumsum(m, out=cs[1:])
        return cs[offsets[1:].astype(np.int64)] - cs[offsets[:-1].astype(np.int64)]


# ------------------------------------------------------------ reference tree

class RefTree:
    """The unmodified reference FKDTree_CPU<float, dim> behind oracle/_ref."""

    def __init__(self, coords: np.ndarray, ids: np.ndarray):
        self.coords = _soa(coords, np.float32)
        self.ids = _soa(ids, np.uint32)
        self.dim, self.n = self.coords.shape
        if self.n == 0:
            raise ValueError("the reference build is undefined for an empty input (FKDTree_cpu.h:226)")
        self.L = ref_lib()
        self.h = self.L.fkdref_create(self.dim, self.n, self.coords, self.ids)
        if not self.h:
            raise ValueError(f"unsupported dimension {self.dim}")
        self.build_seconds = None

    def build(self) -> float:
        self.build_seconds = self.L.fkdref_build(self.h)
        return self.build_seconds

    def tables(self):
        tab = np.empty((self.dim, self.n), dtype=np.float32)
        tid = np.empty(self.n, dtype=np.uint32)
        self.L.fkdref_tables(self.h, tab, tid)
        return tab, tid

    def search(self, mins, maxs, variant: int = RECURSIVE, want_ids: bool = True, threads: int = 0):
        """Returns (counts, offsets, ids, seconds) -- seconds covers the
        parallel search loop only (the ids pass when want_ids)."""
        mins = _soa(mins, np.float32)
        maxs = _soa(maxs, np.float32)
        q = mins.shape[1]
        counts = np.empty(q, dtype=np.uint32)
        secs = C.c_double(0.0)
        self.L.fkdref_search(self.h, variant, q, mins, maxs, _ptr(counts), None, None, threads, C.byref(secs))
        offsets = np.zeros(q + 1, dtype=np.uint64)
        np.cumsum(counts, out=offsets[1:])
        ids = None
        if want_ids:
            ids = np.empty(int(offsets[-1]), dtype=np.uint32)
            self.L.fkdref_search(self.h, variant, q, mins, maxs, None, _ptr(offsets), _ptr(ids), threads,
                                 C.byref(secs))
        return counts, offsets, ids, secs.value

    def search_digest(self, mins, maxs, threads: int = 0):
        """search_in_the_box_recursive of every box on `threads` OpenMP
        threads, each list reduced to (count, digest): returns (counts,
        digests, seconds)."""
        mins = _soa(mins, np.float32)
        maxs = _soa(maxs, np.float32)
        q = mins.shape[1]
        counts = np.empty(q, dtype=np.uint32)
        dig = np.empty(q, dtype=np.uint64)
        sec = self.L.fkdref_search_digest(self.h, q, mins, maxs, counts, dig, threads)
        return counts, dig, float(sec)

    def close(self):
        if self.h:
            self.L.fkdref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host_threads() -> int:
    return len(os.sched_getaffinity(0))
