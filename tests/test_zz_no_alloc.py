"""fkd_build_noalloc, the build entry point that allocates nothing, against
the regular fkd_build + fkd_get_tables and against the oracle.

It exists for callers that may not call cudaMalloc / cudaFree while they
work (a framework that owns all device memory through its own pool, where
those calls would synchronise the device or fail mid-event); it builds one
small tree in a fixed scratch array the library carries.  The tables are
integer data, so the entry points must agree bit for bit -- on calls in a
row, with different inputs, so that scratch left by one call cannot leak
into the next.  This file is collected last so that a run that stops at the
first failure has run every other test first; it also passes on its own."""
import ctypes as C

import numpy as np
import pytest

from fkdtree_b200 import _capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_NAN = 1, 4


def _dev(t):
    return C.c_void_p(t.data_ptr())


def _regular(L, dim, coords_np, ids_np):
    h = C.c_void_p()
    _capi.check(L.fkd_create(dim, 0, None, C.byref(h)))
    try:
        n = ids_np.shape[0]
        _capi.check(L.fkd_build(h, coords_np.ctypes.data_as(C.c_void_p), ids_np.ctypes.data_as(C.c_void_p), n,
                                _capi.MEM_HOST))
        tab = np.empty(dim * n, np.float32)
        tid = np.empty(n, np.uint32)
        _capi.check(L.fkd_get_tables(h, tab.ctypes.data_as(C.c_void_p), tid.ctypes.data_as(C.c_void_p),
                                     _capi.MEM_HOST))
        return tab, tid
    finally:
        L.fkd_destroy(h)


class _Call:
    """Device buffers of one fkd_build_noalloc call, allocated up front so
    that the calls themselves can run back to back with nothing allocated
    between them."""

    def __init__(self, torch, dim, coords_np, ids_np):
        self.dim, self.n = dim, ids_np.shape[0]
        self.coords_np, self.ids_np = coords_np, ids_np
        self.c = torch.from_numpy(coords_np).cuda()
        self.i = torch.from_numpy(ids_np.view(np.int32)).cuda()
        self.tab = torch.full((dim * self.n,), float("nan"), dtype=torch.float32, device="cuda")
        self.tid = torch.full((self.n,), -1, dtype=torch.int32, device="cuda")

    def run(self, L, stream):
        return L.fkd_build_noalloc(self.dim, _dev(self.c), _dev(self.i), self.n, _dev(self.tab), _dev(self.tid),
                                   C.c_void_p(stream))

    def result(self):
        return self.tab.cpu().numpy(), self.tid.cpu().numpy().view(np.uint32)


def _cases(dim, cap, rng):
    out = []
    for n in (cap, 1000, cap, 1, 2, 3, 17):  # different data every call; the first size again after a smaller one
        c = rng.random((dim, n), dtype=np.float32)
        c[-1] = np.round(c[-1] * 16) / 16  # ties, decided by id
        out.append((np.ascontiguousarray(c.reshape(-1)), rng.permutation(n).astype(np.uint32) * 7 + 3))
    return out


@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_noalloc_build_matches_regular_build(cuda, dim):
    import torch
    L = _capi.lib()
    cap = L.fkd_build_noalloc_max_points(dim)
    assert cap == (4096 if dim <= 3 else 3072)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(17 + dim)
    # the first call on the device looks the scratch up (and loads this dim's kernels)
    warm = _Call(torch, dim, *_cases(dim, cap, np.random.default_rng(99))[1])
    _capi.check(warm.run(L, stream))
    calls = [_Call(torch, dim, c, i) for c, i in _cases(dim, cap, rng)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for call in calls:  # back to back: nothing else allocates in between
        _capi.check(call.run(L, stream))
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes across the calls"
    for k, call in enumerate(calls):
        got_tab, got_ids = call.result()
        want_tab, want_ids = _regular(L, dim, call.coords_np, call.ids_np)
        assert np.array_equal(got_tab.view(np.uint32), want_tab.view(np.uint32)), f"call {k}: tables differ"
        assert np.array_equal(got_ids, want_ids), f"call {k}: ids differ"
        otab, oid = O.build(call.coords_np.reshape(dim, -1), call.ids_np)
        assert np.array_equal(got_tab.view(np.uint32), otab.reshape(-1).view(np.uint32)), f"call {k}: vs oracle"
        assert np.array_equal(got_ids, oid), f"call {k}: ids vs oracle"


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    L = _capi.lib()
    for dim in (3, 4):
        n = L.fkd_build_noalloc_max_points(dim) + 1
        c = torch.zeros(dim * n, dtype=torch.float32, device="cuda")
        i = torch.zeros(n, dtype=torch.int32, device="cuda")
        st = L.fkd_build_noalloc(dim, _dev(c), _dev(i), n, _dev(c), _dev(i), None)
        assert st == ERR_ARG
        assert b"exceed" in L.fkd_last_error()


def test_noalloc_rejects_nan_then_builds(cuda):
    import torch
    L = _capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    c, i = _cases(3, 4096, rng)[1]
    bad = c.copy()
    bad[123] = np.nan
    call = _Call(torch, 3, bad, i)
    assert call.run(L, stream) == ERR_NAN
    good = _Call(torch, 3, c, i)
    _capi.check(good.run(L, stream))  # the error word of the failed call does not carry over
    got_tab, got_ids = good.result()
    otab, oid = O.build(c.reshape(3, -1), i)
    assert np.array_equal(got_tab.view(np.uint32), otab.reshape(-1).view(np.uint32)) and np.array_equal(got_ids, oid)
