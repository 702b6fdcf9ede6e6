"""fkd_build_noalloc, the build entry point that allocates nothing, against
the regular fkd_build + fkd_get_tables.

It exists for callers that may not call cudaMalloc / cudaFree while they
work (a framework that owns all device memory through its own pool, where
those calls would synchronise the device or fail mid-event); it builds one
small tree in a fixed scratch array the library carries.  The tables are
integer data, so the two entry points must agree bit for bit -- on two calls
in a row, with different inputs, so that scratch left by one call cannot leak
into the next.  This file is collected last so that a run that stops at the
first failure has run every other test first; it also passes on its own."""
import ctypes as C

import numpy as np
import pytest

from fkdtree_b200 import _capi

pytestmark = pytest.mark.gpu


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


def _noalloc(L, torch, dim, coords_np, ids_np, stream):
    n = ids_np.shape[0]
    c = torch.from_numpy(coords_np).cuda()
    i = torch.from_numpy(ids_np.view(np.int32)).cuda()
    tab = torch.full((dim * n,), float("nan"), dtype=torch.float32, device="cuda")
    tid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    _capi.check(L.fkd_build_noalloc(dim, _dev(c), _dev(i), n, _dev(tab), _dev(tid), C.c_void_p(stream)))
    return tab.cpu().numpy(), tid.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("dim", [3, 4])
def test_noalloc_build_matches_regular_build(cuda, dim):
    import torch
    L = _capi.lib()
    cap = L.fkd_build_noalloc_max_points(dim)
    assert cap == (4096 if dim <= 3 else 3072)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(17 + dim)
    cases = []
    for n in (cap, 1000, cap):  # two calls in a row each with different data, then the first size again
        c = rng.random((dim, n), dtype=np.float32)
        c[-1] = np.round(c[-1] * 16) / 16  # ties, decided by id
        cases.append((np.ascontiguousarray(c.reshape(-1)), rng.permutation(n).astype(np.uint32)))
    free0 = None
    for k, (c, i) in enumerate(cases):
        got_tab, got_ids = _noalloc(L, torch, dim, c, i, stream)
        if k == 0:
            free0 = torch.cuda.mem_get_info()[0]
        want_tab, want_ids = _regular(L, dim, c, i)
        assert np.array_equal(got_tab.view(np.uint32), want_tab.view(np.uint32)), f"call {k}: tables differ"
        assert np.array_equal(got_ids, want_ids), f"call {k}: ids differ"
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    L = _capi.lib()
    n = L.fkd_build_noalloc_max_points(3) + 1
    c = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    i = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = L.fkd_build_noalloc(3, _dev(c), _dev(i), n, _dev(c), _dev(i), None)
    assert st == 1  # FKD_ERR_ARG
    assert b"exceed" in L.fkd_last_error()
