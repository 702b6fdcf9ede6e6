"""ctypes binding of the C ABI declared in include/fkdtree_b200.h.

The shared library is built in-tree (fkdtree_b200/libfkdtree_b200.so, by
fkdtree_b200/csrc/Makefile or __graft_entry__.build()).  There is no fallback:
if the library is missing or the GPU is absent, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfkdtree_b200.so"

FKD_OK = 0
STATUS = {
    0: "FKD_OK", 1: "FKD_ERR_ARG", 2: "FKD_ERR_CUDA", 3: "FKD_ERR_NOMEM", 4: "FKD_ERR_NAN", 5: "FKD_ERR_STATE",
    6: "FKD_ERR_CAPACITY", 7: "FKD_ERR_INTERNAL", 8: "FKD_ERR_TIMEOUT",
}
MEM_HOST, MEM_DEVICE = 0, 1
ERR_CAPACITY = 6
FLAG_ASYNC = 1

# Every entry point include/fkdtree_b200.h declares, with its ctypes signature.
_vp, _u32, _u64, _int = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
SIGNATURES = {
    "fkd_version": ([], C.c_char_p),
    "fkd_last_error": ([], C.c_char_p),
    "fkd_kernel_launches": ([], C.c_uint64),
    "fkd_debug_fail_alloc": ([C.c_int32], None),
    "fkd_create": ([_int, _u32, _vp, C.POINTER(_vp)], _int),
    "fkd_destroy": ([_vp], _int),
    "fkd_set_stream": ([_vp, _vp], _int),
    "fkd_build": ([_vp, _vp, _vp, _u64, _int], _int),
    "fkd_size": ([_vp, C.POINTER(_u64)], _int),
    "fkd_build_noalloc": ([_int, _vp, _vp, _u32, _vp, _vp, _vp], _int),
    "fkd_build_noalloc_max_points": ([_int], _u32),
    "fkd_get_tables": ([_vp, _vp, _vp, _int], _int),
    "fkd_search_count": ([_vp, _vp, _vp, _u64, _vp, _int], _int),
    "fkd_search_write": ([_vp, _vp, _vp, _u64, _vp, _vp, _int, _int], _int),
    "fkd_search": ([_vp, _vp, _vp, _u64, _vp, _vp, _u64, C.POINTER(_u64), _int, _int], _int),
    "fkd_search_digest": ([_vp, _vp, _vp, _u64, _vp, _vp, _int], _int),
    "fkd_build_points": ([_vp, _vp, _u64, _int], _int),
    "fkd_search_radius_count": ([_vp, _vp, _vp, _u64, _vp, _int], _int),
    "fkd_search_radius": ([_vp, _vp, _vp, _u64, _vp, _vp, _u64, C.POINTER(_u64), _int, _int], _int),
    "fkd_search_knn": ([_vp, _vp, _u64, _u32, _vp, _vp, _int], _int),
    "fkd_knn_max_k": ([], _u32),
    "fkd_sync": ([_vp], _int),
    "fkd_batch_create": ([_u32, _vp, _vp, _vp, _u32, _vp, C.POINTER(_vp)], _int),
    "fkd_batch_destroy": ([_vp], _int),
    "fkd_batch_set_param": ([_vp, C.c_char_p, C.c_int64], _int),
    "fkd_set_param": ([_vp, C.c_char_p, C.c_int64], _int),
    "fkd_kernel_times": ([_vp, C.c_uint32, _vp], _int),
    "fkd_batch_build": ([_vp, _vp, _vp, _int], _int),
    "fkd_batch_get_tables": ([_vp, _vp, _vp, _int], _int),
    "fkd_batch_search_digest": ([_vp, _vp, _vp, _vp, _vp, _int], _int),
    "fkd_batch_run": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp], _int),
    "fkd_batch_sync": ([_vp], _int),
    "fkd_mlp_create": ([_u32, C.POINTER(_vp)], _int),
    "fkd_mlp_destroy": ([_vp], _int),
    "fkd_mlp_param_count": ([], _u64),
    "fkd_mlp_get_params": ([_vp, _vp], _int),
    "fkd_mlp_set_params": ([_vp, _vp], _int),
    "fkd_mlp_forward": ([_vp, _vp, _u64, _vp, _int], _int),
    "fkd_mlp_grad": ([_vp, _vp, _vp, _u64, _vp, _vp, _int], _int),
    "fkd_mlp_train": ([_vp, _vp, _vp, _u64, _u32, _u32, C.c_float, _u32, _vp, _int], _int),
    "fkd_set_mlp": ([_vp, _vp, C.c_float], _int),
    "fkd_batch_set_mlp": ([_vp, _vp, C.c_float], _int),
    "fkd_learn_stats": ([_vp, _vp, _int], _int),
    "fkd_batch_learn_stats": ([_vp, _vp, _int], _int),
    "fkd_batch_record": ([_vp, _vp, _vp, _vp, _vp, _u64, _vp, _int], _int),
}


class FKDError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C fkdtree_b200/csrc` "
                              "or __graft_entry__.build(); there is no CPU fallback")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != FKD_OK:
        raise FKDError(status, lib().fkd_last_error().decode(errors="replace"))
