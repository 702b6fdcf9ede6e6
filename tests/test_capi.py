"""The C ABI library loads and exports every entry point include/*.h
declares; argument checks that need no GPU.  CPU only."""
import ctypes as C
import re
from pathlib import Path

from fkdtree_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^FKD_API\s+[\w\s\*]+?\b(fkd_\w+)\s*\(", h.read_text(), re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    names = declared_symbols()
    assert names, "no FKD_API declarations found"
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(_capi.SIGNATURES) >= {n for n in names if n in _capi.SIGNATURES}


def test_version_and_arg_checks_without_gpu():
    L = _capi.lib()
    assert b"sm_100a" in L.fkd_version()
    h = C.c_void_p()
    assert L.fkd_create(7, 0, None, C.byref(h)) == 1  # FKD_ERR_ARG, dim out of range
    assert b"dim" in L.fkd_last_error()
    assert L.fkd_build(None, None, None, 0, 0) == 1
    assert L.fkd_search_count(None, None, None, 0, None, 0) == 1
    assert L.fkd_destroy(None) == 0
