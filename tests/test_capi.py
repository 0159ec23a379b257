"""The C-ABI library loads and exports every entry point include/hgx.h declares (no GPU
compute is called here)."""
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:int|void\s*\*|const char\s*\*)\s+(hgx_\w+)\s*\(",
                                    txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    from hipgisaxs_b200 import _capi
    L = _capi.lib()
    names = _declared()
    assert len(names) >= 10
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_header():
    from hipgisaxs_b200 import _capi
    assert _declared() <= set(_capi.SIGNATURES), sorted(_declared() - set(_capi.SIGNATURES))


def test_status_strings_without_gpu():
    from hipgisaxs_b200 import _capi
    L = _capi.lib()
    assert L.hgx_status_string(0) == b"ok"
    assert L.hgx_version() >= 10000


def test_null_arguments_rejected_without_gpu():
    import ctypes as C
    from hipgisaxs_b200 import _capi
    L = _capi.lib()
    assert L.hgx_create(0, None) == 1  # rejected before any device call
    rc = L.hgx_qgrid_info(None, None, None, None, None, None)
    assert rc == 1 and b"NULL" in L.hgx_last_error()
