"""The C-ABI library loads and exports every function include/gtls_b200.h declares."""
import ctypes
import os
import re

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "gtls_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(gtls_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_declared_symbols():
    from gtls_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert "gtls_search" in names and "gtls_spectra" in names and len(names) >= 8
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.EXPORTS, name
    assert lib.gtls_abi_version() == _lib.ABI_VERSION


def test_context_creation_reports_errors_without_a_gpu():
    import torch
    from gtls_b200 import _lib
    lib = _lib.load()
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = lib.gtls_ctx_create(0, ctypes.byref(h))
    assert rc != 0
    assert len(lib.gtls_last_error(None)) > 0
