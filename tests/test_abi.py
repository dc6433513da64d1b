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


def test_ctypes_descriptors_match_the_c_layout(tmp_path):
    """Size and field offsets of the ctypes mirrors equal the C compiler's."""
    import shutil
    import subprocess
    from gtls_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    structs = {"gtls_search_desc": _lib.SearchDesc, "gtls_batch_desc": _lib.BatchDesc, "gtls_timing": _lib.Timing,
               "gtls_template_desc": _lib.TemplateDesc}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gtls_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            cf = "pass" if fname == "pass_" else fname
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, cf))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_device_status_word_becomes_an_error():
    """A search's non-zero device status word (a chi2 tile copy that did not
    complete within its bounded wait) is reported as GTLS_E_DEVICE with its
    meaning, and the Python layer turns it into GtlsError; 0 is no error."""
    from gtls_b200 import _lib
    lib = _lib.load()
    buf = ctypes.create_string_buffer(128)
    assert lib.gtls_decode_status(0, buf, len(buf)) == 0
    assert lib.gtls_decode_status(1, buf, len(buf)) == 5   # GTLS_E_DEVICE
    assert b"tile copy" in buf.value
    assert lib.gtls_decode_status(5, buf, 16) == 5 and len(buf.value) == 15   # truncated, NUL-terminated
    assert _lib.device_status_error(0) is None
    err = _lib.device_status_error(1)
    assert isinstance(err, _lib.GtlsError) and "tile copy" in str(err)
