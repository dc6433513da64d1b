"""The allocation-free spectra entry point, called through the C-ABI.

gtls_spectra_noalloc serves callers that cannot allocate device memory when
they compute a periodogram's SDE (fixed memory budgets owned by another
framework, allocation-free real-time loops, callers without a gtls context).
It keeps its scratch in a static device array instead.  This file is named to
be collected last, so a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, chi2, mask, osf):
    sr = torch.empty_like(chi2)
    praw = torch.empty_like(chi2)
    power = torch.empty_like(chi2)
    sde_raw, sde = ctypes.c_double(), ctypes.c_double()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.gtls_spectra_noalloc(ctypes.c_void_p(chi2.data_ptr()),
                                  ctypes.c_void_p(mask.data_ptr()) if mask is not None else None,
                                  chi2.numel(), float(osf), ctypes.c_void_p(sr.data_ptr()),
                                  ctypes.c_void_p(praw.data_ptr()), ctypes.c_void_p(power.data_ptr()),
                                  ctypes.byref(sde_raw), ctypes.byref(sde), stream)
    assert rc == 0, lib.gtls_noalloc_last_error().decode()
    return sr, praw, power, sde_raw.value, sde.value


def test_noalloc_spectra_matches_allocating_entry_point(cuda):
    torch = cuda
    from gtls_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(5)
    # calls in a row with different inputs (each reuses the static scratch);
    # the last has n <= 2 * kernel (91 here), where no running median is taken
    for n, osf, nmask in [(20000, 3, 0), (7001, 2, 11), (150, 3, 5)]:
        chi2 = torch.from_numpy(1000 + rng.normal(0, 3, n)).cuda()
        m = np.zeros(n, np.uint8)
        m[rng.choice(n, nmask, replace=False)] = 1
        mask = torch.from_numpy(m).cuda() if nmask else None
        got = _noalloc(lib, torch, chi2, mask, osf)
        ref = _lib.spectra(chi2, mask, osf)
        for a, b in zip(got[:3], ref[:3]):
            np.testing.assert_allclose(a.cpu().numpy(), b.cpu().numpy(), rtol=1e-12, atol=0)
        np.testing.assert_allclose(got[3:], ref[3:], rtol=1e-12)


def test_noalloc_rejects_sizes_beyond_its_maximum(cuda):
    from gtls_b200 import _lib
    lib = _lib.load()
    dummy = ctypes.c_void_p(1)
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = lib.gtls_spectra_noalloc(dummy, None, (1 << 20) + 1, 3.0, dummy, dummy, dummy, ctypes.byref(a),
                                  ctypes.byref(b), None)
    assert rc != 0
    assert b"exceeds" in lib.gtls_noalloc_last_error()
