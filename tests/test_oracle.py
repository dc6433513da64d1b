"""The CPU oracle against the reference itself (no GPU needed).

Pins: the NumPy restatement vs (a) the reference's kernels compiled for the
CPU when oracle/_ref is built, (b) the golden fixtures recorded from the
reference (grid, spectra, kernels).
"""
import numpy as np
import pytest

import tls_oracle as O
import ref_replay as RR
from conftest import golden, search_inputs


def test_period_grid_matches_reference_grid_module():
    g = golden("grid")
    i = 0
    while "case%d_args" % i in g:
        rs, ms, span, pmin, pmax, osf, ntr = g["case%d_args" % i]
        p = O.period_grid(rs, ms, span, pmin, pmax, int(osf), int(ntr))
        np.testing.assert_array_equal(p, g["case%d_periods" % i])
        i += 1
    assert i >= 5


def test_spectra_matches_reference_stats():
    s = golden("spectra")
    for i in range(4):
        n, osf = s["case%d" % i]
        c = np.ma.array(s["case%d_chi2" % i], mask=s["case%d_mask" % i])
        SR, praw, power, sde_raw, sde = O.spectra(c, int(osf))
        np.testing.assert_allclose(np.ma.getdata(power), s["case%d_power" % i], rtol=0, atol=1e-12)
        np.testing.assert_allclose([sde_raw, sde], s["case%d_sde" % i], rtol=1e-13)


def test_numpy_kernels_match_reference_kernel_fixtures():
    k = golden("kernels")
    nb = O.NumpyBackend()
    for i in range(3):
        t, y, dy = k["case%d_t" % i], k["case%d_y" % i], k["case%d_dy" % i]
        widths, os_, tm, maxd = k["case%d_widths" % i], k["case%d_overshoot" % i], k["case%d_templates" % i], \
            int(k["case%d_maxd" % i][0])
        for j, p in enumerate(k["case%d_periods" % i]):
            wmin, wmax = O.duration_ranges(np.array([p]), t.max() - t.min(), len(t))
            m = (widths >= wmin[0]) & (widths <= wmax[0])
            a = nb.main_pass(t, y, dy, p, widths[m], tm[m], os_[m], maxd, 1e-5, 8)
            b = nb.noskip_pass(t, y, dy, p, widths[m], tm[m], os_[m], maxd, 1e-5)
            ref = k["case%d_r64" % i][j]
            assert a[1] == int(ref[1]) and b[1] == int(ref[3])
            np.testing.assert_allclose([a[0], b[0]], [ref[0], ref[2]], rtol=1e-12)


@pytest.mark.skipif(not RR.available("r64_skip8"), reason="oracle/_ref not built (make -C oracle)")
@pytest.mark.parametrize("use_dy", [False, True])
def test_numpy_kernels_match_compiled_reference_kernels(use_dy):
    s = search_inputs(seed=5, n=800, span=5.0, use_dy=use_dy)
    nb = O.NumpyBackend()
    rb = RR.RefKernelBackend("r64", 8)
    span = s["t"].max() - s["t"].min()
    w1 = O.duration_ranges(s["periods"], span, len(s["t"]))
    w2 = rb.duration_ranges(s["periods"], span, len(s["t"]))
    np.testing.assert_array_equal(w1[0], w2[0])
    np.testing.assert_array_equal(w1[1], w2[1])
    for p in s["periods"][::17]:
        args = (s["t"], s["y"], s["dy"], p, s["widths"], s["templates"], s["overshoot"], s["maxd"], 1e-5)
        a, b = nb.main_pass(*args, 8), rb.main_pass(*args, 8)
        assert a[1] == b[1]
        assert abs(a[0] / b[0] - 1) < 1e-12
        a, b = nb.noskip_pass(*args), rb.noskip_pass(*args)
        assert a[1] == b[1]
        assert abs(a[0] / b[0] - 1) < 1e-12


@pytest.mark.skipif(not RR.available("r64_skipnever"), reason="oracle/_ref not built (make -C oracle)")
def test_no_skip_margin_matches_reference():
    """T0_fit_margin = 0 -> SKIP_POINT 0x7f800000: every start evaluated (core.py:598-599)."""
    s = search_inputs(seed=6, n=600, span=4.0)
    nb = O.NumpyBackend()
    rb = RR.RefKernelBackend("r64", O.SKIP_NEVER)
    for p in s["periods"][::40]:
        args = (s["t"], s["y"], s["dy"], p, s["widths"], s["templates"], s["overshoot"], s["maxd"], 1e-5)
        a, b = nb.main_pass(*args, O.SKIP_NEVER), rb.main_pass(*args, O.SKIP_NEVER)
        assert a[1] == b[1] and abs(a[0] / b[0] - 1) < 1e-12


def test_full_flow_runs_and_finds_injected_period():
    s = search_inputs(seed=2, n=1500, span=6.0)
    out = O.search(O.NumpyBackend(), s["periods"], s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                   s["overshoot"], s["dur_u"], s["maxd"], 1e-5, 0.125, 3, batch=12)
    assert abs(out["period"] - 1.7) < 0.02
    assert out["SDE"] > 7
