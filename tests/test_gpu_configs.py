"""Parity at the full sizes of the benchmark workloads (seeded synthetic curves).

* 19,728 samples, 2-min cadence over 27.4 d: the whole default search
  (``gtls(t, y, dy).power()`` with no ``periods``: the Ofir grid, the main pass
  over every period, spectra, the 200 candidates re-searched at every start,
  the harmonics and the best-period finish) against the oracle's host flow
  (core.py:568-999) driving the reference's own kernels compiled for the CPU
  in FP64 (R64).  Identical grid (bit for bit), best period index, duration,
  (duration, start) location and candidate list; chi2, SDE, depth, T0 and
  duration within 1e-9 relative.
* 70,000 samples over 1,470 d (the multi-year phase-fold case; records staged
  in shared-memory tiles, 50 durations up to 8,400 samples): 512 periods
  spread over the whole 0.5-735 d grid (the shortest and the longest among
  them) through the main pass and 8 of them through the all-starts pass,
  against the same reference kernels: identical argmin locations, chi2
  within 1e-9; and the fold ordering of 16 periods equal to NumPy's stable
  argsort of the FP64 phases.
* The reference's own call on the TESS sector-58 2-minute light curve it
  bundles (test1.py:86-150, columns in the golden fixture tess_s58.npz):
  cleaned, normalised by the mean flux and searched with
  ``power(periods=np.linspace(1, 14, 10000))``; the script's wotan detrending
  is left out (wotan is not installed).  Same bars as the 19,728-sample case.
* The FP32-compensated form of the 19,728-sample search on three seeds of
  the mixed-precision workload (depth log-U(100, 2000) ppm, P log-U(1, 500) d)
  against the FP64 oracle: identical best period index and duration, SDE
  within 1e-4 relative, the chi2 spectrum within 2e-6.
"""
import numpy as np
import pytest

import tls_oracle as O

pytestmark = pytest.mark.gpu
RTOL64 = 1e-9
RTOL32 = 2e-6


def _backend():
    import ref_replay as RR
    if not RR.available("r64_skip8"):
        pytest.skip("the CPU build of the reference's kernels (oracle/_ref) is absent")
    return RR.RefKernelBackend("r64", 8)


def _oracle_search(model, res):
    """The oracle's full search over the product's grid, tables and batch size."""
    from gtls_b200 import template
    widths, os_, dd, tm, maxd = template.device_templates(model.lc_arr, model.lc_cache_overview)
    periods = np.asarray(np.ma.getdata(res.periods))
    return O.search(_backend(), periods, model.t, model.y, model.dy, widths, tm, os_, dd, maxd, 1e-5, 0.125, 3,
                    batch=res.diagnostics["batch_periods"])


def _assert_same_search(res, ref, rtol_chi2=RTOL64, rtol_sde=RTOL64):
    assert res.diagnostics["period_index"] == ref["period_index"]
    assert res.period == ref["period"]
    assert res.durationPoints == ref["width"]
    np.testing.assert_allclose(np.ma.getdata(res.chi2), np.ma.getdata(ref["chi2"]), rtol=rtol_chi2)
    np.testing.assert_allclose(res.SDE, ref["SDE"], rtol=rtol_sde)


def test_cfg1_default_search_matches_the_reference_flow(cuda):
    from gtls_b200 import gtls, synthetic
    t, y, dy, _ = synthetic.light_curve_cfg1(seed=0)
    model = gtls(t, y, dy, verbose=False)
    res = model.power(period_min=0.5, period_max=13.7, oversampling_factor=3)
    periods = np.asarray(np.ma.getdata(res.periods))
    span = model.t.max() - model.t.min()
    # the default grid is the reference's grid.period_grid, bit for bit
    np.testing.assert_array_equal(periods, np.sort(O.period_grid(1, 1, span, 0.5, 13.7, 3)))
    assert len(periods) > 2500 and len(model.t) == 19728
    ref = _oracle_search(model, res)
    _assert_same_search(res, ref)
    assert res.diagnostics["loc"] == ref["loc"]
    assert list(res.possiblePeriodsIndices) == list(ref["candidates"])
    np.testing.assert_allclose(res.raw_chi2, ref["raw_chi2"], rtol=RTOL64)
    np.testing.assert_allclose(res.diagnostics["chi2_main"], ref["chi2_main"], rtol=RTOL64)
    np.testing.assert_allclose([res.depth, res.T0, res.duration], [ref["depth"], ref["T0"], ref["duration"]],
                               rtol=RTOL64)
    assert abs(res.period / 3.853 - 1) < 2e-3


def _cfg2_inputs():
    from gtls_b200 import grid as G, synthetic, template, validate as V
    t, y, dy, _ = synthetic.light_curve_cfg2(seed=0)
    t, y, dy = V.validate_inputs(t, y, dy)
    P = G.period_grid(1, 1, t.max() - t.min(), 0.5, 735.0, 3, ascending=True)
    step = G.duration_grid_step_for(P, 1 / len(t), 50)
    durs = G.duration_grid(P, shortest=1 / len(t), log_step=step)
    mw = int(np.max(durs) * len(y))
    mw += mw % 2
    ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    widths, os_, _, tm, maxd = template.device_templates(lc, ov)
    return t, y, dy, P, lc, ov, widths, os_, tm, maxd


def test_cfg2_period_subset_matches_reference_kernels(cuda):
    from gtls_b200 import _lib
    from gtls_b200.core import CurveOnDevice
    t, y, dy, P, lc, ov, widths, os_, tm, maxd = _cfg2_inputs()
    assert len(t) == 70000 and len(widths) == 50 and maxd == 8400 and t.max() - t.min() > 1400
    be = _backend()
    cur = CurveOnDevice(t, y, dy, lc, ov)
    sub = P[np.linspace(0, len(P) - 1, 512).astype(int)]
    chi2, loc = cur.search(sub, 1e-5, 8, 16, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(be, sub, t, y, dy, widths, tm, os_, maxd, 1e-5, 8, 16)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL64)
    np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)
    few = sub[[0, 73, 146, 219, 292, 365, 438, 511]]
    chi2, loc = cur.search(few, 1e-5, 8, 1, _lib.GTLS_PASS_ALL, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(be, few, t, y, dy, widths, tm, os_, maxd, 1e-5, 8, 1, noskip=True)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL64)
    np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)


def test_cfg2_fold_order_is_the_stable_argsort(cuda):
    from gtls_b200 import _lib
    t, y, dy, P, *_ = _cfg2_inputs()
    sub = P[np.linspace(0, len(P) - 1, 16).astype(int)]
    order = _lib.fold_order(cuda.tensor(t, device="cuda"), cuda.tensor(sub, device="cuda")).cpu().numpy()
    for i, p in enumerate(sub):
        np.testing.assert_array_equal(order[i], np.argsort(O.fold_phases(t, p), kind="stable"))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_cfg3_fp32_form_agrees_with_the_fp64_oracle(cuda, seed):
    from gtls_b200 import gtls, synthetic
    t, y, dy, _ = synthetic.light_curve_cfg3(seed)
    model = gtls(t, y, dy, verbose=False)
    res = model.power(period_min=0.5, period_max=13.7, oversampling_factor=3, precision="fp32")
    ref = _oracle_search(model, res)
    _assert_same_search(res, ref, rtol_chi2=RTOL32, rtol_sde=1e-4)
    np.testing.assert_allclose([res.depth, res.T0, res.duration], [ref["depth"], ref["T0"], ref["duration"]],
                               rtol=RTOL64)


def test_tess_sector58_reference_call_matches_the_reference_flow(cuda):
    from conftest import golden
    from gtls_b200 import gtls, validate as V
    f = golden("tess_s58")
    t, y, dy = V.cleaned_array(f["time"], f["pdcsap_flux"], f["pdcsap_flux_err"])
    y = y / np.nanmean(y)
    model = gtls(t, y, dy, verbose=False)
    res = model.power(periods=np.linspace(1, 14, 10000))
    assert len(model.t) > 15000
    ref = _oracle_search(model, res)
    _assert_same_search(res, ref)
    assert res.diagnostics["loc"] == ref["loc"]
    assert list(res.possiblePeriodsIndices) == list(ref["candidates"])
    np.testing.assert_allclose(res.diagnostics["chi2_main"], ref["chi2_main"], rtol=RTOL64)
    np.testing.assert_allclose([res.depth, res.T0, res.duration], [ref["depth"], ref["T0"], ref["duration"]],
                               rtol=RTOL64)
