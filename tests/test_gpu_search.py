"""CUDA search kernels against the oracle and the reference's recorded outputs.

Bars: FP64 chi2 within 1e-9 relative of the FP64 oracle and identical argmin
(duration, start) locations; FP32 chi2 within 2e-6 relative.
"""
import numpy as np
import pytest

import tls_oracle as O
from conftest import golden, search_inputs

pytestmark = pytest.mark.gpu
RTOL64 = 1e-9
RTOL32 = 2e-6


def _curve(s):
    from gtls_b200.core import CurveOnDevice
    return CurveOnDevice(s["t"], s["y"], s["dy"], s["lc"], s["ov"])


def test_period_grid_within_one_ulp_of_reference(cuda):
    from gtls_b200 import grid as G
    g = golden("grid")
    for i in range(6):
        rs, ms, span, pmin, pmax, osf, ntr = g["case%d_args" % i]
        ref = g["case%d_periods" % i]
        if len(ref) < 100:
            continue
        ours = G.period_grid(rs, ms, span, pmin, pmax, int(osf), int(ntr))
        assert len(ours) == len(ref)
        # the device cube is correctly rounded; NumPy's SIMD pow is within ~1 ulp,
        # and 1/f/86400 adds two roundings on both sides
        np.testing.assert_array_almost_equal_nulp(ours, ref, nulp=2)
        assert np.mean(ours == ref) > 0.9


def test_duration_ranges_equal_oracle(cuda):
    from gtls_b200 import _lib
    s = search_inputs(seed=3, n=19728, span=27.4)
    span = s["t"].max() - s["t"].min()
    a = _lib.duration_ranges(s["periods"], span, len(s["t"]))
    b = O.duration_ranges(s["periods"], span, len(s["t"]))
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("use_dy,batch", [(False, 1), (False, 7), (True, 5), (True, 1000)])
def test_main_pass_fp64_matches_oracle(cuda, use_dy, batch):
    from gtls_b200 import _lib
    s = search_inputs(seed=11, n=1100, span=6.0, use_dy=use_dy)
    cur = _curve(s)
    P = s["periods"][::3]
    chi2, loc = cur.search(P, 1e-5, 8, batch, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                    s["overshoot"], s["maxd"], 1e-5, 8, batch)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL64)
    np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)


@pytest.mark.parametrize("use_dy", [False, True])
def test_all_starts_pass_fp64_matches_oracle(cuda, use_dy):
    from gtls_b200 import _lib
    s = search_inputs(seed=12, n=900, span=5.0, use_dy=use_dy)
    cur = _curve(s)
    P = s["periods"][::9]
    chi2, loc = cur.search(P, 1e-5, 8, 4, _lib.GTLS_PASS_ALL, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                    s["overshoot"], s["maxd"], 1e-5, 8, 4, noskip=True)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL64)
    np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)


@pytest.mark.parametrize("skip_point", [O.SKIP_NEVER, 10, 3])
def test_other_skip_points_match_oracle(cuda, skip_point):
    from gtls_b200 import _lib
    s = search_inputs(seed=13, n=700, span=4.0)
    cur = _curve(s)
    P = s["periods"][::11]
    chi2, loc = cur.search(P, 1e-5, skip_point, 3, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                    s["overshoot"], s["maxd"], 1e-5, skip_point, 3)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL64)
    np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)


@pytest.mark.parametrize("skip_point", [2, 5])
def test_small_skips_both_precisions_match_oracle(cuda, skip_point):
    """Skips 1..31 take the lane path: groups whose starts all lie in the tile
    read unclamped (tile pad), the last group of a tile reads clamped."""
    from gtls_b200 import _lib
    s = search_inputs(seed=16, n=1333, span=6.0, use_dy=True)
    cur = _curve(s)
    P = s["periods"][::7]
    c_ref, l_ref = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                    s["overshoot"], s["maxd"], 1e-5, skip_point, 5)
    for prec, rtol in (("fp64", RTOL64), ("fp32", RTOL32)):
        chi2, loc = cur.search(P, 1e-5, skip_point, 5, _lib.GTLS_PASS_MAIN, prec, want_loc=True)
        np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=rtol)
        if prec == "fp64":
            np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)


def test_all_starts_pass_fp32_close_to_oracle(cuda):
    from gtls_b200 import _lib
    s = search_inputs(seed=17, n=1001, span=5.0)
    cur = _curve(s)
    P = s["periods"][::13]
    chi2, _ = cur.search(P, 1e-5, 8, 4, _lib.GTLS_PASS_ALL, "fp32")
    c_ref, _ = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                s["overshoot"], s["maxd"], 1e-5, 8, 4, noskip=True)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL32)


def test_matches_reference_kernel_fixtures(cuda):
    """Against the reference's own kernels (recorded R64 outputs), per period with its own durations."""
    import torch
    from gtls_b200 import _lib
    k = golden("kernels")
    for i in range(3):
        t, y, dy = k["case%d_t" % i], k["case%d_y" % i], k["case%d_dy" % i]
        widths = k["case%d_widths" % i]
        maxd = int(k["case%d_maxd" % i][0])
        tm = np.ones((len(widths), maxd))
        tm[:, : k["case%d_templates" % i].shape[1]] = k["case%d_templates" % i]
        dev = torch.device("cuda")
        curve = dict(t=torch.from_numpy(t).to(dev), y=torch.from_numpy(y).to(dev), dy=torch.from_numpy(dy).to(dev),
                     span=float(np.float32(t.max() - t.min())))
        tables = dict(widths=torch.from_numpy(widths.astype(np.int32)).to(dev),
                      overshoot=torch.from_numpy(k["case%d_overshoot" % i]).to(dev),
                      templates=torch.from_numpy(tm).to(dev), max_width=maxd)
        P = torch.from_numpy(k["case%d_periods" % i]).to(dev)
        ref = k["case%d_r64" % i]
        c1, l1 = _lib.search(curve, P, tables, 1e-5, 8, 1, _lib.GTLS_PASS_MAIN, "fp64")
        c2, l2 = _lib.search(curve, P, tables, 1e-5, 8, 1, _lib.GTLS_PASS_ALL, "fp64")
        np.testing.assert_allclose(c1.cpu().numpy(), ref[:, 0], rtol=RTOL64)
        np.testing.assert_array_equal(l1.cpu().numpy(), ref[:, 1].astype(np.int64))
        np.testing.assert_allclose(c2.cpu().numpy(), ref[:, 2], rtol=RTOL64)
        np.testing.assert_array_equal(l2.cpu().numpy(), ref[:, 3].astype(np.int64))
        c3, _ = _lib.search(curve, P, tables, 1e-5, 8, 1, _lib.GTLS_PASS_MAIN, "fp32")
        np.testing.assert_allclose(c3.cpu().numpy(), ref[:, 0], rtol=RTOL32)


def test_fp32_main_pass_close_to_fp64(cuda):
    from gtls_b200 import _lib
    s = search_inputs(seed=14, n=19728, span=27.4)
    cur = _curve(s)
    P = s["periods"][::5]
    c64, l64 = cur.search(P, 1e-5, 8, 83, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    c32, l32 = cur.search(P, 1e-5, 8, 83, _lib.GTLS_PASS_MAIN, "fp32", want_loc=True)
    c64, c32 = c64.cpu().numpy(), c32.cpu().numpy()
    np.testing.assert_allclose(c32, c64, rtol=RTOL32)
    assert np.mean(l64.cpu().numpy() == l32.cpu().numpy()) > 0.98


def test_empty_union_gives_nan(cuda):
    """A batch whose periods admit none of the widths gets NaN (core.py:722-729)."""
    from gtls_b200 import _lib
    s = search_inputs(seed=15, n=800, span=5.0)
    cur = _curve(s)
    P = np.array([0.6, 0.61, 2.5e4, 2.6e4])   # very long periods: every width above wmax
    chi2, loc = cur.search(P, 1e-5, 8, 2, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    wmin, wmax = O.duration_ranges(P, s["t"].max() - s["t"].min(), len(s["t"]))
    c = chi2.cpu().numpy()
    if np.all(s["widths"].min() > wmax[2:]):
        assert np.all(np.isnan(c[2:])) and np.all(loc.cpu().numpy()[2:] == -1)
    assert np.all(np.isfinite(c[:2]))


def test_spectra_matches_reference_stats(cuda):
    import torch
    from gtls_b200 import _lib
    sp = golden("spectra")
    for i in range(4):
        n, osf = sp["case%d" % i]
        chi2 = torch.from_numpy(sp["case%d_chi2" % i]).cuda()
        m = sp["case%d_mask" % i]
        mask = torch.from_numpy(m.astype(np.uint8)).cuda() if m.any() else None
        SR, praw, power, sde_raw, sde = _lib.spectra(chi2, mask, float(osf))
        np.testing.assert_allclose(SR.cpu().numpy()[~m], sp["case%d_SR" % i][~m], rtol=1e-12)
        np.testing.assert_allclose(power.cpu().numpy()[~m], sp["case%d_power" % i][~m], rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose([sde_raw, sde], sp["case%d_sde" % i], rtol=1e-9)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_all_durations_flag_reproduces_a_batch_union(cuda, precision):
    """Re-searching some periods of a batch over that batch's duration union
    (GTLS_SEARCH_ALL_DURATIONS) gives exactly their values in the full search."""
    import torch
    from gtls_b200 import _lib
    from gtls_b200.core import subset_tables
    s = search_inputs(seed=33, n=1200, span=6.0, use_dy=True)
    cur = _curve(s)
    P = s["periods"][::17][:21]
    S = 7
    full, floc = cur.search(P, 1e-5, 8, S, _lib.GTLS_PASS_ALL, precision, want_loc=True)
    full, floc = full.cpu().numpy(), floc.cpu().numpy()
    span = s["t"].max() - s["t"].min()
    wmin, wmax = O.duration_ranges(P, span, len(s["t"]))
    valid = (s["widths"][None, :] >= wmin[:, None]) & (s["widths"][None, :] <= wmax[:, None])
    for b, sub in [(0, [3, 5]), (1, [7]), (2, [14, 15, 20])]:
        union = np.nonzero(valid[b * S:(b + 1) * S].any(axis=0))[0]
        c, l = cur.search(P[sub], 1e-5, 8, len(sub), _lib.GTLS_PASS_ALL, precision, want_loc=True,
                          tables=subset_tables(cur.tables, union, torch), flags=_lib.GTLS_SEARCH_ALL_DURATIONS)
        np.testing.assert_array_equal(c.cpu().numpy(), full[sub])
        np.testing.assert_array_equal(l.cpu().numpy(), floc[sub])


def test_fp32_form_rechecks_its_best_candidates_in_fp64(cuda):
    from gtls_b200 import gtls, synthetic
    t, y, _ = synthetic.small_curve(seed=34, n=2500, span=9.0, period=1.7, depth=5e-3)
    kw = dict(oversampling_factor=2, batch_periods=40, use_threads=1)
    r32 = gtls(t, y, verbose=False).power(precision="fp32", **kw)
    r64 = gtls(t, y, verbose=False).power(precision="fp64", **kw)
    re = np.asarray(r32.diagnostics["fp64_rechecked"])
    assert len(re) == 32
    assert list(r32.possiblePeriodsIndices) == list(r64.possiblePeriodsIndices)
    c32 = np.ma.filled(r32.chi2, np.nan)
    c64 = np.ma.filled(r64.chi2, np.nan)
    np.testing.assert_array_equal(c32[re], c64[re])
    assert r32.period == r64.period and r32.durationPoints == r64.durationPoints
    assert abs(r32.SDE - r64.SDE) <= 1e-6 * abs(r64.SDE)


def test_search_rejects_invalid_arguments_and_stays_usable(cuda):
    from gtls_b200 import _lib
    s = search_inputs(seed=35, n=600, span=4.0)
    cur = _curve(s)
    P = s["periods"][::20]
    with pytest.raises(_lib.GtlsError, match="flags"):
        cur.search(P, 1e-5, 8, 3, _lib.GTLS_PASS_MAIN, "fp64", flags=4)
    with pytest.raises(_lib.GtlsError, match="pass"):
        cur.search(P, 1e-5, 8, 3, 7, "fp64")
    with pytest.raises(_lib.GtlsError, match="skip_point"):
        cur.search(P, 1e-5, 0, 3, _lib.GTLS_PASS_MAIN, "fp64")
    with pytest.raises(_lib.GtlsError, match="batch"):
        cur.search(P, 1e-5, 8, 0, _lib.GTLS_PASS_MAIN, "fp64")
    with pytest.raises(ValueError):
        cur.search(np.array([0.0, 1.0]), 1e-5, 8, 3, _lib.GTLS_PASS_MAIN, "fp64")
    c, _ = cur.search(P, 1e-5, 8, 3, _lib.GTLS_PASS_MAIN, "fp64")
    c_ref, _ = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                s["overshoot"], s["maxd"], 1e-5, 8, 3)
    np.testing.assert_allclose(c.cpu().numpy(), c_ref, rtol=RTOL64)


def test_fold_order_is_the_stable_argsort_of_the_phases(cuda):
    """The fold ordering, bit for bit: np.argsort(phase, kind="stable") of the
    reference's foldFast phases, including clustered phases (regular cadence,
    periods near multiples of it) and exact ties (repeated times)."""
    import torch
    from gtls_b200 import _lib
    rng = np.random.default_rng(9)
    cad = 10.0 / 1440.0
    cases = [
        np.sort(rng.uniform(100.0, 400.0, 3000)),                      # random sampling
        100.0 + np.arange(5000) * cad,                                  # regular cadence
        np.repeat(100.0 + np.arange(800) * 0.01, 3),                    # exact ties
    ]
    for t in cases:
        P = np.concatenate([np.exp(rng.uniform(np.log(0.5), np.log(50.0), 40)),
                            cad * np.array([72.0, 144.0, 1000.0]) * (1 + np.array([1e-9, -3e-8, 0.0]))])
        dev = torch.device("cuda:0")
        got = _lib.fold_order(torch.from_numpy(t).to(dev), torch.from_numpy(P).to(dev)).cpu().numpy()
        for i, p in enumerate(P):
            ref = np.argsort(O.fold_phases(t, p), kind="stable")
            np.testing.assert_array_equal(got[i], ref, err_msg="period %r" % p)


def test_clustered_phases_take_the_global_ordering_and_match_the_oracle(cuda):
    """12,000 of 40,000 samples within a millisecond: for every period they
    share one phase bucket, more than the shared-memory ordering holds in a
    round, so the period falls back to the global-scatter ordering.  The fold
    order is still the stable argsort, and the FP64 main pass (records and
    prefix from that path) matches the oracle."""
    import torch
    from gtls_b200 import _lib, template, grid as G, validate as V
    from gtls_b200.core import CurveOnDevice
    rng = np.random.default_rng(5)
    t = np.sort(np.concatenate([100.0 + np.arange(28000) * (2.0 / 1440.0), 110.3 + np.arange(12000) * 8.3e-12]))
    y = 1.0 + rng.normal(0, 1e-3, len(t))
    dy = np.full(len(t), 1e-3)
    t, y, dy = V.validate_inputs(t, y, dy)
    P = np.array([0.5, 1.0, 1.7, 3.1, 7.3])
    for p in P:
        assert np.bincount(np.floor(O.fold_phases(t, p) * 16384).astype(int)).max() > 12000 - 100
    dev = torch.device("cuda:0")
    got = _lib.fold_order(torch.from_numpy(t).to(dev), torch.from_numpy(P).to(dev)).cpu().numpy()
    for i, p in enumerate(P):
        np.testing.assert_array_equal(got[i], np.argsort(O.fold_phases(t, p), kind="stable"), err_msg="period %r" % p)
    durs = G.duration_grid(np.sort(O.period_grid(1, 1, t.max() - t.min())), shortest=1 / len(t), log_step=1.1)
    mw = int(np.max(durs) * len(y))
    mw += mw % 2
    ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    widths, os_, _, tm, maxd = template.device_templates(lc, ov)
    cur = CurveOnDevice(t, y, dy, lc, ov)
    chi2, loc = cur.search(P, 1e-5, 8, 5, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(O.NumpyBackend(), P, t, y, dy, widths, tm, os_, maxd, 1e-5, 8, 5)
    np.testing.assert_allclose(chi2.cpu().numpy(), c_ref, rtol=RTOL64)
    np.testing.assert_array_equal(loc.cpu().numpy(), l_ref)
