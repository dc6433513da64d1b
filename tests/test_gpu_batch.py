"""Batched search (gtls_search_batch, gtls_batch) against single-curve searches
and the oracle.

Curves in one batched call are independent searches: every chi2 and argmin
location must equal, bit for bit, what gtls_search gives for that curve
alone, whatever the chunking of the period list, and the FP64 values must
match the oracle within 1e-9 relative.
"""
import numpy as np
import pytest

import tls_oracle as O
from conftest import search_inputs

pytestmark = pytest.mark.gpu
RTOL64 = 1e-9

# (seed, samples, span in days): uneven lengths, grids and duration tables
CURVES = [(21, 1200, 6.0), (22, 700, 4.0), (23, 1900, 9.0), (24, 950, 5.0)]


def _inputs():
    return [search_inputs(seed=s, n=n, span=sp, use_dy=(s % 2 == 0)) for s, n, sp in CURVES]


def _prepared(s, periods):
    return dict(t=s["t"], y=s["y"], dy=s["dy"], periods=periods, span=float(np.float32(s["t"].max() - s["t"].min())),
                widths=s["widths"], overshoot=s["overshoot"], durations=s["dur_u"], tmpl=s["templates"],
                maxd=int(s["maxd"]))


def _single(s):
    from gtls_b200.core import CurveOnDevice
    return CurveOnDevice(s["t"], s["y"], s["dy"], s["lc"], s["ov"])


@pytest.fixture
def budget(cuda):
    from gtls_b200 import _lib
    yield _lib.set_chunk_budget
    _lib.set_chunk_budget(8 << 30)


@pytest.mark.parametrize("precision,pass_name,chunk_mb", [
    ("fp64", "MAIN", 8192), ("fp64", "MAIN", 2), ("fp32", "MAIN", 3), ("fp64", "ALL", 2), ("fp32", "ALL", 8192)])
def test_batch_equals_single_curve_searches(cuda, budget, precision, pass_name, chunk_mb):
    from gtls_b200 import _lib
    from gtls_b200.batch import CurveSetOnDevice
    budget(chunk_mb << 20)
    pass_ = getattr(_lib, "GTLS_PASS_" + pass_name)
    ins = _inputs()
    plist = [s["periods"][i::5] for i, s in enumerate(ins)]
    batches = np.array([1, 7, 3, 1000], dtype=np.int32)
    cs = CurveSetOnDevice([_prepared(s, p) for s, p in zip(ins, plist)])
    off = np.concatenate([[0], np.cumsum([len(p) for p in plist])])
    chi2, loc = cs.search(np.concatenate(plist), off, 1e-5, 8, batches, pass_, precision, want_loc=True)
    chi2, loc = chi2.cpu().numpy(), loc.cpu().numpy()
    for c, s in enumerate(ins):
        c1, l1 = _single(s).search(plist[c], 1e-5, 8, int(batches[c]), pass_, precision, want_loc=True)
        np.testing.assert_array_equal(chi2[off[c]:off[c + 1]], c1.cpu().numpy())
        np.testing.assert_array_equal(loc[off[c]:off[c + 1]], l1.cpu().numpy())


def test_batch_fp64_matches_oracle(cuda, budget):
    from gtls_b200 import _lib
    from gtls_b200.batch import CurveSetOnDevice
    budget(2 << 20)
    ins = _inputs()
    plist = [s["periods"][1::7] for s in ins]
    batches = np.array([5, 2, 9, 1], dtype=np.int32)
    cs = CurveSetOnDevice([_prepared(s, p) for s, p in zip(ins, plist)])
    off = np.concatenate([[0], np.cumsum([len(p) for p in plist])])
    chi2, loc = cs.search(np.concatenate(plist), off, 1e-5, 8, batches, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    chi2, loc = chi2.cpu().numpy(), loc.cpu().numpy()
    for c, s in enumerate(ins):
        c_ref, l_ref = O.search_periods(O.NumpyBackend(), plist[c], s["t"], s["y"], s["dy"], s["widths"],
                                        s["templates"], s["overshoot"], s["maxd"], 1e-5, 8, int(batches[c]))
        np.testing.assert_allclose(chi2[off[c]:off[c + 1]], c_ref, rtol=RTOL64)
        np.testing.assert_array_equal(loc[off[c]:off[c + 1]], l_ref)


def test_batch_with_empty_period_list(cuda):
    """A curve with no periods contributes nothing; the others are unaffected."""
    from gtls_b200 import _lib
    from gtls_b200.batch import CurveSetOnDevice
    ins = _inputs()[:3]
    plist = [ins[0]["periods"][::9], np.zeros(0), ins[2]["periods"][::9]]
    cs = CurveSetOnDevice([_prepared(s, p) for s, p in zip(ins, plist)])
    off = np.concatenate([[0], np.cumsum([len(p) for p in plist])])
    chi2, loc = cs.search(np.concatenate(plist), off, 1e-5, 8, np.array([3, 3, 3], np.int32), _lib.GTLS_PASS_MAIN,
                          "fp64", want_loc=True)
    for c in (0, 2):
        c1, l1 = _single(ins[c]).search(plist[c], 1e-5, 8, 3, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
        np.testing.assert_array_equal(chi2.cpu().numpy()[off[c]:off[c + 1]], c1.cpu().numpy())


def test_batch_rejects_curve_without_durations(cuda):
    from gtls_b200 import _lib
    from gtls_b200.batch import CurveSetOnDevice
    ins = _inputs()[:2]
    plist = [s["periods"][::9] for s in ins]
    cs = CurveSetOnDevice([_prepared(s, p) for s, p in zip(ins, plist)])
    cs.tables["dur_off"] = np.array([0, 0, cs.dur_off[2]], dtype=np.int64)
    off = np.concatenate([[0], np.cumsum([len(p) for p in plist])])
    with pytest.raises(_lib.GtlsError, match="duration"):
        cs.search(np.concatenate(plist), off, 1e-5, 8, np.array([3, 3], np.int32), _lib.GTLS_PASS_MAIN, "fp64")


def _light_curves():
    from gtls_b200 import synthetic
    out = []
    for i, (seed, n, span) in enumerate([(31, 1500, 6.0), (32, 2400, 9.0), (33, 1100, 5.0)]):
        t, y, _ = synthetic.small_curve(seed=seed, n=n, span=span, period=1.3 + 0.4 * i, depth=4e-3)
        out.append((t, y))
    return out


def test_gtls_batch_power_equals_gtls_power(cuda):
    from gtls_b200 import gtls
    from gtls_b200.batch import gtls_batch
    curves = _light_curves()
    kw = dict(precision="fp64", batch_periods=20, oversampling_factor=2, use_threads=1)
    # the same (host-built) template tables on both sides: the batched engine
    # must give bitwise the single-curve results
    res = gtls_batch(curves).power(templates="host", **kw)
    for (t, y), r in zip(curves, res):
        ref = gtls(t, y, verbose=False).power(**kw)
        assert r.period == ref.period
        assert r.SDE == ref.SDE
        assert r.duration == ref.duration
        assert r.depth == ref.depth
        assert r.T0 == ref.T0
        np.testing.assert_array_equal(np.ma.filled(r.power, -1.0), np.ma.filled(ref.power, -1.0))
        np.testing.assert_array_equal(np.ma.filled(r.chi2, -1.0), np.ma.filled(ref.chi2, -1.0))


def test_gtls_batch_full_stats_equal_gtls(cuda):
    from gtls_b200 import gtls
    from gtls_b200.batch import gtls_batch
    curves = _light_curves()[:2]
    kw = dict(precision="fp64", batch_periods=20, oversampling_factor=2, use_threads=1)
    res = gtls_batch(curves).power(full_stats=True, templates="host", **kw)
    for (t, y), r in zip(curves, res):
        ref = gtls(t, y, verbose=False).power(**kw)
        np.testing.assert_array_equal(r.transit_times, ref.transitTimes)
        for a, b in (("snr", "snr"), ("snr_pink", "snrPink"), ("snr_fit", "snrFit"), ("snr_fit_pink", "snrFitPink")):
            assert getattr(r, a) == getattr(ref, b) or (np.isnan(getattr(r, a)) and np.isnan(getattr(ref, b)))


def test_gtls_batch_fp32_finds_the_fp64_period(cuda):
    from gtls_b200.batch import gtls_batch
    curves = _light_curves()
    kw = dict(batch_periods=20, oversampling_factor=2, use_threads=1)
    r32 = gtls_batch(curves).power(precision="fp32", **kw)
    r64 = gtls_batch(curves).power(precision="fp64", **kw)
    for a, b in zip(r32, r64):
        assert a.period_index == b.period_index
        assert a.width == b.width
        assert abs(a.SDE - b.SDE) <= 1e-4 * abs(b.SDE)
