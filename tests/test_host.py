"""Host-side logic against the reference's pure-Python modules (golden fixtures)."""
import numpy as np

from conftest import golden
from gtls_b200 import grid as G, template, validate as V


def test_validate_inputs_matches_reference():
    v = golden("validate")
    t1, y1, dy1 = V.validate_inputs(v["t"].copy(), v["y"].copy(), v["dy"].copy())
    np.testing.assert_array_equal(t1, v["t1"])
    np.testing.assert_array_equal(y1, v["y1"])
    np.testing.assert_array_equal(dy1, v["dy1"])
    t2, y2, dy2 = V.validate_inputs(v["t"].copy(), v["y"].copy(), None)
    np.testing.assert_array_equal(t2, v["t2"])
    np.testing.assert_array_equal(dy2, v["dy2"])


def test_validate_errors():
    import pytest
    with pytest.raises(ValueError):
        V.validate_inputs(np.array([1.0, 2.0]), np.array([1.0, 1.0]), None)
    with pytest.raises(ValueError):
        V.validate_inputs(np.array([1.0, 1.0, 1.0]), np.array([1.0, 1.0, 1.0]), None)

    class A:
        pass
    with pytest.raises(ValueError):
        V.validate_args(A(), {"R_star": -1})
    with pytest.raises(ValueError):
        V.validate_args(A(), {"transit_template": "nope"})
    a, _ = V.validate_args(A(), {"T0_fit_margin": 0.5})
    assert a.T0_fit_margin == 0.125


def test_duration_grid_matches_reference():
    g = golden("grid")
    for i in range(6):
        p = g["case%d_periods" % i]
        d = G.duration_grid(p, shortest=1 / 19728, log_step=1.1)
        np.testing.assert_array_equal(np.asarray(d), g["case%d_durations" % i])


def test_ofir_coefficients_reproduce_reference_grid_within_one_ulp():
    g = golden("grid")
    for i in range(6):
        rs, ms, span, pmin, pmax, osf, ntr = g["case%d_args" % i]
        ref = g["case%d_periods" % i]
        a3, c, npts, _ = G.ofir_coefficients(rs, ms, span, osf, int(ntr))
        X = np.arange(npts) + 1.0
        p = 1 / (a3 * X + c) ** 3 / 86400
        p = p[(p > pmin) & (p <= pmax)]
        if len(ref) >= 100:
            np.testing.assert_array_almost_equal_nulp(p, ref, nulp=1)


def test_default_period_grid_is_bitwise_the_reference_grid():
    """The default (host) evaluation of power()'s grid: the reference's
    grid.period_grid outputs bit for bit, fallback grids included."""
    g = golden("grid")
    for i in range(6):
        rs, ms, span, pmin, pmax, osf, ntr = g["case%d_args" % i]
        ours = G.period_grid(rs, ms, span, pmin, pmax, int(osf), int(ntr))
        np.testing.assert_array_equal(ours, g["case%d_periods" % i])
        asc = G.period_grid(rs, ms, span, pmin, pmax, int(osf), int(ntr), ascending=True)
        np.testing.assert_array_equal(asc, g["case%d_periods" % i][::-1])


def test_template_cache_matches_reference_get_cache():
    c = golden("cache")
    for i in range(2):
        durations = c["case%d_durations" % i]
        mw = int(c["case%d_maxw" % i][0])
        base = template.reference_transit(mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
        np.testing.assert_array_equal(base, c["case%d_base" % i])
        ov, lc = template.get_cache(durations, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
        np.testing.assert_array_equal(ov["width_in_samples"], c["case%d_width" % i])
        np.testing.assert_array_equal(ov["overshoot"], c["case%d_overshoot" % i])
        np.testing.assert_array_equal(np.concatenate(list(lc)), c["case%d_lc" % i])


def test_device_templates_layout():
    c = golden("cache")
    durations = c["case0_durations"]
    mw = int(c["case0_maxw"][0])
    ov, lc = template.get_cache(durations, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    widths, os_, dd, tm, maxd = template.device_templates(lc, ov)
    assert np.all(np.diff(widths) > 0) and maxd % 2 == 0 and maxd >= widths.max()
    for d in range(len(widths)):
        n = len(lc[d])
        np.testing.assert_array_equal(tm[d, :n], 1 - lc[d])
        assert np.all(tm[d, n:] == 1.0)   # 1 - zero padding (core.py:753-754)


def test_candidate_selection_matches_reference_sort():
    import torch
    import tls_oracle as O
    from gtls_b200.core import _candidates
    rng = np.random.default_rng(0)
    for n in (50, 400, 3000):
        periods = np.sort(rng.uniform(0.5, 20, n))
        power = rng.normal(0, 1, n)
        power[rng.integers(0, n, 5)] = power[3]   # ties keep index order
        idx, _ = O.select_candidates(np.ma.array(periods), np.ma.array(power))
        ours = _candidates(torch.from_numpy(power), torch.zeros(n, dtype=torch.uint8), torch.from_numpy(periods),
                           torch)
        assert list(ours) == list(idx)


def test_fp64_recheck_plan_uses_each_batch_union(monkeypatch):
    """The FP32 form re-checks its best candidates over exactly the duration
    union of their batch of the candidate list (core.py:1081-1115 groups the
    candidates in batches of S)."""
    import tls_oracle as O
    from gtls_b200 import _lib, core
    monkeypatch.setattr(_lib, "duration_ranges", lambda p, span, n, device=0: O.duration_ranges(np.asarray(p), span, n))
    rng = np.random.default_rng(5)
    cand_p = np.exp(rng.uniform(np.log(0.6), np.log(300.0), 60))
    power = rng.normal(size=60)
    power[7] = np.nan
    widths = np.unique(rng.integers(5, 4000, 40)).astype(np.int64)
    n, span, S = 20000, np.float32(800.0), 25
    plan = core.recheck_plan(cand_p, power, widths, span, n, S, device=0, k=10)
    chosen = np.sort(np.concatenate([sel for sel, _ in plan]))
    order = np.argsort(np.where(np.isfinite(power), -power, np.inf), kind="stable")
    np.testing.assert_array_equal(chosen, np.sort(order[:10]))
    wmin, wmax = O.duration_ranges(cand_p, span, n)
    valid = (widths[None, :] >= wmin[:, None]) & (widths[None, :] <= wmax[:, None])
    for sel, union in plan:
        g = sel[0] // S
        assert np.all(sel // S == g)
        np.testing.assert_array_equal(union, np.nonzero(valid[g * S:(g + 1) * S].any(axis=0))[0])
    assert 7 not in chosen


def test_phases_accumulate_per_name(monkeypatch):
    """core.Phases: wall-clock seconds per phase name, summed over repeated
    marks; a no-op without a dict (no device synchronisation either)."""
    import torch
    from gtls_b200.core import Phases
    calls = []
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a: calls.append(1))
    out = {}
    ph = Phases(out)
    ph.mark("a")
    ph.mark("b")
    ph.mark("a")
    assert set(out) == {"a", "b"} and all(v >= 0.0 for v in out.values())
    assert len(calls) == 4
    calls.clear()
    Phases(None).mark("x")
    assert calls == []


def _transit_fluxes_by_mask(t, y, mids, dur):
    out = []
    for mid in mids:
        a, b = mid - 0.5 * dur, mid + 0.5 * dur
        out.append(None if np.isnan(a) or np.isnan(b) else y[np.logical_and(t > a, t < b)])
    return out


def test_transit_fluxes_equal_the_mask():
    """stats._transit_fluxes (binary search on sorted times) selects the
    samples the reference's per-transit mask selects, in the same order,
    including bounds that fall exactly on sample times, repeated times,
    transits outside the data, NaN mid-times and unsorted times."""
    from gtls_b200 import stats
    rng = np.random.default_rng(5)
    t = np.sort(rng.uniform(0.0, 30.0, 4000))
    t[100:110] = t[100]                                   # repeated times
    y = rng.normal(1.0, 1e-3, len(t))
    dur = 0.125
    mids = list(np.arange(-1.0, 32.0, 0.7)) + [t[500] + 0.5 * dur, t[900] - 0.5 * dur, np.nan, t[100]]
    for tt in (t, t[rng.permutation(len(t))]):
        yy = y if tt is t else y[np.argsort(np.argsort(tt))]
        got = stats._transit_fluxes(tt, yy, mids, dur)
        want = _transit_fluxes_by_mask(tt, yy, mids, dur)
        assert len(got) == len(want)
        for g, w in zip(got, want):
            assert (g is None) == (w is None)
            if g is not None:
                np.testing.assert_array_equal(g, w)


def test_pink_noise_matches_per_window_std():
    """stats.pink_noise (prefix sums in extended precision) against the
    reference's loop over windows (stats.py:426-431: the mean over windows of
    np.std(window) / sqrt(width)), within 1e-12 relative."""
    import pytest
    from gtls_b200 import stats
    rng = np.random.default_rng(9)
    x = 1.0 + rng.normal(0.0, 1e-3, 5000)
    x[1000:1040] -= 2e-3                                  # a transit-like dip
    for data, width in ((x, 1), (x, 2), (x, 15), (x, 300), (x[:40], 40), (x[:3] * 0 + 1.0, 2)):
        n = len(data) - width + 1
        ref = sum(np.std(data[i:i + width]) / width ** 0.5 for i in range(n)) / n
        got = stats.pink_noise(data, width)
        assert abs(got - ref) <= 1e-12 * abs(ref) + 1e-300, (width, got, ref)
    with pytest.raises(ValueError):
        stats.pink_noise(x[:5], 6)


def test_calls_on_a_new_stream_wait_for_the_previous_one():
    """_lib._stream: a device's calls share one scratch arena, so a call on a
    different stream than the device's previous call first makes its stream
    wait for the previous one (no wait while the stream stays the same)."""
    import types
    from gtls_b200 import _lib

    class FakeStream:
        def __init__(self, h):
            self.cuda_stream = h
            self.waited = []

        def __eq__(self, other):
            return self.cuda_stream == other.cuda_stream

        def __ne__(self, other):
            return not self == other

        def wait_stream(self, other):
            self.waited.append(other.cuda_stream)

    a, b = FakeStream(11), FakeStream(22)
    current = {"s": a}
    fake = types.SimpleNamespace(cuda=types.SimpleNamespace(current_stream=lambda device: current["s"]))
    saved = dict(_lib._last_stream)
    try:
        _lib._last_stream.clear()
        assert _lib._stream(fake, 5).value == 11 and a.waited == []
        assert _lib._stream(fake, 5).value == 11 and a.waited == []
        current["s"] = b
        assert _lib._stream(fake, 5).value == 22 and b.waited == [11]
        assert _lib._stream(fake, 6).value == 22 and b.waited == [11]      # other device: independent
    finally:
        _lib._last_stream.clear()
        _lib._last_stream.update(saved)


def test_bench_clock_summary_reads_throttle_reasons(tmp_path, monkeypatch):
    """bench.Clocks: median SM clock, max clock and the active throttle
    reasons from nvidia-smi's CSV samples; the raw file is kept only when
    GTLS_CLOCKS_DIR names a folder for it."""
    import os
    import sys
    from conftest import ROOT
    sys.path.insert(0, ROOT)
    import bench
    rows = ["0, 1965, 1965, 900.0, 0x0, Not Active, Not Active, Not Active, Active",
            "0, 1900, 1965, 990.0, 0x0, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    for keep in (False, True):
        if keep:
            monkeypatch.setenv("GTLS_CLOCKS_DIR", str(tmp_path))
        else:
            monkeypatch.delenv("GTLS_CLOCKS_DIR", raising=False)
        c = bench.Clocks(0)
        c.proc = object()                     # as if nvidia-smi had been started
        with open(c.path, "w") as f:
            f.write("\n".join(rows) + "\n")
        s = c.summary()
        assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
        assert s["reasons"] == ["sw_power_cap"]
        assert os.path.exists(c.path) == keep
        assert c.summary() == s


def _get_cache_per_duration(durations, mw, *planet):
    """The template cache one duration at a time (the reference's loop,
    transit.py:98-160, with fractional_transit's in-transit part)."""
    from gtls_b200 import constants
    ref = template.reference_transit(mw, *planet)
    dmax = np.max(durations)
    rt = np.linspace(-0.5, 0.5, mw)
    widths, overs, lcs = [], [], []
    for d in durations:
        occ = int((d / dmax) * mw)
        sc = 1 - ((1 - template.interp_linear(np.linspace(-0.5, 0.5, occ), rt, ref)) * constants.SIGNAL_DEPTH)
        full = np.nonzero(sc < 1 - constants.NUMERICAL_STABILITY_CUTOFF)[0]
        sig = sc[full[0]: full[-1] + 1]
        widths.append(int((d / dmax) * mw))
        overs.append(1 / (2 - np.mean(sig) / np.min(sig)))
        lcs.append(sig)
    return np.array(widths), np.array(overs), lcs


def test_template_cache_equals_the_per_duration_loop():
    """template.get_cache interpolates all durations in one pass: bitwise the
    values of the per-duration loop, on random duration grids and widths."""
    planet = (12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    rng = np.random.default_rng(4)
    for _ in range(6):
        mw = int(rng.integers(200, 6000)) * 2
        dmin = rng.uniform(0.002, 0.01)
        durations = dmin * 1.1 ** np.arange(int(rng.integers(5, 45)))
        ov, lc = template.get_cache(durations, mw, *planet, verbose=False)
        w_ref, o_ref, lc_ref = _get_cache_per_duration(durations, mw, *planet)
        np.testing.assert_array_equal(ov["width_in_samples"], w_ref)
        np.testing.assert_array_equal(ov["overshoot"], o_ref)
        np.testing.assert_array_equal(ov["duration"], durations)
        assert len(lc) == len(lc_ref)
        for a, b in zip(lc, lc_ref):
            np.testing.assert_array_equal(a, b)


def test_best_period_statistics_match_reference():
    """Depth, T0, duration, transit times, snr, snr_pink, snrFit and
    snrFitPink of a chi2 minimum (core.finish_stats) and the statistics
    functions one by one, against the reference's own stats.py/helpers.py
    (golden stats.npz).  pink_noise runs in O(N) from prefix sums here, so
    the pink-noise figures carry a 1e-12 bar; the rest is the same arithmetic."""
    from gtls_b200 import core, stats
    f = golden("stats")
    for i in range(3):
        period, loc, width, raw, ovs, maxd = f["case%d_inputs" % i]
        t, y = f["case%d_t" % i], f["case%d_y" % i]
        g = {k[len("case%d_" % i):]: f[k] for k in f.files if k.startswith("case%d_" % i)}
        out = core.finish_stats(t, y, period, int(loc), int(width), raw, ovs, int(maxd))
        for k in ("depth", "T0", "duration", "snr", "snr_fit", "snr_fit_pink"):
            np.testing.assert_allclose(out[k], g[k], rtol=1e-13, err_msg=k)
        np.testing.assert_allclose(out["snr_pink"], g["snr_pink"], rtol=1e-12)
        np.testing.assert_allclose(out["transit_times"], g["transit_times"], rtol=1e-15)
        tt, dur = g["transit_times"], float(g["duration"])
        ins = stats.intransit_stats(t, y, tt, dur)
        np.testing.assert_allclose(np.array(ins[:4], dtype=float), g["intransit"], rtol=1e-13)
        np.testing.assert_array_equal(ins[6], g["per_transit_count"])
        np.testing.assert_allclose(ins[7], g["transit_depths"], rtol=1e-15)
        np.testing.assert_allclose(ins[8], g["depth_uncertainties"], rtol=1e-13)
        snr_pt, snr_pink_pt = stats.snr_stats(t, y, period, raw, float(g["T0"]), tt, dur, ins[6])
        np.testing.assert_allclose(snr_pt, g["snr_per_transit"], rtol=1e-13)
        np.testing.assert_allclose(snr_pink_pt, g["snr_pink_per_transit"], rtol=1e-12)
        mask = stats.transit_mask(t, period, 2 * raw, float(g["T0"]))
        np.testing.assert_array_equal(mask, g["mask"])
        pink = [stats.pink_noise(y[~mask], w) for w in (1, 5, 37)]
        np.testing.assert_allclose(pink, g["pink"], rtol=1e-12, atol=1e-300)


def test_cfg3_oracle_fixture_matches_the_product_grid():
    """The FP64-oracle fixture of the mixed-precision workload (64 seeds)
    was made on the grids power() uses: same period count, and the recorded
    best period is the grid point at the recorded index."""
    from gtls_b200 import synthetic, validate as V
    f = golden("cfg3_oracle")
    assert int(f["n_seeds"]) == 64
    for seed in (0, 31, 63):
        t, y, dy, _ = synthetic.light_curve_cfg3(seed)
        t, y, dy = V.validate_inputs(t, y, dy)
        P = G.period_grid(1, 1, t.max() - t.min(), 0.5, 13.7, 3, 2, ascending=True)
        sc = f["seed%d_scalars" % seed]
        assert len(f["seed%d_chi2" % seed]) == len(P)
        assert P[int(sc[0])] == sc[1]


def test_autotune_sweep_and_choice(monkeypatch):
    """The tuner's sweep and choice, with the library replaced by a fake
    tuning store and made-up stage times: records mode and tile cap are
    swept for every curve, the bucket shift only above 2^17 samples (where
    the global-scatter ordering runs); the default stays unless another
    setting is faster by the margin."""
    from gtls_b200 import _lib, tune

    state = dict(tile_cap_fp32=16384, tile_cap_fp64=8192, bucket_shift=0, records_global=0)
    seen = []

    def set_tuning(device=0, **cfg):
        state.update(cfg)

    monkeypatch.setattr(_lib, "get_tuning", lambda device=0: dict(state))
    monkeypatch.setattr(_lib, "set_tuning", set_tuning)

    def make_run(times):
        def run(tm):
            key = (state["tile_cap_fp64"], state["records_global"], state["bucket_shift"])
            seen.append(key)
            tm.prepare_ms, tm.chi2_ms, tm.finish_ms = 1.0, times.get(key, 10.0), 0.0
        return run

    # a clearly faster global-records setting is chosen
    tune._CACHE.clear()
    best = tune.autotune(make_run({(10240, 1, 0): 8.0}), "fp64", n=70000, maxd=8400)
    assert (best["tile_cap_fp64"], best["records_global"]) == (10240, 1)
    assert {k[2] for k in seen} == {0}                      # no bucket sweep at 70,000 samples
    assert {(k[0], k[1]) for k in seen} == {(c, r) for c in tune.TILE_CAPS["fp64"] for r in (0, 1)}
    # within the margin the default is kept
    seen.clear()
    tune._CACHE.clear()
    best = tune.autotune(make_run({(10240, 1, 0): 9.9}), "fp64", n=70000, maxd=8400)
    assert (best["tile_cap_fp64"], best["records_global"], best["bucket_shift"]) == (8192, 0, 0)
    # above 2^17 samples the bucket shift is swept too
    seen.clear()
    tune._CACHE.clear()
    tune.autotune(make_run({}), "fp64", n=200000, maxd=8400)
    assert {k[2] for k in seen} == set(tune.BUCKET_SHIFTS)
    tune._CACHE.clear()
