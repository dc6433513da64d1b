"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout that has the reference tree and the CPU build of its
kernels (``make -C oracle``); the reference root is the first argument, else
the REFERENCE_ROOT environment variable:

    python tests/golden/make_golden.py [/path/to/reference]

What is recorded, and from which reference code:

* ``grid.npz``     -- grid.period_grid / grid.duration_grid (src/gputls/grid.py)
                     for several stellar parameters, spans and bounds;
* ``validate.npz`` -- validate.validate_inputs (src/gputls/validate.py) on
                     inputs holding NaN, zero, negative and None samples;
* ``spectra.npz``  -- stats.spectra (src/gputls/stats.py), plain and masked;
* ``cache.npz``    -- transit.get_cache (src/gputls/transit.py) with its batman
                     light curve replaced by this project's limb-darkening model
                     (batman is a third-party package outside the reference);
* ``stats.npz``    -- the statistics of the best period: stats.intransit_stats,
                     stats.snr_stats, stats.pink_noise, stats.all_transit_times,
                     stats.calcDurationDays and helpers.transit_mask
                     (src/gputls/stats.py:233-488, helpers.py:62-65), combined
                     as search_single_periods does (core.py:1427-1499: depth,
                     T0, duration, transit times, snr, snr_pink, snrFit,
                     snrFitPink; the snrFit lines are inline in core.py, which
                     imports cupy, so they are restated here in its order);
* ``kernels.npz``  -- per-period chi2 and argmin of the reference's CUDA kernels
                     (src/gputls/GPUFun.cu) compiled for the CPU and launched in
                     core.py's order (oracle/ref_replay.py), R64 and R32, for
                     small seeded curves, main pass and all-starts pass.

The fixtures let tests on machines without the reference tree compare against
the reference's own outputs.
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_reference(ref_root):
    src = os.path.join(ref_root, "src", "gputls")
    pkg = types.ModuleType("gputls")
    pkg.__path__ = [src]
    sys.modules["gputls"] = pkg
    sys.modules.setdefault("batman", types.ModuleType("batman"))   # only used by reference_transit
    mods = {}
    for name in ["version", "constants", "interpolation", "helpers", "grid", "stats", "validate", "transit"]:
        spec = importlib.util.spec_from_file_location("gputls." + name, os.path.join(src, name + ".py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules["gputls." + name] = m
        spec.loader.exec_module(m)
        mods[name] = m
    return mods


def main(ref_root):
    R = load_reference(ref_root)
    from gtls_b200 import synthetic, template, validate as V
    import tls_oracle as O
    import ref_replay as RR

    # ---- grids
    cases = [(1.0, 1.0, 27.4, 0, np.inf, 3, 2), (1.0, 1.0, 6.0, 0, np.inf, 3, 2), (0.5, 0.4, 80.0, 0.7, 20.0, 2, 3),
             (1.8, 1.3, 400.0, 0, np.inf, 1, 2), (1.0, 1.0, 3.0, 0, np.inf, 3, 2), (1.0, 1.0, 27.4, 0.5, 13.7, 3, 2)]
    g = {}
    for i, (rs, ms, span, pmin, pmax, osf, ntr) in enumerate(cases):
        p = R["grid"].period_grid(rs, ms, span, pmin, pmax, osf, ntr)
        g["case%d_args" % i] = np.array([rs, ms, span, pmin, pmax, osf, ntr], dtype=float)
        g["case%d_periods" % i] = np.asarray(p, dtype=float)
        g["case%d_durations" % i] = np.asarray(R["grid"].duration_grid(p, shortest=1 / 19728, log_step=1.1))
    np.savez_compressed(os.path.join(HERE, "grid.npz"), **g)

    # ---- validate_inputs
    rng = np.random.default_rng(3)
    t = np.linspace(1, 10, 50)
    y = 1 + rng.normal(0, 1e-3, 50)
    dy = rng.uniform(0.5e-3, 1.5e-3, 50)
    t[3] = np.nan
    y[7] = -1.0
    y[9] = 0.0
    dy[11] = np.inf
    t[13] = 0.0
    out_dy = R["validate"].validate_inputs(t.copy(), y.copy(), dy.copy())
    out_nody = R["validate"].validate_inputs(t.copy(), y.copy(), None)
    np.savez_compressed(os.path.join(HERE, "validate.npz"), t=t, y=y, dy=dy, t1=out_dy[0], y1=out_dy[1],
                        dy1=out_dy[2], t2=out_nody[0], y2=out_nody[1], dy2=out_nody[2])

    # ---- spectra
    s = {}
    for i, (n, osf, nmask) in enumerate([(2000, 3, 0), (150, 3, 0), (3000, 2, 7), (500, 5, 3)]):
        chi2 = 1000 + rng.normal(0, 3, n)
        chi2[rng.integers(0, n, 3)] -= 40
        mask = np.zeros(n, bool)
        mask[rng.choice(n, nmask, replace=False)] = True
        c = np.ma.array(chi2, mask=mask)
        SR, praw, power, sde_raw, sde = R["stats"].spectra(c, osf)
        s["case%d" % i] = np.array([n, osf])
        s["case%d_chi2" % i] = chi2
        s["case%d_mask" % i] = mask
        s["case%d_SR" % i] = np.ma.getdata(SR)
        s["case%d_praw" % i] = np.ma.getdata(praw)
        s["case%d_power" % i] = np.ma.getdata(power)
        s["case%d_sde" % i] = np.array([sde_raw, sde], dtype=float)
    np.savez_compressed(os.path.join(HERE, "spectra.npz"), **s)

    # ---- template cache through the reference's get_cache
    c = {}
    for i, (maxw, durs) in enumerate([(144, None), (2368, None)]):
        n = 1200 if maxw == 144 else 19728
        P = np.sort(O.period_grid(1, 1, 6.0 if n == 1200 else 27.4))
        durations = R["grid"].duration_grid(P, shortest=1 / n, log_step=1.1)
        mw = int(np.max(durations) * n)
        mw += mw % 2
        args = dict(per=12.9, rp=0.03, a=23.1, inc=89.21, ecc=0, w=90, u=[0.4804, 0.1867], limb_dark="quadratic")
        ours = template.reference_transit(mw, **args)
        R["transit"].reference_transit = lambda samples, **kw: ours
        ov, lc = R["transit"].get_cache(durations, mw, **args, verbose=False)
        c["case%d_durations" % i] = np.asarray(durations)
        c["case%d_maxw" % i] = np.array([mw])
        c["case%d_base" % i] = ours
        c["case%d_width" % i] = ov["width_in_samples"]
        c["case%d_overshoot" % i] = ov["overshoot"]
        c["case%d_lc" % i] = np.concatenate(list(lc))
        c["case%d_lclen" % i] = np.array([len(x) for x in lc])
    np.savez_compressed(os.path.join(HERE, "cache.npz"), **c)

    # ---- reference kernels (CPU build) per period
    k = {}
    rb64 = RR.RefKernelBackend("r64", 8)
    rb32 = RR.RefKernelBackend("r32", 8)
    for i, (seed, n, span, use_dy) in enumerate([(1, 1200, 6.0, False), (2, 900, 4.0, True), (3, 2000, 9.0, False)]):
        t, y, dy = synthetic.small_curve(seed=seed, n=n, span=span, dy=use_dy)
        t, y, dy = V.validate_inputs(t, y, dy)
        P = np.sort(O.period_grid(1, 1, t.max() - t.min()))
        sel = P[:: max(1, len(P) // 24)]
        durs = R["grid"].duration_grid(P, shortest=1 / len(t), log_step=1.1)
        mw = int(np.max(durs) * len(y))
        mw += mw % 2
        ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
        widths, os_, dd, tm, maxd = template.device_templates(lc, ov)
        rows64, rows32 = [], []
        for p in sel:
            wmin, wmax = rb64.duration_ranges(np.array([p]), t.max() - t.min(), len(t))
            m = (widths >= wmin[0]) & (widths <= wmax[0])
            args = (t, y, dy, p, widths[m], tm[m], os_[m], maxd, 1e-5)
            a = rb64.main_pass(*args, 8)
            b = rb64.noskip_pass(*args)
            a3 = rb32.main_pass(*args, 8)
            b3 = rb32.noskip_pass(*args)
            rows64.append([a[0], a[1], b[0], b[1]])
            rows32.append([a3[0], a3[1], b3[0], b3[1]])
        k["case%d_t" % i] = t
        k["case%d_y" % i] = y
        k["case%d_dy" % i] = dy
        k["case%d_periods" % i] = sel
        k["case%d_r64" % i] = np.array(rows64)
        k["case%d_r32" % i] = np.array(rows32)
        k["case%d_widths" % i] = widths
        k["case%d_overshoot" % i] = os_
        k["case%d_templates" % i] = tm
        k["case%d_maxd" % i] = np.array([maxd])
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **k)
    stats_fixture(R)
    print("fixtures written to", HERE)


def reference_best_period_stats(R, t, y, period, loc, width, raw_duration, ovs, maxd):
    """search_single_periods after its chi2 minimum (core.py:1427-1499) with
    the reference's stats and helpers functions."""
    st, hp = R["stats"], R["helpers"]
    tsize = len(t)
    phase = (t % period) / period                      # foldCPU core.py:16-20
    rank = np.argsort(phase)
    best_t, best_f = np.array(t[rank]), y[rank]
    best_f = np.concatenate((best_f, best_f[:maxd]))
    k0 = loc % tsize
    mean = best_f[k0:k0 + width].mean()
    depth = (1 - mean) * ovs
    out_tr = np.concatenate((best_f[0:k0], best_f[k0 + width:]))
    snr_fit = (1 - depth) * (width ** 0.5) / np.std(out_tr)
    csum = np.cumsum(out_tr)
    red = np.std((csum[width:] - csum[:-width]) / width)
    tx = best_t[k0]
    T0 = tx - int((tx - min(t)) / period) * period - period
    tt = st.all_transit_times(T0, t, period)
    snr_fit_pink = (1 - depth) / ((np.std(out_tr) ** 2 / width) + (red ** 2 / len(tt))) ** 0.5
    dur = st.calcDurationDays(t, period, T0, raw_duration)
    T0 = T0 + dur / 2
    tt = np.array(tt) + dur / 2
    if T0 < min(t):
        T0 = T0 + period
    ins = st.intransit_stats(t, y, tt, dur)
    snr_pt, snr_pink_pt = st.snr_stats(t=t, y=y, period=period, duration=raw_duration, T0=T0, transit_times=tt,
                                       transit_duration_in_days=dur, per_transit_count=ins[6])
    f_in = np.concatenate([ins[4], ins[5]])
    mask = hp.transit_mask(t, period, 2 * raw_duration, T0)
    ootr = y[~mask]
    snr = ((1 - np.mean(f_in)) / np.std(ootr)) * len(f_in) ** 0.5
    snr_pink = np.mean(snr_pink_pt) * (len(tt) ** 0.5)
    return dict(depth=depth, T0=T0, duration=dur, transit_times=tt, snr=snr, snr_pink=snr_pink, snr_fit=snr_fit,
                snr_fit_pink=snr_fit_pink, intransit=np.array(ins[:4], dtype=float), per_transit_count=ins[6],
                transit_depths=ins[7], depth_uncertainties=ins[8], snr_per_transit=snr_pt,
                snr_pink_per_transit=snr_pink_pt, mask=mask, ootr=ootr)


def stats_fixture(R):
    """stats.npz: three seeded curves, the chi2 minimum of their true period
    from the oracle, and the reference's statistics of that minimum."""
    from gtls_b200 import synthetic, template, grid as G, validate as V
    import tls_oracle as O
    cases = [synthetic.light_curve_cfg1(seed=4, n=5000, period=1.9, depth=2500e-6)[:2] + (None, 1.9),
             synthetic.small_curve(seed=8, n=1500, span=6.0, dy=True) + (1.7,),
             synthetic.light_curve_cfg1(seed=6, n=14000, period=4.4, depth=800e-6)[:2] + (None, 4.4)]
    f = {}
    for i, (t, y, dy, period) in enumerate(cases):
        t, y, dy = V.validate_inputs(t, y, dy)
        P = np.sort(O.period_grid(1, 1, t.max() - t.min()))
        durs = G.duration_grid(P, shortest=1 / len(t))
        mw = int(np.max(durs) * len(y))
        mw += mw % 2
        ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
        widths, os_, dd, tm, maxd = template.device_templates(lc, ov)
        fin = O.single_period(O.NumpyBackend(), period, t, y, dy, widths, tm, os_, dd, maxd, 1e-5)
        loc, width, raw = fin["loc"], fin["width"], fin["raw_duration"]
        ovs = float(os_[int(np.nonzero(widths == width)[0][0])])
        ref = reference_best_period_stats(R, t, y, period, loc, width, raw, ovs, int(maxd))
        f["case%d_inputs" % i] = np.array([period, loc, width, raw, ovs, maxd], dtype=float)
        f["case%d_t" % i] = t
        f["case%d_y" % i] = y
        ootr = ref.pop("ootr")
        f["case%d_pink" % i] = np.array([R["stats"].pink_noise(ootr, w) for w in (1, 5, 37)])
        for k, v in ref.items():
            f["case%d_%s" % (i, k)] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "stats.npz"), **f)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", "/root/reference"))
