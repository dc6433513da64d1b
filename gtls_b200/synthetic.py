"""Seeded synthetic light curves for the benchmark workloads and the tests.

The reference's own scripts run on TESS/Kepler light curves (a bundled TESS
sector-58 2-minute FITS file, Kepler downloads); these generators stand in for
them with the same shapes, cadences and noise levels.  Every generator takes a
seed and draws from ``numpy.random.default_rng(seed)``.  Transits are injected
with ``ldmodel`` (quadratic limb darkening, circular orbit, impact parameter 0).
"""
import numpy as np

from . import ldmodel

DAY_MIN = 1440.0


def _transit(t, t0, period, depth, duration, u):
    rp, a, inc = ldmodel.transit_params_from_shape(period, depth, duration, u)
    return ldmodel.light_curve(t, t0, period, rp, a, inc, u)


def _times_with_gaps(n, cadence_min, t_start, gaps, rng):
    """``n`` regularly spaced samples, skipping the listed (start_fraction, length_days) gaps."""
    dt = cadence_min / DAY_MIN
    span_guess = n * dt + sum(g[1] for g in gaps)
    edges = sorted((t_start + f * span_guess, t_start + f * span_guess + L) for f, L in gaps)
    out = np.empty(n)
    cur = t_start
    i = 0
    j = 0
    while i < n:
        if j < len(edges) and cur >= edges[j][0]:
            cur = max(cur, edges[j][1])
            j += 1
            continue
        out[i] = cur
        cur += dt
        i += 1
    return out


def light_curve_cfg1(seed=0, depth=1200e-6, period=3.853, duration=2.4 / 24, u=(0.48, 0.19),
                     n=19728, noise=1e-3):
    """19,728 samples at 2-min cadence with a 1.0 d mid-span gap, white noise 1e-3,
    one quadratic-limb-darkened transit train.  Returns (t, y, dy=None, truth)."""
    rng = np.random.default_rng(seed)
    t = _times_with_gaps(n, 2.0, 1000.0, [(0.5, 1.0)], rng)
    t0 = t[0] + rng.uniform(0, period)
    y = 1.0 + rng.normal(0.0, noise, n)
    y *= _transit(t, t0, period, depth, duration, list(u))
    return t, y, None, dict(period=period, t0=t0, depth=depth, duration=duration)


def light_curve_cfg2(seed=0):
    """70,000 samples at 29.4-min cadence over ~1,470 d with 17 gaps of 1-5 d,
    per-sample sigma ~ U(50, 500) ppm plus AR(1) red noise (rho 0.9, 100 ppm),
    one transit P=289.9 d, 490 ppm, 7.4 h, u=(0.40, 0.26).  Returns (t, y, dy, truth)."""
    rng = np.random.default_rng(seed)
    n = 70000
    lengths = rng.uniform(1.0, 5.0, 17)
    # scale the gaps so that the light curve spans 1,470 d
    lengths *= (1470.0 - (n - 1) * 29.4 / DAY_MIN) / lengths.sum()
    gaps = [(f, L) for f, L in zip(rng.uniform(0.02, 0.98, 17), lengths)]
    t = _times_with_gaps(n, 29.4, 1000.0, gaps, rng)
    sigma = rng.uniform(50e-6, 500e-6, n)
    red = np.empty(n)
    innov = rng.normal(0.0, 100e-6 * np.sqrt(1 - 0.9 ** 2), n)
    red[0] = rng.normal(0.0, 100e-6)
    for i in range(1, n):
        red[i] = 0.9 * red[i - 1] + innov[i]
    period = 289.9
    t0 = t[0] + rng.uniform(0, period)
    y = (1.0 + sigma * rng.standard_normal(n) + red) * _transit(t, t0, period, 490e-6, 7.4 / 24,
                                                                  [0.40, 0.26])
    return t, y, sigma, dict(period=period, t0=t0, depth=490e-6, duration=7.4 / 24)


def light_curve_cfg3(seed):
    """Config-1 curve with depth log-U(100, 2000) ppm and P log-U(1, 500) d."""
    rng = np.random.default_rng(10_000 + seed)
    depth = float(np.exp(rng.uniform(np.log(100e-6), np.log(2000e-6))))
    period = float(np.exp(rng.uniform(np.log(1.0), np.log(500.0))))
    return light_curve_cfg1(seed=seed, depth=depth, period=period)


def batch_cfg4_specs(n_curves=4096, seed=0):
    """Per-curve (n, cadence_min, span_days, sigma, has_transit, P, depth, rho_star) of
    the batched workload: n log-U(5k, 70k), cadence in {2, 10, 30} min, span
    clamp(n * cadence, 27, 1470) d, sigma log-U(100, 3000) ppm, half with one
    transit (P log-U(0.5, span/3), depth log-U(200, 5000) ppm, stellar density
    U(0.5, 2) solar setting the duration)."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(5000), np.log(70000), n_curves)).astype(np.int64)
    cad = rng.choice([2.0, 10.0, 30.0], n_curves)
    span = np.clip(n * cad / DAY_MIN, 27.0, 1470.0)
    sigma = np.exp(rng.uniform(np.log(100e-6), np.log(3000e-6), n_curves))
    has = rng.uniform(size=n_curves) < 0.5
    per = np.exp(rng.uniform(np.log(0.5), np.log(span / 3.0)))
    depth = np.exp(rng.uniform(np.log(200e-6), np.log(5000e-6), n_curves))
    rho = rng.uniform(0.5, 2.0, n_curves)
    return dict(n=n, cadence=cad, span=span, sigma=sigma, has_transit=has, period=per, depth=depth,
                rho=rho, seed=seed)


def light_curve_cfg4(specs, i):
    """Curve ``i`` of the batched workload (see ``batch_cfg4_specs``)."""
    rng = np.random.default_rng((specs["seed"] + 1) * 1_000_003 + i)
    n = int(specs["n"][i])
    span = float(specs["span"][i])
    t = np.sort(rng.uniform(0.0, span, n)) + 100.0 if n * specs["cadence"][i] / DAY_MIN < span else \
        100.0 + np.arange(n) * specs["cadence"][i] / DAY_MIN
    y = 1.0 + rng.normal(0.0, specs["sigma"][i], n)
    if specs["has_transit"][i]:
        P = float(specs["period"][i])
        # duration of a central transit for stellar density rho (solar units)
        a = 215.03 * (specs["rho"][i] * (P / 365.25) ** 2) ** (1.0 / 3.0)
        duration = P / np.pi * np.arcsin(min(1.0, 1.0 / a))
        y *= _transit(t, t[0] + rng.uniform(0, P), P, float(specs["depth"][i]), duration, [0.45, 0.2])
    return t, y, None


def small_curve(seed=0, n=1500, span=6.0, period=1.7, depth=3e-3, noise=1e-3, gap=True, dy=False):
    """A short curve for tests: ``n`` samples over ``span`` days with one optional gap."""
    rng = np.random.default_rng(seed)
    cad = (span - (0.4 if gap else 0.0)) / n * DAY_MIN
    t = _times_with_gaps(n, cad, 10.0, [(0.45, 0.4)] if gap else [], rng)
    y = 1.0 + rng.normal(0.0, noise, n)
    t0 = t[0] + rng.uniform(0, period)
    y *= _transit(t, t0, period, depth, 0.08 * period ** (1 / 3) / 3, [0.45, 0.2])
    s = rng.uniform(0.5 * noise, 1.5 * noise, n) if dy else None
    return t, y, s


def refinement_set(n_curves=1024, n=20000, seed=0, noise=1e-3, depth_range=(100e-6, 2000e-6)):
    """Light curves with transits and perturbed starting parameters for the
    adjoint refinement: n samples at 2-min cadence, P log-U(1, 13) d, depth
    log-U(100, 2000) ppm, white noise 1e-3 (dy given).  Starting parameters are
    the truth moved by up to half an Ofir grid step in P, half a cadence in T0,
    5% in duration and 10% in depth, with the default limb darkening.
    Returns (curves [(t, y, dy)], truth (n_curves x 6), start (n_curves x 6),
    scales (6,) per curve)."""
    rng = np.random.default_rng(20_000 + seed)
    cad = 2.0 / DAY_MIN
    curves, truth, start, scales = [], [], [], []
    for c in range(n_curves):
        period = float(np.exp(rng.uniform(np.log(1.0), np.log(13.0))))
        depth = float(np.exp(rng.uniform(np.log(depth_range[0]), np.log(depth_range[1]))))
        t = 100.0 + np.arange(n) * cad
        span = t[-1] - t[0]
        t0 = t[0] + rng.uniform(0.2, 0.8) * period
        dur = 0.13 * period ** (1.0 / 3.0) / 3.0
        u = [0.45, 0.2]
        y = _transit(t, t0, period, depth, dur, u) + rng.normal(0.0, noise, n)
        dy = np.full(n, noise)
        # Ofir spacing at this period for a Sun-like star, oversampling 3
        step_p = period * 2.7e-4 * (period / span) ** (1.0 / 3.0)
        curves.append((t, y, dy))
        truth.append([period, t0, dur, depth, u[0], u[1]])
        start.append([period + rng.uniform(-0.5, 0.5) * step_p, t0 + rng.uniform(-0.5, 0.5) * cad,
                      dur * (1 + rng.uniform(-0.05, 0.05)), depth * (1 + rng.uniform(-0.1, 0.1)), 0.4804, 0.1867])
        scales.append([step_p, cad, 0.05 * dur, 0.1 * depth, 0.05, 0.05])
    return curves, np.array(truth), np.array(start), np.array(scales)
