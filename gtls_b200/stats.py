"""Host statistics of the best period (NumPy, as the reference runs them).

Restated from the reference's ``src/gputls/stats.py``: ``all_transit_times``
(:233-250), ``calcDurationDays`` (:252-275), ``intransit_stats`` (:351-424),
``pink_noise`` (:426-431), ``snr_stats`` (:433-488), and
``helpers.transit_mask`` (helpers.py:62-65).  These are O(N) host steps after
the search: ``pink_noise`` takes its window sums from prefix sums (the
reference loops over the windows in Python, O(N x width)), and the samples of
each transit are found by binary search when the times are sorted (the
reference masks all N samples per transit).
"""
import numpy as np


def _transit_fluxes(t, y, transit_times, transit_duration_in_days):
    """Flux of the samples with mid - d/2 < t < mid + d/2 for every transit
    mid-time (None where a bound is NaN), in index order.  Sorted times: the
    two bounds by binary search (the same samples in the same order as the
    mask); otherwise the mask over all samples."""
    t = np.asarray(t)
    mids = np.asarray(transit_times, dtype=float)
    tmin = mids - 0.5 * transit_duration_in_days
    tmax = mids + 0.5 * transit_duration_in_days
    if len(t) > 1 and np.all(t[1:] >= t[:-1]):
        lo = np.searchsorted(t, tmin, side="right")
        hi = np.searchsorted(t, tmax, side="left")
        return [None if np.isnan(a) or np.isnan(b) else y[i:max(i, j)]
                for a, b, i, j in zip(tmin, tmax, lo, hi)]
    return [None if np.isnan(a) or np.isnan(b) else y[np.logical_and(t > a, t < b)] for a, b in zip(tmin, tmax)]


def transit_mask(t, period, duration, T0):
    return np.abs((t - T0 + 0.5 * period) % period - 0.5 * period) < 0.5 * duration


def all_transit_times(T0, t, period):
    transit_times = [T0 + period] if T0 < np.min(t) else [T0]
    prev = transit_times[0]
    end = np.min(t) + (np.max(t) - np.min(t))
    while True:
        nxt = prev + period
        if nxt < end:
            transit_times.append(nxt)
            prev = nxt
        else:
            break
    return transit_times


def calc_duration_days(times, period, start_t0, raw_duration):
    """Duration in days from the phase-sorted samples after the nearest-to-centre one.

    The end index is clamped to the last sample (the reference indexes past the
    array and raises IndexError when the duration reaches beyond it).
    """
    t0c = start_t0 + period / 2
    phases = (times - t0c) / period - np.floor((times - t0c) / period)
    ps = phases[np.argsort(phases)]
    start = int(np.abs(ps - 0.5).argmin())
    end = min(start + int(np.array(raw_duration) * len(times)), len(times) - 1)
    return (ps[end] - 0.5) * period


def intransit_stats(t, y, transit_times, transit_duration_in_days):
    odd = []
    even = []
    per_transit_count = np.zeros(len(transit_times))
    transit_depths = np.zeros(len(transit_times))
    uncert = np.zeros(len(transit_times))
    for i, flux in enumerate(_transit_fluxes(t, y, transit_times, transit_duration_in_days)):
        if flux is None:
            flux = np.array([])
            mean_flux = np.nan
        else:
            mean_flux = np.mean(flux) if len(flux) > 0 else np.nan
        transit_depths[i] = mean_flux
        uncert[i] = np.std(flux) / np.sqrt(flux.size) if flux.size > 0 else np.nan
        per_transit_count[i] = flux.size
        (even if i % 2 == 0 else odd).append(flux)
    odd = np.concatenate(odd) if odd else np.array([])
    even = np.concatenate(even) if even else np.array([])
    d_odd = np.mean(odd) if len(odd) else np.nan
    d_even = np.mean(even) if len(even) else np.nan
    s_odd = np.std(odd) / len(odd) ** 0.5 if len(odd) else np.nan
    s_even = np.std(even) / len(even) ** 0.5 if len(even) else np.nan
    return d_odd, d_even, s_odd, s_even, odd, even, per_transit_count, transit_depths, uncert


def pink_noise(data, width):
    """Mean standard deviation of all windows of ``width`` samples, / sqrt(width).

    The windows' sums of x and x^2 are differences of prefix sums of the
    data minus its mean, accumulated in extended precision (64-bit
    mantissa), so the windowed variances keep about 1e-13 relative accuracy
    against the per-window two-pass standard deviation at O(N) cost."""
    x = np.asarray(data, dtype=float)
    n = len(x) - width + 1
    if width < 1 or n < 1:
        raise ValueError("pink_noise window does not fit the data")
    if width == 1:
        return 0.0                                        # every one-sample window has std 0
    xl = x.astype(np.longdouble)
    xc = xl - np.mean(xl)
    c1 = np.concatenate((np.zeros(1, dtype=np.longdouble), np.cumsum(xc)))
    c2 = np.concatenate((np.zeros(1, dtype=np.longdouble), np.cumsum(xc * xc)))
    s1 = c1[width:] - c1[:-width]
    s2 = c2[width:] - c2[:-width]
    var = (s2 - s1 * s1 / width) / width
    std = np.sqrt(np.maximum(var, 0)).astype(float)
    return np.sum(std) / (n * width ** 0.5)


def snr_stats(t, y, period, duration, T0, transit_times, transit_duration_in_days, per_transit_count):
    snr_per_transit = np.zeros(len(transit_times))
    snr_pink_per_transit = np.zeros(len(transit_times))
    intransit = transit_mask(t, period, 2 * duration, T0)
    flux_ootr = y[~intransit]
    try:
        pinknoise = pink_noise(flux_ootr, int(np.mean(per_transit_count)))
    except Exception:
        pinknoise = np.nan
    std = np.std(flux_ootr) if len(flux_ootr) > 0 else np.nan
    for i, flux in enumerate(_transit_fluxes(t, y, transit_times, transit_duration_in_days)):
        if flux is None:
            flux = np.array([])
            mean_flux = np.nan
        else:
            mean_flux = np.mean(flux) if len(flux) > 0 else np.nan
        pts = flux.size
        with np.errstate(divide="ignore", invalid="ignore"):
            snr_pink_per_transit[i] = (1 - mean_flux) / pinknoise
            if pts > 0 and not np.isnan(std):
                snr_per_transit[i] = (1 - mean_flux) / (std / pts ** 0.5)
            else:
                snr_per_transit[i] = 0
                snr_pink_per_transit[i] = 0
    return snr_per_transit, snr_pink_per_transit
