"""Transit template cache: one trimmed, depth-scaled template per duration.

Same construction as the reference's ``src/gputls/transit.py``:
``reference_transit`` (:8-42) samples a transit of one day's width on 10,000
points, trims it to the in-transit part, downsamples it to ``maxwidth``
samples by linear interpolation and rescales it to [0, 1];
``fractional_transit`` (:45-95) squeezes it to each trial duration and scales
it to SIGNAL_DEPTH; ``get_cache`` (:98-160) trims each one to the samples
below ``1 - 1e-8`` and records its width in samples and its ``overshoot``.
The light curve of the reference transit comes from ``ldmodel`` (our own
limb-darkened occultation integral) instead of batman, which is a
third-party package outside the reference tree.

The linear interpolation reproduces ``src/gputls/interpolation.py`` (:8-58):
for each new abscissa the bracketing index is the last knot not above it,
clamped to [0, n-2], and the value is ``(1-theta)*y[i] + theta*y[i+1]``.
"""
import numpy as np

from . import constants, ldmodel


def interp_linear(x_new, x, y):
    """Linear interpolation with end extrapolation (interpolation.py:8-58)."""
    x = np.asarray(x, dtype=float)
    x_new = np.asarray(x_new, dtype=float)
    n = len(x)
    i = np.clip(np.searchsorted(x, x_new, side="right") - 1, 0, n - 2)
    theta = (x_new - x[i]) / (x[i + 1] - x[i])
    y = np.asarray(y, dtype=float)
    return (1 - theta) * y[i] + theta * y[i + 1]


def transit_flux(t, per, rp, a, inc, ecc, w, u, limb_dark):
    """Flux of the reference planet at times ``t`` (days from mid-transit)."""
    if ecc != 0:
        raise ValueError("only circular template orbits (ecc=0) are supported")
    if limb_dark == "linear":
        u = [u[0] if len(u) else 0.0, 0.0]
    elif limb_dark != "quadratic":
        raise ValueError("limb_dark must be 'quadratic' or 'linear'")
    return ldmodel.light_curve(t, 0.0, per, rp, a, inc, u)


_FLUX_CACHE = {}


def _supersampled_flux(per, rp, a, inc, ecc, w, u, limb_dark):
    """Flux of the reference planet on the SUPERSAMPLE_SIZE grid over one day.

    It depends only on the planet parameters, so a batch of light curves
    sharing them computes it once (the occultation integral dominates the
    cost of a template set)."""
    key = (float(per), float(rp), float(a), float(inc), float(ecc), float(w),
           tuple(float(v) for v in np.atleast_1d(u)), str(limb_dark))
    hit = _FLUX_CACHE.get(key)
    if hit is None:
        t = np.linspace(-0.5, 0.5, constants.SUPERSAMPLE_SIZE)
        flux = transit_flux(t, per, rp, a, inc, ecc, w, u, limb_dark)
        flux.setflags(write=False)
        if len(_FLUX_CACHE) > 64:
            _FLUX_CACHE.clear()
        hit = _FLUX_CACHE[key] = (t, flux)
    return hit


def reference_transit(samples, per, rp, a, inc, ecc, w, u, limb_dark):
    """Unit-width, unit-depth reference transit on ``samples`` points (transit.py:8-42)."""
    t, flux = _supersampled_flux(per, rp, a, inc, ecc, w, u, limb_dark)
    idx_first = int(np.argmax(flux < 1))
    intransit_flux = flux[idx_first: -idx_first + 1]
    intransit_time = t[idx_first: -idx_first + 1]
    x_new = np.linspace(t[idx_first], t[-idx_first - 1], samples)
    down = interp_linear(x_new, intransit_time, intransit_flux)
    return (np.min(down) - down) / (np.min(down) - 1)


def fractional_transit(duration, maxwidth, depth, samples, reference_flux):
    """Reference transit squeezed to ``duration`` and scaled to ``depth`` (transit.py:45-95)."""
    reference_time = np.linspace(-0.5, 0.5, samples)
    occupied = int((duration / maxwidth) * samples)
    x_new = np.linspace(-0.5, 0.5, occupied)
    y_new = interp_linear(x_new, reference_time, reference_flux)
    missing = samples - occupied
    empty = np.ones(int(missing * 0.5))
    result = np.append(empty, y_new)
    result = np.append(result, empty)
    if np.size(result) < samples:
        result = np.append(result, np.ones(1))
    return 1 - ((1 - result) * depth)


def _linspaces(counts):
    """``np.linspace(-0.5, 0.5, k)`` for every k of ``counts`` (each >= 2),
    concatenated, with numpy's own arithmetic: index * (1 / (k - 1)), then
    + (-0.5), and the last point set to 0.5 exactly."""
    counts = np.asarray(counts, dtype=np.int64)
    off = np.concatenate(([0], np.cumsum(counts)))
    seg = np.repeat(np.arange(len(counts)), counts)
    idx = (np.arange(off[-1]) - off[seg]).astype(float)
    x = idx * (1.0 / (counts - 1).astype(float))[seg]
    x += -0.5
    x[off[1:] - 1] = 0.5
    return x, off


def get_cache(durations, maxwidth_in_samples, per, rp, a, inc, ecc, w, u, limb_dark,
              verbose=True):
    """Template per duration plus (duration, width_in_samples, overshoot) (transit.py:98-160).

    The in-transit part of fractional_transit(duration, dmax, SIGNAL_DEPTH,
    samples, ref) for every duration at once: its padding is
    1 - (1 - 1) * depth = 1 exactly, never below the cutoff, so the trimmed
    signal comes from the squeezed template alone.  The squeezed templates
    of all durations are interpolated in one pass (each value computed as
    the per-duration interpolation computes it)."""
    durations = np.atleast_1d(np.asarray(durations, dtype=float))
    rows = np.size(durations)
    overview = np.zeros(rows, dtype=[("duration", "f8"), ("width_in_samples", "i8"),
                                     ("overshoot", "f8")])
    ref = reference_transit(maxwidth_in_samples, per, rp, a, inc, ecc, w, u, limb_dark)
    dmax = np.max(durations)
    samples = maxwidth_in_samples
    reference_time = np.linspace(-0.5, 0.5, samples)
    cutoff = 1 - constants.NUMERICAL_STABILITY_CUTOFF
    occupied = np.array([int((d / dmax) * samples) for d in durations], dtype=np.int64)
    overview["duration"] = durations
    overview["width_in_samples"] = [int((d / dmax) * maxwidth_in_samples) for d in durations]
    if np.all(occupied >= 2):
        x_new, off = _linspaces(occupied)
        scaled_all = 1 - ((1 - interp_linear(x_new, reference_time, ref)) * constants.SIGNAL_DEPTH)
        segments = [scaled_all[off[r]:off[r + 1]] for r in range(rows)]
    else:
        segments = [1 - ((1 - interp_linear(np.linspace(-0.5, 0.5, k), reference_time, ref))
                         * constants.SIGNAL_DEPTH) for k in occupied]
    lc = np.empty(rows, dtype=object)
    for row, scaled in enumerate(segments):
        full = np.flatnonzero(scaled < cutoff)
        if np.size(full) == 0:
            raise ValueError("transit template of duration %g has no in-transit samples "
                             "(light curve too short for this duration grid)" % durations[row])
        signal = scaled[full[0]: full[-1] + 1].copy()
        lc[row] = signal
        overview["overshoot"][row] = 1 / (2 - np.mean(signal) / np.min(signal))
    return overview, lc


def device_templates(lc_arr, overview):
    """Deduplicate by width and build the template matrix the kernels consume.

    Mirrors core.py:605-614 (unique widths, first occurrence, ascending) and
    the template construction ``1 - pad(lc, 0)`` of core.py:753-754: position
    ``i`` of duration ``d`` holds ``1 - lc[d][i]`` for ``i < len(lc[d])`` and
    ``1`` beyond it (zero padding, then ``1 -``).  Rows are ``width`` long.

    Returns (widths int32[D], overshoot f64[D], durations f64[D],
    templates f64[D, maxw], max_duration_even).
    """
    widths, first = np.unique(overview["width_in_samples"], return_index=True)
    lc = lc_arr[first]
    ov = overview[first]
    maxw = int(np.max(widths))
    max_dur = maxw + (maxw % 2)
    tm = np.ones((len(widths), maxw), dtype=np.float64)
    for d, sig in enumerate(lc):
        n = min(len(sig), maxw)
        tm[d, :n] = 1.0 - np.asarray(sig[:n], dtype=np.float64)
    return (widths.astype(np.int32), ov["overshoot"].astype(np.float64),
            ov["duration"].astype(np.float64), tm, max_dur)
