"""Period and duration grids.

Follows the reference's ``src/gputls/grid.py``: ``T14`` (:7-29),
``duration_grid`` (:32-53) and ``period_grid`` (:56-157, Ofir 2014 optimal
frequency sampling).  The scalar set-up (stellar-parameter clamps, the Ofir
coefficients A and C, the number of grid points) runs on the host exactly as
in the reference.  The per-point evaluation ``P(X) = 1 / (A/3*X + C)^3 / 86400``
and the selection of ``period_min < P <= period_max`` run either on the host
with the reference's own NumPy expression (the default: bit-identical to the
reference's grid on the same host, whose NumPy ``**3`` rounding depends on
the CPU's SIMD pow) or on the GPU (``gtls_period_grid`` in the C-ABI, the cube
correctly rounded, so each period within 2 ulp of NumPy's).
"""
import warnings

import numpy as np
from numpy import pi, sqrt

from . import constants


def T14(R_s, M_s, P, upper_limit=constants.FRACTIONAL_TRANSIT_DURATION_MAX, small=False):
    """Maximum transit duration as a fraction of the period (grid.py:7-29)."""
    P = P * constants.SECONDS_PER_DAY
    R_s = constants.R_sun * R_s
    M_s = constants.M_sun * M_s
    if small:
        T14max = R_s * ((4 * P) / (pi * constants.G * M_s)) ** (1 / 3)
    else:
        T14max = (R_s + 2 * constants.R_jup) * ((4 * P) / (pi * constants.G * M_s)) ** (1 / 3)
    result = T14max / P
    if result > upper_limit:
        result = upper_limit
    return result


def duration_grid(periods, shortest, log_step=constants.DURATION_GRID_STEP):
    """Log-spaced fractional durations between the T14 bounds (grid.py:32-53)."""
    periods = np.asarray(periods, dtype=np.float64)   # min/max of an array: NumPy's, same values
    duration_max = T14(R_s=constants.R_STAR_MAX, M_s=constants.M_STAR_MAX, P=float(np.min(periods)), small=False)
    duration_min = T14(R_s=constants.R_STAR_MIN, M_s=constants.M_STAR_MIN, P=float(np.max(periods)), small=True)
    durations = [duration_min]
    current = duration_min
    while current * log_step < duration_max:
        current = current * log_step
        durations.append(current)
    durations.append(duration_max)
    return durations


def duration_grid_step_for(periods, shortest, count):
    """The ``log_step`` for which ``duration_grid(periods, shortest, log_step)``
    has exactly ``count`` durations (bisection; the count falls as the step
    grows).  Workloads that ask for a number of durations use it."""
    lo, hi = 1.0001, 3.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        c = len(duration_grid(periods, shortest=shortest, log_step=mid))
        if c > count:
            lo = mid
        elif c < count:
            hi = mid
        else:
            return mid
    raise ValueError("no duration grid step gives %d durations" % count)


def ofir_coefficients(R_star, M_star, time_span, oversampling_factor=constants.OVERSAMPLING_FACTOR,
                      n_transits_min=constants.N_TRANSITS_MIN):
    """Clamp the stellar parameters and return (A/3, C, n_points) of the Ofir grid.

    Same expressions and evaluation order as grid.py:68-126; ``n_points`` is
    ``len(numpy.arange(N_opt))``.
    """
    if R_star < 0.01:
        warnings.warn("Warning: R_star was set to 0.01 for period_grid (was unphysical: " + str(R_star) + ")")
        R_star = 0.1
    if R_star > 10000:
        warnings.warn("Warning: R_star was set to 10000 for period_grid (was unphysical: " + str(R_star) + ")")
        R_star = 10000
    if M_star < 0.01:
        warnings.warn("Warning: M_star was set to 0.01 for period_grid (was unphysical: " + str(M_star) + ")")
        M_star = 0.01
    if M_star > 1000:
        warnings.warn("Warning: M_star was set to 1000 for period_grid (was unphysical: " + str(M_star) + ")")
        M_star = 1000
    R_star = R_star * constants.R_sun
    M_star = M_star * constants.M_sun
    time_span = time_span * constants.SECONDS_PER_DAY
    f_min = n_transits_min / time_span
    f_max = 1.0 / (2 * pi) * sqrt(constants.G * M_star / (3 * R_star) ** 3)
    A = ((2 * pi) ** (2.0 / 3) / pi * R_star / (constants.G * M_star) ** (1.0 / 3)
         / (time_span * oversampling_factor))
    C = f_min ** (1.0 / 3) - A / 3.0
    N_opt = (f_max ** (1.0 / 3) - f_min ** (1.0 / 3) + A / 3) * 3 / A
    n_points = len(np.arange(N_opt))
    return np.float64(A / 3), np.float64(C), int(n_points), time_span


def _host_points(a3, c, n_points, period_min, period_max):
    """grid.py:127-133: f_x = (A/3 * X + C)^3, P = 1/f_x/86400, kept where
    period_min < P <= period_max; the same NumPy operations in the same order
    (so the same bits on the same host).  Ascending."""
    X = np.arange(n_points, dtype=np.float64) + 1
    f_x = (a3 * X + c) ** 3
    periods = 1 / f_x / constants.SECONDS_PER_DAY
    sel = np.where(np.logical_and(periods > period_min, periods <= period_max))
    return np.ascontiguousarray(periods[sel][::-1])


def period_grid(R_star, M_star, time_span, period_min=0, period_max=float("inf"),
                oversampling_factor=constants.OVERSAMPLING_FACTOR,
                n_transits_min=constants.N_TRANSITS_MIN, device=0, ascending=False, evaluate="host"):
    """Ofir-optimal trial periods in days.

    ``evaluate``: "host" (default) evaluates the points with the reference's
    NumPy expression, "device" on the GPU (``gtls_period_grid``).  Returns
    the periods in the reference's order (descending, as grid.py:132-157
    returns them) unless ``ascending`` is set.  With fewer than 100 periods
    the grid is rebuilt for R_star = M_star = 1 and a time span of at least 5
    days, with the default bounds, as the reference does.
    """
    if evaluate not in ("host", "device"):
        raise ValueError("evaluate must be 'host' or 'device'")
    a3, c, n_points, span_s = ofir_coefficients(R_star, M_star, time_span, oversampling_factor,
                                                n_transits_min)
    if evaluate == "host":
        periods = _host_points(a3, c, n_points, period_min, period_max)
    else:
        from . import _lib
        periods = _lib.period_grid(a3, c, n_points, float(period_min), float(period_max), device=device)
    if periods.size > 10 ** 6:
        warnings.warn("period_grid generates a very large grid (" + str(periods.size)
                      + "). Recommend to check physical plausibility for stellar mass, radius, "
                      "and time series duration.")
    if periods.size < constants.MINIMUM_PERIOD_GRID_SIZE:
        if span_s < 5 * constants.SECONDS_PER_DAY:
            span_s = 5 * constants.SECONDS_PER_DAY
        warnings.warn("period_grid defaults to R_star=1 and M_star=1 as given density yielded grid "
                      "with too few values")
        return period_grid(R_star=1, M_star=1, time_span=span_s / constants.SECONDS_PER_DAY,
                           device=device, ascending=ascending, evaluate=evaluate)
    return periods if ascending else periods[::-1].copy()
