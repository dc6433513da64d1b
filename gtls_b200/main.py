"""User API: ``gtls(t, y, dy).power(**kwargs)`` (the reference's ``src/gputls/main.py``).

Same constructor, same ``power()`` keywords (constants.VALID_PARAMETERS) and
the same return: a ``gtlsResult`` or, with ``fast=True``, ``(periods, power)``.
The search runs on one GPU (``GPUDeviceID``); ``GPUDeviceIDs`` with more than
one entry shards the main pass over those devices in this process, as the
reference's multi-GPU mode does with a worker process per GPU (contiguous,
batch-aligned period ranges, one host thread per device; every chi2 value is
the unsharded one), and runs the rest on the first of them.  ``distributed``
(below) does the same with one process per GPU started by torchrun.
Extra keywords: ``precision`` ("fp64" plain FP64 search, default; "fp32" FP32
chi2 with float-float prefix sums in the main pass and the candidate
re-search, then an FP64 re-check of the 32 best candidates),
``batch_periods`` (periods per duration-union batch; default: the reference's
free-memory formula, core.py:620-628), ``distributed`` (shard the main pass
over the ranks of the initialised torch.distributed process group, one
process per GPU: batch-aligned period ranges, chi2 all-gathered; every rank
returns the same result) and ``refine`` (move the best peak's period, T0,
duration and depth below grid resolution with the adjoint of the
limb-darkened model chi2; the grid values stay if the chi2 does not
decrease; both are in ``diagnostics["refinement"]``).
"""
import numpy as np

from . import constants, core
from .grid import duration_grid, period_grid
from .results import gtlsResult
from .template import get_cache
from .validate import validate_args, validate_inputs


class gtls(object):
    """Transit least squares of limb-darkened transit models on a B200."""

    def __init__(self, t, y, dy=None, verbose=True):
        self.t, self.y, self.dy = validate_inputs(t, y, dy)
        self.verbose = verbose

    def _grids(self):
        if len(self.periods) == 0:
            periods = period_grid(R_star=self.R_star, M_star=self.M_star,
                                  time_span=np.max(self.t) - np.min(self.t), period_min=self.period_min,
                                  period_max=self.period_max, oversampling_factor=self.oversampling_factor,
                                  n_transits_min=self.n_transits_min, device=self.GPUDeviceID)
        else:
            periods = np.asarray(self.periods, dtype=np.float64)
        return periods

    def power(self, **kwargs):
        """Run the search; see the module docstring for the keywords."""
        self, kwargs = validate_args(self, kwargs)
        devices = None
        if self.GPUDeviceIDs is not None and len(self.GPUDeviceIDs) > 0:
            devices = [int(d) for d in self.GPUDeviceIDs]
            self.GPUDeviceID = devices[0]
        if self.verbose:
            print(constants.BANNER)
        periods = self._grids()
        durations = duration_grid(periods, shortest=1 / len(self.t), log_step=self.duration_grid_step)
        maxwidth = int(np.max(durations) * np.size(self.y))
        if maxwidth % 2 != 0:
            maxwidth = maxwidth + 1
        self.maxwidth_in_samples = maxwidth
        self.lc_cache_overview, self.lc_arr = get_cache(
            durations=durations, maxwidth_in_samples=maxwidth, per=self.per, rp=self.rp, a=self.a,
            inc=self.inc, ecc=self.ecc, w=self.w, u=self.u, limb_dark=self.limb_dark, verbose=self.verbose)
        if self.verbose:
            print("Searching " + str(len(self.y)) + " data points, " + str(len(periods)) + " periods from "
                  + str(round(min(periods), 3)) + " to " + str(round(max(periods), 3)) + " days")
        periods = np.sort(periods)
        out = core.search_multi_periods(
            periods=periods, t=self.t, y=self.y, dy=self.dy, transit_depth_min=self.transit_depth_min,
            lc_arr=self.lc_arr, lc_cache_overview=self.lc_cache_overview, T0_fit_margin=self.T0_fit_margin,
            oversampling_factor=self.oversampling_factor, verbose=self.verbose, GPUDeviceID=self.GPUDeviceID,
            fast=self.fast, precision=self.precision, batch_periods=self.batch_periods,
            distributed=self.distributed, devices=devices)
        if self.fast:
            return out
        (self.periods, self.period, self.rawDuration, durationPoints, self.duration, self.Depth, self.bestT0,
         SDE, chi2, self.transitTimes, power, snr, snrPink, snrFit, snrFitPink, raw_power, raw_chi2,
         cand_idx, cand_p, diag) = out
        self.rawDurations = durations
        if self.refine:
            self._refine(periods, diag)
        return gtlsResult(self.periods, self.period, self.rawDuration, durationPoints, durations, self.duration,
                          self.Depth, self.bestT0, SDE, chi2, self.transitTimes, power, snr, snrPink, snrFit,
                          snrFitPink, raw_power, raw_chi2, cand_idx, cand_p, diag)

    def _refine(self, periods, diag):
        """Sub-grid refinement of the best peak (refine=True): the adjoint of
        the limb-darkened model chi2 from the grid's (period, T0, duration,
        depth) and the template's limb darkening; the refined values replace
        the grid's only if the model chi2 decreased.  ``diagnostics
        ["refinement"]`` keeps both."""
        from . import refine as R
        start, scale = R.grid_start(self.period, self.bestT0, self.duration, self.Depth, self.u, periods, self.t)
        params, chi, chi0, ok = R.refine_peaks([(self.t, self.y, self.dy)], start[None], scale[None],
                                               device=self.GPUDeviceID)
        diag["refinement"] = dict(grid=dict(period=self.period, T0=self.bestT0, duration=self.duration,
                                            depth=self.Depth), params=params[0], chi2=float(chi[0]),
                                  chi2_grid=float(chi0[0]), improved=bool(ok[0]))
        if ok[0]:
            self.period, self.bestT0, self.duration, self.Depth = (float(v) for v in params[0][:4])
            self.transitTimes = R.refined_transit_times(self.transitTimes, self.bestT0, self.period)

    def periodogram(self, **kwargs):
        """The trial periods power() would search (main.py:186-205)."""
        self, kwargs = validate_args(self, kwargs)
        return self._grids()
