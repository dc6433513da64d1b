"""Input cleaning and keyword validation for ``gtls(...).power(**kw)``.

Mirrors the reference's ``src/gputls/validate.py`` (``validate_inputs`` :9-46,
``validate_args`` :49-203) and ``helpers.cleaned_array`` (:16-59): the same
samples are kept, the same defaults are applied, and the same ``ValueError``
messages are raised for the same invalid arguments.  The cleaning is
vectorised (the reference loops over samples in Python) but keeps exactly the
samples the reference keeps: a value is valid when it is not None, not NaN,
strictly positive and finite.
"""
import multiprocessing
import warnings

import numpy as np

from . import constants


def _as_float(x):
    if isinstance(x, np.ma.MaskedArray):
        return np.ma.filled(x.astype(float), np.nan)
    return np.asarray(
        [np.nan if v is None else v for v in x] if isinstance(x, (list, tuple)) else x,
        dtype=float,
    )


def cleaned_array(t, y, dy=None):
    """Drop samples where any of t, y (, dy) is None/NaN/<=0/inf (helpers.py:16-59)."""
    t = _as_float(t)
    y = _as_float(y)
    with np.errstate(invalid="ignore"):
        ok = np.isfinite(t) & (t > 0) & np.isfinite(y) & (y > 0)
        if dy is not None:
            dy = _as_float(dy)
            ok &= np.isfinite(dy) & (dy > 0)
    if dy is None:
        return t[ok].copy(), y[ok].copy()
    return t[ok].copy(), y[ok].copy(), dy[ok].copy()


def impact_to_inclination(b, semimajor_axis):
    """Impact parameter -> inclination in degrees (helpers.py:108-110)."""
    return np.degrees(np.arccos(b / semimajor_axis))


def validate_inputs(t, y, dy):
    """Clean and check (t, y, dy); dy defaults to std(y) (validate.py:9-46)."""
    if dy is None:
        t, y = cleaned_array(t, y)
    else:
        t, y, dy = cleaned_array(t, y, dy)
        dy = dy / np.mean(dy)
    if np.size(t) == 0:
        raise ValueError("Too few values in data set")
    duration = np.max(t) - np.min(t)
    if duration <= 0:
        raise ValueError("Time duration must positive")
    if np.size(y) < 3 or np.size(t) < 3:
        raise ValueError("Too few values in data set")
    if np.mean(y) > 1.01 or np.mean(y) < 0.99:
        warnings.warn(
            "Warning: The mean flux should be normalized to 1, but it was found to be "
            + str(np.mean(y))
        )
    if np.min(y) < 0:
        raise ValueError("Flux values must be positive")
    if np.max(y) >= float("inf"):
        raise ValueError("Flux values must be finite")
    if dy is None:
        dy = np.full(len(y), np.std(y))
    if np.size(t) != np.size(y) or np.size(t) != np.size(dy):
        raise ValueError("Arrays (t, y, dy) must be of the same dimensions")
    if t.ndim != 1:
        raise ValueError("Inputs (t, y, dy) must be 1-dimensional")
    return t, y, dy


def validate_args(self, kwargs):
    """Apply defaults and range checks to power() keywords (validate.py:49-203)."""
    self.useLocalPTXCUBIN = kwargs.get("useLocalPTXCUBIN", False)
    self.GPUDeviceID = kwargs.get("GPUDeviceID", 0)
    self.GPUDeviceIDs = kwargs.get("GPUDeviceIDs", None)
    self.legacy = kwargs.get("legacy", False)
    self.fast = kwargs.get("fast", False)
    self.bar_location = kwargs.get("bar_location", 0)
    for key in kwargs:
        if key not in constants.VALID_PARAMETERS:
            warnings.warn("Ignoring unknown parameter: " + str(key))

    self.show_progress_bar = kwargs.get("show_progress_bar", True)
    self.transit_depth_min = kwargs.get("transit_depth_min", constants.TRANSIT_DEPTH_MIN)
    self.R_star = kwargs.get("R_star", constants.R_STAR)
    self.M_star = kwargs.get("M_star", constants.M_STAR)
    self.oversampling_factor = kwargs.get("oversampling_factor", constants.OVERSAMPLING_FACTOR)
    self.period_max = kwargs.get("period_max", float("inf"))
    self.period_min = kwargs.get("period_min", 0)
    self.periods = kwargs.get("periods", [])
    self.n_transits_min = kwargs.get("n_transits_min", constants.N_TRANSITS_MIN)
    self.R_star_min = kwargs.get("R_star_min", constants.R_STAR_MIN)
    self.R_star_max = kwargs.get("R_star_max", constants.R_STAR_MAX)
    self.M_star_min = kwargs.get("M_star_min", constants.M_STAR_MIN)
    self.M_star_max = kwargs.get("M_star_max", constants.M_STAR_MAX)
    self.duration_grid_step = kwargs.get("duration_grid_step", constants.DURATION_GRID_STEP)
    self.use_threads = kwargs.get("use_threads", multiprocessing.cpu_count())
    self.per = kwargs.get("per", constants.DEFAULT_PERIOD)
    self.rp = kwargs.get("rp", constants.DEFAULT_RP)
    self.a = kwargs.get("a", constants.DEFAULT_A)
    self.T0_fit_margin = kwargs.get("T0_fit_margin", constants.T0_FIT_MARGIN)
    # precision: "fp64" (plain FP64 search) or "fp32" (FP32 chi2 with
    # compensated prefix sums; candidates re-evaluated in FP64)
    self.precision = kwargs.get("precision", "fp64")
    if self.precision not in ("fp64", "fp32"):
        raise ValueError('precision must be "fp64" or "fp32"')
    self.batch_periods = kwargs.get("batch_periods", None)
    # distributed: shard the search over the ranks of the initialised
    # torch.distributed process group (one process per GPU)
    self.distributed = bool(kwargs.get("distributed", False))
    # refine: move the best peak below grid resolution with the adjoint of
    # the limb-darkened model chi2 (the grid result is kept if chi2 does not
    # decrease)
    self.refine = bool(kwargs.get("refine", False))

    if "b" in kwargs:
        self.b = kwargs.get("b")
        self.inc = impact_to_inclination(b=self.b, semimajor_axis=self.a)
    else:
        self.inc = kwargs.get("inc", constants.DEFAULT_INC)
    self.ecc = kwargs.get("ecc", constants.DEFAULT_ECC)
    self.w = kwargs.get("w", constants.DEFAULT_W)
    self.u = kwargs.get("u", constants.DEFAULT_U)
    self.limb_dark = kwargs.get("limb_dark", constants.DEFAULT_LIMB_DARK)

    self.transit_template = kwargs.get("transit_template", "default")
    if self.transit_template == "default":
        self.per = constants.DEFAULT_PERIOD
        self.rp = constants.DEFAULT_RP
        self.a = constants.DEFAULT_A
        self.inc = constants.DEFAULT_INC
    elif self.transit_template == "grazing":
        self.b = constants.GRAZING_B
        self.inc = impact_to_inclination(b=self.b, semimajor_axis=self.a)
    elif self.transit_template == "box":
        self.per = constants.BOX_PERIOD
        self.rp = constants.BOX_RP
        self.a = constants.BOX_A
        self.b = constants.BOX_B
        self.inc = constants.BOX_INC
        self.u = constants.BOX_U
        self.limb_dark = constants.BOX_LIMB_DARK
    else:
        raise ValueError('Unknown transit_template. Known values: "default", "grazing", "box"')

    if self.R_star <= 0 or self.R_star >= float("inf"):
        raise ValueError("R_star must be positive")
    if self.R_star_min > self.R_star:
        raise ValueError("R_star_min <= R_star is required")
    if self.R_star_min <= 0 or self.R_star_min >= float("inf"):
        raise ValueError("R_star_min must be positive")
    if self.R_star_max < self.R_star:
        raise ValueError("R_star_max >= R_star is required")
    if self.R_star_max <= 0 or self.R_star_max >= float("inf"):
        raise ValueError("R_star_max must be positive")
    if self.M_star <= 0 or self.M_star >= float("inf"):
        raise ValueError("M_star must be positive")
    if self.M_star_min > self.M_star:
        raise ValueError("M_star_min <= M_star is required")
    if self.M_star_min <= 0 or self.M_star_min >= float("inf"):
        raise ValueError("M_star_min must be positive")
    if self.M_star_max < self.M_star:
        raise ValueError("M_star_max >= M_star required")
    if self.M_star_max <= 0 or self.M_star_max >= float("inf"):
        raise ValueError("M_star_max must be positive")
    if self.period_min < 0:
        raise ValueError("period_min >= 0 required")
    if self.period_min >= self.period_max:
        raise ValueError("period_min < period_max required")
    if not isinstance(self.n_transits_min, int):
        raise ValueError("n_transits_min must be an integer value")
    if self.n_transits_min < 1:
        raise ValueError("n_transits_min must be an integer value >= 1")
    if not isinstance(self.use_threads, int) or self.use_threads < 1:
        raise ValueError("use_threads must be an integer value >= 1")
    if self.T0_fit_margin < 0:
        self.T0_fit_margin = 0
    elif self.T0_fit_margin > 0.125:
        self.T0_fit_margin = 0.125
    return self, kwargs
