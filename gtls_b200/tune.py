"""Autotuning of the search's launch shapes on the caller's own data.

The tile of starts per chi2 CTA, where the chi2 kernel reads the folded
records from (a shared-memory tile, or global memory through a large L1),
and the number of phase buckets of the global-scatter fold ordering change
only the time of a search, never its result (every chi2 value and argmin
location is the same; ``tests/test_gpu_tune.py``).  Which setting is fastest
depends on the curves: the tile against the longest duration (halo re-reads
versus work per CTA; in the FP64 form on a 70,000-sample, 8,400-width curve
the records read through L1, in tiles of 10,240 starts, beat the staged tile
by 7.5%), the bucket count against how clustered the folded phases are (it
matters only for curves above 2^17 samples, which take the global-scatter
ordering).  ``autotune`` times the main pass of a sample of the trial
periods under each candidate setting, with the library's own CUDA-event
stage timing, and keeps the fastest for the context (``gtls_set_tuning``).
Results are cached per (precision, samples rounded to a power of two,
longest width rounded to a power of two).
"""
import itertools

import numpy as np

from . import _lib

TILE_CAPS = {"fp32": (8192, 12288, 16384, 24576), "fp64": (4096, 8192, 10240, 12288)}
BUCKET_SHIFTS = (0, -1)
RECORDS_GLOBAL = (0, 1)
PACKED_MAX_N = 1 << 17   # curves up to this many samples order their phases in shared memory
DEFAULT_CAP = {"fp32": 16384, "fp64": 8192}
MARGIN = 0.02   # a setting must beat the default by this fraction to be chosen
_CACHE = {}


def _key(precision, n, maxd):
    return precision, int(np.ceil(np.log2(max(n, 2)))), int(np.ceil(np.log2(max(maxd, 2))))


def autotune(run_main_pass, precision, n, maxd, device=0, repeats=2):
    """Pick the fastest (tile cap, records mode, bucket shift) for ``precision``.

    ``run_main_pass(timing)`` runs the main pass of a representative sample
    of periods and fills the ``_lib.Timing`` it is given.  Returns the chosen
    setting (a dict) and leaves it set on ``device``."""
    key = _key(precision, n, maxd)
    if key in _CACHE:
        best = _CACHE[key]
    else:
        prev = _lib.get_tuning(device)
        trials = []
        shifts = BUCKET_SHIFTS if n > PACKED_MAX_N else (0,)
        for cap, rg, shift in itertools.product(TILE_CAPS[precision], RECORDS_GLOBAL, shifts):
            cfg = dict(prev)
            cfg["tile_cap_" + precision] = cap
            cfg["records_global"] = rg
            cfg["bucket_shift"] = shift
            _lib.set_tuning(device=device, **cfg)
            ms = []
            for _ in range(repeats):
                tm = _lib.Timing()
                run_main_pass(tm)
                ms.append(tm.prepare_ms + tm.chi2_ms + tm.finish_ms)
            trials.append((min(ms), cap, rg, shift, cfg))
        trials.sort(key=lambda x: (x[0], x[1], x[2], -x[3]))
        best = trials[0][4]
        # keep the default unless another setting is clearly faster (timing noise
        # would otherwise make the choice differ from run to run)
        dflt = [x for x in trials if x[1] == DEFAULT_CAP[precision] and x[2] == 0 and x[3] == 0]
        if dflt and trials[0][0] > (1.0 - MARGIN) * dflt[0][0]:
            best = dflt[0][4]
        _CACHE[key] = best
    _lib.set_tuning(device=device, **best)
    return dict(best)


def tune_curve_set(cs, precision, n_sample=600, device=None):
    """``autotune`` for a ``batch.CurveSetOnDevice``: the main pass over every
    k-th period of the curve set's largest curve (by samples x periods)."""
    device = cs.device if device is None else device
    counts = np.diff(cs.period_off)
    c = int(np.argmax(cs.n * counts))
    a, b = int(cs.period_off[c]), int(cs.period_off[c + 1])
    step = max(1, (b - a) // n_sample)
    sub = np.arange(a, b, step)[:n_sample]
    periods = cs.periods[sub]
    p_dev = cs.periods_dev[a:b:step][:n_sample].contiguous()
    # a one-curve set view: only curve c has periods
    off = np.zeros(len(cs) + 1, dtype=np.int64)
    off[c + 1:] = len(periods)
    batches = np.full(len(cs), 50, dtype=np.int32)

    def run(tm):
        cs.search(periods, off, 1e-5, 8, batches, _lib.GTLS_PASS_MAIN, precision, timing=tm, periods_dev=p_dev)

    return autotune(run, precision, int(cs.n[c]), int(cs.max_width[c]), device=device)


def tune_curve(cur, periods, precision, n_sample=600, batch=50):
    """``autotune`` for one ``core.CurveOnDevice``: the main pass over every
    k-th of its sorted trial ``periods`` (host array)."""
    periods = np.asarray(periods, dtype=np.float64)
    step = max(1, len(periods) // n_sample)
    sub = np.ascontiguousarray(periods[::step][:n_sample])

    def run(tm):
        cur.search(sub, 1e-5, 8, batch, _lib.GTLS_PASS_MAIN, precision, timing=tm)

    return autotune(run, precision, cur.n, cur.maxd, device=cur.device)
