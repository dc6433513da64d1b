"""Batched search: many light curves, one independent TLS search each.

``gtls_batch(curves).power(**kw)`` runs, for every curve, the same search
``gtls(t, y, dy).power(**kw)`` runs for it alone (the sequence of
``core.search_multi_periods`` in the reference's ``src/gputls/core.py``), but
each GPU pass covers all curves at once: one ``gtls_search_batch`` call for
the main pass over every curve's own period grid, one for the re-search of
every curve's candidates, one for the harmonics and one for the best period.
The per-curve steps between the passes (outlier mask, spectra, candidate
choice) and the host statistics of the best period stay per curve.

The reference has no batched form; it searches one curve per ``gtls``
object.  ``precision`` defaults to "fp32" here (FP32 chi2 with float-float
prefix sums in the main pass and the candidate re-search, then an FP64
re-check of each curve's best 32 candidates; harmonics and the best period in
FP64).
"""
import types

import numpy as np

from . import _lib, constants, core, template
from .grid import duration_grid, period_grid
from .validate import validate_args, validate_inputs

_h2d = _lib.h2d
_d2h = _lib.d2h


class CurveSetOnDevice:
    """Light curves and their duration tables, concatenated on one GPU.

    Curve ``c`` owns samples ``[sample_off[c], sample_off[c+1])`` and
    durations ``[dur_off[c], dur_off[c+1])``; its template rows (``1 -
    template``, padded with 1 to its own ``max_width``) start at
    ``tmpl_off[c]``."""

    def __init__(self, prepared, device=0):
        import torch
        self.torch = torch
        self.device = device
        self.dev = torch.device("cuda:%d" % device)
        self.prepared = prepared
        C = len(prepared)
        self.n = np.array([len(p["t"]) for p in prepared], dtype=np.int64)
        self.sample_off = np.concatenate([[0], np.cumsum(self.n)]).astype(np.int64)
        self.span = np.array([p["span"] for p in prepared], dtype=np.float32)
        self.t_max = np.array([np.max(np.abs(p["t"])) for p in prepared])
        D = np.array([len(p["widths"]) for p in prepared], dtype=np.int64)
        if np.any(D > _lib.MAX_DURATIONS):
            raise ValueError("at most %d distinct durations are supported" % _lib.MAX_DURATIONS)
        self.dur_off = np.concatenate([[0], np.cumsum(D)]).astype(np.int64)
        self.max_width = np.array([p["maxd"] for p in prepared], dtype=np.int32)
        sizes = D * self.max_width
        self.tmpl_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if C else np.zeros(0, np.int64)
        cat = lambda k, dt: np.concatenate([np.asarray(p[k], dtype=dt) for p in prepared])
        on_device = [p["tmpl"] is None for p in prepared]
        if any(on_device) and not all(on_device):
            raise ValueError("a curve set's templates are all built on the host or all on the device")
        if all(on_device):
            # every curve's template rows and overshoots built on the GPU in one call
            planets = {p["planet"] for p in prepared}
            if len(planets) != 1:
                raise ValueError("one template planet per curve set")
            tm_dev = torch.empty(int(np.sum(sizes)), dtype=torch.float64, device=self.dev)
            ov_dev = torch.empty(int(self.dur_off[-1]), dtype=torch.float64, device=self.dev)
            _lib.template_cache(planets.pop(), [p["samples"] for p in prepared], self.dur_off, cat("widths", np.int32),
                                self.tmpl_off, self.max_width, ov_dev, tm_dev, device=device)
            ov = _d2h(ov_dev)
            for c, p in enumerate(prepared):
                p["overshoot"] = ov[self.dur_off[c]:self.dur_off[c + 1]]
        else:
            tm = np.empty(int(np.sum(sizes)), dtype=np.float64)
            for c, p in enumerate(prepared):
                rows = np.pad(p["tmpl"], ((0, 0), (0, p["maxd"] - p["tmpl"].shape[1])), constant_values=1.0)
                tm[self.tmpl_off[c]:self.tmpl_off[c] + sizes[c]] = rows.ravel()
            tm_dev = _h2d(torch, tm, self.dev)
            ov_dev = _h2d(torch, cat("overshoot", np.float64), self.dev)
        self.curves = dict(t=_h2d(torch, cat("t", np.float64), self.dev),
                           y=_h2d(torch, cat("y", np.float64), self.dev),
                           dy=_h2d(torch, cat("dy", np.float64), self.dev),
                           sample_off=self.sample_off, span=self.span)
        self.tables = dict(widths=_h2d(torch, cat("widths", np.int32), self.dev), overshoot=ov_dev,
                           templates=tm_dev,
                           dur_off=self.dur_off, tmpl_off=self.tmpl_off, max_width=self.max_width)
        # every curve's own trial periods (ascending), resident for the main pass
        self.period_off = np.concatenate([[0], np.cumsum([len(p["periods"]) for p in prepared])]).astype(np.int64)
        self.periods = cat("periods", np.float64)
        self.periods_dev = _h2d(torch, self.periods, self.dev)

    def __len__(self):
        return len(self.prepared)

    def curve_view(self, c):
        """Curve ``c`` as the (curve, tables) dicts of a single-curve ``_lib.search``
        (views of the concatenated device arrays, no copies)."""
        a, b = int(self.sample_off[c]), int(self.sample_off[c + 1])
        d0, d1 = int(self.dur_off[c]), int(self.dur_off[c + 1])
        mw = int(self.max_width[c])
        t0 = int(self.tmpl_off[c])
        curve = dict(t=self.curves["t"][a:b], y=self.curves["y"][a:b], dy=self.curves["dy"][a:b],
                     span=float(self.span[c]))
        tables = dict(widths=self.tables["widths"][d0:d1], overshoot=self.tables["overshoot"][d0:d1],
                      templates=self.tables["templates"][t0:t0 + (d1 - d0) * mw].view(d1 - d0, mw), max_width=mw)
        return curve, tables

    def search(self, periods, period_off, depth_min, skip_point, batches, pass_, precision, want_loc=False,
               timing=None, periods_dev=None):
        """One ``gtls_search_batch`` pass over host ``periods`` (curve c at
        ``period_off[c]:period_off[c+1]``); ``periods_dev`` is the same array
        already on the device, if the caller has it."""
        periods = np.asarray(periods, dtype=np.float64)
        period_off = np.asarray(period_off, dtype=np.int64)
        for c in range(len(self)):
            seg = periods[period_off[c]:period_off[c + 1]]
            if len(seg) and (not np.min(seg) > 0 or self.t_max[c] / np.min(seg) >= 2.0 ** 31):
                # the fold truncates t/P to a 32-bit int (GPUFun.py:39)
                raise ValueError("periods must be > 0 and max|t| / min(period) < 2^31")
        if periods_dev is None:
            periods_dev = _h2d(self.torch, periods, self.dev)
        return _lib.search_batch(self.curves, periods_dev, period_off, self.tables, depth_min, skip_point, batches,
                                 pass_, precision, device=self.device, want_loc=want_loc, timing=timing)


def template_planet(opts):
    """(per, rp, a, inc, u1, u2) of the template planet of ``opts`` (the
    reference's "default", "grazing" or "box" template after validate_args);
    linear limb darkening has u2 = 0."""
    u = list(np.atleast_1d(opts.u))
    if opts.limb_dark == "linear":
        u = [u[0] if len(u) else 0.0, 0.0]
    elif opts.limb_dark != "quadratic":
        raise ValueError("limb_dark must be 'quadratic' or 'linear'")
    if opts.ecc != 0:
        raise ValueError("only circular template orbits (ecc=0) are supported")
    return (float(opts.per), float(opts.rp), float(opts.a), float(opts.inc), float(u[0]), float(u[1]))


def prepare_curve(t, y, dy, opts, device=0, templates="host"):
    """Clean one curve and build its grids and templates as ``gtls.power`` does
    (main.py:86-148 of the reference): period grid, duration grid, template
    cache deduplicated by width.  ``templates="device"`` leaves the template
    rows and overshoots to ``CurveSetOnDevice`` (built on the GPU for all
    curves at once, ``gtls_template_cache``); the widths and durations, which
    depend on the grids alone, are set here."""
    t, y, dy = validate_inputs(t, y, dy)
    if len(opts.periods) == 0:
        periods = period_grid(R_star=opts.R_star, M_star=opts.M_star, time_span=np.max(t) - np.min(t),
                              period_min=opts.period_min, period_max=opts.period_max,
                              oversampling_factor=opts.oversampling_factor, n_transits_min=opts.n_transits_min,
                              device=device, ascending=True)
    else:
        periods = np.sort(np.asarray(opts.periods, dtype=np.float64))
    durations = duration_grid(periods, shortest=1 / len(t), log_step=opts.duration_grid_step)
    maxwidth = int(np.max(durations) * np.size(y))
    if maxwidth % 2 != 0:
        maxwidth = maxwidth + 1
    if templates == "device":
        # get_cache's widths (transit.py:119-121) and device_templates' dedup (core.py:605-614)
        dur = np.asarray(durations, dtype=np.float64)
        occupied = np.array([int((d / np.max(dur)) * maxwidth) for d in dur], dtype=np.int64)
        widths, first = np.unique(occupied, return_index=True)
        widths = widths.astype(np.int32)
        durs = dur[first]
        overshoot, tmpl = None, None
        maxd = int(np.max(widths)) + int(np.max(widths)) % 2
        planet = template_planet(opts)
    else:
        overview, lc_arr = template.get_cache(durations=durations, maxwidth_in_samples=maxwidth, per=opts.per,
                                              rp=opts.rp, a=opts.a, inc=opts.inc, ecc=opts.ecc, w=opts.w, u=opts.u,
                                              limb_dark=opts.limb_dark, verbose=False)
        widths, overshoot, durs, tmpl, maxd = template.device_templates(lc_arr, overview)
        planet = None
    return dict(t=np.ascontiguousarray(t, dtype=np.float64), y=np.ascontiguousarray(y, dtype=np.float64),
                dy=np.ascontiguousarray(dy, dtype=np.float64), periods=np.ascontiguousarray(periods),
                span=float(np.float32(np.max(t) - np.min(t))), widths=widths, overshoot=overshoot,
                durations=durs, tmpl=tmpl, maxd=int(maxd), duration_grid=np.asarray(durations),
                samples=int(maxwidth), planet=planet)


def _offsets(counts):
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


class gtls_batch(object):
    """Transit least squares of many light curves on one B200.

    ``curves``: a sequence of ``(t, y)`` or ``(t, y, dy)``.  ``power(**kw)``
    takes the keywords of ``gtls.power`` (applied to every curve) plus
    ``full_stats`` (default False: period, duration, depth, T0 and SDE only;
    True adds transit times and the SNRs) and ``keep_spectra`` (default
    True: each result carries its periods, power and chi2) and ``autotune``
    (default True: launch shapes timed and chosen on the data, see
    ``gtls_b200.tune``; results do not depend on them), ``templates``
    ("device", default: every curve's template tables built on the GPU in one
    call, ``gtls_template_cache``; "host": the reference's host construction,
    ``template.get_cache``; the two agree to about 1e-15); ``refine=True``
    refines every curve's best peak in one batched adjoint run (see
    ``refine_results``).  With
    ``distributed=True`` under an initialised torch.distributed process group
    (one process per GPU) every rank searches a work-balanced share of the
    curves and all ranks return every curve's result."""

    def __init__(self, curves, verbose=False):
        self.curves = [tuple(c) + (None,) * (3 - len(c)) for c in curves]
        if not self.curves:
            raise ValueError("no light curves given")
        self.verbose = verbose

    def power(self, **kwargs):
        full_stats = bool(kwargs.pop("full_stats", False))
        autotune = bool(kwargs.pop("autotune", True))
        keep_spectra = bool(kwargs.pop("keep_spectra", True))
        templates = kwargs.pop("templates", "device")
        if templates not in ("device", "host"):
            raise ValueError('templates must be "device" or "host"')
        timing = kwargs.pop("timing", None)
        phases = kwargs.pop("phases", None)
        kwargs.setdefault("precision", "fp32")
        opts = types.SimpleNamespace()
        opts, kwargs = validate_args(opts, kwargs)
        device = opts.GPUDeviceID
        if opts.GPUDeviceIDs:
            device = opts.GPUDeviceIDs[0]
        per_curve_batch = opts.batch_periods is not None and np.ndim(opts.batch_periods) > 0
        if per_curve_batch and len(opts.batch_periods) != len(self.curves):
            raise ValueError("batch_periods must be one value or one per curve")

        def search_subset(indices):
            sub = opts
            if per_curve_batch:
                sub = types.SimpleNamespace(**vars(opts))
                sub.batch_periods = np.asarray(opts.batch_periods)[list(indices)]
            ph = core.Phases(phases)
            prepared = [prepare_curve(*self.curves[i], sub, device=device, templates=templates) for i in indices]
            ph.mark("prepare_curves")
            out = search_prepared(prepared, sub, device=device, full_stats=full_stats,
                                  keep_spectra=keep_spectra, timing=timing, autotune=autotune, phases=phases)
            if opts.refine and out:
                ph = core.Phases(phases)
                refine_results(out, prepared, opts.u, device)
                ph.mark("refine")
            return out

        if opts.distributed:
            # each rank searches a share of the curves balanced by estimated
            # work (samples x time span, which the period count follows)
            from . import shard
            costs = [len(c[0]) * float(np.ptp(np.asarray(c[0], dtype=np.float64))) for c in self.curves]
            return shard.sharded_curves(costs, search_subset)
        return search_subset(list(range(len(self.curves))))


def refine_results(out, prepared, u, device):
    """power(refine=True): every curve's best peak refined in one batched run
    of the adjoint of the limb-darkened model chi2 (``refine.refine_peaks``);
    a result takes the refined period, T0, duration and depth only where the
    model chi2 decreased, and ``r.refinement`` keeps both."""
    from . import refine as R
    starts, scales = [], []
    for r, p in zip(out, prepared):
        a, b = R.grid_start(r.period, r.T0, r.duration, r.depth, u, p["periods"], p["t"])
        starts.append(a)
        scales.append(b)
    params, chi, chi0, ok = R.refine_peaks([(p["t"], p["y"], p["dy"]) for p in prepared], np.array(starts),
                                           np.array(scales), device=device)
    for c, r in enumerate(out):
        r.refinement = dict(grid=dict(period=r.period, T0=r.T0, duration=r.duration, depth=r.depth),
                            params=params[c], chi2=float(chi[c]), chi2_grid=float(chi0[c]), improved=bool(ok[c]))
        if ok[c]:
            r.period, r.T0, r.duration, r.depth = (float(v) for v in params[c][:4])
            if hasattr(r, "transit_times"):
                r.transit_times = R.refined_transit_times(r.transit_times, r.T0, r.period)


def _recheck_fp64(cs, cand, cand_p, c_off, spectra, chi2_dev, p_off, S, depth_min, skip, torch):
    """FP64 re-check of every curve's best ``core.FP64_RECHECK`` candidates
    (``core.recheck_plan``), as one batched FP64 search: entry c of the call
    is curve c restricted to its re-checked candidates and their batch's
    duration union (a curve whose re-checked candidates span several batches
    of the candidate list adds one more single-curve call per extra batch)."""
    dev = cs.dev
    C = len(cs)
    plans = []
    for c in range(C):
        if len(cand[c]) == 0:
            plans.append([])
            continue
        _, _, power_dev, _, _ = spectra(c)
        ci = torch.as_tensor(cand[c], device=dev)
        plans.append(core.recheck_plan(cand_p[c_off[c]:c_off[c + 1]], _d2h(power_dev[ci]), cs.prepared[c]["widths"],
                                       float(cs.span[c]), int(cs.n[c]), int(S[c]), cs.device))
    # first batch of every curve's plan in one call
    widths, overshoot, templ, periods, dur_n, tmpl_n, per_n, gidx = [], [], [], [], [], [], [], []
    for c in range(C):
        d0 = int(cs.dur_off[c])
        mw = int(cs.max_width[c])
        t0 = int(cs.tmpl_off[c])
        if plans[c]:
            sel, union = plans[c][0]
        else:
            sel, union = np.zeros(0, dtype=np.int64), np.zeros(1, dtype=np.int64)   # no periods: any duration
        u = torch.as_tensor(union, device=dev)
        widths.append(cs.tables["widths"][d0 + u])
        overshoot.append(cs.tables["overshoot"][d0 + u])
        rows = cs.tables["templates"][t0:t0 + (int(cs.dur_off[c + 1]) - d0) * mw].view(-1, mw)
        templ.append(rows[u].reshape(-1))
        dur_n.append(len(union))
        tmpl_n.append(len(union) * mw)
        periods.append(cand_p[c_off[c]:c_off[c + 1]][sel])
        per_n.append(len(sel))
        gidx.append(cand[c][sel] + p_off[c])
    if sum(per_n):
        tables = dict(widths=torch.cat(widths).contiguous(), overshoot=torch.cat(overshoot).contiguous(),
                      templates=torch.cat(templ).contiguous(), dur_off=_offsets(dur_n),
                      tmpl_off=_offsets(tmpl_n)[:-1], max_width=cs.max_width)
        pc = np.concatenate(periods)
        c64, _ = _lib.search_batch(cs.curves, _h2d(torch, pc, dev), _offsets(per_n), tables, depth_min, skip,
                                   np.maximum(np.array(per_n), 1).astype(np.int32), _lib.GTLS_PASS_ALL, "fp64",
                                   device=cs.device, want_loc=False, flags=_lib.GTLS_SEARCH_ALL_DURATIONS)
        chi2_dev[_h2d(torch, np.concatenate(gidx), dev)] = c64
    # further batches (rare): one single-curve call each
    for c in range(C):
        for sel, union in plans[c][1:]:
            curve_c, tables_c = cs.curve_view(c)
            ch, _ = _lib.search(curve_c, _h2d(torch, cand_p[c_off[c]:c_off[c + 1]][sel], dev),
                                core.subset_tables(tables_c, union, torch), depth_min, skip, len(sel),
                                _lib.GTLS_PASS_ALL, "fp64", device=cs.device, want_loc=False,
                                flags=_lib.GTLS_SEARCH_ALL_DURATIONS)
            chi2_dev[_h2d(torch, cand[c][sel] + p_off[c], dev)] = ch


def search_prepared(prepared, opts, device=0, full_stats=False, keep_spectra=True, timing=None, autotune=False,
                    phases=None):
    """The batched search of curves already prepared by ``prepare_curve``.

    Returns one ``types.SimpleNamespace`` per curve with period, duration,
    depth, T0, SDE, SDE_raw, period_index, width, rawDuration and (with
    ``keep_spectra``) periods, power and chi2 as masked arrays.  With
    ``autotune`` the launch shapes are first tuned on the set's largest
    curve (``tune.tune_curve_set``; cached per shape, results unchanged)."""
    ph = core.Phases(phases)
    cs = CurveSetOnDevice(prepared, device=device)
    ph.mark("upload")
    if autotune:
        from . import tune
        tune.tune_curve_set(cs, opts.precision)
        ph.mark("tune")
    return search_on_device(cs, opts, full_stats=full_stats, keep_spectra=keep_spectra, timing=timing, phases=phases)


def search_on_device(cs, opts, full_stats=False, keep_spectra=True, timing=None, phases=None):
    """The batched search of a ``CurveSetOnDevice`` (see ``search_prepared``).
    ``phases``: optional dict receiving the wall-clock seconds of each phase."""
    import torch
    ph = core.Phases(phases)
    prepared = cs.prepared
    device = cs.device
    dev = cs.dev
    C = len(cs)
    skip = core.skip_point_of(opts.T0_fit_margin)
    osf = opts.oversampling_factor
    depth_min = opts.transit_depth_min
    np_c = np.diff(cs.period_off)
    p_off = cs.period_off
    if opts.batch_periods is None:
        free = torch.cuda.mem_get_info(device)[0]
        S = np.array([core.reference_batch_size(int(np_c[c]), int(cs.n[c]), int(cs.max_width[c]),
                                                int(cs.dur_off[c + 1] - cs.dur_off[c]), free) for c in range(C)],
                     dtype=np.int32)
    else:
        S = np.broadcast_to(np.asarray(opts.batch_periods, dtype=np.int32), (C,)).copy()
    periods_h = cs.periods
    periods_dev = cs.periods_dev

    # main pass
    chi2_dev, _ = cs.search(periods_h, p_off, depth_min, skip, S, _lib.GTLS_PASS_MAIN, opts.precision,
                            timing=timing, periods_dev=periods_dev)
    ph.mark("main_pass")
    raw_chi2 = _d2h(chi2_dev)
    mask = np.zeros(len(raw_chi2), dtype=bool)
    for c in range(C):
        seg = raw_chi2[p_off[c]:p_off[c + 1]]
        mask[p_off[c]:p_off[c + 1]] = seg > (100 * np.median(seg))
    mask_dev = _h2d(torch, mask.astype(np.uint8), dev)

    def spectra(c):
        a, b = int(p_off[c]), int(p_off[c + 1])
        return core._spectra(chi2_dev[a:b], mask_dev[a:b], osf, device)

    # candidates of every curve re-searched at every start: in FP64, or (FP32
    # form) in FP32 followed by an FP64 re-check of each curve's best
    # core.FP64_RECHECK candidates over their batch's duration union
    cand = []
    for c in range(C):
        a, b = int(p_off[c]), int(p_off[c + 1])
        _, _, power_dev, _, _ = spectra(c)
        cand.append(core._candidates(power_dev, mask_dev[a:b], periods_dev[a:b], torch))
    c_off = _offsets([len(x) for x in cand])
    cand_p = np.concatenate([prepared[c]["periods"][cand[c]] for c in range(C)])
    fp32 = opts.precision == "fp32"
    ph.mark("mask_spectra_candidates")
    again, _ = cs.search(cand_p, c_off, depth_min, skip, S, _lib.GTLS_PASS_ALL, "fp32" if fp32 else "fp64")
    gidx = _h2d(torch, np.concatenate([cand[c] + p_off[c] for c in range(C)]), dev)
    chi2_dev[gidx] = again
    mask_dev[gidx] = 0
    ph.mark("candidate_research")
    if fp32:
        _recheck_fp64(cs, cand, cand_p, c_off, spectra, chi2_dev, p_off, S, depth_min, skip, torch)
        ph.mark("fp64_recheck")
    period = np.empty(C)
    h_idx = []
    for c in range(C):
        _, _, power_dev, _, _ = spectra(c)
        ci = torch.as_tensor(cand[c], device=dev)
        best = int(cand[c][int(torch.argmax(power_dev[ci]).item())])
        P = prepared[c]["periods"][best]
        idx, _ = core.find_nearest_indices([P * r for r in (0.5, 1, 2, 2 / 3, 3 / 2)], prepared[c]["periods"])
        h_idx.append(idx)

    ph.mark("best_candidate")
    # harmonics
    h_off = _offsets([len(x) for x in h_idx])
    h_p = np.concatenate([prepared[c]["periods"][h_idx[c]] for c in range(C)])
    again2, _ = cs.search(h_p, h_off, depth_min, skip, S, _lib.GTLS_PASS_ALL, "fp64")
    gidx = _h2d(torch, np.concatenate([h_idx[c] + p_off[c] for c in range(C)]), dev)
    chi2_dev[gidx] = again2
    mask_dev[gidx] = 0
    ph.mark("harmonics_research")
    best_idx = np.empty(C, dtype=np.int64)
    sde = np.empty(C)
    sde_raw = np.empty(C)
    power_all = []
    for c in range(C):
        _, _, power_dev, sde_raw[c], sde[c] = spectra(c)
        hi = torch.as_tensor(h_idx[c], device=dev)
        best_idx[c] = int(h_idx[c][int(torch.argmax(power_dev[hi]).item())])
        period[c] = float(prepared[c]["periods"][best_idx[c]])
        if keep_spectra:
            power_all.append(power_dev)

    ph.mark("spectra_best_harmonic")
    # best period of every curve at every start and duration of its range
    one = np.ones(C, dtype=np.int32)
    chi2_b, loc_b = cs.search(period, _offsets(one), depth_min, 1, one, _lib.GTLS_PASS_ALL, "fp64", want_loc=True)
    loc_h = _d2h(loc_b)
    ph.mark("best_period_search")
    chi2_bh = _d2h(chi2_b)
    chi2_h = _d2h(chi2_dev) if keep_spectra else None
    mask_h = _d2h(mask_dev).astype(bool) if keep_spectra else None
    out = []
    for c in range(C):
        p = prepared[c]
        fin = core.finish_period(p["widths"], p["durations"], p["overshoot"], p["maxd"], p["span"], period[c],
                                 int(loc_h[c]), p["t"], p["y"], device=device, full_stats=full_stats)
        r = types.SimpleNamespace(period=period[c], period_index=int(best_idx[c]), SDE=float(sde[c]),
                                  SDE_raw=float(sde_raw[c]), duration=fin["duration"], depth=fin["depth"],
                                  T0=fin["T0"], width=fin["width"], rawDuration=fin["raw_duration"],
                                  loc=fin["loc"], chi2_best=float(chi2_bh[c]), batch_periods=int(S[c]))
        if full_stats:
            for k in ("transit_times", "snr", "snr_pink", "snr_fit", "snr_fit_pink"):
                setattr(r, k, fin[k])
        if keep_spectra:
            a, b = int(p_off[c]), int(p_off[c + 1])
            m = mask_h[a:b]
            r.periods = np.ma.array(p["periods"], mask=m)
            r.power = np.ma.array(_d2h(power_all[c]), mask=m)
            r.chi2 = np.ma.array(chi2_h[a:b], mask=m)
            r.chi2_main = raw_chi2[a:b]
        out.append(r)
    ph.mark("finish_host")
    return out
