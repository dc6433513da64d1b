"""Search driver: the sequence of ``core.search_multi_periods`` on the GPU.

Follows the reference's ``src/gputls/core.py``:

* main pass over the period grid with per-batch duration unions
  (:568-875) -> ``gtls_search`` (pass MAIN);
* outlier mask ``chi2 > 100 * median`` and spectra (:890-898) ->
  ``gtls_spectra``;
* candidates: top 100 by power, then the next 100 with P > 1 d (:904-915);
* re-search of the candidates with every phase start (:930-950,
  ``search_multi_periods_again`` :1001-1247) -> ``gtls_search`` (pass ALL);
* harmonics {1/2, 1, 2, 2/3, 3/2} x P re-searched (:952-981);
* best period: duration index, T0 index, depth, T0, duration in days and SNRs
  (``search_single_periods`` :1250-1505): the chi2 part on the GPU, the
  rest on the host as in the reference.

All device buffers stay resident between the passes; the host sees only the
chi2/power arrays it returns and the candidate indices.
"""
import numpy as np
import numpy.ma as ma

from . import _lib, constants, stats, template

TRANSFER = _lib.TRANSFER
_h2d = _lib.h2d
_d2h = _lib.d2h


def skip_point_of(T0_fit_margin):
    """SKIP_POINT of the kernels (core.py:597-601)."""
    return constants.SKIP_POINT_NEVER if T0_fit_margin == 0 else int(1 / T0_fit_margin)


def reference_batch_size(n_periods, n_samples, maxd, n_durations, free_bytes):
    """Periods per duration-union batch as core.py:620-628 sizes it (at least 1)."""
    m = n_samples + maxd
    cap = free_bytes / (5 * (m * 2 + 2 + n_durations * m * 4 + 2 * n_durations))
    s = int(np.min([np.floor(cap), n_periods / 30]))
    if s < 15:
        s = int(s / 1.1)
    return max(1, s)


class Phases:
    """Wall-clock time per phase of a search (a dict given by the caller),
    with a device synchronisation at each boundary; no-op when the caller
    gives none."""

    def __init__(self, out):
        self.out = out
        self.t = None
        if out is not None:
            import time
            import torch
            self._time, self._sync = time.perf_counter, torch.cuda.synchronize
            self._sync()
            self.t = self._time()

    def mark(self, name):
        if self.out is None:
            return
        self._sync()
        now = self._time()
        self.out[name] = self.out.get(name, 0.0) + (now - self.t)
        self.t = now


def find_nearest_indices(a, b):
    """Nearest element of ``b`` to each value of ``a``, first occurrence (core.py:34-46)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    idx = np.array([int(np.argmin(np.abs(b - v))) for v in a], dtype=int)
    return idx, b[idx]


class CurveOnDevice:
    """A light curve and its duration tables resident on one GPU."""

    def __init__(self, t, y, dy, lc_arr, lc_cache_overview, device=0):
        import torch
        self.torch = torch
        self.device = device
        dev = torch.device("cuda:%d" % device)
        self.dev = dev
        self.t_host = np.ascontiguousarray(t, dtype=np.float64)
        self.n = len(self.t_host)
        span = np.max(self.t_host) - np.min(self.t_host)
        self.t_max = float(np.max(np.abs(self.t_host)))
        self.curve = dict(
            t=_h2d(torch, self.t_host, dev),
            y=_h2d(torch, np.asarray(y, dtype=np.float64), dev),
            dy=_h2d(torch, np.asarray(dy, dtype=np.float64), dev),
            span=float(np.float32(span)),
        )
        widths, overshoot, durations, tmpl, maxd = template.device_templates(lc_arr, lc_cache_overview)
        if len(widths) > _lib.MAX_DURATIONS:
            raise ValueError("at most %d distinct durations are supported" % _lib.MAX_DURATIONS)
        self.widths = widths
        self.overshoot = overshoot
        self.durations = durations
        self.maxd = int(maxd)
        self.tables = dict(
            widths=_h2d(torch, widths, dev),
            overshoot=_h2d(torch, overshoot, dev),
            templates=_h2d(torch, np.pad(tmpl, ((0, 0), (0, maxd - tmpl.shape[1])), constant_values=1.0), dev),
            max_width=self.maxd,
        )

    def on_device(self, device):
        """The same curve and tables on another device (self for the same one)."""
        if device == self.device:
            return self
        import copy
        other = copy.copy(self)
        other.device = device
        other.dev = self.torch.device("cuda:%d" % device)
        other.curve = {k: (v.to(other.dev) if hasattr(v, "to") else v) for k, v in self.curve.items()}
        other.tables = {k: (v.to(other.dev) if hasattr(v, "to") else v) for k, v in self.tables.items()}
        return other

    def search(self, periods, depth_min, skip_point, batch, pass_, precision, want_loc=False, timing=None,
               tables=None, flags=0):
        torch = self.torch
        if isinstance(periods, torch.Tensor):
            p = periods.to(self.dev, dtype=torch.float64).contiguous()
        else:
            p = _h2d(torch, np.asarray(periods, dtype=np.float64), self.dev)
        pmin = float(p.min().item())
        if not pmin > 0 or self.t_max / pmin >= 2.0 ** 31:
            # the fold truncates t/P to a 32-bit int (GPUFun.py:39)
            raise ValueError("periods must be > 0 and max|t| / min(period) < 2^31")
        return _lib.search(self.curve, p, self.tables if tables is None else tables, depth_min, skip_point, batch,
                           pass_, precision, device=self.device, want_loc=want_loc, timing=timing, flags=flags)


# candidates re-evaluated in FP64 after the FP32 form's candidate re-search
FP64_RECHECK = 32


def subset_tables(tables, idx, torch):
    """The duration tables restricted to the durations ``idx`` (ascending)."""
    ii = torch.as_tensor(np.asarray(idx, dtype=np.int64), device=tables["widths"].device)
    return dict(widths=tables["widths"][ii].contiguous(), overshoot=tables["overshoot"][ii].contiguous(),
                templates=tables["templates"][ii].contiguous(), max_width=tables["max_width"])


def recheck_plan(cand_p, power_cand, widths, span, n, batch, device, k=FP64_RECHECK):
    """Which candidates the FP32 form re-checks in FP64, and over which durations.

    The candidate re-search groups the candidate list in batches of
    ``batch`` and searches each candidate over its batch's duration union
    (core.py:1081-1115).  The ``k`` candidates of highest power (``power_cand``,
    host, in candidate-list order) are re-searched in FP64 over exactly their
    batch's union (``GTLS_SEARCH_ALL_DURATIONS`` with the union's durations),
    so that each gets the value an FP64 re-search of the whole list gives.
    Returns a list of (positions in the candidate list, union duration
    indices), one entry per batch that holds re-checked candidates."""
    if len(cand_p) == 0:
        return []
    key = np.where(np.isfinite(power_cand), -power_cand, np.inf)
    top = np.argsort(key, kind="stable")[:k]
    wmin, wmax = _lib.duration_ranges(np.asarray(cand_p, dtype=np.float64), span, n, device=device)
    valid = (widths[None, :] >= wmin[:, None]) & (widths[None, :] <= wmax[:, None])
    group = np.arange(len(cand_p)) // batch
    plan = []
    for g in np.unique(group[top]):
        union = np.nonzero(valid[group == g].any(axis=0))[0]
        if len(union):
            plan.append((np.sort(top[group[top] == g]), union))
    return plan


def fp64_recheck(search, cand_p, power_cand, widths, span, n, batch, device, k=FP64_RECHECK):
    """Run ``recheck_plan``: ``search(periods, union)`` is the FP64 search of
    those periods over those durations (returns a chi2 tensor).  Returns
    (positions in the candidate list, their FP64 chi2, host)."""
    pos_out, val_out = [], []
    for sel, union in recheck_plan(cand_p, power_cand, widths, span, n, batch, device, k):
        pos_out.append(sel)
        val_out.append(_d2h(search(np.asarray(cand_p)[sel], union)))
    if not pos_out:
        return np.zeros(0, dtype=np.int64), np.zeros(0)
    return np.concatenate(pos_out), np.concatenate(val_out)


def _spectra(chi2_dev, mask_dev, osf, device):
    sr, praw, power, sde_raw, sde = _lib.spectra(chi2_dev, mask_dev, osf, device=device)
    return sr, praw, power, sde_raw, sde


def _candidates(power_dev, mask_dev, periods_dev, torch):
    """core.py:904-915 with a stable sort by -power (masked entries last)."""
    key = -power_dev
    key = torch.where(mask_dev.bool(), torch.full_like(key, float("inf")), key)
    order = torch.sort(key, stable=True).indices
    top = order[:100]
    rest = order[100:]
    ok = (periods_dev[rest] > 1) & ~mask_dev.bool()[rest]
    nxt = rest[ok][:100]
    idx = torch.cat([top, nxt]).cpu().numpy().astype(np.int64)
    return idx


def search_multi_periods(periods, t, y, dy, transit_depth_min, lc_arr, lc_cache_overview, T0_fit_margin,
                         oversampling_factor, verbose=False, GPUDeviceID=0, fast=False, precision="fp64",
                         batch_periods=None, distributed=False, devices=None):
    """GPU counterpart of core.search_multi_periods (core.py:568-999).

    Returns the reference's 19 values (periods, period, rawDuration,
    durationPoints, duration, depth, T0, SDE, chi2, transitTimes, power, snr,
    snrPink, snrFit, snrFitPink, raw_power, raw_chi2, candidate indices,
    candidate periods) plus a dict of diagnostics, or (periods, power) when
    ``fast``.  ``devices``: more than one CUDA device ids shard the main pass
    over them in this process (the reference's ``GPUDeviceIDs``); the rest
    runs on ``GPUDeviceID``.
    """
    import torch
    periods = np.sort(np.asarray(periods, dtype=np.float64))
    cur = CurveOnDevice(t, y, dy, lc_arr, lc_cache_overview, device=GPUDeviceID)
    periods_dev = _h2d(torch, periods, cur.dev)
    return run_search(cur, periods, periods_dev, t, y, dy, transit_depth_min, T0_fit_margin, oversampling_factor,
                      fast=fast, precision=precision, batch_periods=batch_periods, distributed=distributed,
                      devices=devices)


def run_search(cur, periods, periods_dev, t, y, dy, transit_depth_min, T0_fit_margin, oversampling_factor,
               fast=False, precision="fp64", batch_periods=None, timing=None, distributed=False, group=None,
               phases=None, devices=None):
    """The search on a curve already resident on the device (see search_multi_periods).

    ``periods``: sorted host array, ``periods_dev`` the same on the device.
    ``timing``: optional ``_lib.Timing`` receiving the main pass's stage times.
    ``distributed``: shard the main pass over the ranks of the initialised
    process group ``group`` (batch-aligned period ranges, chi2 all-gathered);
    every rank then finishes the search and returns the same result.
    ``phases``: optional dict receiving the wall-clock seconds of each phase
    (a device synchronisation at each boundary).
    """
    import torch
    from . import shard
    ph = Phases(phases)
    device = cur.device
    skip = skip_point_of(T0_fit_margin)
    rank, world = shard.world_info(group) if distributed else (0, 1)
    if batch_periods is None:
        free = torch.cuda.mem_get_info(device)[0]
        batch_periods = reference_batch_size(len(periods), cur.n, cur.maxd, len(cur.widths), free)
        if world > 1:
            # every rank must use rank 0's batch size (the free memory differs)
            import torch.distributed as dist
            obj = [batch_periods]
            dist.broadcast_object_list(obj, src=0, group=group)
            batch_periods = obj[0]
    S = int(batch_periods)
    dev = cur.dev

    if world > 1:
        import torch.distributed as dist
        nccl = dist.get_backend(group) == "nccl"

        def main_pass(p0, p1):
            c, _ = cur.search(periods_dev[p0:p1], transit_depth_min, skip, S, _lib.GTLS_PASS_MAIN, precision,
                              timing=timing)
            return c if nccl else c.cpu()

        chi2_dev = shard.sharded_period_pass(len(periods), S, main_pass, group=group,
                                             device=dev if nccl else None).to(dev)
    elif devices is not None and len(devices) > 1:
        curves = {int(d): cur.on_device(int(d)) for d in devices}

        def main_pass_on(d, p0, p1):
            c, _ = curves[d].search(periods[p0:p1], transit_depth_min, skip, S, _lib.GTLS_PASS_MAIN, precision)
            return _d2h(c)

        chi2_dev = _h2d(torch, shard.multi_device_period_pass(len(periods), S, list(devices), main_pass_on), dev)
    else:
        chi2_dev, _ = cur.search(periods_dev, transit_depth_min, skip, S, _lib.GTLS_PASS_MAIN, precision,
                                 timing=timing)
    ph.mark("main_pass")
    raw_chi2 = _d2h(chi2_dev)
    median = np.median(raw_chi2)
    mask = raw_chi2 > (100 * median)
    mask_dev = _h2d(torch, mask.astype(np.uint8), dev)
    _, _, power_dev, sde_raw, sde = _spectra(chi2_dev, mask_dev, oversampling_factor, device)
    raw_power = ma.array(_d2h(power_dev), mask=mask)
    mperiods = ma.array(periods, mask=mask)
    ph.mark("spectra")
    if fast:
        return mperiods, raw_power

    # candidates re-searched at every phase start: in FP64, or (FP32 form) in
    # FP32 followed by an FP64 re-check of the best FP64_RECHECK of them
    cand_idx = _candidates(power_dev, mask_dev, periods_dev, torch)
    TRANSFER["d2h"] += cand_idx.nbytes
    cand_p = periods[cand_idx]
    ph.mark("candidates")
    again, _ = cur.search(cand_p, transit_depth_min, skip, S, _lib.GTLS_PASS_ALL,
                          "fp32" if precision == "fp32" else "fp64")
    ph.mark("candidate_search")
    ci = _h2d(torch, cand_idx, dev)
    chi2_dev[ci] = again
    mask_dev[ci] = 0
    _, _, power_dev, sde_raw, sde = _spectra(chi2_dev, mask_dev, oversampling_factor, device)
    ph.mark("spectra")
    rechecked = np.zeros(0, dtype=np.int64)
    if precision == "fp32":
        def search64(p, union):
            c, _ = cur.search(p, transit_depth_min, skip, len(p), _lib.GTLS_PASS_ALL, "fp64",
                              tables=subset_tables(cur.tables, union, torch), flags=_lib.GTLS_SEARCH_ALL_DURATIONS)
            return c
        pos, val = fp64_recheck(search64, cand_p, _d2h(power_dev[ci]), cur.widths, cur.curve["span"], cur.n, S,
                                device)
        if len(pos):
            chi2_dev[_h2d(torch, cand_idx[pos], dev)] = _h2d(torch, val, dev)
            _, _, power_dev, sde_raw, sde = _spectra(chi2_dev, mask_dev, oversampling_factor, device)
        rechecked = cand_idx[pos]
        again = chi2_dev[ci]
        ph.mark("fp64_recheck")
    pw = power_dev[ci]
    best = int(cand_idx[int(torch.argmax(pw).item())])
    period = periods[best]

    rates = [0.5, 1, 2, 2 / 3, 3 / 2]
    h_idx, h_p = find_nearest_indices([period * r for r in rates], periods)
    again2, _ = cur.search(h_p, transit_depth_min, skip, S, _lib.GTLS_PASS_ALL, "fp64")
    hi = _h2d(torch, h_idx, dev)
    chi2_dev[hi] = again2
    mask_dev[hi] = 0
    _, _, power_dev, sde_raw, sde = _spectra(chi2_dev, mask_dev, oversampling_factor, device)
    best = int(h_idx[int(torch.argmax(power_dev[hi]).item())])
    period = float(periods[best])
    ph.mark("harmonics")

    fin = single_period(cur, period, t, y, dy, transit_depth_min, phases=ph)

    chi2_h = _d2h(chi2_dev)
    # core.py:892-895 wraps raw_chi2 in a masked array without copying, so the
    # re-searched values written into chi2 (core.py:942,973) also land in the
    # returned raw_chi2; the main-pass values stay available as chi2_main.
    chi2_main = raw_chi2
    raw_chi2 = chi2_h.copy()
    mask_h = _d2h(mask_dev).astype(bool)
    power_h = _d2h(power_dev)
    chi2_m = ma.array(chi2_h, mask=mask_h)
    power_m = ma.array(power_h, mask=mask_h)
    periods_m = ma.array(periods, mask=mask_h)
    ph.mark("outputs")
    diag = dict(batch_periods=S, period_index=best, sde_raw=sde_raw, again=_d2h(again), chi2_main=chi2_main,
                fp64_rechecked=rechecked,
                harmonic_indices=h_idx, chi2_harmonics=_d2h(again2), loc=fin["loc"],
                skip_point=skip, precision=precision)
    return (periods_m, period, fin["raw_duration"], fin["width"], fin["duration"], fin["depth"], fin["T0"],
            float(sde), chi2_m, fin["transit_times"], power_m, fin["snr"], fin["snr_pink"], fin["snr_fit"],
            fin["snr_fit_pink"], raw_power, raw_chi2, list(cand_idx), list(cand_p), diag)


def single_period(cur, period, t, y, dy, transit_depth_min, phases=None):
    """core.search_single_periods (core.py:1250-1505): chi2 over the period's own
    duration range at every start on the GPU, then the host statistics.
    ``phases``: optional ``Phases`` marking the two parts."""
    chi2, loc = cur.search(np.array([period]), transit_depth_min, 1, 1, _lib.GTLS_PASS_ALL, "fp64",
                           want_loc=True)
    loc = int(_d2h(loc)[0])
    if phases is not None:
        phases.mark("best_period_search")
    fin = finish_period(cur.widths, cur.durations, cur.overshoot, cur.maxd, cur.curve["span"], period, loc, t, y,
                        device=cur.device)
    if phases is not None:
        phases.mark("best_period_stats")
    fin["chi2"] = float(_d2h(chi2)[0])
    return fin


def finish_period(widths, durations, overshoot, maxd, span, period, loc, t, y, device=0, full_stats=True):
    """Host part of core.search_single_periods (core.py:1420-1505) for the chi2
    minimum ``loc`` (= duration position * n + start) of ``period``: width,
    duration, depth, T0 and, with ``full_stats``, transit times and SNRs."""
    t = np.asarray(t, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = len(t)
    wmin, wmax = _lib.duration_ranges(np.array([period]), span, n, device=device)
    sel = (widths <= wmax[0]) & (widths >= wmin[0])
    w_sel = widths[sel]
    didx = loc // n
    width = int(w_sel[didx])
    raw_duration = float(durations[sel][didx])
    ovs = float(overshoot[sel][didx])
    return finish_stats(t, y, period, loc, width, raw_duration, ovs, maxd, full_stats=full_stats)


def finish_stats(t, y, period, loc, width, raw_duration, ovs, maxd, full_stats=True):
    """Host statistics of the best period (core.py:1427-1499) given its chi2
    minimum ``loc`` (= duration position * n + start), the width, duration
    and overshoot of that duration: depth, T0, duration in days and, with
    ``full_stats``, transit times, snr, snr_pink, snrFit and snrFitPink."""
    t = np.asarray(t, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = len(t)
    phase = (t % period) / period                       # foldCPU core.py:16-20
    rank = np.argsort(phase)
    best_t = np.array(t[rank])
    best_y = y[rank]
    best_y = np.concatenate((best_y, best_y[:maxd]))
    k0 = loc % n
    mean = best_y[k0:k0 + width].mean()
    depth = float((1 - mean) * ovs)
    tx = best_t[k0]
    t_min = float(np.min(t))
    T0 = tx - int((tx - t_min) / period) * period - period
    dur_days = float(stats.calc_duration_days(t, period, T0, raw_duration))
    out = dict(raw_duration=raw_duration, width=width, duration=dur_days, depth=depth, loc=loc)
    if not full_stats:
        T0 = T0 + dur_days / 2
        if T0 < t_min:
            T0 = T0 + period
        out["T0"] = float(T0)
        return out
    out_tr = np.concatenate((best_y[0:k0], best_y[k0 + width:]))
    snr_fit = (1 - depth) * (width ** 0.5) / np.std(out_tr)
    csum = np.cumsum(out_tr)
    red = np.std((csum[width:] - csum[:-width]) / width)
    transit_times = np.array(stats.all_transit_times(T0, t, period))
    snr_fit_pink = (1 - depth) / ((np.std(out_tr) ** 2 / width) + (red ** 2 / len(transit_times))) ** 0.5
    T0 = T0 + dur_days / 2
    transit_times = transit_times + dur_days / 2
    if T0 < t_min:
        T0 = T0 + period
    d_odd, d_even, s_odd, s_even, f_odd, f_even, per_count, _, _ = stats.intransit_stats(
        t, y, transit_times, dur_days)
    snr_pt, snr_pink_pt = stats.snr_stats(t, y, period, raw_duration, T0, transit_times, dur_days, per_count)
    f_in = np.concatenate([f_odd, f_even])
    intransit = stats.transit_mask(t, period, 2 * raw_duration, T0)
    flux_ootr = y[~intransit]
    with np.errstate(divide="ignore", invalid="ignore"):
        snr = ((1 - np.mean(f_in)) / np.std(flux_ootr)) * len(f_in) ** 0.5
        snr_pink = np.mean(snr_pink_pt) * (len(transit_times) ** 0.5)
    out.update(T0=float(T0), transit_times=transit_times, snr=float(snr), snr_pink=float(snr_pink),
               snr_fit=float(snr_fit), snr_fit_pink=float(snr_fit_pink))
    return out
