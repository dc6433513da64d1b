"""CPU oracle of the reference TLS search -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``gtls_b200``) imports this module; only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, as the
checker.  It restates, in NumPy float64, the arithmetic of the reference's
kernels and the host sequence that drives them:

* kernels (``src/gputls/GPUFun.py``): ``foldFast`` :30-41,
  ``durationsGrid`` :47-86, ``durationBool`` :91-105, ``patchData`` :110-129,
  ``calcInverseSquaredPatchedDy`` :134-142, ``calcEdgeEffectCorrections``
  :147-168, ``calcAllFullSum`` :173-201, ``calcAllFullSum_v2`` :207-232,
  ``calcAllOutOfTransitResiduals_step1/2`` :237-284, ``calculate_base_error``
  :293-312, ``calculate_final_ootr_v3`` :317-359, ``calcAverageFromCumsum``
  :366-375, ``calcAllLowestResidualsGPUB_SignalTiled_v2`` :382-438,
  ``calcAllLowestResidualsGPUBNoSkip`` :646-695 and ``...NoSkipTemp`` :819-873;
* host sequence (``src/gputls/core.py``): ``search_multi_periods`` :568-999,
  ``search_multi_periods_again`` :1001-1247, ``search_single_periods``
  :1250-1505, ``foldCPU`` :16-20, ``find_nearest_indices`` :34-46;
* statistics (``src/gputls/stats.py``): ``spectra`` :95-122,
  ``all_transit_times`` :233-250, ``calcDurationDays`` :252-275, and
  ``helpers.running_median`` :91-106.

"R64" means the kernels' formulas with every ``float`` promoted to
``double`` (what core.py's float64 host buffers intend).  cupy's argsort is
taken as a stable sort, its cumsum as a sequential prefix sum and its argmin
as first-occurrence; the reference tests pin none of these.  The per-batch
numerics are behind a small backend interface so that the same host flow can
also drive the reference's own kernel source compiled for the CPU
(``oracle/ref_replay.py``), which is how this restatement is pinned.
"""
import numpy as np
import numpy.ma as ma

# constants restated from src/gputls/constants.py and the GPUFun.py #defines
SECONDS_PER_DAY = 86400
R_SUN = 695508000
R_JUP = 69911000
DEV_RS_MIN = R_SUN * 0.05
DEV_RS_MAX = R_SUN * 4.0
DEV_PI_GM_MAX = 416970
DEV_PI_GM_MIN = 20848
DEV_SCALE = 1000000000000000.0
DEV_FRAC_MAX = 0.15
SDE_MEDIAN_KERNEL_SIZE = 30
SKIP_NEVER = 0x7F800000


# --------------------------------------------------------------------------
# kernels restated
# --------------------------------------------------------------------------
def fold_phases(t, period):
    """foldFast (GPUFun.py:30-41): t/P minus its (int) truncation."""
    x = np.asarray(t, dtype=np.float64) / np.float64(period)
    return x - np.trunc(x)


def duration_ranges(periods, span, n_samples):
    """durationsGrid (GPUFun.py:47-86) -> (wmin, wmax) int arrays.

    ``span`` is rounded to float32 first: the only type-consistent caller,
    ``_worker.py:107,132``, passes the time span as float32.
    """
    length = np.float64(np.float32(span))
    P = np.asarray(periods, dtype=np.float64)
    nt = length / P
    corr = (nt + 1.0) / nt
    ps = P * SECONDS_PER_DAY
    fmin = (4.0 * ps) / (DEV_PI_GM_MIN * DEV_SCALE)
    fmax = (4.0 * ps) / (DEV_PI_GM_MAX * DEV_SCALE)
    t14min = DEV_RS_MIN * np.power(fmin, 1.0 / 3.0)
    t14max = (DEV_RS_MAX + R_JUP * 2.0) * np.power(fmax, 1.0 / 3.0)
    dmin = np.minimum(t14min / ps, DEV_FRAC_MAX)
    dmax = np.minimum(t14max / ps, DEV_FRAC_MAX)
    wmin = np.floor(dmin * n_samples).astype(np.int64)
    wmax = np.ceil(dmax * n_samples * corr).astype(np.int64)
    return wmin, wmax


def duration_masks(wmin, wmax, widths):
    """durationBool (GPUFun.py:91-105): bool[P, D]."""
    w = np.asarray(widths)[None, :]
    return (w >= np.asarray(wmin)[:, None]) & (w <= np.asarray(wmax)[:, None])


def batch_unions(masks, batch):
    """OR of the duration masks over each batch of ``batch`` periods (core.py:693-716)."""
    n = masks.shape[0]
    nb = (n + batch - 1) // batch
    return np.stack([np.any(masks[b * batch: min((b + 1) * batch, n)], axis=0) for b in range(nb)])


def skip_point_of(margin):
    """SKIP_POINT substitution of core.py:597-601."""
    return SKIP_NEVER if margin == 0 else int(1 / margin)


def _patched(t, y, dy, period, maxd):
    """Stable fold order + patchData (GPUFun.py:110-129) + 1/dy^2 (:134-142)."""
    order = np.argsort(fold_phases(t, period), kind="stable")
    order = np.concatenate([order, order[:maxd]])
    yp = np.asarray(y, dtype=np.float64)[order]
    dyp = np.asarray(dy, dtype=np.float64)[order]
    return yp, 1.0 / (dyp * dyp)


def _edge(yp, wp, n):
    """calcEdgeEffectCorrections (GPUFun.py:147-168): tail sum, double accumulator."""
    tail_y = yp[n:]
    return float(np.sum((1.0 + tail_y * tail_y - 2.0 * tail_y) * wp[n:]))


def _window_means(cy, k, w):
    """calcAverageFromCumsum (GPUFun.py:366-375)."""
    end = cy[k + w - 1]
    start = np.where(k == 0, 0.0, cy[np.maximum(k - 1, 0)])
    return np.where(k == 0, 1.0 - cy[w - 1] / w, 1.0 - (end - start) / w)


def _intransit(yp, wp, sig, rs, ks, w):
    """In-transit residual loop of GPUFun.py:425-429 for the starts ``ks``."""
    if ks.size == 0:
        return np.zeros(0)
    out = np.empty(ks.size)
    step = max(1, int(4_000_000 // max(w, 1)))
    win_y = np.lib.stride_tricks.sliding_window_view(yp, w)
    win_w = np.lib.stride_tricks.sliding_window_view(wp, w)
    for a in range(0, ks.size, step):
        kk = ks[a:a + step]
        sigi = sig[None, :w] * rs[a:a + step, None]
        loss = win_y[kk] - (1.0 - sigi)
        out[a:a + step] = np.sum(loss * loss * win_w[kk], axis=1)
    return out


class NumpyBackend:
    """R64 restatement of the per-period kernel arithmetic."""

    name = "numpy-r64"

    def main_pass(self, t, y, dy, period, widths, tmpl, overshoot, maxd, depth_min, skip_point):
        """Per-period (min, argmin) of the main pass (core.py:770-875)."""
        n = len(t)
        yp, wp = _patched(t, y, dy, period, maxd)
        m = n + maxd
        diff = 1.0 - yp
        e = diff * diff * wp                       # calculate_base_error :310-311
        E = np.cumsum(e)
        cy = np.cumsum(yp)
        edge = _edge(yp, wp, n)
        k = np.arange(n)
        vals = []
        for d, w in enumerate(widths):
            w = int(w)
            full = E[m - 1] - E[w - 1]             # calcAllFullSum_v2 :224-231
            ootr = full + (E[k] - (E[k + w] - E[w - 1]))   # final_ootr_v3 :344-358
            mean = _window_means(cy, k, w)
            skip = (w // skip_point) if w > skip_point else 1
            ok = (mean > depth_min) & (k % skip == 0)
            stat = np.full(n, float(n))
            ks = k[ok]
            rs = mean[ok] * overshoot[d] * 2.0
            intr = _intransit(yp, wp, tmpl[d], rs, ks, w)
            prev = np.where(ks == 0, full, ootr[np.maximum(ks - 1, 0)])
            frac = float(w) / (((w - 1) // 1) + 1)
            stat[ok] = intr * frac + prev - edge
            vals.append(stat)
        flat = np.concatenate(vals)
        loc = int(np.argmin(flat))
        return float(flat[loc]), loc

    def noskip_pass(self, t, y, dy, period, widths, tmpl, overshoot, maxd, depth_min):
        """Every start evaluated, step1/cumsum/step2 OOTR (core.py:1184-1237, 1378-1418)."""
        n = len(t)
        yp, wp = _patched(t, y, dy, period, maxd)
        diff = 1.0 - yp
        e = diff * diff * wp
        total = float(np.cumsum(e)[-1])            # calcAllFullSum :183-187 (sequential)
        cy = np.cumsum(yp)
        edge = _edge(yp, wp, n)
        k = np.arange(n)
        vals = []
        for d, w in enumerate(widths):
            w = int(w)
            full = total - float(np.cumsum(e[:w])[-1])   # :190-199
            temp = e[k] - e[k + w]                 # step1 :253-263
            ootr = np.cumsum(temp) + full          # cumsum, step2 :283
            mean = _window_means(cy, k, w)
            ok = mean > depth_min
            stat = np.full(n, float(n))
            ks = k[ok]
            rs = mean[ok] * overshoot[d] * 2.0
            intr = _intransit(yp, wp, tmpl[d], rs, ks, w)
            prev = np.where(ks == 0, full, ootr[np.maximum(ks - 1, 0)])
            stat[ok] = intr + prev - edge
            vals.append(stat)
        flat = np.concatenate(vals)
        loc = int(np.argmin(flat))
        return float(flat[loc]), loc


# --------------------------------------------------------------------------
# host sequence restated
# --------------------------------------------------------------------------
def reference_batch_size(n_periods, n_samples, maxd, n_durations, free_bytes):
    """singleCalcPeriods of core.py:620-628 for a given free-memory figure."""
    m = n_samples + maxd
    cap = free_bytes / (5 * (m * 2 + 2 + n_durations * m * 4 + 2 * n_durations))
    s = int(np.min([np.floor(cap), n_periods / 30]))
    if s < 15:
        s = int(s / 1.1)
    return s


def search_periods(backend, periods, t, y, dy, widths, tmpl, overshoot, maxd, depth_min,
                   skip_point, batch, noskip=False):
    """chi2 and argmin per period with batch-union durations.

    Main pass: core.py:691-875; candidate pass (``noskip``): core.py:1081-1237.
    A batch whose union is empty gets NaN (core.py:722-729).
    """
    periods = np.asarray(periods, dtype=np.float64)
    span = np.max(t) - np.min(t)
    wmin, wmax = duration_ranges(periods, span, len(t))
    unions = batch_unions(duration_masks(wmin, wmax, widths), batch)
    chi2 = np.full(len(periods), np.nan)
    loc = np.full(len(periods), -1, dtype=np.int64)
    for p, period in enumerate(periods):
        sel = unions[p // batch]
        if not np.any(sel):
            continue
        args = (t, y, dy, period, widths[sel], tmpl[sel], overshoot[sel], maxd, depth_min)
        if noskip:
            chi2[p], loc[p] = backend.noskip_pass(*args)
        else:
            chi2[p], loc[p] = backend.main_pass(*args, skip_point)
    return chi2, loc


def running_median(data, kernel):
    """helpers.running_median (helpers.py:91-106)."""
    idx = np.arange(kernel) + np.arange(len(data) - kernel + 1)[:, None]
    idx = idx.astype(int)
    med = np.ma.median(data[idx], axis=1)
    first_values = med[0]
    last_values = med[-1]
    missing_values = len(data) - len(med)
    values_front = int(missing_values * 0.5)
    values_end = missing_values - values_front
    med = np.append(np.full(values_front, first_values), med)
    med = np.append(med, np.full(values_end, last_values))
    return med


def spectra(chi2, oversampling_factor):
    """stats.spectra (stats.py:95-122) on a (masked) chi2 array."""
    SR = np.min(chi2) / chi2
    SDE_raw = (1 - np.mean(SR)) / np.std(SR)
    power_raw = SR - np.mean(SR)
    scale = SDE_raw / np.max(power_raw)
    power_raw = power_raw * scale
    kernel = oversampling_factor * SDE_MEDIAN_KERNEL_SIZE
    if kernel % 2 == 0:
        kernel = kernel + 1
    if len(power_raw) > 2 * kernel:
        my_median = running_median(power_raw, kernel)
        power = power_raw - my_median
        power = power - np.mean(power)
        SDE = np.max(power / np.std(power))
        scale = SDE / np.max(power)
        power = power * scale
    else:
        power = power_raw
        SDE = SDE_raw
    return SR, power_raw, power, SDE_raw, SDE


def select_candidates(periods, power):
    """Top-100 by power, then the next 100 with period > 1 d (core.py:904-915)."""
    combined = list(enumerate(zip(periods, -power)))
    sorted_combined = sorted(combined, key=lambda x: x[1][1])
    top = [item[0] for item in sorted_combined[:100]]
    top_p = [item[1][0] for item in sorted_combined[:100]]
    topset = set(top)
    rem = [item for item in sorted_combined if item[0] not in topset]
    rem1 = sorted([item for item in rem if item[1][0] > 1], key=lambda x: x[1][1])
    nxt = [item[0] for item in rem1[:100]]
    nxt_p = [item[1][0] for item in rem1[:100]]
    return top + nxt, top_p + nxt_p


def find_nearest_indices(a, b):
    """core.py:34-46."""
    a = np.array(a)
    b = np.array(b)
    idx = np.zeros(a.shape, dtype=int)
    el = np.zeros(a.shape)
    for i, val in enumerate(a):
        j = np.argmin(np.abs(b - val))
        idx[i] = j
        el[i] = b[j]
    return idx, el


def all_transit_times(T0, t, period):
    """stats.all_transit_times (stats.py:233-250)."""
    transit_times = [T0 + period] if T0 < min(t) else [T0]
    prev = transit_times[0]
    while True:
        nxt = prev + period
        if nxt < (np.min(t) + (np.max(t) - np.min(t))):
            transit_times.append(nxt)
            prev = nxt
        else:
            break
    return transit_times


def calc_duration_days(times, period, start_t0, raw_duration):
    """stats.calcDurationDays (stats.py:252-275); the end index is clamped to the data."""
    t0c = start_t0 + period / 2
    phases = (times - t0c) / period - np.floor((times - t0c) / period)
    ps = phases[np.argsort(phases)]
    start = int(np.abs(ps - 0.5).argmin())
    end = min(start + int(np.array(raw_duration) * len(times)), len(times) - 1)
    return (ps[end] - 0.5) * period


def single_period(backend, period, t, y, dy, widths, tmpl, overshoot, durations, maxd, depth_min):
    """search_single_periods (core.py:1250-1471) up to duration/depth/T0."""
    wmin, wmax = duration_ranges(np.array([period]), np.max(t) - np.min(t), len(t))
    sel = (widths <= wmax[0]) & (widths >= wmin[0])
    w_sel = widths[sel]
    _, loc = backend.noskip_pass(t, y, dy, period, w_sel, tmpl[sel], overshoot[sel], maxd, depth_min)
    n = len(t)
    didx = loc // n
    width = int(w_sel[didx])
    raw_duration = float(durations[sel][didx])
    phase = (t % period) / period                      # foldCPU core.py:16-20
    rank = np.argsort(phase)
    best_t = np.array(t[rank])
    best_y = y[rank]
    best_y = np.concatenate((best_y, best_y[:maxd]))
    k0 = loc % n
    mean = best_y[k0:k0 + width].mean()
    depth = float((1 - mean) * overshoot[sel][didx])
    tx = best_t[k0]
    T0 = tx - int((tx - min(t)) / period) * period - period
    transit_times = np.array(all_transit_times(T0, t, period))
    dur_days = calc_duration_days(t, period, T0, raw_duration)
    T0 = T0 + dur_days / 2
    transit_times = transit_times + dur_days / 2
    if T0 < min(t):
        T0 = T0 + period
    return dict(raw_duration=raw_duration, width=width, duration=float(dur_days), depth=depth,
                T0=float(T0), transit_times=transit_times, loc=int(loc))


def search(backend, periods, t, y, dy, widths, tmpl, overshoot, durations, maxd, depth_min,
           T0_fit_margin, oversampling_factor, batch, fast=False):
    """search_multi_periods (core.py:568-999) without the SNR statistics."""
    periods = np.sort(np.asarray(periods, dtype=np.float64))
    skip = skip_point_of(T0_fit_margin)
    chi2_main, _ = search_periods(backend, periods, t, y, dy, widths, tmpl, overshoot, maxd,
                                  depth_min, skip, batch)
    raw_chi2 = chi2_main.copy()
    median = np.median(raw_chi2)
    mask = raw_chi2 > (100 * median)
    chi2 = ma.array(raw_chi2, mask=mask)
    mperiods = ma.array(periods, mask=mask)
    SR, power_raw, power, SDE_raw, SDE = spectra(chi2, oversampling_factor)
    raw_power = power.copy()
    out = dict(periods=mperiods, raw_chi2=raw_chi2, raw_power=raw_power)
    if fast:
        out.update(power=power)
        return out
    cand_idx, cand_p = select_candidates(mperiods, power)
    again, _ = search_periods(backend, np.array(cand_p, dtype=np.float64), t, y, dy, widths, tmpl,
                              overshoot, maxd, depth_min, skip, batch, noskip=True)
    chi2[cand_idx] = again
    SR, power_raw, power, SDE_raw, SDE = spectra(chi2, oversampling_factor)
    power_again = power[cand_idx]
    best = cand_idx[int(np.argmax(power_again))]
    period = mperiods[best]
    rates = [0.5, 1, 2, 2 / 3, 3 / 2]
    h_idx, h_p = find_nearest_indices([period * r for r in rates], mperiods)
    again2, _ = search_periods(backend, h_p, t, y, dy, widths, tmpl, overshoot, maxd, depth_min,
                               skip, batch, noskip=True)
    chi2[h_idx] = again2
    SR, power_raw, power, SDE_raw, SDE = spectra(chi2, oversampling_factor)
    best = h_idx[int(np.argmax(power[h_idx]))]
    period = float(mperiods.data[best])
    fin = single_period(backend, period, t, y, dy, widths, tmpl, overshoot, durations, maxd,
                        depth_min)
    out.update(period=period, period_index=int(best), chi2=chi2, power=power, SDE=float(SDE),
               SDE_raw=float(SDE_raw), SR=SR, candidates=cand_idx, candidate_periods=cand_p,
               chi2_main=chi2_main, chi2_again=again, harmonic_indices=h_idx,
               chi2_harmonics=again2, **fin)
    return out


def period_grid(R_star, M_star, time_span, period_min=0, period_max=float("inf"),
                oversampling_factor=3, n_transits_min=2):
    """grid.period_grid (grid.py:56-157) in NumPy (descending periods, days)."""
    G = 6.673e-11
    R_sun = 695508000
    M_sun = 1.989 * 10 ** 30
    if R_star < 0.01:
        R_star = 0.1
    if R_star > 10000:
        R_star = 10000
    if M_star < 0.01:
        M_star = 0.01
    if M_star > 1000:
        M_star = 1000
    R_star = R_star * R_sun
    M_star = M_star * M_sun
    time_span = time_span * SECONDS_PER_DAY
    f_min = n_transits_min / time_span
    f_max = 1.0 / (2 * np.pi) * np.sqrt(G * M_star / (3 * R_star) ** 3)
    A = ((2 * np.pi) ** (2.0 / 3) / np.pi * R_star / (G * M_star) ** (1.0 / 3)
         / (time_span * oversampling_factor))
    C = f_min ** (1.0 / 3) - A / 3.0
    N_opt = (f_max ** (1.0 / 3) - f_min ** (1.0 / 3) + A / 3) * 3 / A
    X = np.arange(N_opt) + 1
    f_x = (A / 3 * X + C) ** 3
    periods = 1 / f_x / SECONDS_PER_DAY
    sel = np.where(np.logical_and(periods > period_min, periods <= period_max))
    if np.size(periods[sel]) < 100:
        if time_span < 5 * SECONDS_PER_DAY:
            time_span = 5 * SECONDS_PER_DAY
        return period_grid(1, 1, time_span / SECONDS_PER_DAY)
    return periods[sel]
