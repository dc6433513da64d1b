"""ctypes binding of ``libgtls_b200.so`` (declared in ``include/gtls_b200.h``).

The library is loaded from the package directory.  There is no fallback:
if the library is missing or no CUDA device is present every call raises.
Device buffers are torch tensors (torch is used for device memory and
streams only); calls run on torch's current CUDA stream.
"""
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgtls_b200.so")

ABI_VERSION = 2
GTLS_FP64, GTLS_FP32 = 0, 1
GTLS_PASS_MAIN, GTLS_PASS_ALL = 0, 1
GTLS_SEARCH_ALL_DURATIONS = 1
MAX_DURATIONS = 1024

_lib = None
_lock = threading.Lock()
_ctxs = {}

# bytes copied host->device and device->host by this package (accounting)
TRANSFER = {"h2d": 0, "d2h": 0}


def h2d(torch, arr, dev):
    arr = np.ascontiguousarray(arr)
    TRANSFER["h2d"] += arr.nbytes
    return torch.from_numpy(arr).to(dev)


def d2h(tensor):
    TRANSFER["d2h"] += tensor.numel() * tensor.element_size()
    return tensor.cpu().numpy()


class GtlsError(RuntimeError):
    """A gtls_* C-ABI call returned a non-zero status."""


class Timing(ctypes.Structure):
    """Mirror of ``gtls_timing``."""
    _fields_ = [
        ("chunks", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("setup_ms", ctypes.c_double),
        ("prepare_ms", ctypes.c_double),
        ("chi2_ms", ctypes.c_double),
        ("finish_ms", ctypes.c_double),
        ("chi2_starts", ctypes.c_int64),
        ("chi2_fma", ctypes.c_int64),
        ("chi2_active_fma", ctypes.c_int64),
        ("chi2_issued_fma", ctypes.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class SearchDesc(ctypes.Structure):
    """Mirror of ``gtls_search_desc``."""
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("pass_", ctypes.c_int32),
        ("n", ctypes.c_int32),
        ("t", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("dy", ctypes.c_void_p),
        ("n_periods", ctypes.c_int64),
        ("periods", ctypes.c_void_p),
        ("n_durations", ctypes.c_int32),
        ("max_width", ctypes.c_int32),
        ("widths", ctypes.c_void_p),
        ("overshoot", ctypes.c_void_p),
        ("templates", ctypes.c_void_p),
        ("depth_min", ctypes.c_double),
        ("skip_point", ctypes.c_int32),
        ("batch", ctypes.c_int32),
        ("span", ctypes.c_float),
        ("flags", ctypes.c_int32),
        ("chi2_out", ctypes.c_void_p),
        ("loc_out", ctypes.c_void_p),
        ("timing", ctypes.c_void_p),
    ]


class Tuning(ctypes.Structure):
    """Mirror of ``gtls_tuning``."""
    _fields_ = [
        ("tile_cap_fp32", ctypes.c_int32),
        ("tile_cap_fp64", ctypes.c_int32),
        ("bucket_shift", ctypes.c_int32),
        ("records_global", ctypes.c_int32),
    ]


class BatchDesc(ctypes.Structure):
    """Mirror of ``gtls_batch_desc``."""
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("pass_", ctypes.c_int32),
        ("n_curves", ctypes.c_int32),
        ("sample_off", ctypes.c_void_p),
        ("period_off", ctypes.c_void_p),
        ("dur_off", ctypes.c_void_p),
        ("tmpl_off", ctypes.c_void_p),
        ("max_width", ctypes.c_void_p),
        ("batch", ctypes.c_void_p),
        ("span", ctypes.c_void_p),
        ("t", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("dy", ctypes.c_void_p),
        ("periods", ctypes.c_void_p),
        ("widths", ctypes.c_void_p),
        ("overshoot", ctypes.c_void_p),
        ("templates", ctypes.c_void_p),
        ("depth_min", ctypes.c_double),
        ("skip_point", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("chi2_out", ctypes.c_void_p),
        ("loc_out", ctypes.c_void_p),
        ("timing", ctypes.c_void_p),
    ]


class TemplateDesc(ctypes.Structure):
    """Mirror of ``gtls_template_desc``."""
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("n_curves", ctypes.c_int32),
        ("per", ctypes.c_double),
        ("rp", ctypes.c_double),
        ("a", ctypes.c_double),
        ("inc", ctypes.c_double),
        ("u1", ctypes.c_double),
        ("u2", ctypes.c_double),
        ("samples", ctypes.c_void_p),
        ("row_off", ctypes.c_void_p),
        ("widths", ctypes.c_void_p),
        ("tmpl_off", ctypes.c_void_p),
        ("row_len", ctypes.c_void_p),
        ("overshoot", ctypes.c_void_p),
        ("templates", ctypes.c_void_p),
    ]


EXPORTS = {
    "gtls_ctx_create": ([ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "gtls_ctx_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "gtls_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "gtls_abi_version": ([], ctypes.c_int),
    "gtls_launch_count": ([ctypes.c_void_p], ctypes.c_int64),
    "gtls_decode_status": ([ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "gtls_set_chunk_budget": ([ctypes.c_void_p, ctypes.c_uint64], ctypes.c_int),
    "gtls_set_tuning": ([ctypes.c_void_p, ctypes.POINTER(Tuning)], ctypes.c_int),
    "gtls_get_tuning": ([ctypes.c_void_p, ctypes.POINTER(Tuning)], ctypes.c_int),
    "gtls_period_grid": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                          ctypes.c_double, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p],
                         ctypes.c_int),
    "gtls_duration_ranges": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_int32,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "gtls_search": ([ctypes.c_void_p, ctypes.POINTER(SearchDesc), ctypes.c_void_p], ctypes.c_int),
    "gtls_fold_order": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
                         ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "gtls_search_batch": ([ctypes.c_void_p, ctypes.POINTER(BatchDesc), ctypes.c_void_p], ctypes.c_int),
    "gtls_template_cache": ([ctypes.c_void_p, ctypes.POINTER(TemplateDesc), ctypes.c_void_p], ctypes.c_int),
    "gtls_spectra": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                      ctypes.POINTER(ctypes.c_double), ctypes.c_void_p], ctypes.c_int),
    "gtls_spectra_noalloc": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(ctypes.c_double), ctypes.c_void_p], ctypes.c_int),
    "gtls_noalloc_last_error": ([], ctypes.c_char_p),
    "gtls_model_chi2": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                         ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "gtls_model_chi2_grad": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                             ctypes.c_int),
}


def load():
    """Load the library and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise GtlsError(LIB_PATH + " is missing: build it with `python -m gtls_b200.build`")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in EXPORTS.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = res
            if lib.gtls_abi_version() != ABI_VERSION:
                raise GtlsError("libgtls_b200.so ABI version mismatch")
            _lib = lib
    return _lib


def context(device=0):
    """The (cached) gtls context of CUDA device ``device``."""
    lib = load()
    with _lock:
        c = _ctxs.get(device)
        if c is None:
            h = ctypes.c_void_p()
            rc = lib.gtls_ctx_create(device, ctypes.byref(h))
            if rc != 0:
                raise GtlsError("gtls_ctx_create failed (%d): %s" % (rc, lib.gtls_last_error(None).decode()))
            c = _ctxs[device] = h
    return c


def _check(rc, ctx, what):
    if rc != 0:
        msg = load().gtls_last_error(ctx).decode(errors="replace")
        raise GtlsError("%s failed (%d): %s" % (what, rc, msg))


def device_status_error(word):
    """GtlsError for a non-zero device status word of a search (its meaning
    from gtls_decode_status), None for 0."""
    buf = ctypes.create_string_buffer(256)
    rc = load().gtls_decode_status(int(word), buf, len(buf))
    if rc == 0:
        return None
    return GtlsError("device status %d (%d): %s" % (int(word), rc, buf.value.decode(errors="replace")))


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise GtlsError("gtls_b200 needs a CUDA device (none is visible)")
    return torch


_last_stream = {}


def _stream(torch, device):
    """The current stream of ``device`` for the next call, as a void*.  A
    device's calls share its context's scratch arena, so when the stream
    differs from the one of the previous call on the device, the new stream
    first waits for the old one."""
    cur = torch.cuda.current_stream(device)
    prev = _last_stream.get(device)
    if prev is not None and prev != cur:
        cur.wait_stream(prev)
    _last_stream[device] = cur
    return ctypes.c_void_p(cur.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def period_grid(a_over_3, c, n_points, period_min, period_max, device=0):
    """Ascending Ofir periods from the device (gtls_period_grid)."""
    torch = _torch()
    ctx = context(device)
    out = torch.empty(max(int(n_points), 1), dtype=torch.float64, device="cuda:%d" % device)
    cnt = ctypes.c_int64()
    pmax = float(period_max) if np.isfinite(period_max) else float("inf")
    rc = load().gtls_period_grid(ctx, float(a_over_3), float(c), int(n_points), float(period_min), pmax,
                                 _ptr(out), ctypes.byref(cnt), _stream(torch, device))
    _check(rc, ctx, "gtls_period_grid")
    return d2h(out[: cnt.value])


def duration_ranges(periods, span, n_samples, device=0):
    """(wmin, wmax) per period (gtls_duration_ranges), as numpy int arrays."""
    torch = _torch()
    ctx = context(device)
    p = h2d(torch, np.asarray(periods, dtype=np.float64), "cuda:%d" % device)
    wmin = torch.empty(len(p), dtype=torch.int32, device=p.device)
    wmax = torch.empty_like(wmin)
    rc = load().gtls_duration_ranges(ctx, _ptr(p), len(p), float(np.float32(span)), int(n_samples), _ptr(wmin),
                                     _ptr(wmax), _stream(torch, device))
    _check(rc, ctx, "gtls_duration_ranges")
    return d2h(wmin).astype(np.int64), d2h(wmax).astype(np.int64)


def launch_count(device=0):
    """Kernels launched so far through the device's context."""
    return int(load().gtls_launch_count(context(device)))


def set_chunk_budget(nbytes, device=0):
    """Per-chunk scratch budget of the searches on ``device`` (bytes)."""
    ctx = context(device)
    _check(load().gtls_set_chunk_budget(ctx, int(nbytes)), ctx, "gtls_set_chunk_budget")


def fold_order(t, periods, device=0):
    """gtls_fold_order: the stable phase order of device float64 tensor ``t``
    for every period of device float64 tensor ``periods``; returns an int32
    tensor [len(periods), len(t)]."""
    torch = _torch()
    ctx = context(device)
    n, npd = int(t.numel()), int(periods.numel())
    out = torch.empty((npd, n), dtype=torch.int32, device=t.device)
    rc = load().gtls_fold_order(ctx, t.data_ptr(), n, periods.data_ptr(), npd, out.data_ptr(),
                                _stream(torch, device))
    _check(rc, ctx, "gtls_fold_order")
    return out


def template_cache(planet, samples, row_off, widths, tmpl_off, row_len, overshoot, templates, device=0):
    """gtls_template_cache: fill the device tensors ``overshoot`` [rows] and
    ``templates`` with the template tables of every curve.  ``planet`` =
    (per, rp, a, inc, u1, u2); the other arguments are host arrays (see the
    C header)."""
    torch = _torch()
    ctx = context(device)
    keep = [np.ascontiguousarray(samples, dtype=np.int32), np.ascontiguousarray(row_off, dtype=np.int64),
            np.ascontiguousarray(widths, dtype=np.int32), np.ascontiguousarray(tmpl_off, dtype=np.int64),
            np.ascontiguousarray(row_len, dtype=np.int32)]
    d = TemplateDesc()
    d.abi_version = ABI_VERSION
    d.n_curves = len(keep[0])
    d.per, d.rp, d.a, d.inc, d.u1, d.u2 = (float(v) for v in planet)
    d.samples, d.row_off, d.widths, d.tmpl_off, d.row_len = (a.ctypes.data for a in keep)
    d.overshoot = overshoot.data_ptr()
    d.templates = templates.data_ptr()
    rc = load().gtls_template_cache(ctx, ctypes.byref(d), _stream(torch, device))
    _check(rc, ctx, "gtls_template_cache")


def set_tuning(tile_cap_fp32=0, tile_cap_fp64=0, bucket_shift=0, records_global=0, device=0):
    """Launch-shape parameters of the searches on ``device`` (0 = default);
    results do not depend on them."""
    ctx = context(device)
    t = Tuning(int(tile_cap_fp32), int(tile_cap_fp64), int(bucket_shift), int(records_global))
    _check(load().gtls_set_tuning(ctx, ctypes.byref(t)), ctx, "gtls_set_tuning")


def get_tuning(device=0):
    """The current ``Tuning`` of ``device`` as a dict."""
    ctx = context(device)
    t = Tuning()
    _check(load().gtls_get_tuning(ctx, ctypes.byref(t)), ctx, "gtls_get_tuning")
    return dict(tile_cap_fp32=t.tile_cap_fp32, tile_cap_fp64=t.tile_cap_fp64, bucket_shift=t.bucket_shift,
                records_global=t.records_global)


def search(curve, periods, tables, depth_min, skip_point, batch, pass_, precision, device=0,
           want_loc=True, timing=None, flags=0):
    """Run gtls_search for one curve.

    ``curve``: dict of device tensors t, y, dy (float64) and ``span`` (float).
    ``tables``: dict of device tensors widths (int32), overshoot (float64),
    templates (float64, D x max_width) and int ``max_width``.
    ``periods``: device float64 tensor.  ``timing``: an optional ``Timing``
    filled with CUDA-event stage times.  Returns (chi2, loc) device tensors.
    """
    torch = _torch()
    ctx = context(device)
    n_periods = int(periods.numel())
    chi2 = torch.empty(n_periods, dtype=torch.float64, device=periods.device)
    loc = torch.empty(n_periods, dtype=torch.int64, device=periods.device) if want_loc else None
    d = SearchDesc()
    d.abi_version = ABI_VERSION
    d.precision = GTLS_FP32 if precision == "fp32" else GTLS_FP64
    d.pass_ = pass_
    d.n = int(curve["t"].numel())
    d.t = curve["t"].data_ptr()
    d.y = curve["y"].data_ptr()
    d.dy = curve["dy"].data_ptr()
    d.n_periods = n_periods
    d.periods = periods.data_ptr()
    d.n_durations = int(tables["widths"].numel())
    d.max_width = int(tables["max_width"])
    d.widths = tables["widths"].data_ptr()
    d.overshoot = tables["overshoot"].data_ptr()
    d.templates = tables["templates"].data_ptr()
    d.depth_min = float(depth_min)
    d.skip_point = int(skip_point)
    d.batch = int(batch)
    d.span = float(curve["span"])
    d.chi2_out = chi2.data_ptr()
    d.loc_out = loc.data_ptr() if loc is not None else None
    d.timing = ctypes.addressof(timing) if timing is not None else None
    d.flags = int(flags)
    rc = load().gtls_search(ctx, ctypes.byref(d), _stream(torch, device))
    _check(rc, ctx, "gtls_search")
    return chi2, loc


def search_batch(curves, periods, period_off, tables, depth_min, skip_point, batches, pass_, precision,
                 device=0, want_loc=True, timing=None, flags=0):
    """Run gtls_search_batch over many curves.

    ``curves``: dict of concatenated device tensors t, y, dy (float64), host
    int64 ``sample_off`` [C+1] and host float32 ``span`` [C].
    ``periods``: concatenated device float64 tensor, ``period_off`` host
    int64 [C+1].  ``tables``: concatenated device tensors widths (int32),
    overshoot (float64), templates (float64), host int64 ``dur_off`` [C+1]
    and ``tmpl_off`` [C], host int32 ``max_width`` [C].  ``batches``: host
    int32 [C] periods per duration-union batch.  Returns (chi2, loc) device
    tensors over all curves' periods.
    """
    torch = _torch()
    ctx = context(device)
    n_curves = len(curves["span"])
    total = int(period_off[-1])
    dev = periods.device
    chi2 = torch.empty(total, dtype=torch.float64, device=dev)
    loc = torch.empty(total, dtype=torch.int64, device=dev) if want_loc else None
    host = dict(
        sample_off=np.ascontiguousarray(curves["sample_off"], dtype=np.int64),
        period_off=np.ascontiguousarray(period_off, dtype=np.int64),
        dur_off=np.ascontiguousarray(tables["dur_off"], dtype=np.int64),
        tmpl_off=np.ascontiguousarray(tables["tmpl_off"], dtype=np.int64),
        max_width=np.ascontiguousarray(tables["max_width"], dtype=np.int32),
        batch=np.ascontiguousarray(batches, dtype=np.int32),
        span=np.ascontiguousarray(curves["span"], dtype=np.float32),
    )
    for k, a in host.items():
        want = n_curves + 1 if k in ("sample_off", "period_off", "dur_off") else n_curves
        if a.shape != (want,):
            raise ValueError("%s must hold %d values" % (k, want))
    d = BatchDesc()
    d.abi_version = ABI_VERSION
    d.precision = GTLS_FP32 if precision == "fp32" else GTLS_FP64
    d.pass_ = pass_
    d.n_curves = n_curves
    for k, a in host.items():
        setattr(d, k, a.ctypes.data)
    d.t = curves["t"].data_ptr()
    d.y = curves["y"].data_ptr()
    d.dy = curves["dy"].data_ptr()
    d.periods = periods.data_ptr()
    d.widths = tables["widths"].data_ptr()
    d.overshoot = tables["overshoot"].data_ptr()
    d.templates = tables["templates"].data_ptr()
    d.depth_min = float(depth_min)
    d.skip_point = int(skip_point)
    d.chi2_out = chi2.data_ptr()
    d.loc_out = loc.data_ptr() if loc is not None else None
    d.timing = ctypes.addressof(timing) if timing is not None else None
    d.flags = int(flags)
    rc = load().gtls_search_batch(ctx, ctypes.byref(d), _stream(torch, device))
    _check(rc, ctx, "gtls_search_batch")
    return chi2, loc


def spectra(chi2, mask, oversampling_factor, device=0):
    """gtls_spectra on a device chi2 tensor; returns (SR, power_raw, power, SDE_raw, SDE)."""
    torch = _torch()
    ctx = context(device)
    n = int(chi2.numel())
    sr = torch.empty_like(chi2)
    praw = torch.empty_like(chi2)
    power = torch.empty_like(chi2)
    sde_raw = ctypes.c_double()
    sde = ctypes.c_double()
    rc = load().gtls_spectra(ctx, _ptr(chi2), _ptr(mask), n, float(oversampling_factor), _ptr(sr), _ptr(praw),
                             _ptr(power), ctypes.byref(sde_raw), ctypes.byref(sde), _stream(torch, device))
    _check(rc, ctx, "gtls_spectra")
    return sr, praw, power, sde_raw.value, sde.value


def model_chi2(t, y, w, off, params, device=0):
    """gtls_model_chi2: chi2 per curve (device tensors, float64; off int64)."""
    torch = _torch()
    ctx = context(device)
    n_curves = int(off.numel()) - 1
    out = torch.empty(n_curves, dtype=torch.float64, device=params.device)
    rc = load().gtls_model_chi2(ctx, _ptr(t), _ptr(y), _ptr(w), _ptr(off), n_curves, _ptr(params), _ptr(out),
                                _stream(torch, device))
    _check(rc, ctx, "gtls_model_chi2")
    return out


def model_chi2_grad(t, y, w, off, params, grad_chi2, device=0):
    """gtls_model_chi2_grad: d(sum_c g_c chi2_c)/d params, shape (n_curves, 6)."""
    torch = _torch()
    ctx = context(device)
    n_curves = int(off.numel()) - 1
    out = torch.empty((n_curves, 6), dtype=torch.float64, device=params.device)
    rc = load().gtls_model_chi2_grad(ctx, _ptr(t), _ptr(y), _ptr(w), _ptr(off), n_curves, _ptr(params),
                                     _ptr(grad_chi2), _ptr(out), _stream(torch, device))
    _check(rc, ctx, "gtls_model_chi2_grad")
    return out
