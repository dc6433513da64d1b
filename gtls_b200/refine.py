"""Sub-grid refinement of search peaks with the adjoint of the model chi2.

``ModelChi2`` is a ``torch.autograd.Function`` over the C-ABI kernels
``gtls_model_chi2`` (forward) and ``gtls_model_chi2_grad`` (backward, model
recomputed).  The model is the search's own template model: a central
transit of an opaque disk across a quadratically limb-darkened star
(``ldmodel``), parameterised by (P, T0, D, depth, u1, u2) with D the
first-to-fourth-contact duration and depth the central depth.  ``refine``
runs batched Adam on the six parameters of many light curves at once, in a
scaled parameterisation, and keeps the grid result of any curve whose chi2
did not improve.  ``grid_start`` and ``refine_peaks`` start it from search
results (``power(refine=True)``).  No counterpart in the reference.
"""
import numpy as np

from . import _lib

PARAMS = ("P", "T0", "D", "depth", "u1", "u2")


def _torch():
    import torch
    return torch


class ModelChi2:
    """Namespace for the autograd Function (built lazily so torch imports late)."""
    fn = None


def model_chi2_function():
    torch = _torch()
    if ModelChi2.fn is None:
        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, params, t, y, w, off):
                p = params.detach().contiguous()
                ctx.save_for_backward(p, t, y, w, off)
                return _lib.model_chi2(t, y, w, off, p, device=p.device.index or 0)

            @staticmethod
            def backward(ctx, grad_out):
                p, t, y, w, off = ctx.saved_tensors
                g = _lib.model_chi2_grad(t, y, w, off, p, grad_out.contiguous(), device=p.device.index or 0)
                return g, None, None, None, None

        ModelChi2.fn = _F
    return ModelChi2.fn


def pack_curves(curves, device):
    """Concatenate [(t, y, dy), ...] into device tensors (t, y, w, off).

    The weights w = 1 / (dy * dy) are formed on the device from the copied
    uncertainties (one IEEE multiply and divide: the values the host would
    compute, without a host pass over every sample)."""
    torch = _torch()
    lens = [len(c[0]) for c in curves]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    t = np.concatenate([np.asarray(c[0], dtype=np.float64) for c in curves])
    y = np.concatenate([np.asarray(c[1], dtype=np.float64) for c in curves])
    dy = np.concatenate([np.asarray(c[2], dtype=np.float64) for c in curves])
    dev = torch.device(device)
    dy_d = torch.from_numpy(dy).to(dev)
    w = 1.0 / (dy_d * dy_d)
    return torch.from_numpy(t).to(dev), torch.from_numpy(y).to(dev), w, torch.from_numpy(off).to(dev)


def refine(params0, scales, t, y, w, off, steps=50, lr=0.05):
    """Batched Adam on ``params0`` (n_curves x 6) in units of ``scales``.

    Returns (params, chi2, improved): curves whose chi2 did not decrease keep
    their starting (grid) parameters.
    """
    torch = _torch()
    F = model_chi2_function()
    p0 = params0.detach().clone()
    delta = torch.zeros_like(p0, requires_grad=True)
    opt = torch.optim.Adam([delta], lr=lr)
    with torch.no_grad():
        chi0 = F.apply(p0, t, y, w, off)
    for _ in range(steps):
        opt.zero_grad(set_to_none=True)
        chi = F.apply(p0 + delta * scales, t, y, w, off)
        chi.sum().backward()
        opt.step()
    with torch.no_grad():
        p1 = p0 + delta.detach() * scales
        chi1 = F.apply(p1, t, y, w, off)
        better = chi1 < chi0
        out = torch.where(better[:, None], p1, p0)
        chi = torch.where(better, chi1, chi0)
    return out, chi, better


def grid_start(period, T0, duration, depth, u, periods, t):
    """Starting parameters (P, T0, D, depth, u1, u2) of a grid peak and the
    Adam scales: the local spacing of the period grid at P, the median
    cadence, 5% of D, 10% of the depth and 0.05 for each limb-darkening
    coefficient."""
    periods = np.sort(np.asarray(periods, dtype=np.float64))
    t = np.asarray(t, dtype=np.float64)
    i = int(np.clip(np.searchsorted(periods, period), 0, len(periods) - 1))
    lo, hi = max(i - 1, 0), min(i + 1, len(periods) - 1)
    step = (periods[hi] - periods[lo]) / max(hi - lo, 1) if hi > lo else abs(period) * 1e-4
    cad = float(np.median(np.diff(np.sort(t)))) if len(t) > 1 else 1e-3
    u1 = float(u[0]) if len(u) > 0 else 0.0
    u2 = float(u[1]) if len(u) > 1 else 0.0
    start = np.array([period, T0, duration, depth, u1, u2], dtype=np.float64)
    scale = np.array([step, cad, 0.05 * abs(duration), 0.1 * abs(depth), 0.05, 0.05], dtype=np.float64)
    return start, scale


def refine_peaks(curves, starts, scales, device=0, steps=50, lr=0.05):
    """Refine the grid peaks of ``curves`` [(t, y, dy)] (host arrays) from
    ``starts``/``scales`` (n_curves x 6) in one batched run.  Returns host
    arrays (params, chi2, chi2_grid, improved); a curve whose chi2 did not
    decrease keeps its starting (grid) parameters."""
    torch = _torch()
    dev = "cuda:%d" % device
    t, y, w, off = pack_curves(curves, dev)
    p0 = torch.as_tensor(np.asarray(starts, dtype=np.float64), device=dev)
    sc = torch.as_tensor(np.asarray(scales, dtype=np.float64), device=dev)
    with torch.no_grad():
        chi0 = model_chi2_function().apply(p0, t, y, w, off)
    out, chi, better = refine(p0, sc, t, y, w, off, steps=steps, lr=lr)
    return (out.detach().cpu().numpy(), chi.detach().cpu().numpy(), chi0.cpu().numpy(),
            better.cpu().numpy().astype(bool))


def refined_transit_times(transit_times, T0, period):
    """The grid's transit times moved to a refined (T0, P), epoch by epoch."""
    tt = np.asarray(transit_times, dtype=np.float64)
    if tt.size == 0:
        return tt
    epochs = np.round((tt - T0) / period)
    return T0 + epochs * period
