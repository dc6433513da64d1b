"""Sub-grid refinement of search peaks with the adjoint of the model chi2.

``ModelChi2`` is a ``torch.autograd.Function`` over the C-ABI kernels
``gtls_model_chi2`` (forward) and ``gtls_model_chi2_grad`` (backward, model
recomputed).  ``refine`` runs batched Adam on the six parameters
(P, T0, D, depth, u1, u2) of many light curves at once, in a scaled
parameterisation, and keeps the grid result of any curve whose chi2 did not
improve.  No counterpart in the reference.
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
