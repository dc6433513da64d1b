"""Torch-autograd and finite-difference references of the model chi2 -- TEST INFRASTRUCTURE ONLY.

The same model as the C-ABI's gtls_model_chi2 (its definition is in
include/gtls_b200.h), written with torch operations in float64 so that
torch.autograd provides an independent gradient, plus central finite
differences.  Used only by tests and the bench's checks.
"""
import numpy as np
import torch

EDGE = 0.05
SOFT_K = 200.0


def _softplus_k(x):
    """log(1 + exp(k x)) / k, evaluated as the kernel does."""
    kx = SOFT_K * x
    big = x + torch.log1p(torch.exp(-kx.clamp(min=0.0))) / SOFT_K
    small = torch.log1p(torch.exp(kx.clamp(max=30.0))) / SOFT_K
    return torch.where(kx > 30.0, big, small)


def model(t, params):
    """t: (n,) float64 tensor; params: (6,) float64 tensor -> model flux (n,)."""
    P, T0, D, depth, u1, u2 = params
    x = t - T0
    ep = torch.round((x / P).detach())
    tau = x - ep * P
    s = 2.0 * tau / D
    q = 1.0 - s * s
    B = torch.sigmoid(q / EDGE)
    mu = torch.sqrt(_softplus_k(q).clamp(min=1e-300))
    om = 1.0 - mu
    I = 1.0 - u1 * om - u2 * om * om
    mu0 = torch.sqrt(_softplus_k(torch.ones((), dtype=t.dtype, device=t.device)))
    om0 = 1.0 - mu0
    I0 = 1.0 - u1 * om0 - u2 * om0 * om0
    return 1.0 - depth * B * I / I0


def chi2(t, y, w, params):
    r = y - model(t, params)
    return torch.sum(w * r * r)


def autograd_grad(t, y, w, params):
    p = params.clone().detach().requires_grad_(True)
    c = chi2(t, y, w, p)
    (g,) = torch.autograd.grad(c, p)
    return c.detach(), g


def finite_difference_grad(t, y, w, params, rel=1e-6):
    """Central differences with step rel * |param|.  For T0 the magnitude is its
    offset from the first sample (the epoch within the data): an absolute time
    stamp of ~1e2-1e3 d would make a 1e-6 relative step span many seconds."""
    g = torch.empty_like(params)
    for k in range(params.numel()):
        scale = abs(float(params[k]) - float(t[0])) if k == 1 else abs(float(params[k]))
        h = rel * max(scale, 1e-12)
        pp = params.clone()
        pm = params.clone()
        pp[k] += h
        pm[k] -= h
        g[k] = (chi2(t, y, w, pp) - chi2(t, y, w, pm)) / (2 * h)
    return g


def richardson_grad(t, y, w, params, rel=1e-6):
    """Central differences at steps h and h/2 combined as (4 D(h/2) - D(h)) / 3,
    which cancels the h^2 truncation term."""
    d1 = finite_difference_grad(t, y, w, params, rel)
    d2 = finite_difference_grad(t, y, w, params, rel / 2)
    return (4 * d2 - d1) / 3
